"""BackwardEuler with the state kept by the host (b200fem_backward_euler_step_host).

A host that owns the state (ArtiSynth's Java side) hands x and v over every
step and takes the new ones back in the same call.  The engine keeps its own
velocity history for the PCG warm start, so
* when the host hands back exactly the state it received, every step equals
  the device-resident step bit for bit (positions, velocities, iterations);
* when the host changes the state between steps, the step still solves to
  the PCG tolerance: positions agree with a b200fem_set_state + step run
  within 1e-8 relative (only the initial guess differs).
"""
import numpy as np
import pytest

from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import MechSystemSolver, NeoHookeanMaterial

from helpers import rel_err

pytestmark = pytest.mark.gpu


def _wl():
    wl = W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45), cells=(8, 3, 3), widths=(1.0, 0.3, 0.3))
    wl.build_mesh()
    return wl


def test_host_state_steps_equal_device_steps(b200):
    wl = _wl()
    a = wl.model()
    sa = MechSystemSolver(a, tol=1e-10)
    b = wl.model()
    sb = MechSystemSolver(b, tol=1e-10)
    x = np.ascontiguousarray(wl.rest.reshape(-1).copy())
    v = np.zeros_like(x)
    for step in range(6):
        sa.backwardEuler(wl.h, 1)
        ia = sa.stats.iterations
        sb.backwardEulerHost(wl.h, x, v)
        assert sb.stats.iterations == ia, step
        xa, va = a.getState()
        assert np.array_equal(x, xa.reshape(-1)) and np.array_equal(v, va.reshape(-1)), step


def test_host_changed_state_solves_to_tolerance(b200):
    wl = _wl()
    a = wl.model()
    sa = MechSystemSolver(a, tol=1e-10)
    b = wl.model()
    sb = MechSystemSolver(b, tol=1e-10)
    x = np.ascontiguousarray(wl.rest.reshape(-1).copy())
    v = np.zeros_like(x)
    for _ in range(3):
        sb.backwardEulerHost(wl.h, x, v)
    sa.backwardEuler(wl.h, 3)
    v *= 0.5  # the host damps the velocities between steps
    xa, _ = a.getState()
    a.setState(xa, v.reshape(-1, 3))
    for _ in range(2):
        sa.backwardEuler(wl.h, 1)
        sb.backwardEulerHost(wl.h, x, v)
    xa, _ = a.getState()
    assert rel_err(x, xa.reshape(-1)) <= 1e-8


def _pinned(a):
    import torch
    t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
    p = t.numpy()
    p[:] = a
    return t, p


def test_page_locked_host_state_one_graph(b200):
    """Page-locked x and v take the single-graph path (copies in, step, copies
    out, status in one launch): bit-identical to device-resident steps and to
    the pageable path, also when the host hands over other page-locked
    buffers, or pageable ones, between calls."""
    wl = _wl()
    a = wl.model()
    sa = MechSystemSolver(a, tol=1e-10)
    b = wl.model()
    sb = MechSystemSolver(b, tol=1e-10)
    x0 = np.ascontiguousarray(wl.rest.reshape(-1).copy())
    keep = []
    tx, x = _pinned(x0)
    tv, v = _pinned(np.zeros_like(x0))
    keep += [tx, tv]
    for step in range(8):
        if step == 3:  # other page-locked buffers (captured again)
            tx, x2 = _pinned(x)
            tv, v2 = _pinned(v)
            keep += [tx, tv]
            x, v = x2, v2
        if step == 5:  # pageable buffers (copies issued one by one)
            x, v = np.ascontiguousarray(x.copy()), np.ascontiguousarray(v.copy())
        if step == 7:  # page-locked again
            tx, x2 = _pinned(x)
            tv, v2 = _pinned(v)
            keep += [tx, tv]
            x, v = x2, v2
        sa.backwardEuler(wl.h, 1)
        sb.backwardEulerHost(wl.h, x, v)
        assert sb.stats.iterations == sa.stats.iterations, step
        xa, va = a.getState()
        assert np.array_equal(x, xa.reshape(-1)) and np.array_equal(v, va.reshape(-1)), step
        asm, solve = sb.lastTiming()
        assert asm > 0 and solve > 0
