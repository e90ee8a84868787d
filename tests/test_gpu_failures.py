"""Failure detection without faulting the GPU.

* A PCG grid-barrier wait that runs out: the test knob
  B200FEM_OPT_TEST_SKIP_ARRIVAL makes one CTA not arrive at the first
  barrier (a flag that nothing sets), B200FEM_OPT_BARRIER_TIMEOUT_MS bounds
  every wait at 200 ms; the step returns B200FEM_ERR_TIMEOUT and the same
  handle, and the device, keep working afterwards.
* abortOnInvertedElems (FemModel3d.java:2991-3001: a step with inverted
  elements throws NumericalException("Inverted elements")): the step returns
  B200FEM_ERR_INVERTED before the solve and leaves the state as it was.
* Non-finite caller input (positions, velocities, external forces, rest
  positions, material and step parameters) is refused on the host with
  B200FEM_ERR_INVALID_ARG before anything reaches the device.
"""
import ctypes

import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (LinearMaterial, MechSystemSolver, NeoHookeanMaterial,
                                          StVenantKirchoffMaterial)

pytestmark = pytest.mark.gpu


def _model(wl):
    wl.build_mesh()
    return wl.model()


def _status(fn, *args):
    with pytest.raises(L.B200FemError) as ei:
        fn(*args)
    return ei.value.status


def test_barrier_timeout_reports_status_and_recovers(b200):
    import torch

    wl = W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45), cells=(6, 2, 2))
    m = _model(wl)
    ref = _model(wl)
    e = m.engine()
    e.call("b200fem_set_option", L.OPT_BARRIER_TIMEOUT_MS, 200)
    e.call("b200fem_set_option", L.OPT_TEST_SKIP_ARRIVAL, 1)  # CTA 0 never arrives
    ms = MechSystemSolver(m, tol=1e-12)
    st = _status(ms.backwardEuler, wl.h, 1)
    assert st == L.ERR_TIMEOUT
    assert b"timed out" in L.lib().b200fem_last_error(e.h)
    # the device context is intact: torch work and further steps succeed
    t = torch.arange(1000, dtype=torch.float64, device="cuda:0")
    assert float(t.sum().item()) == 499500.0
    e.call("b200fem_set_option", L.OPT_TEST_SKIP_ARRIVAL, 0)
    v = np.zeros_like(wl.rest)
    m.setState(wl.rest, v)
    ms.backwardEuler(wl.h, 3)
    MechSystemSolver(ref, tol=1e-12).backwardEuler(wl.h, 3)
    x1, v1 = m.getState()
    x2, v2 = ref.getState()
    # same layout, same inputs: bit-identical to a handle that never failed
    assert np.array_equal(x1, x2) and np.array_equal(v1, v2)
    out = ctypes.c_int()
    e.call("b200fem_get_option", L.OPT_BARRIER_TIMEOUT_MS, ctypes.byref(out))
    assert out.value == 200


def _invert_one_element(rest, conn, fixed):
    """Reflect a free node of some tet through the plane of the tet's other
    three nodes: that tet's Jacobian determinant changes sign."""
    x = rest.copy()
    for e in range(conn.shape[0]):
        for a in range(4):
            n = conn[e, a]
            if fixed[n]:
                continue
            others = [conn[e, b] for b in range(4) if b != a]
            p0, p1, p2 = (x[o] for o in others)
            nrm = np.cross(p1 - p0, p2 - p0)
            nrm /= np.linalg.norm(nrm)
            d = np.dot(x[n] - p0, nrm)
            x[n] = x[n] - 2.0 * d * nrm
            return x
    raise AssertionError("no free node")


def test_abort_on_inverted_elements(b200):
    # a non-linear material: the reference counts inverted elements where it
    # forms the Jacobian, which linear materials skip (below)
    wl = W.small_tet_beam(StVenantKirchoffMaterial(5e4, 0.3))
    m = _model(wl)
    x_bad = _invert_one_element(wl.rest, wl.conn, wl.fixed)
    v0 = np.zeros_like(x_bad)
    m.setState(x_bad, v0)
    ms = MechSystemSolver(m, tol=1e-12)
    ms.abort_on_inverted = True
    assert _status(ms.backwardEuler, wl.h, 1) == L.ERR_INVERTED
    assert b"inverted" in L.lib().b200fem_last_error(m.engine().h)
    x, v = m.getState()
    assert np.array_equal(x, x_bad) and np.array_equal(v, v0)  # the step did not run
    # without the abort the step runs and reports the inverted elements in
    # its statistics (filled also when the solve misses its tolerance)
    ms.abort_on_inverted = False
    try:
        ms.backwardEuler(wl.h, 1)
    except L.B200FemError as err:
        assert err.status == L.ERR_NO_CONVERGE
    assert ms.stats.num_inverted >= 1 and ms.stats.min_detJ < 0


def test_linear_material_counts_no_inverted_elements(b200):
    """Linear materials leave computeStressAndStiffness before any Jacobian
    (FemModel3d.java:3356-3394: the warper's cached stiffness, then the early
    return), so an inverted element neither aborts the step nor is counted."""
    wl = W.small_tet_beam(LinearMaterial(5e4, 0.33, True))
    m = _model(wl)
    m.setState(_invert_one_element(wl.rest, wl.conn, wl.fixed), np.zeros_like(wl.rest))
    ms = MechSystemSolver(m, tol=1e-12)
    ms.abort_on_inverted = True
    st = ms.backwardEuler(wl.h, 1)
    assert st.num_inverted == 0


def test_non_finite_inputs_rejected(b200):
    wl = W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33))
    m = _model(wl)
    e = m.engine()
    lib = L.lib()
    n = wl.rest.size
    good_x = np.ascontiguousarray(wl.rest.reshape(-1))
    good_v = np.zeros(n)
    for bad in (np.nan, np.inf, -np.inf):
        xb = good_x.copy()
        xb[7] = bad
        assert lib.b200fem_set_state(e.h, L.dptr(xb), L.dptr(good_v)) == L.ERR_INVALID_ARG
        assert lib.b200fem_set_state(e.h, L.dptr(good_x), L.dptr(xb)) == L.ERR_INVALID_ARG
        assert lib.b200fem_set_external_forces(e.h, L.dptr(xb)) == L.ERR_INVALID_ARG
        assert lib.b200fem_update_stress_stiffness(e.h, L.dptr(xb), None, None, None) == L.ERR_INVALID_ARG
        ms = MechSystemSolver(m, tol=1e-12)
        p = ms.params(wl.h)
        st = L.Stats()
        assert lib.b200fem_backward_euler_step_host(e.h, ctypes.byref(p), 1, xb.ctypes.data, good_v.ctypes.data,
                                                    ctypes.byref(st)) == L.ERR_INVALID_ARG
        p.gravity[2] = bad
        assert lib.b200fem_backward_euler_step(e.h, ctypes.byref(p), 1, ctypes.byref(st)) == L.ERR_INVALID_ARG
        assert b"non-finite" in lib.b200fem_last_error(e.h)
    # a fresh handle refuses a non-finite mesh or material
    cfg = L.Config(0, L.PREC_FP64)
    h = lib.b200fem_create(ctypes.byref(cfg))
    assert h
    try:
        rb = good_x.copy()
        rb[0] = np.nan
        conn = np.ascontiguousarray(wl.conn.reshape(-1))
        assert lib.b200fem_set_mesh(h, wl.elem_type, wl.rest.shape[0], L.dptr(rb), wl.conn.shape[0],
                                    L.iptr(conn), L.iptr(wl.fixed)) == L.ERR_INVALID_ARG
        prm = np.zeros(8)
        prm[:2] = (np.inf, 0.3)
        assert lib.b200fem_set_material(h, L.MAT_NEOHOOKEAN, L.dptr(prm), 1000.0, L.INCOMP_AUTO) == L.ERR_INVALID_ARG
    finally:
        lib.b200fem_destroy(h)
    # nothing reached the device: the model still steps to the same result
    # as an untouched one
    ref = _model(wl)
    MechSystemSolver(m, tol=1e-12).backwardEuler(wl.h, 2)
    MechSystemSolver(ref, tol=1e-12).backwardEuler(wl.h, 2)
    assert np.array_equal(m.getState()[0], ref.getState()[0])
