"""Mixed-precision form (FP32 element kinematics, stress, tangent and stored
solve matrix; FP64 PCG vectors, dot products, residual and state update)
against the FP64 oracle.

Bars: stiffness blocks within 2e-6 of max|K| and positions after the stepped
runs within 1e-6 relative of the FP64 oracle (the stated target of the
mixed form); forces within 1e-5 of the force scale max|K|*|x - x_rest|.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (LinearMaterial, MechSystemSolver, MooneyRivlinMaterial,
                                          NeoHookeanMaterial)

from helpers import deformed, oracle_model, rel_err

pytestmark = pytest.mark.gpu


def _cases():
    return {
        "linear_corotated_tet": W.linear_tet_beam(),
        "neohookean_tet": W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33)),
        "neohookean_hex": W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45)),
        "mooneyrivlin_tet_nodal": W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5)),
    }


@pytest.fixture(scope="module")
def cases(b200):
    return _cases()


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_mixed_update_stress_stiffness(name, cases, oracle):
    wl = cases[name]
    m = wl.model(precision=L.PREC_MIXED)
    om = oracle_model(oracle, wl)
    x = deformed(wl.rest, seed=5)
    f, K = m.updateStressAndStiffness(x)
    of, oK, _ = om.update_stress_stiffness(x)
    assert rel_err(K, oK) <= 2e-6, rel_err(K, oK)
    fscale = np.abs(oK).max() * np.abs(x - wl.rest).max()
    assert np.abs(f - of).max() <= 1e-5 * fscale, np.abs(f - of).max() / fscale


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_mixed_backward_euler(name, cases, oracle):
    wl = cases[name]
    m = wl.model(precision=L.PREC_MIXED)
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(wl.steps):
        st, _, _ = om.be_step(wl.h, x, v, alpha=wl.mass_damping, beta=wl.stiffness_damping,
                              gravity=wl.gravity, fext=None, solver=1)
        assert st == 0
    ms = MechSystemSolver(m, tol=1e-12, max_iter=20000)
    ms.backwardEuler(wl.h, wl.steps)
    xg, _ = m.getState()
    err = rel_err(xg, x)
    assert err <= 1e-6, (name, err)


def test_mixed_mooneyrivlin_block_steps(oracle):
    """The MooneyRivlin block workload (NODAL) on a 12x6x6 block, 5 steps,
    mixed form against the FP64 oracle."""
    wl = W.mooneyrivlin_tet_block()
    wl.cells = (12, 6, 6)
    wl.build_mesh()
    m = wl.model(precision=L.PREC_MIXED)
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(5):
        om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=0, tol=1e-14)
    MechSystemSolver(m, tol=1e-12, max_iter=20000).backwardEuler(wl.h, 5)
    xg, _ = m.getState()
    assert rel_err(xg, x) <= 1e-6, rel_err(xg, x)
