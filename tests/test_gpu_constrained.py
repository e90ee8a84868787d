"""ConstrainedBackwardEuler with particle-plane constraints on single nodes
(b200fem_set_plane_constraints) against the oracle's dense KKT step
(MechSystemSolver.constrainedBackwardEuler with ParticlePlaneConstraint):
positions 1e-8 relative (FP64; mixed 1e-6), constrained nodes on their planes,
normal velocities zero; BackwardEuler ignores the constraints."""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import MechSystemSolver, NeoHookeanMaterial

from helpers import oracle_model, rel_err

pytestmark = pytest.mark.gpu


def _setup(tilt):
    wl = W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), cells=(6, 2, 2), widths=(1.0, 0.3, 0.3))
    wl.build_mesh()
    tip = np.where(wl.rest[:, 0] >= wl.rest[:, 0].max() - 1e-9)[0]
    n = np.array([0.0, 1.0, 1.0]) / np.sqrt(2) if tilt else np.array([0.0, 0.0, 1.0])
    nrm = np.tile(n, (tip.size, 1))
    off = (nrm * wl.rest[tip]).sum(axis=1)
    return wl, tip, nrm, off


@pytest.mark.parametrize("precision,tilt", [(L.PREC_FP64, True), (L.PREC_FP64, False), (L.PREC_MIXED, True)])
def test_constrained_backward_euler_matches_kkt_oracle(b200, oracle, precision, tilt):
    wl, tip, nrm, off = _setup(tilt)
    steps = 6
    m = wl.model(precision=precision)
    m.setPlaneConstraints(tip, nrm, off)
    ms = MechSystemSolver(m, tol=1e-12, max_iter=20000, integrator=L.INTEGRATOR_CONSTRAINED_BACKWARD_EULER)
    om = oracle_model(oracle, wl)
    x, v = wl.rest.copy(), np.zeros_like(wl.rest)
    for _ in range(steps):
        ms.backwardEuler(wl.h, 1)
        assert om.cbe_step(wl.h, x, v, tip, nrm, off, alpha=wl.mass_damping, gravity=wl.gravity) == 0
    xg, vg = m.getState()
    tol = 1e-8 if precision == L.PREC_FP64 else 1e-6
    assert rel_err(xg, x) <= tol, rel_err(xg, x)
    assert np.abs((nrm * xg[tip]).sum(axis=1) - off).max() <= 1e-12
    assert np.abs((nrm * vg[tip]).sum(axis=1)).max() <= 1e-8 * np.abs(vg).max()
    assert rel_err(vg, v) <= (1e-6 if precision == L.PREC_FP64 else 1e-4)


def test_backward_euler_ignores_plane_constraints(b200):
    wl, tip, nrm, off = _setup(True)
    a = wl.model()
    a.setPlaneConstraints(tip, nrm, off)
    b = wl.model()
    sa = MechSystemSolver(a, tol=1e-12)
    sb = MechSystemSolver(b, tol=1e-12)
    sa.backwardEuler(wl.h, 4)
    sb.backwardEuler(wl.h, 4)
    assert np.array_equal(a.getState()[0], b.getState()[0])
