"""LinearPointConstraints (constraints coupling several nodes) under the
ConstrainedBackwardEuler integrator against the oracle's dense KKT step
(orc_cbe_step_points): positions within the parity bar after several
steps, the constraints held after the position correction, BackwardEuler
ignoring them, and the refusal of plane and point constraints together."""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import MechSystemSolver, MooneyRivlinMaterial, NeoHookeanMaterial

from helpers import oracle_model, rel_err

pytestmark = pytest.mark.gpu


def _constraints(rest):
    """The mean of the tip face held at its rest value (one constraint over
    every tip node, equal weights), and a rigid link: the difference of a tip
    node and an interior node held at its rest value (weights 1, -1)."""
    tip = np.nonzero(rest[:, 0] >= rest[:, 0].max() - 1e-9)[0]
    inner = int(np.argmin(np.abs(rest[:, 0] - np.median(rest[:, 0])) + np.abs(rest[:, 1]) + np.abs(rest[:, 2])))
    ptr = np.array([0, tip.size, tip.size + 2], dtype=np.int32)
    nodes = np.concatenate([tip, [tip[0], inner]]).astype(np.int32)
    w = np.concatenate([np.full(tip.size, 1.0 / tip.size), [1.0, -1.0]])
    targets = np.concatenate([rest[tip].mean(axis=0), rest[tip[0]] - rest[inner]])
    return ptr, nodes, w, targets


@pytest.mark.parametrize("precision,maker,mat", [
    (L.PREC_FP64, W.small_tet_beam, NeoHookeanMaterial(5e4, 0.33)),
    (L.PREC_FP64, W.small_hex_beam, MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
    (L.PREC_MIXED, W.small_tet_beam, NeoHookeanMaterial(5e4, 0.33))])
def test_point_constraints_vs_oracle(b200, oracle, precision, maker, mat):
    wl = maker(mat, cells=(6, 2, 2))
    wl.build_mesh()
    ptr, nodes, w, targets = _constraints(wl.rest)
    steps = 5
    m = wl.model(precision=precision)
    m.setPointConstraints(ptr, nodes, w, targets)
    ms = MechSystemSolver(m, tol=1e-13, max_iter=20000, integrator=L.INTEGRATOR_CONSTRAINED_BACKWARD_EULER)
    ms.backwardEuler(wl.h, steps)
    xg, vg = m.getState()
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(steps):
        assert om.cbe_step_points(wl.h, x, v, ptr, nodes, w, targets, alpha=wl.mass_damping,
                                  gravity=wl.gravity) == 0
    tol = 1e-8 if precision == L.PREC_FP64 else 1e-6
    assert rel_err(xg, x) <= tol, rel_err(xg, x)
    assert rel_err(xg - wl.rest, x - wl.rest) <= (1e-6 if precision == L.PREC_FP64 else 1e-4)
    for c in range(ptr.size - 1):
        sl = slice(ptr[c], ptr[c + 1])
        held = (w[sl, None] * xg[nodes[sl]]).sum(axis=0)
        assert np.abs(held - targets[3 * c:3 * c + 3]).max() <= 1e-12
    assert np.abs(xg - wl.rest).max() > 1e-5  # the beam moves under gravity


def test_backward_euler_ignores_point_constraints(b200):
    wl = W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33))
    wl.build_mesh()
    a, b = wl.model(), wl.model()
    a.setPointConstraints(*_constraints(wl.rest))
    MechSystemSolver(a, tol=1e-12).backwardEuler(wl.h, 3)
    MechSystemSolver(b, tol=1e-12).backwardEuler(wl.h, 3)
    assert np.array_equal(a.getState()[0], b.getState()[0])


def test_plane_and_point_constraints_refused_together(b200):
    wl = W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33))
    wl.build_mesh()
    m = wl.model()
    m.setPointConstraints(*_constraints(wl.rest))
    free = np.nonzero(wl.fixed == 0)[0][:1]
    m.setPlaneConstraints(free, np.array([[0.0, 0.0, 1.0]]), wl.rest[free, 2])
    ms = MechSystemSolver(m, tol=1e-12, integrator=L.INTEGRATOR_CONSTRAINED_BACKWARD_EULER)
    with pytest.raises(L.B200FemError) as ei:
        ms.backwardEuler(wl.h, 1)
    assert ei.value.status == L.ERR_UNSUPPORTED
