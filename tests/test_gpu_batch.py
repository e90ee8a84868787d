"""Batched form: several uneven models in one pack (one launch per phase,
per-model PCG scalars and convergence).

* every model of an FP64 pack matches its own oracle run (positions 1e-8);
* a model's result in the pack equals its result stepped alone (1e-9: only
  the dot-product partition differs);
* per-model stats report each model's iterations and true residual.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import FemPack, MechSystemSolver

from helpers import oracle_model, rel_err

pytestmark = pytest.mark.gpu


def _beams(count=6, seed=5):
    bs = W.batched_beams(count=count, seed=seed)
    for b in bs:  # keep the oracle runs short
        b.cells = (min(b.cells[0], 12), b.cells[1], b.cells[2])
        b.widths = (b.cells[0] * 0.05, b.widths[1], b.widths[2])
        b.build_mesh()
    return bs


@pytest.fixture(scope="module")
def beams(b200):
    return _beams()


def test_pack_matches_oracle(beams, oracle):
    steps = 5
    pack = FemPack([b.model() for b in beams], precision=L.PREC_FP64)
    pack.backwardEuler(beams[0].h, steps, tol=1e-12)
    states = pack.getStates()
    for b, (xg, vg) in zip(beams, states):
        om = oracle_model(oracle, b)
        x = b.rest.copy()
        v = np.zeros_like(x)
        for _ in range(steps):
            st, _, _ = om.be_step(b.h, x, v, alpha=b.mass_damping, gravity=b.gravity, solver=1)
            assert st == 0
        assert rel_err(xg, x) <= 1e-8, (b.name, rel_err(xg, x))
    it, rr = pack.modelStats()
    assert np.all(it > 0) and np.all(rr <= 1e-12)


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_pack_result_equals_alone(beams, precision):
    steps = 4
    pack = FemPack([b.model() for b in beams], precision=precision)
    pack.backwardEuler(beams[0].h, steps, tol=1e-12)
    states = pack.getStates()
    for b, (xg, _) in zip(beams, states):
        m = b.model(precision=precision)
        MechSystemSolver(m, tol=1e-12).backwardEuler(b.h, steps)
        xa, _ = m.getState()
        assert rel_err(xg, xa) <= 1e-9, (b.name, rel_err(xg, xa))


def test_pack_of_mixed_materials(b200, oracle):
    """Models with different materials form element groups inside one pack."""
    from artisynth_core_b200.femmodel import MooneyRivlinMaterial, NeoHookeanMaterial, LinearMaterial
    wls = [W.small_tet_beam(NeoHookeanMaterial(3e4, 0.4)), W.small_tet_beam(LinearMaterial(2e4, 0.3, True)),
           W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5)),
           W.small_tet_beam(NeoHookeanMaterial(8e4, 0.3))]
    for w in wls:
        w.build_mesh()
    pack = FemPack([w.model() for w in wls], precision=L.PREC_FP64)
    pack.backwardEuler(wls[0].h, 3, tol=1e-12)
    for w, (xg, _) in zip(wls, pack.getStates()):
        om = oracle_model(oracle, w)
        x = w.rest.copy()
        v = np.zeros_like(x)
        for _ in range(3):
            om.be_step(w.h, x, v, alpha=w.mass_damping, gravity=w.gravity, solver=1)
        assert rel_err(xg, x) <= 1e-8
