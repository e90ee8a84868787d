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
    from artisynth_core_b200.femmodel import (MooneyRivlinMaterial, NeoHookeanMaterial, LinearMaterial,
                                              StVenantKirchoffMaterial)
    wls = [W.small_tet_beam(NeoHookeanMaterial(3e4, 0.4)), W.small_tet_beam(LinearMaterial(2e4, 0.3, True)),
           W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5)),
           W.small_tet_beam(NeoHookeanMaterial(8e4, 0.3)), W.small_tet_beam(StVenantKirchoffMaterial(4e4, 0.3))]
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


@pytest.mark.parametrize("beam", ["wedge", "pyramid", "quadtet", "quadhex", "quadwedge", "quadpyramid"])
def test_pack_of_wedges_or_pyramids(b200, oracle, beam):
    """A pack of one of the multi-point element types: uneven beams with
    different materials (element groups), every model against its oracle run."""
    from artisynth_core_b200.femmodel import (MooneyRivlinMaterial, NeoHookeanMaterial, LinearMaterial,
                                              StVenantKirchoffMaterial)
    mk = {"wedge": W.small_wedge_beam, "pyramid": W.small_pyramid_beam, "quadtet": W.small_quadtet_beam,
          "quadhex": W.small_quadhex_beam, "quadwedge": W.small_quadwedge_beam,
          "quadpyramid": W.small_quadpyramid_beam}[beam]
    wls = [mk(NeoHookeanMaterial(3e4, 0.4)), mk(LinearMaterial(2e4, 0.3, True), cells=(6, 2, 2)),
           mk(MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370), cells=(3, 3, 2)),
           mk(StVenantKirchoffMaterial(4e4, 0.3), cells=(5, 2, 3))]
    for w in wls:
        w.build_mesh()
        if beam in ("quadhex", "quadwedge"):  # several pressure values per element
            w.incomp = L.INCOMP_ELEMENT
    models = []
    for w in wls:
        mdl = w.model()
        if hasattr(w, "incomp"):
            mdl.setSoftIncompMethod(w.incomp)
        models.append(mdl)
    pack = FemPack(models, precision=L.PREC_FP64)
    pack.backwardEuler(wls[0].h, 3, tol=1e-12)
    for w, (xg, _) in zip(wls, pack.getStates()):
        om = oracle_model(oracle, w)
        x = w.rest.copy()
        v = np.zeros_like(x)
        for _ in range(3):
            om.be_step(w.h, x, v, alpha=w.mass_damping, gravity=w.gravity, solver=1)
        assert rel_err(xg, x) <= 1e-8, (beam, w.material, rel_err(xg, x))


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("variant", [L.PCG_AUTO, L.PCG_CLASSIC])
def test_strided_split_equals_alone(beams, precision, variant):
    """The strided split (models cut into short pieces dealt over the CTAs,
    iterations compacted to the models still iterating) gives each model the
    result it gets alone."""
    steps = 4
    opts = {L.OPT_PCG_SPLIT: L.SPLIT_STRIDED, L.OPT_PIECE_ROWS: 8, L.OPT_PCG_CTAS: 7}
    pack = FemPack([b.model() for b in beams], precision=precision, options=opts)
    assert pack.option(L.OPT_PCG_SPLIT) == L.SPLIT_STRIDED
    assert pack.option(L.OPT_PCG_CTAS) == 7
    pack.backwardEuler(beams[0].h, steps, tol=1e-12, pcg_variant=variant)
    it, rr = pack.modelStats()
    assert np.all(rr <= 1e-12)
    assert len(set(it.tolist())) > 1  # models converge at different iterations
    for b, (xg, _) in zip(beams, pack.getStates()):
        m = b.model(precision=precision)
        MechSystemSolver(m, tol=1e-12).backwardEuler(b.h, steps)
        xa, _ = m.getState()
        assert rel_err(xg, xa) <= 1e-9, (b.name, rel_err(xg, xa))


def test_strided_many_pieces_per_cta(b200):
    """More than one warp's worth of pieces on each CTA (the per-CTA piece
    tables span two warps), on a pack whose models converge at different
    iterations: every model matches its solve alone."""
    bs = W.batched_beams(count=24, seed=9)
    for b in bs:
        b.cells = (min(b.cells[0], 10), b.cells[1], b.cells[2])
        b.widths = (b.cells[0] * 0.05, b.widths[1], b.widths[2])
        b.build_mesh()
    steps = 3
    # 40-row pieces over 6 CTAs: about 45 pieces per CTA (270 in all)
    opts = {L.OPT_PCG_SPLIT: L.SPLIT_STRIDED, L.OPT_PIECE_ROWS: 40, L.OPT_PCG_CTAS: 6}
    for precision in (L.PREC_FP64, L.PREC_MIXED):
        pack = FemPack([b.model() for b in bs], precision=precision, options=opts)
        pack.backwardEuler(bs[0].h, steps, tol=1e-12)
        _, rr = pack.modelStats()
        assert np.all(rr <= 1e-12)
        for b, (xg, _) in zip(bs, pack.getStates()):
            m = b.model(precision=precision)
            MechSystemSolver(m, tol=1e-12).backwardEuler(b.h, steps)
            xa, _ = m.getState()
            assert rel_err(xg, xa) <= 1e-9, (b.name, precision, rel_err(xg, xa))
        pack.close()


def test_layout_options_agree(beams):
    """Contiguous and strided splits, CTA counts and SpMV row widths change
    only the rounding of the dot products."""
    steps = 3
    ref = None
    for opts in ({}, {L.OPT_PCG_SPLIT: L.SPLIT_CONTIGUOUS, L.OPT_PCG_CTAS: 3},
                 {L.OPT_PCG_SPLIT: L.SPLIT_STRIDED, L.OPT_ROW_LANES: 8},
                 {L.OPT_PCG_SPLIT: L.SPLIT_STRIDED, L.OPT_ROW_LANES: 32, L.OPT_PIECE_ROWS: 5}):
        pack = FemPack([b.model() for b in beams], precision=L.PREC_FP64, options=opts)
        pack.backwardEuler(beams[0].h, steps, tol=1e-12)
        x = np.concatenate([xg for xg, _ in pack.getStates()])
        if L.OPT_ROW_LANES in opts:
            assert pack.option(L.OPT_ROW_LANES) == opts[L.OPT_ROW_LANES]
        pack.close()
        if ref is None:
            ref = x
        else:
            assert rel_err(x, ref) <= 1e-9, opts


def test_row_lanes_change_after_build(beams):
    pack = FemPack([b.model() for b in beams], precision=L.PREC_FP64)
    pack.backwardEuler(beams[0].h, 2, tol=1e-12)
    for lanes in (8, 32):
        pack.setOption(L.OPT_ROW_LANES, lanes)
        assert pack.option(L.OPT_ROW_LANES) == lanes
    with pytest.raises(L.B200FemError):
        pack.setOption(L.OPT_PCG_SPLIT, L.SPLIT_STRIDED)  # layout options precede the build
    pack.backwardEuler(beams[0].h, 1, tol=1e-12)
    assert np.all(np.isfinite(np.concatenate([xg for xg, _ in pack.getStates()])))


def test_autotune_sets_options_and_keeps_results(beams, tmp_path):
    from artisynth_core_b200 import autotune
    models = [b.model() for b in beams]

    def make(opts):
        o = dict(opts)
        o[L.OPT_PCG_SPLIT] = L.SPLIT_STRIDED
        p = FemPack(models, precision=L.PREC_FP64, options=o)
        p.engine()
        return p

    cache = autotune.TuneCache(str(tmp_path / "tune.json"))
    pack, res, hit = autotune.tune_pack(make, models, L.PREC_FP64, beams[0].h, 1e-12, cache=cache)
    assert not hit and pack.option(L.OPT_ROW_LANES) == res["row_lanes"]
    assert pack.option(L.OPT_ELEM_TILE) == res["elem_tile"]
    for x, v in pack.getStates():
        assert np.all(v == 0)  # the tuning steps were undone
    pack.backwardEuler(beams[0].h, 3, tol=1e-12)
    ref = FemPack([b.model() for b in beams], precision=L.PREC_FP64)
    ref.backwardEuler(beams[0].h, 3, tol=1e-12)
    for (xa, _), (xb, _) in zip(pack.getStates(), ref.getStates()):
        assert rel_err(xa, xb) <= 1e-9
