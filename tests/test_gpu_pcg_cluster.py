"""The cluster split of the pack PCG (B200FEM_OPT_PCG_SPLIT 3: one
thread-block cluster per model, models from a queue largest first).

* every model of an FP64 pack against its oracle run (positions 1e-8);
* a model in the pack against the same model stepped alone, and against the
  strided split (1e-9 at PCG 1e-12: the algorithms and the dot-product
  partitions differ, the solution does not);
* bit-reproducible run to run; models masked out keep their state;
* plane constraints, refinement sweeps, the stand-alone PCG call and the
  non-convergence status on the cluster split.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import FemPack, MechSystemSolver, NeoHookeanMaterial

from helpers import oracle_model, rel_err

pytestmark = pytest.mark.gpu


def _beams(count=20, seed=9, cap=14):
    bs = W.batched_beams(count=count, seed=seed)
    for b in bs:
        b.cells = (min(b.cells[0], cap), b.cells[1], b.cells[2])
        b.widths = (b.cells[0] * 0.05, b.widths[1], b.widths[2])
        b.build_mesh()
    return bs


@pytest.fixture(scope="module")
def beams(b200):
    return _beams()


def _pack(bs, precision, split=L.SPLIT_CLUSTER, **opts):
    o = {L.OPT_PCG_SPLIT: split}
    o.update(opts)
    p = FemPack([b.model() for b in bs], precision=precision, options=o)
    assert p.option(L.OPT_PCG_SPLIT) == split
    return p


def test_cluster_pack_matches_oracle(beams, oracle):
    steps = 4
    pack = _pack(beams, L.PREC_FP64)
    pack.backwardEuler(beams[0].h, steps, tol=1e-12)
    states = pack.getStates()
    it, rr = pack.modelStats()
    pack.close()
    for b, (xg, _) in zip(beams, states):
        om = oracle_model(oracle, b)
        x = b.rest.copy()
        v = np.zeros_like(x)
        for _ in range(steps):
            st, _, _ = om.be_step(b.h, x, v, alpha=b.mass_damping, gravity=b.gravity, solver=0, tol=1e-14)
            assert st == 0
        assert rel_err(xg, x) <= 1e-8, (b.name, rel_err(xg, x))
        assert rel_err(xg - b.rest, x - b.rest) <= 1e-6, (b.name, rel_err(xg - b.rest, x - b.rest))
    assert np.all(it > 0) and np.all(rr <= 1e-12)


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
def test_cluster_equals_alone_and_strided(beams, precision):
    steps = 4
    res = {}
    for split in (L.SPLIT_CLUSTER, L.SPLIT_STRIDED):
        pack = _pack(beams, precision, split)
        pack.backwardEuler(beams[0].h, steps, tol=1e-12)
        res[split] = [x for x, _ in pack.getStates()]
        pack.close()
    for i, b in enumerate(beams):
        m = b.model(precision=precision)
        MechSystemSolver(m, tol=1e-12).backwardEuler(b.h, steps)
        xa, _ = m.getState()
        m._invalidate()
        assert rel_err(res[L.SPLIT_CLUSTER][i], xa) <= 1e-9, (b.name, rel_err(res[L.SPLIT_CLUSTER][i], xa))
        assert rel_err(res[L.SPLIT_CLUSTER][i], res[L.SPLIT_STRIDED][i]) <= 1e-9


def test_cluster_deterministic_and_masks(beams):
    out = []
    for _ in range(2):
        pack = _pack(beams, L.PREC_MIXED)
        pack.backwardEuler(beams[0].h, 2, tol=1e-10)
        before = pack.getStates()
        mask = np.array([i % 3 != 0 for i in range(len(beams))], dtype=np.int32)
        pack.setActive(mask)
        pack.backwardEuler(beams[0].h, 2, tol=1e-10)
        it, _ = pack.modelStats()
        after = pack.getStates()
        for i in range(len(beams)):
            if not mask[i]:
                assert np.array_equal(after[i][0], before[i][0]) and it[i] == 0
        pack.setActive(None)
        pack.backwardEuler(beams[0].h, 1, tol=1e-10)
        out.append(pack.getStates())
        pack.close()
    for (x0, v0), (x1, v1) in zip(*out):
        assert np.array_equal(x0, x1) and np.array_equal(v0, v1)


def test_cluster_refinement_and_pcg_call(beams):
    """One refinement sweep per step on the cluster split reaches the FP64
    result; b200fem_pcg_solve on the pack's matrix solves every model."""
    steps = 3
    pack = FemPack([b.model() for b in beams[:8]], precision=L.PREC_MIXED,
                   options={L.OPT_PCG_SPLIT: L.SPLIT_CLUSTER, L.OPT_REFINE: 1})
    pack.backwardEuler(beams[0].h, steps, tol=1e-10)
    xs = [x for x, _ in pack.getStates()]
    ref = FemPack([b.model() for b in beams[:8]], precision=L.PREC_FP64,
                  options={L.OPT_PCG_SPLIT: L.SPLIT_CLUSTER})
    ref.backwardEuler(beams[0].h, steps, tol=1e-12)
    xr = [x for x, _ in ref.getStates()]
    for b, x, y in zip(beams[:8], xs, xr):
        assert rel_err(x - b.rest, y - b.rest) <= 1e-6, (b.name, rel_err(x - b.rest, y - b.rest))
    # stand-alone solve on the last step's matrix
    import ctypes
    e = ref.engine()
    n = sum(a for (_, _, a) in ref.offsets) * 3
    rng = np.random.default_rng(2)
    xt = rng.standard_normal(n)
    y = np.zeros(n)
    e.call("b200fem_spmv", L.dptr(xt), L.dptr(y))
    x = np.zeros(n)
    st = L.Stats()
    e.call("b200fem_pcg_solve", L.dptr(y), L.dptr(x), 1e-13, 20000, ctypes.byref(st))
    assert rel_err(x, xt) <= 1e-8
    pack.close()
    ref.close()


def test_cluster_no_convergence_status(beams):
    pack = _pack(beams[:4], L.PREC_FP64)
    with pytest.raises(L.B200FemError) as ei:
        pack.backwardEuler(beams[0].h, 1, tol=1e-14, max_iter=2)
    assert ei.value.status == L.ERR_NO_CONVERGE
    pack.backwardEuler(beams[0].h, 1, tol=1e-10)  # the pack still steps
    pack.close()


def test_cluster_plane_constraints_vs_oracle(b200, oracle):
    """ConstrainedBackwardEuler on a pack on the cluster split: a model with
    tip nodes held on tilted planes against the oracle's KKT solve."""
    import ctypes

    wls = [W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), cells=(6, 2, 2), seed=s) for s in (1, 2, 3)]
    for w in wls:
        w.build_mesh()
    pack = FemPack([w.model() for w in wls], precision=L.PREC_FP64,
                   options={L.OPT_PCG_SPLIT: L.SPLIT_CLUSTER})
    e = pack.engine()
    w = wls[1]
    free = np.nonzero(w.fixed == 0)[0]
    tip = free[np.argsort(w.rest[free, 0])[-3:]]
    nrm = np.tile([0.0, 0.3, 1.0], (tip.size, 1))
    off = (nrm * w.rest[tip]).sum(axis=1)
    node0 = pack.offsets[1][0]
    nodes = np.ascontiguousarray((tip + node0).astype(np.int32))
    e.call("b200fem_set_plane_constraints", tip.size, L.iptr(nodes), L.dptr(np.ascontiguousarray(nrm.reshape(-1))),
           L.dptr(np.ascontiguousarray(off)))
    p = L.StepParams()
    p.h = w.h
    p.alpha_m = w.mass_damping
    for i in range(3):
        p.gravity[i] = w.gravity[i]
    p.tol = 1e-13
    p.max_iter = 20000
    p.integrator = L.INTEGRATOR_CONSTRAINED_BACKWARD_EULER
    st = L.Stats()
    steps = 4
    e.call("b200fem_backward_euler_step", ctypes.byref(p), steps, ctypes.byref(st))
    xg = pack.getStates()[1][0]
    pack.close()
    om = oracle_model(oracle, w)
    x = w.rest.copy()
    v = np.zeros_like(x)
    for _ in range(steps):
        assert om.cbe_step(w.h, x, v, tip, nrm / np.linalg.norm(nrm, axis=1)[:, None],
                           off / np.linalg.norm(nrm, axis=1), alpha=w.mass_damping, gravity=w.gravity) == 0
    assert rel_err(xg, x) <= 1e-8
