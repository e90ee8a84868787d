"""The oracle on meshes that mix element types in one model (hexes, wedges
and pyramids along the beam; tets and hexes): the stiffness and forces of
the mixed model are the sums of those of its single-type parts (assembly is
additive per element; masses too), the stiffness matches finite
differences of the forces, and AUTO soft incompressibility resolves as the
reference does (NODAL allowed for tets, hexes, wedges and pyramids)."""
import numpy as np
import pytest

from helpers import deformed


def _blocks(om, K):
    rp, col = om.pattern()
    sidx = om.solve_index()
    node_of = {int(r): n for n, r in enumerate(sidx) if r >= 0}
    out = {}
    for r in range(rp.size - 1):
        for p in range(rp[r], rp[r + 1]):
            out[(node_of[r], node_of[int(col[p])])] = K[p]
    return out


@pytest.mark.parametrize("kinds", [(1, 2, 3), (0, 1, 0)])
@pytest.mark.parametrize("mat,params,incomp", [(1, [5e4, 0.4], 0), (2, [1e4, 2e3, 0, 0, 0, 1e5, 0, 0], 3),
                                               (3, [5e4, 0.3], 0), (0, [5e4, 0.3, 1], 0)])
def test_mixed_equals_sum_of_parts(oracle, kinds, mat, params, incomp):
    xyz, types, conn = oracle.mixed_grid((1.2, 0.4, 0.4), (6, 2, 2), jitter=0.03, seed=4, kinds=kinds)
    fixed = (xyz[:, 0] <= -0.6 + 1e-9).astype(np.int32)
    m = oracle.OracleModel(types, xyz, conn, fixed, mat, params, 1000.0, incomp)
    assert m.E == types.size and len(set(types.tolist())) == len(set(kinds))
    x = deformed(xyz, seed=2, noise=0.005)
    f, K, _ = m.update_stress_stiffness(x)
    whole = _blocks(m, K)
    fsum = np.zeros_like(f)
    msum = np.zeros(len(xyz))
    parts = {}
    offs = np.concatenate([[0], np.cumsum([oracle.ELEM_NODES[int(t)] for t in types])])
    for t in sorted(set(types.tolist())):
        sel = np.nonzero(types == t)[0]
        c = np.concatenate([conn[offs[e]:offs[e + 1]] for e in sel])
        pm = oracle.OracleModel(t, xyz, c, fixed, mat, params, 1000.0, incomp)
        pf, pK, _ = pm.update_stress_stiffness(x)
        fsum += pf
        msum += pm.masses()
        for key, blk in _blocks(pm, pK).items():
            parts[key] = parts.get(key, 0) + blk
    scale = max(np.abs(b).max() for b in whole.values())
    assert set(parts) <= set(whole)
    for key, blk in whole.items():
        assert np.abs(blk - parts.get(key, 0)).max() <= 1e-12 * scale, key
    assert np.abs(f - fsum).max() <= 1e-12 * np.abs(f).max()
    assert np.abs(m.masses() - msum).max() <= 1e-14 * msum.max()


@pytest.mark.parametrize("mat,params,incomp", [(1, [5e4, 0.45], 0), (2, [1e4, 2e3, 0, 0, 0, 1e5, 0, 0], 1),
                                               (2, [1e4, 2e3, 0, 0, 0, 1e5, 0, 1], 3)])
def test_mixed_stiffness_matches_force_fd(oracle, mat, params, incomp):
    xyz, types, conn = oracle.mixed_grid((1.0, 0.4, 0.4), (6, 2, 2), jitter=0.04, seed=3)
    fixed = (xyz[:, 0] <= -0.5 + 1e-9).astype(np.int32)
    m = oracle.OracleModel(types, xyz, conn, fixed, mat, params, 1000.0, incomp)
    assert m.incomp == incomp
    x = deformed(xyz, seed=1, rot_deg=15, bend=0.05, noise=0.01)
    _, K, _ = m.update_stress_stiffness(x)
    sidx = m.solve_index()
    rp, col = m.pattern()
    act = np.where(sidx >= 0)[0]
    h = 1e-7
    rng = np.random.default_rng(4)
    for _ in range(6):
        n = act[rng.integers(act.size)]
        c = rng.integers(3)
        xp = x.copy(); xp[n, c] += h
        xm = x.copy(); xm[n, c] -= h
        df = (m.update_stress_stiffness(xp)[0] - m.update_stress_stiffness(xm)[0]) / (2 * h)
        bj = sidx[n]
        for bi in range(m.nact):
            for p in range(rp[bi], rp[bi + 1]):
                if col[p] == bj:
                    assert np.abs(K[p][:, c] - df[act[bi]]).max() <= 1e-5 * np.abs(K).max()


def test_mixed_incompressibility_resolution(oracle):
    xyz, types, conn = oracle.mixed_grid((1.0, 0.4, 0.4), (6, 2, 2))
    fixed = (xyz[:, 0] <= -0.5 + 1e-9).astype(np.int32)
    mr = [1e4, 2e3, 0, 0, 0, 1e5, 0, 0]
    m = oracle.OracleModel(types, xyz, conn, fixed, 2, mr, 1000.0, oracle.INCOMP_AUTO)
    expect = oracle.INCOMP_NODAL if m.E > m.nact else oracle.INCOMP_ELEMENT
    assert m.incomp == expect
    assert oracle.OracleModel(types, xyz, conn, fixed, 2, mr, 1000.0, oracle.INCOMP_NODAL).incomp == \
        oracle.INCOMP_NODAL
