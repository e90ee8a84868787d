"""The decomposition behind the factored NODAL solve matrix, checked on the
oracle (CPU): the NODAL stiffness K (the reference's 2-ring pattern) equals
the element blocks of direct neighbours plus the dilational term
sum_n kp_n d_n d_n^T of computeNodalIncompressibility (FemModel3d.java:
2632-2669), so that

* every block between nodes that share no element (the 2-ring part of the
  pattern) is exactly the dilational term, and
* the two-phase product the PCG forms -- t_n = kp_n (d_n . v) over each
  active node's neighbour slots, then y_i = sum_n t_n d_n(i) over the
  (node, slot) entries of row i -- equals the dilational blocks times v.
"""
import numpy as np
import pytest

from helpers import deformed


def _model(oracle, etype, params, cells=(5, 3, 3)):
    xyz, conn = oracle.grid(etype, (1.0, 0.4, 0.4), cells, jitter=0.04, seed=9)
    fixed = (xyz[:, 0] <= -0.5 + 1e-9).astype(np.int32)
    m = oracle.OracleModel(etype, xyz, conn, fixed, 2, params, 1000.0, oracle.INCOMP_NODAL)
    assert m.incomp == oracle.INCOMP_NODAL
    return m, xyz, conn


def _dilational_blocks(m, ptr, idx, kp, div):
    sidx = m.solve_index()
    out = {}
    for n in range(m.N):
        if sidx[n] < 0 or kp[n] == 0:
            continue
        for a in range(ptr[n], ptr[n + 1]):
            ra = sidx[idx[a]]
            if ra < 0:
                continue
            for b in range(ptr[n], ptr[n + 1]):
                rb = sidx[idx[b]]
                if rb < 0:
                    continue
                key = (int(ra), int(rb))
                out[key] = out.get(key, 0) + kp[n] * np.outer(div[a], div[b])
    return out


@pytest.mark.parametrize("etype,params", [(0, [1000.0, 500.0, 0, 0, 0, 1e5, 0, 0]),
                                          (1, [1037.0, 120.0, 0, 486.0, 0, 1.037e4, 0, 1])])
def test_indirect_blocks_are_the_dilational_term(oracle, etype, params):
    m, xyz, conn = _model(oracle, etype, params)
    x = deformed(xyz, seed=4, noise=0.01)
    _, K, _ = m.update_stress_stiffness(x)
    ptr, idx, kp, div = m.nodal_factors()
    sidx = m.solve_index()
    rp, col = m.pattern()
    dil = _dilational_blocks(m, ptr, idx, kp, div)
    # direct pairs: nodes sharing an element
    direct = set()
    for e in np.asarray(conn).reshape(len(conn), -1):
        for a in e:
            for b in e:
                if sidx[a] >= 0 and sidx[b] >= 0:
                    direct.add((int(sidx[a]), int(sidx[b])))
    scale = np.abs(K).max()
    n_indirect = 0
    for r in range(m.nact):
        for p in range(rp[r], rp[r + 1]):
            key = (r, int(col[p]))
            if key in direct:
                continue
            n_indirect += 1
            assert np.abs(K[p] - dil[key]).max() <= 1e-12 * scale, key
    assert n_indirect > 0 and len(direct) < rp[-1]
    # every dilational block lies in the pattern
    pat = {(r, int(col[p])) for r in range(m.nact) for p in range(rp[r], rp[r + 1])}
    assert set(dil) <= pat


def test_two_phase_product_equals_the_blocks(oracle):
    m, xyz, _ = _model(oracle, 0, [1000.0, 500.0, 0, 0, 0, 1e5, 0, 0])
    x = deformed(xyz, seed=5, noise=0.01)
    m.update_stress_stiffness(x)
    ptr, idx, kp, div = m.nodal_factors()
    sidx = m.solve_index()
    dil = _dilational_blocks(m, ptr, idx, kp, div)
    v = np.random.default_rng(2).standard_normal((m.nact, 3))
    ref = np.zeros_like(v)
    for (ra, rb), blk in dil.items():
        ref[ra] += blk @ v[rb]
    # phase 1: t_n over the node's active neighbour slots
    t = np.zeros(m.N)
    for n in range(m.N):
        if sidx[n] < 0:
            continue
        s = 0.0
        for a in range(ptr[n], ptr[n + 1]):
            r = sidx[idx[a]]
            if r >= 0:
                s += div[a] @ v[r]
        t[n] = kp[n] * s
    # phase 2: row i adds t_n d_n(i) over the active nodes n of its own
    # neighbour list (i is in nbr(n) exactly when n is in nbr(i))
    y = np.zeros_like(v)
    act_node = np.nonzero(sidx >= 0)[0]
    for r, i in enumerate(act_node):
        for a in range(ptr[i], ptr[i + 1]):
            n = idx[a]
            if sidx[n] < 0:
                continue
            slot = ptr[n] + int(np.searchsorted(idx[ptr[n]:ptr[n + 1]], i))
            assert idx[slot] == i
            y[r] += t[n] * div[slot]
    assert np.abs(y - ref).max() <= 1e-12 * np.abs(ref).max()


def test_bench_factored_byte_counts(oracle):
    """bench.py's counts for the factored roofline: direct blocks between
    active nodes (the 1-ring pattern, as the oracle builds it without NODAL)
    and the neighbour slots of the active nodes (the divBlk rows)."""
    import bench
    m, xyz, conn = _model(oracle, 0, [1000.0, 500.0, 0, 0, 0, 1e5, 0, 0])
    fixed = (xyz[:, 0] <= -0.5 + 1e-9).astype(np.int32)
    nnzb1, slots = bench.direct_counts(np.asarray(conn).reshape(len(conn), -1), fixed)
    off = oracle.OracleModel(0, xyz, conn, fixed, 2, [1000.0, 500.0, 0, 0, 0, 1e5, 0, 0], 1000.0,
                             oracle.INCOMP_OFF)
    assert nnzb1 == off.nnzb
    m.update_stress_stiffness(xyz)
    ptr, _, _, _ = m.nodal_factors()
    act = np.nonzero(fixed == 0)[0]
    assert slots == int(np.sum(ptr[act + 1] - ptr[act]))
