"""The oracle with per-element materials (FemElement.setMaterial;
FemModel3d.getElementMaterial, FemModel3d.java:608-614): each element is
assembled with its own material, else the model's.  A model whose elements
carry several materials equals the sum of one-material models over the same
elements (assembly is additive per element; masses follow the density, not
the material), the stiffness matches finite differences of the forces, soft
incompressibility resolves as the reference does (ELEMENT for incompressible
elements of a compressible model, OFF per compressible element), and NODAL
pressures use the model's bulk modulus."""
import numpy as np
import pytest

from helpers import deformed

LIN_C = (0, [3e4, 0.3, 1])
LIN = (0, [6e4, 0.25, 0])
NH = (1, [5e4, 0.4])
NH2 = (1, [2e4, 0.35])
STVK = (3, [4e4, 0.3])
MR = (2, [1e4, 2e3, 0, 0, 0, 1e5, 0, 0])
MR_LOG = (2, [2e4, 1e3, 0, 0, 0, 5e4, 0, 1])
CYCLE = [None, LIN_C, LIN, NH2, STVK, MR, MR_LOG]


def _blocks(om, K):
    rp, col = om.pattern()
    sidx = om.solve_index()
    node_of = {int(r): n for n, r in enumerate(sidx) if r >= 0}
    out = {}
    for r in range(rp.size - 1):
        for p in range(rp[r], rp[r + 1]):
            out[(node_of[r], node_of[int(col[p])])] = K[p]
    return out


def _mesh(oracle, etype, cells=(6, 2, 2)):
    xyz, conn = oracle.grid(etype, (1.2, 0.4, 0.4), cells, jitter=0.03, seed=6)
    fixed = (xyz[:, 0] <= -0.6 + 1e-9).astype(np.int32)
    return xyz, conn, fixed


def _assign(E, cycle=CYCLE):
    return [cycle[e % len(cycle)] for e in range(E)]


@pytest.mark.parametrize("etype", [0, 1, 2])
def test_element_materials_equal_sum_of_parts(oracle, etype):
    xyz, conn, fixed = _mesh(oracle, etype)
    conn = conn.reshape(len(conn), -1)
    m = oracle.OracleModel(etype, xyz, conn, fixed, NH[0], NH[1], 1000.0, oracle.INCOMP_AUTO)
    mats = _assign(m.E)
    m.set_element_materials(mats)
    # the model's material is compressible: its incompressible elements run with ELEMENT
    assert m.incomp == oracle.INCOMP_ELEMENT
    x = deformed(xyz, seed=2, noise=0.005)
    f, K, _ = m.update_stress_stiffness(x)
    whole = _blocks(m, K)
    fsum = np.zeros_like(f)
    msum = np.zeros(len(xyz))
    parts = {}
    for mat in CYCLE:
        sel = [e for e in range(m.E) if mats[e] == mat]
        kind, prm = NH if mat is None else mat
        pm = oracle.OracleModel(etype, xyz, conn[sel], fixed, kind, prm, 1000.0, oracle.INCOMP_ELEMENT)
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


def test_model_material_everywhere_is_unchanged(oracle):
    """Elements given the model's own material, or None, assemble exactly as
    without element materials."""
    xyz, conn, fixed = _mesh(oracle, 1)
    a = oracle.OracleModel(1, xyz, conn, fixed, MR[0], MR[1], 1000.0, oracle.INCOMP_NODAL)
    b = oracle.OracleModel(1, xyz, conn, fixed, MR[0], MR[1], 1000.0, oracle.INCOMP_NODAL)
    b.set_element_materials([MR if e % 2 else None for e in range(b.E)])
    x = deformed(xyz, seed=3, noise=0.01)
    fa, Ka, _ = a.update_stress_stiffness(x)
    fb, Kb, _ = b.update_stress_stiffness(x)
    assert np.array_equal(fa, fb) and np.array_equal(Ka, Kb)
    b.set_element_materials(None)
    assert np.array_equal(b.update_stress_stiffness(x)[1], Ka)


@pytest.mark.parametrize("etype,model,incomp", [(0, NH, 2), (1, MR, 3), (2, LIN, 2), (1, MR, 1)])
def test_element_materials_stiffness_matches_force_fd(oracle, etype, model, incomp):
    xyz, conn, fixed = _mesh(oracle, etype)
    m = oracle.OracleModel(etype, xyz, conn, fixed, model[0], model[1], 1000.0, incomp)
    if incomp == oracle.INCOMP_NODAL:
        cycle = [None, MR_LOG, (2, [5e3, 4e3, 0, 0, 0, 1e5, 0, 0])]  # NODAL: every element incompressible
    else:
        # (the corotated linear stiffness R K0 R^T leaves out dR/dx: not an exact tangent)
        cycle = [c for c in CYCLE if c is not LIN_C]
    m.set_element_materials(_assign(m.E, cycle))
    # AUTO on a compressible model: its incompressible elements run with ELEMENT
    assert m.incomp == (oracle.INCOMP_ELEMENT if incomp == oracle.INCOMP_AUTO else incomp)
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


def test_nodal_uses_the_models_kappa(oracle):
    """Under NODAL the nodal pressures and the dilational stiffness use the
    model's material (updateNodalPressures / computeNodalIncompressibility
    take myMaterial, FemModel3d.java:2471-2515, 2632-2669): elements that
    differ from the model only in kappa assemble as the model alone."""
    xyz, conn, fixed = _mesh(oracle, 0)
    a = oracle.OracleModel(0, xyz, conn, fixed, MR[0], MR[1], 1000.0, oracle.INCOMP_NODAL)
    b = oracle.OracleModel(0, xyz, conn, fixed, MR[0], MR[1], 1000.0, oracle.INCOMP_NODAL)
    other_kappa = (2, [1e4, 2e3, 0, 0, 0, 3e6, 0, 1])
    b.set_element_materials([other_kappa] * b.E)
    assert a.incomp == b.incomp == oracle.INCOMP_NODAL
    x = deformed(xyz, seed=3, noise=0.01)
    fa, Ka, _ = a.update_stress_stiffness(x)
    fb, Kb, _ = b.update_stress_stiffness(x)
    assert np.array_equal(fa, fb) and np.array_equal(Ka, Kb)


def test_incompressibility_resolution(oracle):
    xyz, conn, fixed = _mesh(oracle, 0)
    m = oracle.OracleModel(0, xyz, conn, fixed, NH[0], NH[1], 1000.0, oracle.INCOMP_AUTO)
    assert m.incomp == oracle.INCOMP_OFF
    m.set_element_materials([MR if e == 3 else None for e in range(m.E)])
    assert m.incomp == oracle.INCOMP_ELEMENT  # the model's material is compressible: no NODAL
    m.set_element_materials(None)
    assert m.incomp == oracle.INCOMP_OFF
    # an incompressible model with more elements than active nodes: AUTO -> NODAL,
    # refused when an element's material is compressible
    mr = oracle.OracleModel(0, xyz, conn, fixed, MR[0], MR[1], 1000.0, oracle.INCOMP_AUTO)
    assert mr.incomp == oracle.INCOMP_NODAL
    mr.set_element_materials([MR_LOG] * mr.E)
    assert mr.incomp == oracle.INCOMP_NODAL
    with pytest.raises(ValueError):
        mr.set_element_materials([NH if e == 0 else None for e in range(mr.E)])
    el = oracle.OracleModel(0, xyz, conn, fixed, MR[0], MR[1], 1000.0, oracle.INCOMP_ELEMENT)
    el.set_element_materials([NH if e == 0 else None for e in range(el.E)])
    assert el.incomp == oracle.INCOMP_ELEMENT
