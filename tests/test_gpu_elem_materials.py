"""Per-element materials (b200fem_set_element_materials; FemElement.setMaterial,
FemModel3d.getElementMaterial, FemModel3d.java:608-614) against the oracle,
which assembles every element with its own material, else the model's.

The engine holds each model's elements sorted by type, material kind and
corotation; the scatter map, forces and stiffness are those of the caller's
element order.  Bars: pattern, CRS indices, slot map, scatter map and solve
indices bit-exact; masses 1e-14; forces and stiffness blocks 1e-10 of the
oracle's scale; positions after 10 BackwardEuler steps 1e-8 relative.
"""
import ctypes

import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200.femmodel import (FemModel3d, FemPack, LinearMaterial, MechSystemSolver,
                                          MooneyRivlinMaterial, NeoHookeanMaterial, StVenantKirchoffMaterial)

from helpers import deformed, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10
LIN_C = LinearMaterial(3e4, 0.3, True)
LIN = LinearMaterial(6e4, 0.25, False)
NH = NeoHookeanMaterial(5e4, 0.4)
NH2 = NeoHookeanMaterial(2e4, 0.35)
STVK = StVenantKirchoffMaterial(4e4, 0.3)
MR = MooneyRivlinMaterial(1e4, 2e3, 0, 0, 0, 1e5)
MR_LOG = MooneyRivlinMaterial(2e4, 1e3, 0, 0, 0, 5e4, 0.0, 1)
MR_SOFT = MooneyRivlinMaterial(5e3, 4e3, 0, 0, 0, 1e5)
CYCLE = [None, LIN_C, LIN, NH2, STVK, MR, MR_LOG]

# name: element type (or mixed kinds), model material, soft incompressibility, element cycle
CASES = {
    "tet_neohookean_all_kinds": (L.ELEM_TET, NH, L.INCOMP_AUTO, CYCLE),
    "hex_linear_all_kinds": (L.ELEM_HEX, LIN, L.INCOMP_AUTO, CYCLE),
    "wedge_stvk_all_kinds": (L.ELEM_WEDGE, STVK, L.INCOMP_AUTO, CYCLE),
    "hex_mooneyrivlin_nodal": (L.ELEM_HEX, MR, L.INCOMP_NODAL, [None, MR_LOG, MR_SOFT]),
    "tet_mooneyrivlin_element": (L.ELEM_TET, MR, L.INCOMP_ELEMENT, CYCLE),
    "quadhex_mooneyrivlin_element": (L.ELEM_QUADHEX, MR, L.INCOMP_AUTO, [None, NH2, MR_LOG]),
    "mixed_hwp_neohookean": ((L.ELEM_HEX, L.ELEM_WEDGE, L.ELEM_PYRAMID), NH, L.INCOMP_AUTO, CYCLE),
}


def _oracle_mats(mats):
    return [None if m is None else (m.kind, m.params()) for m in mats]


def _pair(oracle, name, precision=L.PREC_FP64):
    et, mat, inc, cycle = CASES[name]
    cells = (4, 2, 2) if et == L.ELEM_QUADHEX else (6, 2, 2)
    if isinstance(et, tuple):
        xyz, types, conn = oracle.mixed_grid((1.2, 0.4, 0.4), cells, jitter=0.03, seed=4, kinds=et)
        etype = types
    else:
        xyz, conn = oracle.grid(et, (1.2, 0.4, 0.4), cells, jitter=0.03, seed=6)
        etype = et
    fixed = (xyz[:, 0] <= -0.6 + 1e-9).astype(np.int32)
    m = FemModel3d()
    m.setMesh(etype, xyz, conn, fixed)
    m.setMaterial(mat)
    m.setDensity(1000.0)
    m.setPrecision(precision)
    m.setSoftIncompMethod(inc)
    mats = [cycle[e % len(cycle)] for e in range(m.numElements())]
    m.setElementMaterials(mats)
    om = oracle.OracleModel(etype, xyz, conn, fixed, mat.kind, mat.params(), 1000.0, inc)
    om.set_element_materials(_oracle_mats(mats))
    return m, om, xyz, etype, np.asarray(conn).reshape(-1)


@pytest.mark.parametrize("name", list(CASES))
def test_elem_materials_pattern_and_maps(name, b200, oracle):
    m, om, xyz, etype, conn = _pair(oracle, name)
    assert m.getSoftIncompMethod() == om.incomp
    rp, col = m.getBlockPattern()
    orp, ocol = om.pattern()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(m.getSolveIndices(), om.solve_index())
    for part in (L.PART_FULL, L.PART_UPPER):
        ro, ci = m.getCRSIndices(part)
        oro, oci, osl = om.crs(part)
        assert np.array_equal(ro, oro) and np.array_equal(ci, oci)
        assert np.array_equal(m.createCrsBlockSlotMap(part), osl)
    # the scatter map in the caller's element order, although storage is sorted by material
    types = etype if np.ndim(etype) else np.full(m.numElements(), etype)
    sidx = om.solve_index()
    ref, off = [], 0
    for t in types:
        k = L.ELEM_NODES[int(t)]
        nodes = conn[off:off + k]
        off += k
        for a in range(k):
            for b in range(k):
                ra, rb = sidx[nodes[a]], sidx[nodes[b]]
                ref.append(orp[ra] + np.searchsorted(ocol[orp[ra]:orp[ra + 1]], rb) if ra >= 0 and rb >= 0 else -1)
    assert np.array_equal(np.asarray(m.getScatterMap()).reshape(-1), np.array(ref, dtype=np.int32))
    assert rel_err(m.getNodeMasses(), om.masses()) <= 1e-14


@pytest.mark.parametrize("name", list(CASES))
def test_elem_materials_update_stress_stiffness(name, b200, oracle):
    m, om, xyz, _, _ = _pair(oracle, name)
    x = deformed(xyz, seed=5)
    f, K, crs = m.updateStressAndStiffness(x, want_crs=True)
    of, oK, _ = om.update_stress_stiffness(x)
    assert rel_err(f, of) <= TOL, rel_err(f, of)
    assert rel_err(K, oK) <= TOL, rel_err(K, oK)
    slots = m.createCrsBlockSlotMap(L.PART_FULL)
    assert np.array_equal(crs[slots], K.reshape(-1))


@pytest.mark.parametrize("name", ["tet_neohookean_all_kinds", "hex_mooneyrivlin_nodal", "tet_mooneyrivlin_element",
                                  "mixed_hwp_neohookean"])
def test_elem_materials_backward_euler(name, b200, oracle):
    m, om, xyz, _, _ = _pair(oracle, name)
    h, steps = 0.01, 10
    x, v = xyz.copy(), np.zeros_like(xyz)
    for _ in range(steps):
        st, _, _ = om.be_step(h, x, v, alpha=2.0, gravity=(0, 0, -9.8), solver=1, tol=1e-14)
        assert st == 0
    m.setGravity(0, 0, -9.8)
    MechSystemSolver(m, tol=1e-13, max_iter=20000).backwardEuler(h, steps)
    xg, _ = m.getState()
    assert rel_err(xg, x) <= 1e-8
    assert np.abs((xg - xyz) - (x - xyz)).max() <= 1e-7 * np.abs(x - xyz).max()
    assert (x - xyz)[:, 2].min() < -1e-4  # the beam sags


def test_elem_materials_mixed_precision(b200, oracle):
    m, om, xyz, _, _ = _pair(oracle, "tet_neohookean_all_kinds", precision=L.PREC_MIXED)
    x = deformed(xyz, seed=5)
    f, K = m.updateStressAndStiffness(x)
    of, oK, _ = om.update_stress_stiffness(x)
    assert rel_err(K, oK) <= 2e-6
    assert rel_err(f, of) <= 1e-5


@pytest.mark.parametrize("tet_assembly", [0, 1])
def test_pack_with_elem_materials(tet_assembly, b200, oracle):
    """A pack of a plain model and two with element materials, each against
    its own oracle run; the node-row tet assembly (asked for with 0) stays on
    the element path when a model's elements form several groups."""
    specs = [("tet_neohookean_all_kinds", True), ("tet_mooneyrivlin_element", True),
             ("tet_neohookean_all_kinds", False)]
    models, oms, rests = [], [], []
    for name, own in specs:
        m, om, xyz, _, _ = _pair(oracle, name)
        if not own:
            m.setElementMaterials(None)
            om.set_element_materials(None)
        m.setGravity(0, 0, -9.8)
        models.append(m)
        oms.append(om)
        rests.append(xyz)
    steps, h = 5, 0.01
    pack = FemPack(models, precision=L.PREC_FP64, options={L.OPT_TET_ASSEMBLY: tet_assembly})
    pack.backwardEuler(h, steps, tol=1e-13)
    assert pack.option(L.OPT_TET_ASSEMBLY) == 1
    for om, xyz, (xg, _) in zip(oms, rests, pack.getStates()):
        x, v = xyz.copy(), np.zeros_like(xyz)
        for _ in range(steps):
            st, _, _ = om.be_step(h, x, v, alpha=2.0, gravity=(0, 0, -9.8), solver=1, tol=1e-14)
            assert st == 0
        assert rel_err(xg, x) <= 1e-8, rel_err(xg, x)


def test_elem_materials_refusals(b200, oracle):
    """NODAL with an element of a compressible material is refused at the
    build (ERR_UNSUPPORTED); a wrong element count or an unknown kind at the
    call (ERR_INVALID_ARG); B200FEM_MAT_MODEL everywhere equals no element
    materials."""
    xyz, conn = oracle.grid(L.ELEM_HEX, (1.2, 0.4, 0.4), (6, 2, 2), jitter=0.03, seed=6)
    fixed = (xyz[:, 0] <= -0.6 + 1e-9).astype(np.int32)
    lib = L.lib()
    h = lib.b200fem_create(ctypes.byref(L.Config(0, L.PREC_FP64)))
    assert h
    try:
        rest = np.ascontiguousarray(xyz.reshape(-1))
        c = np.ascontiguousarray(conn.reshape(-1))
        E = conn.shape[0]
        assert lib.b200fem_set_mesh(h, L.ELEM_HEX, xyz.shape[0], L.dptr(rest), E, L.iptr(c), L.iptr(fixed)) == L.OK
        prm = np.zeros(8)
        prm[: len(MR.params())] = MR.params()
        assert lib.b200fem_set_material(h, L.MAT_MOONEYRIVLIN, L.dptr(prm), 1000.0, L.INCOMP_NODAL) == L.OK
        kinds = np.full(E, L.MAT_MODEL, dtype=np.int32)
        eprm = np.zeros((E, 8))
        kinds[5] = L.MAT_NEOHOOKEAN
        eprm[5, :2] = (5e4, 0.4)
        assert lib.b200fem_set_element_materials(h, 0, E - 1, kinds.ctypes.data, eprm.ctypes.data) == \
            L.ERR_INVALID_ARG
        bad = kinds.copy()
        bad[2] = 17
        assert lib.b200fem_set_element_materials(h, 0, E, bad.ctypes.data, eprm.ctypes.data) == L.ERR_INVALID_ARG
        assert lib.b200fem_set_element_materials(h, 0, E, kinds.ctypes.data, eprm.ctypes.data) == L.OK
        assert lib.b200fem_build(h) == L.ERR_UNSUPPORTED
        assert b"compressible" in lib.b200fem_last_error(h)
        assert lib.b200fem_set_element_materials(h, 0, E, None, None) == L.OK
        assert lib.b200fem_build(h) == L.OK
    finally:
        lib.b200fem_destroy(h)


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("option,value", [(L.OPT_TET_ASSEMBLY, 0), (L.OPT_FUSED_ASSEMBLY, 1)])
def test_one_kind_paths_with_elem_materials(option, value, precision, b200, oracle):
    """Elements of one kind with different parameters keep a model in one
    group, so the node-row tet assembly and the fused assembly stay in force;
    both read each element's row of the material table.  10 steps against
    the oracle: 1e-8 in FP64, 1e-5 in the mixed form."""
    xyz, conn = oracle.grid(L.ELEM_TET, (1.2, 0.4, 0.4), (6, 3, 3), jitter=0.03, seed=6)
    fixed = (xyz[:, 0] <= -0.6 + 1e-9).astype(np.int32)
    mats = [[None, NH2, NeoHookeanMaterial(8e4, 0.45)][e % 3] for e in range(conn.shape[0])]
    m = FemModel3d()
    m.setMesh(L.ELEM_TET, xyz, conn, fixed)
    m.setMaterial(NH)
    m.setDensity(1000.0)
    m.setPrecision(precision)
    m.setElementMaterials(mats)
    m.setGravity(0, 0, -9.8)
    m.options = {option: value}
    h, steps = 0.01, 10
    MechSystemSolver(m, tol=1e-13, max_iter=20000).backwardEuler(h, steps)
    o = ctypes.c_int()
    m.engine().call("b200fem_get_option", option, ctypes.byref(o))
    assert o.value == value  # the path asked for is in force
    om = oracle.OracleModel(L.ELEM_TET, xyz, conn, fixed, NH.kind, NH.params(), 1000.0, L.INCOMP_AUTO)
    om.set_element_materials(_oracle_mats(mats))
    x, v = xyz.copy(), np.zeros_like(xyz)
    for _ in range(steps):
        st, _, _ = om.be_step(h, x, v, alpha=2.0, gravity=(0, 0, -9.8), solver=1, tol=1e-14)
        assert st == 0
    xg, _ = m.getState()
    assert rel_err(xg, x) <= (1e-8 if precision == L.PREC_FP64 else 1e-5), rel_err(xg, x)
