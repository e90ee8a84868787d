"""Meshes whose elements are of several types in one model
(b200fem_set_mesh_mixed), and packs of models of different types, against
the oracle (which assembles the same elements in the caller's order).

Bars: pattern, CRS indices, slot map, scatter map and solve indices
bit-exact; masses 1e-14; forces and stiffness blocks 1e-10 of the oracle's
scale; positions after 10 BackwardEuler steps 1e-8 relative, displacements
1e-7 of the largest displacement.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (FemModel3d, FemPack, LinearMaterial, MechSystemSolver,
                                          MooneyRivlinMaterial, NeoHookeanMaterial, StVenantKirchoffMaterial)

from helpers import deformed, oracle_model, rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-10
HEX_WEDGE_PYR = (L.ELEM_HEX, L.ELEM_WEDGE, L.ELEM_PYRAMID)
TET_HEX_TET = (L.ELEM_TET, L.ELEM_HEX, L.ELEM_TET)

CASES = {
    "neohookean_hwp": (HEX_WEDGE_PYR, NeoHookeanMaterial(5e4, 0.45), None),
    "linear_corotated_hwp": (HEX_WEDGE_PYR, LinearMaterial(2e4, 0.3, True), None),
    "linear_plain_tht": (TET_HEX_TET, LinearMaterial(2e4, 0.3, False), None),
    "stvk_hwp": (HEX_WEDGE_PYR, StVenantKirchoffMaterial(5e4, 0.3), None),
    "neohookean_tht": (TET_HEX_TET, NeoHookeanMaterial(5e4, 0.4), None),
    "mooneyrivlin_hwp_element": (HEX_WEDGE_PYR, MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370), L.INCOMP_AUTO),
    "mooneyrivlin_hwp_nodal": (HEX_WEDGE_PYR, MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370), L.INCOMP_NODAL),
    "mooneyrivlin_tht_nodal_log": (TET_HEX_TET, MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5, 0.0, 1),
                                   L.INCOMP_AUTO),
    "mooneyrivlin_tht_element": (TET_HEX_TET, MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5), L.INCOMP_ELEMENT),
}


def _mesh(oracle, kinds):
    xyz, types, conn = oracle.mixed_grid((1.2, 0.4, 0.4), (6, 2, 2), jitter=0.03, seed=4, kinds=kinds)
    fixed = (xyz[:, 0] <= -0.6 + 1e-9).astype(np.int32)
    return xyz, types, conn, fixed


def _pair(oracle, name, precision=L.PREC_FP64):
    kinds, mat, incomp = CASES[name]
    xyz, types, conn, fixed = _mesh(oracle, kinds)
    m = FemModel3d()
    m.setMesh(types, xyz, conn, fixed)
    m.setMaterial(mat)
    m.setDensity(1000.0)
    m.setPrecision(precision)
    inc = L.INCOMP_AUTO if incomp is None else incomp
    m.setSoftIncompMethod(inc)
    om = oracle.OracleModel(types, xyz, conn, fixed, mat.kind, mat.params(), 1000.0, inc)
    return m, om, xyz, types, conn


@pytest.mark.parametrize("name", list(CASES))
def test_mixed_pattern_and_masses(name, b200, oracle):
    m, om, xyz, types, conn = _pair(oracle, name)
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
    smap = m.getScatterMap()
    sidx = om.solve_index()
    ref, q, off = [], 0, 0
    for t in types:
        k = L.ELEM_NODES[int(t)]
        nodes = conn[off:off + k]
        off += k
        for a in range(k):
            for b in range(k):
                ra, rb = sidx[nodes[a]], sidx[nodes[b]]
                ref.append(orp[ra] + np.searchsorted(ocol[orp[ra]:orp[ra + 1]], rb) if ra >= 0 and rb >= 0 else -1)
    assert np.array_equal(smap, np.array(ref, dtype=np.int32))
    assert rel_err(m.getNodeMasses(), om.masses()) <= 1e-14


@pytest.mark.parametrize("name", list(CASES))
def test_mixed_update_stress_stiffness(name, b200, oracle):
    m, om, xyz, _, _ = _pair(oracle, name)
    x = deformed(xyz, seed=5)
    f, K, crs = m.updateStressAndStiffness(x, want_crs=True)
    of, oK, _ = om.update_stress_stiffness(x)
    assert rel_err(f, of) <= TOL, rel_err(f, of)
    assert rel_err(K, oK) <= TOL, rel_err(K, oK)
    slots = m.createCrsBlockSlotMap(L.PART_FULL)
    assert np.array_equal(crs[slots], K.reshape(-1))


@pytest.mark.parametrize("name", ["neohookean_hwp", "linear_corotated_hwp", "mooneyrivlin_hwp_element",
                                  "mooneyrivlin_hwp_nodal", "mooneyrivlin_tht_nodal_log", "neohookean_tht"])
def test_mixed_backward_euler(name, b200, oracle):
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


def test_mixed_precision_mixed_mesh(b200, oracle):
    """The mixed-precision form on a mesh of several types: stiffness within
    2e-6 of the FP64 oracle's scale (FP32 tangent blocks)."""
    m, om, xyz, _, _ = _pair(oracle, "neohookean_hwp", precision=L.PREC_MIXED)
    x = deformed(xyz, seed=5)
    f, K = m.updateStressAndStiffness(x)
    of, oK, _ = om.update_stress_stiffness(x)
    assert rel_err(K, oK) <= 2e-6
    assert rel_err(f, of) <= 1e-5


def test_pack_of_different_types(b200, oracle):
    """Models of different element types in one pack: each matches its own
    oracle run."""
    wls = [W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33)), W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45)),
           W.small_wedge_beam(NeoHookeanMaterial(5e4, 0.45)), W.small_pyramid_beam(LinearMaterial(2e4, 0.3, True))]
    steps = 5
    pack = FemPack([wl.model() for wl in wls], precision=L.PREC_FP64)
    pack.backwardEuler(wls[0].h, steps, tol=1e-13)
    for wl, (xg, _) in zip(wls, pack.getStates()):
        om = oracle_model(oracle, wl)
        x, v = wl.rest.copy(), np.zeros_like(wl.rest)
        for _ in range(steps):
            st, _, _ = om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=1, tol=1e-14)
            assert st == 0
        assert rel_err(xg, x) <= 1e-8, rel_err(xg, x)


def test_mixed_mesh_rejects_bad_input(b200, oracle):
    """An unknown element type or a connectivity index out of range is refused
    (ERR_INVALID_ARG at b200fem_set_mesh_mixed or at the build)."""
    import ctypes
    xyz, types, conn, fixed = _mesh(oracle, HEX_WEDGE_PYR)
    lib = L.lib()
    h = lib.b200fem_create(ctypes.byref(L.Config(0, L.PREC_FP64)))
    assert h
    try:
        rest = np.ascontiguousarray(xyz.reshape(-1))
        bad = types.copy()
        bad[3] = 42
        assert lib.b200fem_set_mesh_mixed(h, xyz.shape[0], L.dptr(rest), types.size, L.iptr(bad), L.iptr(conn),
                                          L.iptr(fixed)) == L.ERR_INVALID_ARG
        c2 = conn.copy()
        c2[7] = xyz.shape[0] + 5
        assert lib.b200fem_set_mesh_mixed(h, xyz.shape[0], L.dptr(rest), types.size, L.iptr(types), L.iptr(c2),
                                          L.iptr(fixed)) == L.OK
        prm = np.zeros(8)
        prm[:2] = (5e4, 0.45)
        assert lib.b200fem_set_material(h, L.MAT_NEOHOOKEAN, L.dptr(prm), 1000.0, L.INCOMP_AUTO) == L.OK
        assert lib.b200fem_build(h) == L.ERR_INVALID_ARG
        assert b"out of range" in lib.b200fem_last_error(h)
    finally:
        lib.b200fem_destroy(h)
