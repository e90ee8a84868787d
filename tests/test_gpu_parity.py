"""Parity of the sm_100a engine (through the C ABI) with the CPU oracle.

Bars (stated here, checked below):
* pattern, CRS indices, slot map, scatter map, solve indices: bit-exact;
* nodal forces and stiffness blocks: max |gpu - oracle| <= 1e-10 * max |oracle|;
* positions after the stepped run: <= 1e-8 relative to the oracle's.
"""
import ctypes

import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (LinearMaterial, MechSystemSolver, MooneyRivlinMaterial,
                                          NeoHookeanMaterial, StVenantKirchoffMaterial)

from helpers import deformed, oracle_model, rel_err

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-10
POS_TOL = 1e-8


def _cases():
    return {
        "linear_corotated_tet": W.linear_tet_beam(),
        "linear_plain_tet": W.small_tet_beam(LinearMaterial(5e4, 0.33, False)),
        "linear_corotated_hex": W.small_hex_beam(LinearMaterial(2e4, 0.3, True)),
        "neohookean_tet": W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33)),
        "neohookean_hex": W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45)),
        "stvk_tet": W.small_tet_beam(StVenantKirchoffMaterial(5e4, 0.3)),
        "stvk_hex": W.small_hex_beam(StVenantKirchoffMaterial(5e4, 0.3)),
        "mooneyrivlin_tet_off": W.small_tet_beam(MooneyRivlinMaterial(1e4, 2e3, 0, 0, 0, 1e5)),
        "mooneyrivlin_hex_full": W.small_hex_beam(MooneyRivlinMaterial(1037, 120, 30, 486, 20, 10370)),
        "mooneyrivlin_tet_nodal": W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5)),
        "mooneyrivlin_hex_nodal": W.small_hex_beam(MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370)),
        "mooneyrivlin_tet_nodal_log": W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5, 0.0, 1)),
        # ELEMENT soft incompressibility: AUTO picks it for the hex beam
        # (16 elements <= 36 active nodes); requested for the tet beam
        "mooneyrivlin_hex_element": W.small_hex_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        "mooneyrivlin_hex_element_log": W.small_hex_beam(MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370, 0.0, 1)),
        "mooneyrivlin_tet_element": W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5)),
        # wedges (6 points) and pyramids (5 points, unequal weights)
        "linear_corotated_wedge": W.small_wedge_beam(LinearMaterial(2e4, 0.3, True)),
        "linear_corotated_pyramid": W.small_pyramid_beam(LinearMaterial(2e4, 0.3, True)),
        "neohookean_wedge": W.small_wedge_beam(NeoHookeanMaterial(5e4, 0.45)),
        "neohookean_pyramid": W.small_pyramid_beam(NeoHookeanMaterial(5e4, 0.45)),
        "stvk_wedge": W.small_wedge_beam(StVenantKirchoffMaterial(5e4, 0.3)),
        "stvk_pyramid": W.small_pyramid_beam(StVenantKirchoffMaterial(5e4, 0.3)),
        "mooneyrivlin_wedge_nodal": W.small_wedge_beam(MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370)),
        "mooneyrivlin_pyramid_nodal": W.small_pyramid_beam(MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370)),
        "mooneyrivlin_wedge_element": W.small_wedge_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        "mooneyrivlin_pyramid_element_log": W.small_pyramid_beam(
            MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370, 0.0, 1)),
        # quadratic tets (10 nodes, 4 points; AUTO resolves to ELEMENT)
        "linear_corotated_quadtet": W.small_quadtet_beam(LinearMaterial(2e4, 0.3, True)),
        "neohookean_quadtet": W.small_quadtet_beam(NeoHookeanMaterial(5e4, 0.45)),
        "stvk_quadtet": W.small_quadtet_beam(StVenantKirchoffMaterial(5e4, 0.3)),
        "mooneyrivlin_quadtet_element": W.small_quadtet_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        # quadratic hexes (20 nodes, 14 points; compressible forms)
        "linear_corotated_quadhex": W.small_quadhex_beam(LinearMaterial(2e4, 0.3, True)),
        "neohookean_quadhex": W.small_quadhex_beam(NeoHookeanMaterial(5e4, 0.45)),
        "stvk_quadhex": W.small_quadhex_beam(StVenantKirchoffMaterial(5e4, 0.3)),
        "mooneyrivlin_quadhex_off": W.small_quadhex_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        # ELEMENT with several pressure values (AUTO resolves to it): quadratic
        # hexes 4, quadratic wedges 2; QUADRATIC and LOGARITHMIC potentials
        "mooneyrivlin_quadhex_element": W.small_quadhex_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        "mooneyrivlin_quadhex_element_log": W.small_quadhex_beam(
            MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370, 0.0, 1)),
        "mooneyrivlin_quadwedge_element": W.small_quadwedge_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        "mooneyrivlin_quadwedge_element_log": W.small_quadwedge_beam(
            MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370, 0.0, 1)),
        # quadratic wedges (15 nodes, 9 points) and pyramids (13 nodes, 5 points)
        "linear_corotated_quadwedge": W.small_quadwedge_beam(LinearMaterial(2e4, 0.3, True)),
        "neohookean_quadwedge": W.small_quadwedge_beam(NeoHookeanMaterial(5e4, 0.45)),
        "linear_corotated_quadpyramid": W.small_quadpyramid_beam(LinearMaterial(2e4, 0.3, True)),
        "stvk_quadpyramid": W.small_quadpyramid_beam(StVenantKirchoffMaterial(5e4, 0.3)),
        "mooneyrivlin_quadpyramid_element": W.small_quadpyramid_beam(
            MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
    }


def _incomp_off(wl):
    wl.incomp = L.INCOMP_OFF
    return wl


@pytest.fixture(scope="module")
def cases(b200):
    cs = _cases()
    for k in ("mooneyrivlin_tet_off", "mooneyrivlin_hex_full", "mooneyrivlin_quadhex_off"):
        _incomp_off(cs[k])
    # more hexes than active nodes is needed for AUTO -> NODAL; request it
    cs["mooneyrivlin_hex_nodal"].incomp = L.INCOMP_NODAL
    cs["mooneyrivlin_tet_element"].incomp = L.INCOMP_ELEMENT
    for k in ("mooneyrivlin_wedge_nodal", "mooneyrivlin_pyramid_nodal"):
        cs[k].incomp = L.INCOMP_NODAL
    for k in ("mooneyrivlin_wedge_element", "mooneyrivlin_pyramid_element_log"):
        cs[k].incomp = L.INCOMP_ELEMENT
    return cs


def _gpu_model(wl):
    m = wl.model()
    if hasattr(wl, "incomp"):
        m.setSoftIncompMethod(wl.incomp)
    return m


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_pattern_bit_exact(name, cases, oracle):
    wl = cases[name]
    m = _gpu_model(wl)
    om = oracle_model(oracle, wl)
    rp, col = m.getBlockPattern()
    orp, ocol = om.pattern()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(m.getSolveIndices(), om.solve_index())
    for part in (L.PART_FULL, L.PART_UPPER):
        ro, ci = m.getCRSIndices(part)
        oro, oci, osl = om.crs(part)
        assert np.array_equal(ro, oro) and np.array_equal(ci, oci)
        assert np.array_equal(m.createCrsBlockSlotMap(part), osl)
    # scatter map: element pair (i, j) -> block of (sidx_i, sidx_j)
    smap = m.getScatterMap()
    sidx = om.solve_index()
    nen = wl.conn.shape[1]
    ref = np.full_like(smap, -1)
    for e in range(wl.conn.shape[0]):
        for a in range(nen):
            for b in range(nen):
                ra, rb = sidx[wl.conn[e, a]], sidx[wl.conn[e, b]]
                if ra >= 0 and rb >= 0:
                    k = orp[ra] + np.searchsorted(ocol[orp[ra]:orp[ra + 1]], rb)
                    ref[e, a, b] = k
    assert np.array_equal(smap, ref)
    assert rel_err(m.getNodeMasses(), om.masses()) <= 1e-14


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_update_stress_stiffness(name, cases, oracle):
    wl = cases[name]
    m = _gpu_model(wl)
    om = oracle_model(oracle, wl)
    for seed, x in ((0, wl.rest), (1, deformed(wl.rest, seed=5))):
        f, K, crs = m.updateStressAndStiffness(x, want_crs=True)
        of, oK, _ = om.update_stress_stiffness(x)
        if seed == 0:
            # at rest the force is round-off of the cancelling terms
            assert np.abs(f).max() <= 1e-9 * np.abs(oK).max() * np.ptp(wl.rest)
        else:
            assert rel_err(f, of) <= FORCE_TOL, (name, seed, rel_err(f, of))
        assert rel_err(K, oK) <= FORCE_TOL, (name, seed, rel_err(K, oK))
        # full-partition CRS export lands every block entry in its slot
        slots = m.createCrsBlockSlotMap(L.PART_FULL)
        assert np.array_equal(crs[slots], K.reshape(-1))


def _run_pair(wl, oracle, steps, solver, tol_gpu):
    m = _gpu_model(wl)
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    fext = wl.fext if wl.traction is not None else None
    for _ in range(steps):
        st, it, rr = om.be_step(wl.h, x, v, alpha=wl.mass_damping, beta=wl.stiffness_damping,
                                gravity=wl.gravity, fext=fext, solver=solver, tol=1e-14)
        assert st == 0
    ms = MechSystemSolver(m, tol=tol_gpu, max_iter=20000)
    ms.backwardEuler(wl.h, steps)
    xg, vg = m.getState()
    return xg, vg, x, v, ms


def test_backward_euler_linear_tet_beam(cases, oracle):
    """Corotated linear tet beam, 100 BackwardEuler steps (dense oracle solve)."""
    wl = cases["linear_corotated_tet"]
    xg, vg, x, v, ms = _run_pair(wl, oracle, wl.steps, 1, 1e-13)
    assert rel_err(xg, x) <= POS_TOL, rel_err(xg, x)
    assert np.abs(xg - x).max() <= POS_TOL * np.abs(x).max()
    assert x[:, 2].min() < -0.05  # the beam sags (FemModel3dTest.runCorotatedBeamStep)


@pytest.mark.parametrize("name", ["neohookean_tet", "neohookean_hex", "stvk_tet", "stvk_hex", "mooneyrivlin_tet_off",
                                  "linear_plain_tet", "linear_corotated_hex", "mooneyrivlin_hex_full",
                                  "mooneyrivlin_tet_nodal", "mooneyrivlin_hex_nodal",
                                  "mooneyrivlin_tet_nodal_log", "mooneyrivlin_hex_element",
                                  "mooneyrivlin_hex_element_log", "mooneyrivlin_tet_element",
                                  "linear_corotated_wedge", "linear_corotated_pyramid", "neohookean_wedge",
                                  "neohookean_pyramid", "stvk_wedge", "stvk_pyramid", "mooneyrivlin_wedge_nodal",
                                  "mooneyrivlin_pyramid_nodal", "mooneyrivlin_wedge_element",
                                  "mooneyrivlin_pyramid_element_log", "linear_corotated_quadtet",
                                  "neohookean_quadtet", "stvk_quadtet", "mooneyrivlin_quadtet_element",
                                  "linear_corotated_quadhex", "neohookean_quadhex", "stvk_quadhex",
                                  "mooneyrivlin_quadhex_off", "mooneyrivlin_quadhex_element",
                                  "mooneyrivlin_quadhex_element_log", "mooneyrivlin_quadwedge_element",
                                  "mooneyrivlin_quadwedge_element_log", "linear_corotated_quadwedge",
                                  "neohookean_quadwedge", "linear_corotated_quadpyramid", "stvk_quadpyramid",
                                  "mooneyrivlin_quadpyramid_element"])
def test_backward_euler_small(name, cases, oracle):
    wl = cases[name]
    xg, vg, x, v, ms = _run_pair(wl, oracle, wl.steps, 1, 1e-13)
    assert rel_err(xg, x) <= POS_TOL, (name, rel_err(xg, x))
    assert rel_err(vg, v) <= 1e-6, (name, rel_err(vg, v))


def test_backward_euler_neohookean_hex_beam_steps(oracle):
    """The 40x10x10 NeoHookean hex beam with traction: 5 steps against the
    oracle's tight CG, and PCG at the workload's 1e-10 tolerance."""
    wl = W.neohookean_hex_beam()
    wl.build_mesh()
    xg, vg, x, v, ms = _run_pair(wl, oracle, 5, 0, wl.tol)
    assert rel_err(xg - wl.rest, x - wl.rest) <= 1e-6
    assert rel_err(xg, x) <= POS_TOL
    assert ms.stats.rel_residual <= 1.5 * wl.tol


def test_deterministic(cases):
    wl = cases["neohookean_tet"]
    out = []
    for _ in range(2):
        m = _gpu_model(wl)
        MechSystemSolver(m, tol=1e-12).backwardEuler(wl.h, 5)
        out.append(m.getState())
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_no_convergence_reports_status(cases):
    wl = cases["neohookean_hex"]
    m = _gpu_model(wl)
    ms = MechSystemSolver(m, tol=1e-14, max_iter=1)
    with pytest.raises(L.B200FemError) as ei:
        ms.backwardEuler(wl.h, 1)
    assert ei.value.status == L.ERR_NO_CONVERGE


def test_spmv_and_pcg_solve(cases):
    wl = cases["neohookean_hex"]
    m = _gpu_model(wl)
    ms = MechSystemSolver(m, tol=1e-12)
    ms.backwardEuler(wl.h, 2)
    n = m.sizes()["n_active"] * 3
    rng = np.random.default_rng(0)
    xt = rng.standard_normal(n)
    b = ms.spmv(xt)
    x, st = ms.pcg(b, tol=1e-13, max_iter=5000)
    assert rel_err(x, xt) <= 1e-9
    assert st.rel_residual <= 1e-12


def test_nodal_resolution_and_pattern(cases, oracle):
    """AUTO resolves to NODAL for the MooneyRivlin tet beam (more elements than
    active nodes) and the 2-ring pattern is bit-exact."""
    wl = cases["mooneyrivlin_tet_nodal"]
    m = _gpu_model(wl)
    om = oracle_model(oracle, wl)
    assert m.getSoftIncompMethod() == L.INCOMP_NODAL == om.incomp
    rp, col = m.getBlockPattern()
    orp, ocol = om.pattern()
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    direct = W.small_tet_beam(NeoHookeanMaterial(1e4, 0.3)).model()
    assert col.size > direct.sizes()["nnzb"]  # the 2-ring adds blocks


def test_mooneyrivlin_block_nodal_steps(oracle):
    """The MooneyRivlin block workload's material and NODAL incompressibility
    on a 12x6x6 block (z-min fixed, gravity): 5 steps against the oracle."""
    wl = W.mooneyrivlin_tet_block()
    wl.cells = (12, 6, 6)
    wl.build_mesh()
    xg, vg, x, v, ms = _run_pair(wl, oracle, 5, 0, 1e-12)
    assert rel_err(xg, x) <= POS_TOL
    assert rel_err(xg - wl.rest, x - wl.rest) <= 1e-6


@pytest.mark.parametrize("variant", [1, 2])
def test_pcg_variants_agree_with_oracle(cases, oracle, variant):
    """Classic (two barriers) and pipelined-only PCG both reach the oracle."""
    wl = cases["neohookean_hex"]
    m = _gpu_model(wl)
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(wl.steps):
        om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=1)
    MechSystemSolver(m, tol=1e-13, max_iter=20000, pcg_variant=variant).backwardEuler(wl.h, wl.steps)
    xg, _ = m.getState()
    assert rel_err(xg, x) <= POS_TOL


def test_stiff_beam_reaches_tight_tolerance(b200, oracle):
    """A stiff beam (E = 9.6e5 Pa at h = 0.01, Jacobi-PCG needs thousands of
    iterations) at 1e-12: the auto variant falls back to classic PCG when the
    pipelined recurrences stall, and matches the dense oracle."""
    wl = W.batched_beams(count=6, seed=5)[4]
    wl.cells = (12, wl.cells[1], wl.cells[2])
    wl.widths = (12 * 0.05, wl.widths[1], wl.widths[2])
    wl.build_mesh()
    m = _gpu_model(wl)
    ms = MechSystemSolver(m, tol=1e-12, max_iter=20000)
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(3):
        om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=1)
        ms.backwardEuler(wl.h, 1)
        assert ms.stats.rel_residual <= 1e-12
    xg, _ = m.getState()
    assert rel_err(xg, x) <= POS_TOL


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("name", ["neohookean_tet", "neohookean_hex", "mooneyrivlin_tet_off",
                                  "mooneyrivlin_hex_full"])
def test_fused_assembly_matches_gather(name, precision, cases):
    """The fused row-chunk assembly forms the same solve matrix as the element
    kernel + block gather (same sums in the same order): stepped positions and
    the inverted-element statistics agree."""
    wl = cases[name]
    out = []
    for fused in (1, 0):
        m = _gpu_model(wl)
        m.precision = precision
        m.options = {L.OPT_FUSED_ASSEMBLY: fused}
        ms = MechSystemSolver(m, tol=1e-13)
        ms.backwardEuler(wl.h, 4)
        out.append((m.getState()[0], ms.stats.num_inverted, ms.stats.min_detJ))
        o = ctypes.c_int()
        m.engine().call("b200fem_get_option", L.OPT_FUSED_ASSEMBLY, ctypes.byref(o))
        assert o.value == fused  # after the build: 1 when the fused path is in force
        m._invalidate()
    (xa, ia, da), (xb, ib, db) = out
    assert rel_err(xa, xb) <= (1e-11 if precision == L.PREC_FP64 else 1e-7), rel_err(xa, xb)
    assert ia == ib == 0
    assert abs(da - db) <= 1e-5 * abs(db)


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("name", ["neohookean_tet", "stvk_tet", "mooneyrivlin_tet_off", "mooneyrivlin_tet_nodal",
                                  "mooneyrivlin_tet_element"])
def test_tet_kernels_agree(name, precision, cases):
    """The one-thread-per-tetrahedron kernel and the shared-memory staged
    kernel give the same steps (same formulas; the former keeps kinematics
    and stress in FP64 in both forms)."""
    wl = cases[name]
    xs = []
    for tile in (0, 1):
        m = _gpu_model(wl)
        m.precision = precision
        m.options = {L.OPT_ELEM_TILE: tile}
        ms = MechSystemSolver(m, tol=1e-13)
        ms.backwardEuler(wl.h, 4)
        xs.append(m.getState()[0])
        assert ms.stats.num_inverted == 0
        m._invalidate()
    assert rel_err(xs[0], xs[1]) <= (1e-11 if precision == L.PREC_FP64 else 1e-6), rel_err(xs[0], xs[1])


@pytest.mark.parametrize("maker", [W.small_quadhex_beam, W.small_quadwedge_beam])
def test_multi_pressure_resolution(b200, oracle, maker):
    """Quadratic hexes and wedges: AUTO and NODAL resolve to ELEMENT (their
    points do not map to nodes, FemModel3d.java:462-481), as in the oracle."""
    wl = maker(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)).build_mesh()
    for req in (L.INCOMP_AUTO, L.INCOMP_NODAL):
        wl.incomp = req
        m = _gpu_model(wl)
        assert m.getSoftIncompMethod() == L.INCOMP_ELEMENT == oracle_model(oracle, wl).incomp
        m._invalidate()
