"""Parity at the benchmark workloads' full sizes and step counts.

* NeoHookean hex beam, 40x10x10 hexes (14,520 DOF): all 200 BackwardEuler
  steps against the oracle (Jacobi-PCG to 1e-14), the engine at the
  workload's PCG tolerance (1e-10) and at 1e-13.
* MooneyRivlin tet block, 60x30x30 cells (270,000 tets; AUTO resolves to
  NODAL incompressibility, FemModel3d.java:462-481): the 2-ring block
  pattern (3,935,980 blocks), scalar CRS indices and slot maps bit-exact;
  3 FP64 steps against the oracle; 50 mixed-precision steps against 50 FP64
  steps of the engine.
* The 256-beam pack (uneven NeoHookean tet beams) in FP64, 20 steps: a
  sample of its models against the oracle stepping each model alone; and
  the largest model of the served distribution (120x8x8 cells, 38,400 tets)
  against the oracle.

Bars: positions <= 1e-8 relative to the oracle's (the library's parity bar);
displacements (x - rest) relative to the oracle's displacements as stated
per test; mixed precision <= 1e-6 relative position error against FP64.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import FemPack, MechSystemSolver, NeoHookeanMaterial

from helpers import oracle_model, rel_err

pytestmark = pytest.mark.gpu

POS_TOL = 1e-8


def _oracle_run(om, wl, steps, tol=1e-14, x=None, v=None):
    x = wl.rest.copy() if x is None else x
    v = np.zeros_like(x) if v is None else v
    fext = wl.fext if wl.traction is not None else None
    for _ in range(steps):
        st, it, rr = om.be_step(wl.h, x, v, alpha=wl.mass_damping, beta=wl.stiffness_damping,
                                gravity=wl.gravity, fext=fext, solver=0, tol=tol)
        assert st == 0, (st, it, rr)
    return x, v


def _gpu_run(wl, steps, tol, precision=L.PREC_FP64):
    m = wl.model(precision=precision)
    ms = MechSystemSolver(m, tol=tol, max_iter=20000)
    ms.backwardEuler(wl.h, steps)
    x, v = m.getState()
    rr = ms.stats.rel_residual
    m._invalidate()
    return x, v, rr


@pytest.fixture(scope="module")
def hex_beam_oracle(b200, oracle):
    wl = W.neohookean_hex_beam()
    wl.build_mesh()
    om = oracle_model(oracle, wl)
    x, v = _oracle_run(om, wl, wl.steps)
    return wl, x, v


def test_hex_beam_200_steps_at_workload_tolerance(hex_beam_oracle):
    """The whole 200-step run at PCG 1e-10 (the workload's tolerance)."""
    wl, x, v = hex_beam_oracle
    xg, vg, rr = _gpu_run(wl, wl.steps, wl.tol)
    pos = rel_err(xg, x)
    disp = rel_err(xg - wl.rest, x - wl.rest)
    print(f"hex beam 200 steps, PCG 1e-10: position {pos:.2e}, displacement {disp:.2e}")
    assert pos <= POS_TOL, pos
    # a 1e-10 relative residual per step leaves ~1e-8 of the velocity per
    # step; over 200 steps the displacement stays within 1e-6 of the oracle's
    assert disp <= 1e-6, disp
    assert rr <= 1.5 * wl.tol
    assert np.abs(x - wl.rest).max() > 1e-5  # the traction moves the tip


def test_hex_beam_200_steps_tight(hex_beam_oracle):
    """The same run with the engine's PCG at 1e-13: displacements within
    1e-7 of the oracle's."""
    wl, x, v = hex_beam_oracle
    xg, vg, rr = _gpu_run(wl, wl.steps, 1e-13)
    pos = rel_err(xg, x)
    disp = rel_err(xg - wl.rest, x - wl.rest)
    print(f"hex beam 200 steps, PCG 1e-13: position {pos:.2e}, displacement {disp:.2e}")
    assert pos <= POS_TOL, pos
    assert disp <= 1e-7, disp
    assert rel_err(vg, v) <= 1e-6


@pytest.fixture(scope="module")
def block(b200, oracle):
    wl = W.mooneyrivlin_tet_block()
    wl.build_mesh()
    om = oracle_model(oracle, wl)
    return wl, om


def test_block_pattern_bit_exact(block):
    """NODAL 2-ring pattern, solve indices, scalar CRS indices and slot maps
    of the full block, bit for bit."""
    wl, om = block
    assert wl.conn.shape == (270000, 4) and wl.rest.shape == (58621, 3)
    m = wl.model()
    assert m.getSoftIncompMethod() == L.INCOMP_NODAL == om.incomp
    rp, col = m.getBlockPattern()
    orp, ocol = om.pattern()
    assert col.size == 3935980
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(m.getSolveIndices(), om.solve_index())
    assert m.sizes()["n_active"] * 3 == 170190
    for part in (L.PART_FULL, L.PART_UPPER):
        ro, ci = m.getCRSIndices(part)
        oro, oci, osl = om.crs(part)
        assert np.array_equal(ro, oro) and np.array_equal(ci, oci)
        assert np.array_equal(m.createCrsBlockSlotMap(part), osl)
    assert rel_err(m.getNodeMasses(), om.masses()) <= 1e-14
    m._invalidate()


def test_block_fp64_steps_vs_oracle(block):
    """Three FP64 steps of the full block against the oracle's 1e-14 CG."""
    wl, om = block
    x, v = _oracle_run(om, wl, 3)
    xg, vg, rr = _gpu_run(wl, 3, 1e-12)
    pos = rel_err(xg, x)
    disp = rel_err(xg - wl.rest, x - wl.rest)
    print(f"block 3 FP64 steps: position {pos:.2e}, displacement {disp:.2e}")
    assert pos <= POS_TOL, pos
    assert disp <= 1e-6, disp
    assert rr <= 1.5e-12


def test_block_mixed_50_steps_vs_fp64(block):
    """The block's 50-step run in the mixed form (FP32 element tangents and
    SpMV, FP64 residual/dots/update) against the plain FP64 form, both at
    PCG 1e-10: position error within 1e-6 (the mixed form's bound)."""
    wl, _ = block
    x64, _, _ = _gpu_run(wl, wl.steps, wl.tol)
    xmx, _, _ = _gpu_run(wl, wl.steps, wl.tol, precision=L.PREC_MIXED)
    pos = rel_err(xmx, x64)
    disp = rel_err(xmx - wl.rest, x64 - wl.rest)
    print(f"block 50 steps mixed vs FP64: position {pos:.2e}, displacement {disp:.2e}")
    assert pos <= 1e-6, pos
    assert disp <= 1e-4, disp
    assert np.abs(x64 - wl.rest).max() > 1e-4  # gravity sags the block


def test_pack_256_fp64_vs_oracle(b200, oracle):
    """All 256 beams in one FP64 pack, 20 steps; every 16th model (and the
    largest) against the oracle stepping it alone."""
    bs = W.batched_beams()
    for b in bs:
        b.build_mesh()
    pack = FemPack([b.model() for b in bs], precision=L.PREC_FP64)
    pack.backwardEuler(bs[0].h, bs[0].steps, tol=1e-12)
    xs = [x for x, _ in pack.getStates()]
    pack.close()
    sizes = [b.conn.shape[0] for b in bs]
    sample = sorted(set(range(0, len(bs), 16)) | {int(np.argmax(sizes))})
    worst = (0.0, 0.0)
    for i in sample:
        b = bs[i]
        x, _ = _oracle_run(oracle_model(oracle, b), b, b.steps)
        pos = rel_err(xs[i], x)
        disp = rel_err(xs[i] - b.rest, x - b.rest)
        worst = (max(worst[0], pos), max(worst[1], disp))
        assert pos <= POS_TOL, (i, b.name, pos)
        assert disp <= 1e-5, (i, b.name, disp)
    print(f"256-beam FP64 pack, {len(sample)} models vs oracle: position {worst[0]:.2e}, "
          f"displacement {worst[1]:.2e}")


def test_largest_served_model_vs_oracle(b200, oracle):
    """The largest beam of the served distribution (n = 120, m = 8: 38,400
    tets), 10 steps (one request) in FP64 against the oracle."""
    wl = W.Workload("beam_120x8x8", L.ELEM_TET, (120, 8, 8), (6.0, 0.4, 0.4), 0.05, 4242,
                    NeoHookeanMaterial(2e5, 0.45), 1000.0, "xmin", (0.0, 0.0, -9.81), 0.01, 10, tol=1e-10)
    wl.build_mesh()
    assert wl.conn.shape[0] == 38400
    x, v = _oracle_run(oracle_model(oracle, wl), wl, wl.steps)
    xg, vg, rr = _gpu_run(wl, wl.steps, 1e-12)
    pos = rel_err(xg, x)
    disp = rel_err(xg - wl.rest, x - wl.rest)
    print(f"120x8x8 beam 10 steps: position {pos:.2e}, displacement {disp:.2e}")
    assert pos <= POS_TOL, pos
    assert disp <= 1e-6, disp
