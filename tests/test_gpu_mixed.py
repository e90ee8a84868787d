"""Mixed-precision form (FP32 element kinematics, stress, tangent and stored
solve matrix; FP64 PCG vectors, dot products, residual and state update)
against the FP64 oracle.

Bars: stiffness blocks within 2e-6 of max|K| and positions after the stepped
runs within 1e-6 relative of the FP64 oracle (the stated target of the
mixed form); forces within 1e-5 of the force scale max|K|*|x - x_rest|.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (LinearMaterial, MechSystemSolver, MooneyRivlinMaterial,
                                          NeoHookeanMaterial)

from helpers import deformed, oracle_model, rel_err

pytestmark = pytest.mark.gpu


def _cases():
    return {
        "linear_corotated_tet": W.linear_tet_beam(),
        "neohookean_tet": W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33)),
        "neohookean_hex": W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45)),
        "mooneyrivlin_tet_nodal": W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5)),
        "neohookean_wedge": W.small_wedge_beam(NeoHookeanMaterial(5e4, 0.45)),
        "neohookean_pyramid": W.small_pyramid_beam(NeoHookeanMaterial(5e4, 0.45)),
        # AUTO: ELEMENT on the wedge beam (32 elements <= 36 active nodes),
        # NODAL on the pyramid beam (48 > 36)
        "mooneyrivlin_wedge_auto": W.small_wedge_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        "mooneyrivlin_pyramid_auto": W.small_pyramid_beam(MooneyRivlinMaterial(1037, 0, 0, 486, 0, 10370)),
        "neohookean_quadtet": W.small_quadtet_beam(NeoHookeanMaterial(5e4, 0.45)),
        "mooneyrivlin_quadtet_auto": W.small_quadtet_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        "neohookean_quadhex": W.small_quadhex_beam(NeoHookeanMaterial(5e4, 0.45)),
        "neohookean_quadwedge": W.small_quadwedge_beam(NeoHookeanMaterial(5e4, 0.45)),
        "mooneyrivlin_quadpyramid_auto": W.small_quadpyramid_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        # AUTO resolves to ELEMENT with four (quadratic hex) and two
        # (quadratic wedge) pressure values per element
        "mooneyrivlin_quadhex_auto": W.small_quadhex_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
        "mooneyrivlin_quadwedge_auto": W.small_quadwedge_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370)),
    }


@pytest.fixture(scope="module")
def cases(b200):
    return _cases()


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_mixed_update_stress_stiffness(name, cases, oracle):
    wl = cases[name]
    m = wl.model(precision=L.PREC_MIXED)
    om = oracle_model(oracle, wl)
    x = deformed(wl.rest, seed=5)
    f, K = m.updateStressAndStiffness(x)
    of, oK, _ = om.update_stress_stiffness(x)
    assert rel_err(K, oK) <= 2e-6, rel_err(K, oK)
    fscale = np.abs(oK).max() * np.abs(x - wl.rest).max()
    assert np.abs(f - of).max() <= 1e-5 * fscale, np.abs(f - of).max() / fscale


@pytest.mark.parametrize("name", list(_cases().keys()))
def test_mixed_backward_euler(name, cases, oracle):
    wl = cases[name]
    m = wl.model(precision=L.PREC_MIXED)
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(wl.steps):
        st, _, _ = om.be_step(wl.h, x, v, alpha=wl.mass_damping, beta=wl.stiffness_damping,
                              gravity=wl.gravity, fext=None, solver=1)
        assert st == 0
    ms = MechSystemSolver(m, tol=1e-12, max_iter=20000)
    ms.backwardEuler(wl.h, wl.steps)
    xg, _ = m.getState()
    err = rel_err(xg, x)
    assert err <= 1e-6, (name, err)


def test_mixed_mooneyrivlin_block_steps(oracle):
    """The MooneyRivlin block workload (NODAL) on a 12x6x6 block, 5 steps,
    mixed form against the FP64 oracle."""
    wl = W.mooneyrivlin_tet_block()
    wl.cells = (12, 6, 6)
    wl.build_mesh()
    m = wl.model(precision=L.PREC_MIXED)
    om = oracle_model(oracle, wl)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(5):
        om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=0, tol=1e-14)
    MechSystemSolver(m, tol=1e-12, max_iter=20000).backwardEuler(wl.h, 5)
    xg, _ = m.getState()
    assert rel_err(xg, x) <= 1e-6, rel_err(xg, x)


@pytest.mark.parametrize("name", ["neohookean_tet", "neohookean_hex"])
def test_refinement_recovers_fp64(name, cases):
    """Refinement sweeps against the FP64 residual bring the mixed form's
    positions to the plain FP64 result: the error falls by orders of
    magnitude and the stats report the sweeps."""
    wl = cases[name]
    steps = 6
    ref = wl.model(precision=L.PREC_FP64)
    MechSystemSolver(ref, tol=1e-12).backwardEuler(wl.h, steps)
    x64, _ = ref.getState()
    errs = {}
    for sweeps in (0, 2):
        m = wl.model(precision=L.PREC_MIXED)
        m.options = {L.OPT_REFINE: sweeps}
        ms = MechSystemSolver(m, tol=1e-12)
        ms.backwardEuler(wl.h, steps)
        assert ms.stats.refinements == sweeps
        x, _ = m.getState()
        errs[sweeps] = rel_err(x - wl.rest, x64 - wl.rest)
        m._invalidate()
    assert errs[2] <= 1e-9 and errs[2] <= 1e-2 * errs[0], errs


def test_refinement_in_a_pack_equals_alone(b200):
    """A refined pack (strided split, masked models) gives each active model
    its refined result alone and leaves the masked ones untouched."""
    from artisynth_core_b200.femmodel import FemPack
    bs = W.batched_beams(count=5, seed=6)
    for b in bs:
        b.cells = (min(b.cells[0], 8), b.cells[1], b.cells[2])
        b.widths = (b.cells[0] * 0.05, b.widths[1], b.widths[2])
        b.build_mesh()
    pack = FemPack([b.model() for b in bs], precision=L.PREC_MIXED,
                   options={L.OPT_REFINE: 2, L.OPT_PCG_SPLIT: L.SPLIT_STRIDED, L.OPT_PIECE_ROWS: 8})
    mask = np.array([1, 0, 1, 1, 0], dtype=np.int32)
    pack.setActive(mask)
    pack.backwardEuler(bs[0].h, 3, tol=1e-12)
    for i, (b, (x, v)) in enumerate(zip(bs, pack.getStates())):
        if not mask[i]:
            assert np.array_equal(x, b.rest) and not v.any()
            continue
        m = b.model(precision=L.PREC_MIXED)
        m.options = {L.OPT_REFINE: 2}
        MechSystemSolver(m, tol=1e-12).backwardEuler(b.h, 3)
        xa, _ = m.getState()
        assert rel_err(x, xa) <= 1e-9, (i, rel_err(x, xa))
