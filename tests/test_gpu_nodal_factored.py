"""The factored NODAL solve matrix (B200FEM_OPT_NODAL_FACTORED 2): the
direct-neighbour blocks assembled, the dilational term (h^2 + h beta)
sum_n kp_n d_n d_n^T (FemModel3d.computeNodalIncompressibility,
FemModel3d.java:2632-2669) applied from the divBlk rows inside every SpMV of
the PCG.  The operator equals the assembled 2-ring matrix (option 1) to
rounding, so BackwardEuler steps agree with the oracle at the bars of the
assembled path (positions after 10 steps 1e-8 relative) and with the
assembled path itself to the PCG tolerance; b200fem_spmv applies the same
operator (1e-12 of the assembled result).
"""
import ctypes

import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (FemModel3d, FemPack, MechSystemSolver, MooneyRivlinMaterial,
                                          NeoHookeanMaterial)

from helpers import oracle_model, rel_err

pytestmark = pytest.mark.gpu

MR = MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5)
MR_LOG = MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5, 0.0, 1)


def _option(m, key):
    v = ctypes.c_int()
    m.engine().call("b200fem_get_option", key, ctypes.byref(v))
    return v.value


def _grid_model(oracle, etype, mat, cells=(6, 3, 3), types=None, precision=L.PREC_FP64, factored=2, beta=0.0):
    if types is not None:
        xyz, t, conn = oracle.mixed_grid((1.2, 0.4, 0.4), cells, jitter=0.03, seed=4, kinds=types)
        etype = t
    else:
        xyz, conn = oracle.grid(etype, (1.2, 0.4, 0.4), cells, jitter=0.03, seed=6)
    fixed = (xyz[:, 0] <= -0.6 + 1e-9).astype(np.int32)
    m = FemModel3d()
    m.setMesh(etype, xyz, conn, fixed)
    m.setMaterial(mat)
    m.setDensity(1000.0)
    m.setPrecision(precision)
    m.setSoftIncompMethod(L.INCOMP_NODAL)
    m.setGravity(0, 0, -9.8)
    m.setStiffnessDamping(beta)
    m.options = {L.OPT_NODAL_FACTORED: factored}
    om = oracle.OracleModel(etype, xyz, conn, fixed, mat.kind, mat.params(), 1000.0, L.INCOMP_NODAL)
    return m, om, xyz


CASES = {
    "tet": (L.ELEM_TET, MR, None),
    "tet_log": (L.ELEM_TET, MR_LOG, None),
    "hex": (L.ELEM_HEX, MR, None),
    "tet_hex_mixed": (None, MR, (L.ELEM_TET, L.ELEM_HEX, L.ELEM_TET)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_factored_steps_match_oracle(name, b200, oracle):
    etype, mat, types = CASES[name]
    m, om, xyz = _grid_model(oracle, etype, mat, types=types)
    assert om.incomp == L.INCOMP_NODAL
    h, steps = 0.01, 10
    MechSystemSolver(m, tol=1e-13, max_iter=20000).backwardEuler(h, steps)
    assert _option(m, L.OPT_NODAL_FACTORED) == 2
    x, v = xyz.copy(), np.zeros_like(xyz)
    for _ in range(steps):
        st, _, _ = om.be_step(h, x, v, alpha=2.0, gravity=(0, 0, -9.8), solver=1, tol=1e-14)
        assert st == 0
    xg, _ = m.getState()
    assert rel_err(xg, x) <= 1e-8, rel_err(xg, x)
    assert (x - xyz)[:, 2].min() < -1e-4


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("beta", [0.0, 0.01])
def test_factored_equals_assembled(precision, beta, b200, oracle):
    """Both forms of the solve matrix step the same (stiffness damping
    included: its h beta scale is part of the factored coefficient), and the
    standalone SpMV of the last step's matrix agrees."""
    states, ys = [], []
    for factored in (2, 1):
        m, _, xyz = _grid_model(oracle, L.ELEM_TET, MR, precision=precision, factored=factored, beta=beta)
        ms = MechSystemSolver(m, tol=1e-12, max_iter=20000)
        ms.backwardEuler(0.01, 5)
        assert _option(m, L.OPT_NODAL_FACTORED) == factored
        states.append(m.getState()[0])
        n = m.sizes()["n_active"]
        vec = np.random.default_rng(3).standard_normal(3 * n)
        ys.append(ms.spmv(vec))
    tol = 1e-9 if precision == L.PREC_FP64 else 1e-5
    assert rel_err(states[0], states[1]) <= tol, rel_err(states[0], states[1])
    assert rel_err(ys[0], ys[1]) <= (1e-12 if precision == L.PREC_FP64 else 1e-5), rel_err(ys[0], ys[1])


def test_factored_pcg_solve_and_stale_after_update(b200, oracle):
    """b200fem_pcg_solve runs on the factored matrix of the last step (its
    solution satisfies the assembled matrix); after
    b200fem_update_stress_stiffness that matrix is stale and spmv reports
    ERR_STATE until the next step."""
    m, _, xyz = _grid_model(oracle, L.ELEM_HEX, MR, factored=2)
    ref, _, _ = _grid_model(oracle, L.ELEM_HEX, MR, factored=1)
    for mm in (m, ref):
        MechSystemSolver(mm, tol=1e-12).backwardEuler(0.01, 3)
    n = m.sizes()["n_active"]
    b = np.random.default_rng(5).standard_normal(3 * n)
    x, _ = MechSystemSolver(m, tol=1e-12).pcg(b, tol=1e-12)
    r = MechSystemSolver(ref, tol=1e-12).spmv(x) - b
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(b)
    m.updateStressAndStiffness(xyz)
    y = np.zeros(3 * n)
    xx = np.ascontiguousarray(b)
    assert L.lib().b200fem_spmv(m.engine().h, L.dptr(xx), L.dptr(y)) == L.ERR_STATE
    MechSystemSolver(m, tol=1e-12).backwardEuler(0.01, 1)
    MechSystemSolver(m, tol=1e-12).spmv(b)


def test_factored_pack_with_plain_models(b200, oracle):
    """A pack of NODAL and non-NODAL models: the NODAL rows take the
    dilational term, the others none; each model matches its own oracle run."""
    wls = [W.small_tet_beam(MR, cells=(6, 3, 3)), W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33)),
           W.small_hex_beam(MR)]
    models = []
    for wl in wls:
        wl.incomp = L.INCOMP_NODAL  # (read by oracle_model; OFF for the compressible material)
        mm = wl.model()
        mm.setSoftIncompMethod(L.INCOMP_NODAL)
        models.append(mm)
    steps = 5
    pack = FemPack(models, precision=L.PREC_FP64, options={L.OPT_NODAL_FACTORED: 2})
    pack.backwardEuler(wls[0].h, steps, tol=1e-13)
    assert pack.option(L.OPT_NODAL_FACTORED) == 2
    for wl, mm, (xg, _) in zip(wls, models, pack.getStates()):
        om = oracle_model(oracle, wl)
        x, v = wl.rest.copy(), np.zeros_like(wl.rest)
        for _ in range(steps):
            st, _, _ = om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=1, tol=1e-14)
            assert st == 0
        assert rel_err(xg, x) <= 1e-8, rel_err(xg, x)


def test_factored_pack_with_inactive_models(b200):
    """Continuous batching on a pack with NODAL models: steps with some
    models left out (b200fem_set_active_models) agree between the factored
    and the assembled solve matrix."""
    wls = [W.small_tet_beam(MR, cells=(6, 3, 3), seed=4), W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), seed=1),
           W.small_hex_beam(MR_LOG, seed=2), W.small_tet_beam(MR, cells=(5, 2, 2), seed=3)]
    res = []
    for factored in (2, 1):
        models = []
        for w in wls:
            m = w.model()
            m.setSoftIncompMethod(L.INCOMP_NODAL)
            models.append(m)
        pack = FemPack(models, precision=L.PREC_FP64, options={L.OPT_NODAL_FACTORED: factored})
        pack.backwardEuler(wls[0].h, 2, tol=1e-12)
        pack.setActive([0, 1, 1, 0])
        pack.backwardEuler(wls[0].h, 2, tol=1e-12)
        pack.setActive(None)
        pack.backwardEuler(wls[0].h, 2, tol=1e-12)
        assert pack.option(L.OPT_NODAL_FACTORED) == factored
        res.append(pack.getStates())
        pack.close()
    for (x0, _), (x1, _) in zip(*res):
        assert rel_err(x0, x1) <= 1e-9, rel_err(x0, x1)
