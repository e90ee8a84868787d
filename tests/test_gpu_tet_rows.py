"""The node-row assembly of tetrahedral packs (B200FEM_OPT_TET_ASSEMBLY 0,
the default) against the element kernel + block gather (option 1): the
node-row kernel repeats the element path's arithmetic expression for
expression and sums in the same orders, so the BackwardEuler steps agree to
rounding (the two kernels are compiled apart, and the compiler may fuse a
different product of an expression into an FMA: NeoHookean steps differ in
the last bit, StVenantKirchhoff and MooneyRivlin ones do not) -- bars 1e-13
relative on positions and 1e-11 on velocities (a last-bit change of S and b
moves the PCG's iterates by round-off amplified by the condition number;
measured 2e-16 and 2e-14), same PCG iterations -- and against the
oracle where the element path has no counterpart run (a node with 48
incident tets, which takes the 64-lane tasks).
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (FemPack, LinearMaterial, MechSystemSolver, MooneyRivlinMaterial,
                                          NeoHookeanMaterial, StVenantKirchoffMaterial)

from helpers import oracle_model, rel_err

pytestmark = pytest.mark.gpu

AGREE_X, AGREE_V = 1e-13, 1e-11


def _agree(s0, s1):
    (x0, v0), (x1, v1) = s0, s1
    return rel_err(x0, x1) <= AGREE_X and rel_err(v0, v1) <= AGREE_V


def _model(wl, path, precision=L.PREC_FP64, incomp=None):
    m = wl.model(precision=precision)
    # (the element path with the NODAL solve matrix assembled, as the
    # node-row path builds it: the factored form agrees only to rounding)
    m.options = {L.OPT_TET_ASSEMBLY: path, L.OPT_NODAL_FACTORED: 1}
    if incomp is not None:
        m.setSoftIncompMethod(incomp)
    return m


def _path_in_force(eng):
    import ctypes
    v = ctypes.c_int()
    eng.call("b200fem_get_option", L.OPT_TET_ASSEMBLY, ctypes.byref(v))
    return v.value


CASES = {
    "neohookean": (lambda: W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), cells=(6, 3, 3)), None),
    "stvk": (lambda: W.small_tet_beam(StVenantKirchoffMaterial(5e4, 0.3), cells=(6, 3, 3)), None),
    "mooneyrivlin_nodal": (lambda: W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5),
                                                    cells=(6, 3, 3)), L.INCOMP_NODAL),
    "mooneyrivlin_element": (lambda: W.small_tet_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370),
                                                      cells=(6, 3, 3)), L.INCOMP_ELEMENT),
    "mooneyrivlin_off": (lambda: W.small_tet_beam(MooneyRivlinMaterial(1e4, 2e3, 0, 0, 0, 1e5), cells=(6, 3, 3)),
                         L.INCOMP_OFF),
}


@pytest.mark.parametrize("precision", [L.PREC_FP64, L.PREC_MIXED])
@pytest.mark.parametrize("name", list(CASES))
def test_node_rows_equal_element_path(b200, name, precision):
    make, incomp = CASES[name]
    wl = make()
    wl.build_mesh()
    out = []
    for path in (0, 1):
        m = _model(wl, path, precision, incomp)
        ms = MechSystemSolver(m, tol=1e-12, max_iter=20000)
        ms.backwardEuler(wl.h, 6)
        assert _path_in_force(m.engine()) == path
        out.append((m.getState(), ms.stats.iterations))
        m._invalidate()
    s0, it0 = out[0]
    s1, it1 = out[1]
    assert it0 == it1
    assert _agree(s0, s1), (name, rel_err(s0[0], s1[0]), rel_err(s0[1], s1[1]))


def test_linear_material_keeps_element_path(b200):
    wl = W.small_tet_beam(LinearMaterial(5e4, 0.33, True))
    wl.build_mesh()
    m = _model(wl, 0)
    m.engine()
    assert _path_in_force(m.engine()) == 1  # corotated linear tets: element path


def test_pack_of_mixed_materials_and_masks(b200):
    """A pack of NeoHookean, StVenantKirchhoff and MooneyRivlin (NODAL) tet
    beams of different sizes; part of the models masked out of some steps
    (continuous batching)."""
    wls = [W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), cells=(5, 2, 2), seed=1),
           W.small_tet_beam(NeoHookeanMaterial(2e5, 0.45), cells=(8, 3, 3), seed=2),
           W.small_tet_beam(StVenantKirchoffMaterial(5e4, 0.3), cells=(4, 2, 2), seed=3),
           W.small_tet_beam(MooneyRivlinMaterial(1000.0, 500.0, 0, 0, 0, 1e5), cells=(6, 3, 3), seed=4),
           W.small_tet_beam(NeoHookeanMaterial(1e4, 0.3), cells=(7, 2, 2), seed=5)]
    for w in wls:
        w.build_mesh()
    wls[3].incomp = L.INCOMP_NODAL
    res = []
    for path in (0, 1):
        models = []
        for w in wls:
            m = w.model(precision=L.PREC_MIXED)
            if hasattr(w, "incomp"):
                m.setSoftIncompMethod(w.incomp)
            models.append(m)
        pack = FemPack(models, precision=L.PREC_MIXED,
                       options={L.OPT_TET_ASSEMBLY: path, L.OPT_NODAL_FACTORED: 1})
        pack.backwardEuler(wls[0].h, 2, tol=1e-12)
        pack.setActive([1, 0, 1, 0, 1])
        pack.backwardEuler(wls[0].h, 2, tol=1e-12)
        pack.setActive(None)
        pack.backwardEuler(wls[0].h, 2, tol=1e-12)
        assert pack.option(L.OPT_TET_ASSEMBLY) == path
        res.append(pack.getStates())
        pack.close()
    for s0, s1 in zip(*res):
        assert _agree(s0, s1)


def test_plane_constraints_on_node_rows(b200):
    """ConstrainedBackwardEuler: the node-row path projects the initial guess
    onto the constraint planes like the element path."""
    wl = W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), cells=(6, 2, 2))
    wl.build_mesh()
    free = np.nonzero(wl.fixed == 0)[0]
    tip = free[np.argsort(wl.rest[free, 0])[-3:]]
    nrm = np.tile([0.0, 0.3, 1.0], (tip.size, 1))
    off = (nrm * wl.rest[tip]).sum(axis=1)
    out = []
    for path in (0, 1):
        m = _model(wl, path)
        m.setPlaneConstraints(tip, nrm, off)
        ms = MechSystemSolver(m, tol=1e-12, integrator=L.INTEGRATOR_CONSTRAINED_BACKWARD_EULER)
        ms.backwardEuler(wl.h, 4)
        out.append(m.getState())
        m._invalidate()
    assert _agree(out[0], out[1])


def _fan_mesh():
    """Tets fanned around one centre node: the faces of a cube, each cut into
    2 x 2 squares of two triangles, joined to the centre (48 tets at the
    centre node: the 64-lane tasks)."""
    k = 2
    pts = {}
    tris = []

    def pid(p):
        key = tuple(np.round(p, 9))
        if key not in pts:
            pts[key] = len(pts) + 1
        return pts[key]

    for ax in range(3):
        for sgn in (-1.0, 1.0):
            u, v = [a for a in range(3) if a != ax]
            for i in range(k):
                for j in range(k):
                    def corner(di, dj):
                        p = np.zeros(3)
                        p[ax] = sgn
                        p[u] = -1 + 2 * (i + di) / k
                        p[v] = -1 + 2 * (j + dj) / k
                        return pid(p)
                    a, b, c, d = corner(0, 0), corner(1, 0), corner(1, 1), corner(0, 1)
                    tris += [(a, b, c), (a, c, d)]
    xyz = np.zeros((len(pts) + 1, 3))
    for key, i in pts.items():
        xyz[i] = key
    xyz *= 0.1
    conn = []
    for a, b, c in tris:
        t = [0, a, b, c]
        vol = np.linalg.det(np.array([xyz[t[1]] - xyz[t[0]], xyz[t[2]] - xyz[t[0]], xyz[t[3]] - xyz[t[0]]]))
        if vol < 0:
            t = [0, a, c, b]
        conn.append(t)
    return xyz, np.array(conn, dtype=np.int32)


def test_high_valence_node_vs_oracle(b200, oracle):
    xyz, conn = _fan_mesh()
    assert conn.shape[0] == 48 and np.all(np.bincount(conn.ravel())[0] == 48)
    fixed = (xyz[:, 2] <= -0.1 + 1e-9).astype(np.int32)
    wl = W.Workload("fan", L.ELEM_TET, (1, 1, 1), (0.2, 0.2, 0.2), 0.0, 0, NeoHookeanMaterial(5e4, 0.4), 1000.0,
                    "zmin", (0.0, 0.0, -9.81), 0.01, 5, tol=1e-13)
    wl.rest, wl.conn, wl.fixed, wl.fext = xyz, conn, fixed, np.zeros_like(xyz)
    states = []
    for path in (0, 1):
        m = _model(wl, path)
        ms = MechSystemSolver(m, tol=1e-13)
        ms.backwardEuler(wl.h, wl.steps)
        assert _path_in_force(m.engine()) == path
        states.append(m.getState())
        m._invalidate()
    assert _agree(states[0], states[1])
    om = oracle_model(oracle, wl)
    x = xyz.copy()
    v = np.zeros_like(x)
    for _ in range(wl.steps):
        st, _, _ = om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, solver=1)
        assert st == 0
    assert rel_err(states[0][0], x) <= 1e-8
    assert rel_err(states[0][0] - xyz, x - xyz) <= 1e-6
