"""Host-side mirror of the reference interface for the FEM hot path.

Names follow ArtiSynth: ``FemFactory.createTetGrid/createHexGrid``,
``FemModel3d`` (setMaterial, setDensity, setMassDamping,
setStiffnessDamping, setGravity, updateStressAndStiffness, ...),
``LinearMaterial`` / ``NeoHookeanMaterial`` / ``MooneyRivlinMaterial`` and
``MechSystemSolver.backwardEuler``.  Every numerical operation is a call
into libb200fem.so (sm_100a kernels); this module only marshals arrays.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L


# ---------------------------------------------------------------- materials
@dataclass
class LinearMaterial:
    """LinearMaterial(E, nu) is corotated by default (LinearMaterial.java:53-55)."""

    E: float = 500000.0
    nu: float = 0.33
    corotated: bool = True

    kind = L.MAT_LINEAR

    def params(self):
        return [self.E, self.nu, 1.0 if self.corotated else 0.0]

    def isIncompressible(self):
        return False


@dataclass
class NeoHookeanMaterial:
    E: float = 500000.0
    nu: float = 0.33

    kind = L.MAT_NEOHOOKEAN

    def params(self):
        return [self.E, self.nu]

    def isIncompressible(self):
        return False


@dataclass
class StVenantKirchoffMaterial:
    """StVenantKirchoffMaterial(E, nu) (StVenantKirchoffMaterial.java:60-64):
    the reference's FEBio form, sigma = ((lam trE - mu)/J) B + (mu/J) B^2."""
    E: float = 500000.0
    nu: float = 0.33

    kind = L.MAT_STVK

    def params(self):
        return [self.E, self.nu]

    def isIncompressible(self):
        return False


@dataclass
class MooneyRivlinMaterial:
    """MooneyRivlinMaterial(c10, c01, c11, c20, c02, kappa)
    (MooneyRivlinMaterial.java:98-108); bulk potential QUADRATIC by default
    (IncompressibleMaterialBase.java:13-14)."""

    c10: float = 150000.0
    c01: float = 0.0
    c11: float = 0.0
    c20: float = 0.0
    c02: float = 0.0
    kappa: float = 100000.0
    jlimit: float = 0.0
    bulk_potential: int = 0  # 0 QUADRATIC, 1 LOGARITHMIC

    kind = L.MAT_MOONEYRIVLIN

    def params(self):
        return [self.c10, self.c01, self.c11, self.c20, self.c02, self.kappa, self.jlimit,
                float(self.bulk_potential)]

    def isIncompressible(self):
        return True


# ------------------------------------------------------------------ factory
def grid_dims(elem_type, nx, ny, nz):
    nn, ne = ctypes.c_int(), ctypes.c_int()
    L.check(L.lib().b200fem_grid_dims(elem_type, nx, ny, nz, ctypes.byref(nn), ctypes.byref(ne)))
    return nn.value, ne.value


def create_grid(elem_type, wx, wy, wz, nx, ny, nz):
    nn, ne = grid_dims(elem_type, nx, ny, nz)
    nen = L.ELEM_NODES[elem_type]
    xyz = np.zeros(3 * nn)
    conn = np.zeros(nen * ne, dtype=np.int32)
    L.check(L.lib().b200fem_create_grid(elem_type, wx, wy, wz, nx, ny, nz, L.dptr(xyz), L.iptr(conn)))
    return xyz.reshape(-1, 3), conn.reshape(-1, nen)


def quadratic_tet_mesh(xyz, conn):
    """FemFactory.createQuadraticModel of a linear tet mesh (host only)."""
    x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
    c = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1)
    n = ctypes.c_int()
    lib = L.lib()
    L.check(lib.b200fem_quadratic_tet_mesh(x.size // 3, L.dptr(x), c.size // 4, L.iptr(c), ctypes.byref(n), None, None))
    ox = np.zeros(3 * n.value)
    oc = np.zeros(10 * (c.size // 4), dtype=np.int32)
    L.check(lib.b200fem_quadratic_tet_mesh(x.size // 3, L.dptr(x), c.size // 4, L.iptr(c), ctypes.byref(n),
                                           L.dptr(ox), L.iptr(oc)))
    return ox.reshape(-1, 3), oc.reshape(-1, 10)


def jitter_grid(xyz, nx, ny, nz, wx, wy, wz, frac, seed):
    flat = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1).copy()
    L.check(L.lib().b200fem_jitter_grid(nx, ny, nz, wx, wy, wz, float(frac), ctypes.c_ulonglong(seed),
                                        L.dptr(flat)))
    return flat.reshape(-1, 3)


class FemFactory:
    """FemFactory.createTetGrid / createHexGrid / createWedgeGrid /
    createPyramidGrid (FemFactory.java:86-310)."""

    @staticmethod
    def createTetGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_TET, wx, wy, wz, nx, ny, nz)
        return m

    @staticmethod
    def createHexGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_HEX, wx, wy, wz, nx, ny, nz)
        return m

    @staticmethod
    def createQuadtetGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_QUADTET, wx, wy, wz, nx, ny, nz)
        return m

    @staticmethod
    def createQuadwedgeGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_QUADWEDGE, wx, wy, wz, nx, ny, nz)
        return m

    @staticmethod
    def createQuadpyramidGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_QUADPYRAMID, wx, wy, wz, nx, ny, nz)
        return m

    @staticmethod
    def createQuadhexGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_QUADHEX, wx, wy, wz, nx, ny, nz)
        return m

    @staticmethod
    def createWedgeGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_WEDGE, wx, wy, wz, nx, ny, nz)
        return m

    @staticmethod
    def createPyramidGrid(model, wx, wy, wz, nx, ny, nz):
        m = model if model is not None else FemModel3d()
        m._set_grid(L.ELEM_PYRAMID, wx, wy, wz, nx, ny, nz)
        return m


# ------------------------------------------------------------------- engine
class FemEngine:
    """Owns one libb200fem handle (CuDssJNI-style opaque handle)."""

    def __init__(self, device: int = 0, precision: int = L.PREC_FP64):
        cfg = L.Config(device, precision)
        h = L.lib().b200fem_create(ctypes.byref(cfg))
        if not h:
            msg = L.lib().b200fem_last_error(None)
            raise L.B200FemError(L.ERR_CUDA, (msg or b"").decode())
        self.h = ctypes.c_void_p(h)

    def close(self):
        if getattr(self, "h", None):
            L.lib().b200fem_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def call(self, name, *args):
        return L.check(getattr(L.lib(), name)(self.h, *args), self.h)


# -------------------------------------------------------------------- model
class FemModel3d:
    """FemModel3d restricted to the hot path: tet, hex, wedge and pyramid
    elements, linear or quadratic (one type, or any mix of them), the model's
    material and optional per-element materials, lumped mass, fixed nodes and
    the BackwardEuler data."""

    def __init__(self):
        self.elem_type = L.ELEM_TET
        self.rest = None
        self.conn = None
        self.fixed = None
        self.material = LinearMaterial()
        self.elem_materials = None  # per element: None (the model's material) or its own
        self.density = 1000.0
        self.mass_damping = 2.0      # FemModel.DEFAULT_MASS_DAMPING (FemModel.java:304)
        self.stiffness_damping = 0.0  # FemModel.DEFAULT_STIFFNESS_DAMPING (:303)
        self.gravity = np.array([0.0, 0.0, -9.8])  # MechModel default (MechModel.java:125)
        self.soft_incomp = L.INCOMP_AUTO  # FemModel3d.DEFAULT_SOFT_INCOMP (:196)
        self.fext = None
        self._grid = None
        self._engine = None
        self.precision = L.PREC_FP64
        self.device = 0

    # --- construction
    def _set_grid(self, elem_type, wx, wy, wz, nx, ny, nz):
        self.elem_type = elem_type
        xyz, conn = create_grid(elem_type, wx, wy, wz, nx, ny, nz)
        self.rest = xyz
        self.conn = conn
        self.fixed = np.zeros(xyz.shape[0], dtype=np.int32)
        self._grid = (nx, ny, nz, wx, wy, wz)
        self._invalidate()

    def setMesh(self, elem_type, rest, conn, fixed=None):
        """elem_type: one B200FEM_ELEM_* type for every element (conn: E x nen),
        or a sequence of one type per element (conn: every element's nodes
        concatenated in element order)."""
        self.rest = np.ascontiguousarray(rest, dtype=np.float64).reshape(-1, 3)
        if np.ndim(elem_type) == 0:
            self.elem_type = int(elem_type)
            nen = L.ELEM_NODES[self.elem_type]
            self.conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, nen)
        else:
            self.elem_type = np.ascontiguousarray(elem_type, dtype=np.int32).reshape(-1)
            self.conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1)
            if self.conn.size != sum(L.ELEM_NODES[int(t)] for t in self.elem_type):
                raise ValueError("connectivity size does not match the element types")
        self.fixed = (np.zeros(self.rest.shape[0], dtype=np.int32) if fixed is None
                      else np.ascontiguousarray(fixed, dtype=np.int32))
        self._grid = None
        self.elem_materials = None
        self._invalidate()

    def jitterInterior(self, frac, seed):
        """Seeded jitter of interior grid nodes, applied to rest and current
        positions before setup."""
        if self._grid is None:
            raise ValueError("jitter needs a grid built by FemFactory")
        nx, ny, nz, wx, wy, wz = self._grid
        self.rest = jitter_grid(self.rest, nx, ny, nz, wx, wy, wz, frac, seed)
        self._invalidate()

    def numNodes(self):
        return self.rest.shape[0]

    def numElements(self):
        return self.elem_type.size if self.isMixed() else self.conn.shape[0]

    def isMixed(self):
        """True when the elements are of several types (one type per element)."""
        return np.ndim(self.elem_type) > 0

    def setMaterial(self, mat):
        self.material = mat
        self._invalidate()

    def setElementMaterial(self, e, mat):
        """FemElement.setMaterial for element e; None restores the model's
        material (FemModel3d.getElementMaterial, FemModel3d.java:608-614)."""
        if self.elem_materials is None:
            self.elem_materials = [None] * self.numElements()
        self.elem_materials[int(e)] = mat
        self._invalidate()

    def setElementMaterials(self, mats):
        """One entry per element (None: the model's material), or None for
        the model's material everywhere."""
        if mats is not None and len(mats) != self.numElements():
            raise ValueError("one material per element")
        self.elem_materials = None if mats is None else list(mats)
        self._invalidate()

    def getElementMaterial(self, e):
        m = None if self.elem_materials is None else self.elem_materials[int(e)]
        return self.material if m is None else m

    def _element_material_arrays(self):
        kinds = np.full(self.numElements(), L.MAT_MODEL, dtype=np.int32)
        prm = np.zeros((self.numElements(), 8))
        for e, m in enumerate(self.elem_materials):
            if m is not None:
                kinds[e] = m.kind
                p = m.params()
                prm[e, : len(p)] = p
        return kinds, prm

    def setDensity(self, d):
        self.density = float(d)
        self._invalidate()

    def setMassDamping(self, d):
        self.mass_damping = float(d)

    setParticleDamping = setMassDamping

    def setStiffnessDamping(self, d):
        self.stiffness_damping = float(d)

    def setGravity(self, gx, gy=None, gz=None):
        self.gravity = np.array([gx, gy, gz] if gy is not None else gx, dtype=np.float64).reshape(3)

    def setSoftIncompMethod(self, method):
        self.soft_incomp = int(method)
        self._invalidate()

    def fixNodes(self, mask):
        """node.setDynamic(false) for every node where mask is true."""
        self.fixed = np.ascontiguousarray(np.asarray(mask).astype(np.int32))
        self._invalidate()

    def setExternalForces(self, fext):
        self.fext = None if fext is None else np.ascontiguousarray(fext, dtype=np.float64).reshape(-1, 3)
        if self._engine is not None:
            self._push_fext()

    def setPrecision(self, precision):
        self.precision = int(precision)
        self._invalidate()

    # --- engine
    def _invalidate(self):
        if self._engine is not None:
            self._engine.close()
        self._engine = None

    def _push_fext(self):
        f = self.fext.reshape(-1).copy() if self.fext is not None else None
        self._engine.call("b200fem_set_external_forces", L.dptr(f))

    def engine(self) -> FemEngine:
        if self._engine is None:
            eng = FemEngine(self.device, self.precision)
            rest = np.ascontiguousarray(self.rest.reshape(-1))
            conn = np.ascontiguousarray(self.conn.reshape(-1))
            if self.isMixed():
                eng.call("b200fem_set_mesh_mixed", self.numNodes(), L.dptr(rest), self.numElements(),
                         L.iptr(self.elem_type), L.iptr(conn), L.iptr(self.fixed))
            else:
                eng.call("b200fem_set_mesh", self.elem_type, self.numNodes(), L.dptr(rest), self.numElements(),
                         L.iptr(conn), L.iptr(self.fixed))
            prm = np.zeros(8)
            p = self.material.params()
            prm[: len(p)] = p
            eng.call("b200fem_set_material", self.material.kind, L.dptr(prm), self.density, self.soft_incomp)
            if self.elem_materials is not None:
                kinds, eprm = self._element_material_arrays()
                eng.call("b200fem_set_element_materials", 0, self.numElements(), kinds.ctypes.data,
                         eprm.ctypes.data)
            for k, v in getattr(self, "options", {}).items():
                eng.call("b200fem_set_option", int(k), int(v))
            att = getattr(self, "attachments", None)
            if att is not None:
                nf, nd, fr, hb = att
                eng.call("b200fem_set_frame_attachments", nf, int(nd.size), L.iptr(nd), L.iptr(fr), L.dptr(hb))
            eng.call("b200fem_build")
            self._engine = eng
            if self.fext is not None:
                self._push_fext()
        return self._engine

    # --- queries
    def sizes(self):
        e = self.engine()
        a, b, c, d = (ctypes.c_int() for _ in range(4))
        e.call("b200fem_get_sizes", ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
        return dict(n_active=a.value, nnzb=b.value, crs_nnz_full=c.value, crs_nnz_upper=d.value)

    def getSolveIndices(self):
        out = np.zeros(self.numNodes(), dtype=np.int32)
        self.engine().call("b200fem_get_solve_index", L.iptr(out))
        return out

    def getBlockPattern(self):
        s = self.sizes()
        rp = np.zeros(s["n_active"] + 1, dtype=np.int32)
        col = np.zeros(s["nnzb"], dtype=np.int32)
        self.engine().call("b200fem_get_pattern", L.iptr(rp), L.iptr(col))
        return rp, col

    def getCRSIndices(self, partition=L.PART_FULL):
        s = self.sizes()
        nnz = s["crs_nnz_full"] if partition == L.PART_FULL else s["crs_nnz_upper"]
        ro = np.zeros(3 * s["n_active"] + 1, dtype=np.int32)
        ci = np.zeros(nnz, dtype=np.int32)
        self.engine().call("b200fem_get_crs_indices", partition, L.iptr(ro), L.iptr(ci))
        return ro, ci

    def createCrsBlockSlotMap(self, partition=L.PART_FULL):
        s = self.sizes()
        slots = np.zeros(9 * s["nnzb"], dtype=np.int32)
        self.engine().call("b200fem_get_slot_map", partition, L.iptr(slots))
        return slots

    def getScatterMap(self):
        """Block index of every element's (i, j) node pair: E x nen x nen, or
        for a mesh of several types a flat array of nen_e * nen_e entries per
        element in element order."""
        if self.isMixed():
            out = np.zeros(sum(L.ELEM_NODES[int(t)] ** 2 for t in self.elem_type), dtype=np.int32)
            self.engine().call("b200fem_get_scatter_map", L.iptr(out))
            return out
        nen = self.conn.shape[1]
        out = np.zeros(self.numElements() * nen * nen, dtype=np.int32)
        self.engine().call("b200fem_get_scatter_map", L.iptr(out))
        return out.reshape(self.numElements(), nen, nen)

    def getNodeMasses(self):
        out = np.zeros(self.numNodes())
        self.engine().call("b200fem_get_masses", L.dptr(out))
        return out

    def getSoftIncompMethod(self):
        out = ctypes.c_int()
        self.engine().call("b200fem_get_incomp_method", ctypes.byref(out))
        return out.value

    # --- state
    def setState(self, x=None, v=None):
        xe = None if x is None else np.ascontiguousarray(x, dtype=np.float64).reshape(-1).copy()
        ve = None if v is None else np.ascontiguousarray(v, dtype=np.float64).reshape(-1).copy()
        self.engine().call("b200fem_set_state", L.dptr(xe), L.dptr(ve))

    def getState(self):
        x = np.zeros(3 * self.numNodes())
        v = np.zeros(3 * self.numNodes())
        self.engine().call("b200fem_get_state", L.dptr(x), L.dptr(v))
        return x.reshape(-1, 3), v.reshape(-1, 3)

    def setPointConstraints(self, ptr, nodes, weights, targets):
        """LinearPointConstraints: constraint c holds the weighted sum of the
        positions of nodes[ptr[c]:ptr[c+1]] at targets[c] (enforced by the
        ConstrainedBackwardEuler integrator)."""
        pt = np.ascontiguousarray(np.asarray(ptr, dtype=np.int32).reshape(-1))
        nd = np.ascontiguousarray(np.asarray(nodes, dtype=np.int32).reshape(-1))
        wt = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
        tg = np.ascontiguousarray(np.asarray(targets, dtype=np.float64).reshape(-1))
        self.engine().call("b200fem_set_point_constraints", int(pt.size - 1), L.iptr(pt), L.iptr(nd), L.dptr(wt),
                           L.dptr(tg))

    def setFrameAttachments(self, n_frames, nodes, frames, H):
        """PointFrameAttachment of `nodes` to active frames (FemModel3d.
        getGpuNodeReduction, FemModel3d.java:4356-4387): H holds each
        attachment's 6x3 master block.  The stiffness and pattern queries
        then describe the reduced system P^T K P over the free nodes and two
        block rows per frame."""
        nd = np.ascontiguousarray(np.asarray(nodes, dtype=np.int32).reshape(-1))
        fr = np.ascontiguousarray(np.asarray(frames, dtype=np.int32).reshape(-1))
        hb = np.ascontiguousarray(np.asarray(H, dtype=np.float64).reshape(-1))
        assert hb.size == 18 * nd.size and fr.size == nd.size
        self.attachments = (int(n_frames), nd, fr, hb)
        self._invalidate()

    def setPlaneConstraints(self, nodes, normals, offsets):
        """ParticlePlaneConstraint on single nodes: node nodes[i] is held on
        the plane normals[i] . x = offsets[i] by the ConstrainedBackwardEuler
        integrator (b200fem_set_plane_constraints); empty lists remove them."""
        nd = np.ascontiguousarray(nodes, dtype=np.int32).reshape(-1)
        nr = np.ascontiguousarray(normals, dtype=np.float64).reshape(-1)
        of = np.ascontiguousarray(offsets, dtype=np.float64).reshape(-1)
        if nr.size != 3 * nd.size or of.size != nd.size:
            raise ValueError("one normal (3 values) and one offset per node")
        self.engine().call("b200fem_set_plane_constraints", int(nd.size), L.iptr(nd), L.dptr(nr), L.dptr(of))

    # --- hot path
    def updateStressAndStiffness(self, x=None, want_crs=False):
        """Internal force (N,3), stiffness blocks (nnzb,3,3) in block-CSR
        order and optionally the full-partition CRS values."""
        s = self.sizes()
        xe = None if x is None else np.ascontiguousarray(x, dtype=np.float64).reshape(-1).copy()
        f = np.zeros(3 * self.numNodes())
        K = np.zeros(9 * s["nnzb"])
        crs = np.zeros(s["crs_nnz_full"]) if want_crs else None
        self.engine().call("b200fem_update_stress_stiffness", L.dptr(xe), L.dptr(f), L.dptr(K), L.dptr(crs))
        out = (f.reshape(-1, 3), K.reshape(-1, 3, 3))
        return out + (crs,) if want_crs else out


class MechSystemSolver:
    """BackwardEuler integration of one FemModel3d on the device
    (MechSystemSolver.backwardEuler, MechSystemSolver.java:2171-2476)."""

    def __init__(self, model: FemModel3d, tol: float = 1e-10, max_iter: int = 10000, pcg_variant: int = 0,
                 integrator: int = L.INTEGRATOR_BACKWARD_EULER):
        self.model = model
        self.tol = tol
        self.max_iter = max_iter
        self.pcg_variant = pcg_variant
        # MechSystemSolver.setIntegrator: BackwardEuler ignores constraints,
        # ConstrainedBackwardEuler enforces the model's plane constraints
        self.integrator = integrator
        self.abort_on_inverted = False
        self.stats = L.Stats()

    def params(self, h):
        m = self.model
        p = L.StepParams()
        p.h = h
        p.alpha_m = m.mass_damping
        p.beta_k = m.stiffness_damping
        for i in range(3):
            p.gravity[i] = m.gravity[i]
        p.tol = self.tol
        p.max_iter = self.max_iter
        p.abort_on_inverted = 1 if self.abort_on_inverted else 0
        p.pcg_variant = self.pcg_variant
        p.integrator = self.integrator
        return p

    def backwardEuler(self, h, nsteps=1):
        p = self.params(h)
        self.model.engine().call("b200fem_backward_euler_step", ctypes.byref(p), int(nsteps),
                                 ctypes.byref(self.stats))
        return self.stats

    def backwardEulerHost(self, h, x, v, nsteps=1):
        """nsteps steps from the host state x, v (float64 arrays of 3N
        values, updated in place): the call a host that keeps the state makes
        every step (b200fem_backward_euler_step_host)."""
        n3 = 3 * self.model.numNodes()
        for a in (x, v):
            if a.dtype != np.float64 or not a.flags["C_CONTIGUOUS"] or a.size != n3:
                raise ValueError("x and v must be C-contiguous float64 arrays of 3N values")
        # the step parameters and the bound entry point are kept between
        # calls: this is the per-step call of a host that keeps the state
        m = self.model
        key = (h, m.mass_damping, m.stiffness_damping, tuple(m.gravity), self.tol, self.max_iter,
               self.abort_on_inverted, self.pcg_variant, self.integrator)
        cache = getattr(self, "_host_call", None)
        eng = m.engine()
        if cache is None or cache[0] != key or cache[1] is not eng:
            p = self.params(h)
            cache = (key, eng, p, ctypes.byref(p), ctypes.byref(self.stats),
                     L.lib().b200fem_backward_euler_step_host)
            self._host_call = cache
        st = cache[5](eng.h, cache[3], int(nsteps), x.ctypes.data, v.ctypes.data, cache[4])
        if st != L.OK:
            L.check(st, eng.h)
        return self.stats

    def spmv(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1).copy()
        y = np.zeros_like(x)
        self.model.engine().call("b200fem_spmv", L.dptr(x), L.dptr(y))
        return y

    def pcg(self, b, x0=None, tol=1e-10, max_iter=10000):
        b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1).copy()
        x = np.zeros_like(b) if x0 is None else np.ascontiguousarray(x0, dtype=np.float64).reshape(-1).copy()
        st = L.Stats()
        self.model.engine().call("b200fem_pcg_solve", L.dptr(b), L.dptr(x), float(tol), int(max_iter),
                                 ctypes.byref(st))
        return x, st

    def lastTiming(self):
        a, s = ctypes.c_double(), ctypes.c_double()
        self.model.engine().call("b200fem_last_timing", ctypes.byref(a), ctypes.byref(s))
        return a.value, s.value


class FemPack:
    """Batched form: several independent models stepped together in one
    engine (one pack).  Every kernel launch covers all models; each model
    keeps its own material, PCG scalars and convergence test."""

    def __init__(self, models, precision=L.PREC_MIXED, device=0, options=None):
        self.models = list(models)
        self.precision = precision
        self.device = device
        self.options = dict(options or {})  # B200FEM_OPT_* key -> value, applied before the build
        self._engine = None
        self.offsets = None
        self.stats = L.Stats()

    def engine(self) -> FemEngine:
        if self._engine is None:
            eng = FemEngine(self.device, self.precision)
            for m in self.models:
                if m.isMixed():
                    raise ValueError("a pack takes models of one element type each")
                prm = np.zeros(8)
                p = m.material.params()
                prm[: len(p)] = p
                rest = np.ascontiguousarray(m.rest.reshape(-1))
                conn = np.ascontiguousarray(m.conn.reshape(-1))
                idx = ctypes.c_int()
                eng.call("b200fem_add_model", m.elem_type, m.numNodes(), L.dptr(rest), m.numElements(),
                         L.iptr(conn), L.iptr(m.fixed), m.material.kind, L.dptr(prm), m.density, m.soft_incomp,
                         ctypes.byref(idx))
                if m.elem_materials is not None:
                    kinds, eprm = m._element_material_arrays()
                    eng.call("b200fem_set_element_materials", idx.value, m.numElements(), kinds.ctypes.data,
                             eprm.ctypes.data)
            for k, v in self.options.items():
                eng.call("b200fem_set_option", int(k), int(v))
            eng.call("b200fem_build")
            self._engine = eng
            self.offsets = []
            for i in range(len(self.models)):
                o, n, a = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
                eng.call("b200fem_model_range", i, ctypes.byref(o), ctypes.byref(n), ctypes.byref(a))
                self.offsets.append((o.value, n.value, a.value))
            fext = [m.fext if m.fext is not None else np.zeros((m.numNodes(), 3)) for m in self.models]
            if any(m.fext is not None for m in self.models):
                f = np.ascontiguousarray(np.concatenate(fext).reshape(-1))
                eng.call("b200fem_set_external_forces", L.dptr(f))
        return self._engine

    def close(self):
        if self._engine is not None:
            self._engine.close()
            self._engine = None

    def deviceBytes(self) -> int:
        """Device memory held by the pack."""
        v = ctypes.c_ulonglong()
        self.engine().call("b200fem_memory_usage", ctypes.byref(v))
        return v.value

    def setActive(self, active=None):
        """Mask of the models the next steps advance (None: all)."""
        if active is None:
            self.engine().call("b200fem_set_active_models", None)
        else:
            a = np.ascontiguousarray(np.asarray(active, dtype=np.int32))
            assert a.shape == (len(self.models),)
            self.engine().call("b200fem_set_active_models", L.iptr(a))

    def option(self, key) -> int:
        """The value of a B200FEM_OPT_* option in force (resolved after the build)."""
        v = ctypes.c_int()
        self.engine().call("b200fem_get_option", int(key), ctypes.byref(v))
        return v.value

    def setOption(self, key, value):
        """Options that may change after the build (ROW_LANES)."""
        if self._engine is not None:
            self._engine.call("b200fem_set_option", int(key), int(value))
        self.options[key] = value

    def total_nodes(self):
        return sum(m.numNodes() for m in self.models)

    def setStates(self, xs=None, vs=None):
        e = self.engine()
        xe = None if xs is None else np.ascontiguousarray(np.concatenate([np.asarray(x).reshape(-1, 3) for x in xs]).reshape(-1))
        ve = None if vs is None else np.ascontiguousarray(np.concatenate([np.asarray(v).reshape(-1, 3) for v in vs]).reshape(-1))
        e.call("b200fem_set_state", L.dptr(xe), L.dptr(ve))

    def getStates(self):
        e = self.engine()
        n = self.total_nodes()
        x = np.zeros(3 * n)
        v = np.zeros(3 * n)
        e.call("b200fem_get_state", L.dptr(x), L.dptr(v))
        x = x.reshape(-1, 3)
        v = v.reshape(-1, 3)
        return [(x[o:o + k], v[o:o + k]) for (o, k, _) in self.offsets]

    def backwardEuler(self, h, nsteps=1, tol=1e-10, max_iter=20000, alpha=None, beta=None, gravity=None,
                      pcg_variant=0):
        m0 = self.models[0]
        p = L.StepParams()
        p.h = h
        p.alpha_m = m0.mass_damping if alpha is None else alpha
        p.beta_k = m0.stiffness_damping if beta is None else beta
        g = m0.gravity if gravity is None else gravity
        for i in range(3):
            p.gravity[i] = g[i]
        p.tol = tol
        p.max_iter = max_iter
        p.pcg_variant = pcg_variant
        self.engine().call("b200fem_backward_euler_step", ctypes.byref(p), int(nsteps), ctypes.byref(self.stats))
        return self.stats

    def modelStats(self):
        n = len(self.models)
        it = np.zeros(n, dtype=np.int32)
        rr = np.zeros(n)
        self.engine().call("b200fem_get_model_stats", L.iptr(it), L.dptr(rr))
        return it, rr

    def lastTiming(self):
        a, s = ctypes.c_double(), ctypes.c_double()
        self.engine().call("b200fem_last_timing", ctypes.byref(a), ctypes.byref(s))
        return a.value, s.value
