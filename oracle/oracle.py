"""ctypes front end of the CPU FP64 oracle (``oracle/fem_oracle.cpp``).

TEST INFRASTRUCTURE ONLY: tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it as the checker.  The product package
never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libfemoracle.so")
_lib = None
# the reference's device assembly kernels (cudssBridgeKernels.cu), compiled
# from the reference tree by `make ref` where that tree is present; its
# location comes from the caller or from $ARTISYNTH_REFERENCE
REF_LIB_PATH = os.path.join(_HERE, "_ref", "libref_kernels.so")

ELEM_TET, ELEM_HEX, ELEM_WEDGE, ELEM_PYRAMID, ELEM_QUADTET, ELEM_QUADHEX, ELEM_QUADWEDGE, ELEM_QUADPYRAMID = range(8)
ELEM_NODES = {ELEM_TET: 4, ELEM_HEX: 8, ELEM_WEDGE: 6, ELEM_PYRAMID: 5, ELEM_QUADTET: 10, ELEM_QUADHEX: 20,
              ELEM_QUADWEDGE: 15, ELEM_QUADPYRAMID: 13}
MAT_LINEAR, MAT_NEOHOOKEAN, MAT_MOONEYRIVLIN, MAT_STVK = 0, 1, 2, 3
INCOMP_OFF, INCOMP_NODAL, INCOMP_AUTO, INCOMP_ELEMENT = 0, 1, 2, 3

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def build_ref(source_root: str | None = None) -> str | None:
    """Compile the reference's kernels into oracle/_ref/ from the reference
    tree at `source_root` (default: $ARTISYNTH_REFERENCE) when that tree is
    present; elsewhere (a GPU box gets the prebuilt library) return the
    library path if it exists, else None."""
    root = source_root or os.environ.get("ARTISYNTH_REFERENCE")
    if root and os.path.isdir(root):
        subprocess.run(["make", "-s", "-C", _HERE, "ref", "REF=" + root], check=True)
    return REF_LIB_PATH if os.path.exists(REF_LIB_PATH) else None


def ref_kernels():
    """ctypes handle of the reference kernels library, or None when it was
    not built.  Entry points used: addMaterialStiffness3_launch
    (cudssBridgeKernels.cu:244-253), addMaterialStiffness3Element_launch
    (:436-449), addLinearElasticStiffness3Element_launch (:518-530) and
    addDilationalStiffness3Element_launch (:725-739)."""
    if not os.path.exists(REF_LIB_PATH):
        return None
    R = ctypes.CDLL(REF_LIB_PATH)
    vp = ctypes.c_void_p
    R.addMaterialStiffness3_launch.argtypes = [ctypes.c_int, vp, vp, vp, vp, vp, vp, ctypes.c_double, vp, vp]
    R.addMaterialStiffness3_launch.restype = None
    R.addLinearElasticStiffness3Element_launch.argtypes = [ctypes.c_int] + [vp] * 9 + [ctypes.c_double, vp, vp]
    R.addLinearElasticStiffness3Element_launch.restype = None
    R.addDilationalStiffness3Element_launch.argtypes = [ctypes.c_int] + [vp] * 12 + [ctypes.c_double, vp, vp]
    R.addDilationalStiffness3Element_launch.restype = None
    R.addMaterialStiffness3Element_launch.argtypes = [ctypes.c_int] + [vp] * 13 + [ctypes.c_double, vp, vp]
    R.addMaterialStiffness3Element_launch.restype = None
    return R


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        vp = ctypes.c_void_p
        L.orc_num_threads.argtypes = [ctypes.c_int]
        L.orc_grid_dims.argtypes = [ctypes.c_int] * 4 + [ctypes.POINTER(ctypes.c_int)] * 2
        L.orc_create_grid.argtypes = [ctypes.c_int] + [ctypes.c_double] * 3 + [ctypes.c_int] * 3 + [_dp, _ip]
        for fn in ("orc_quadratic_tets", "orc_quadratic_hexes"):
            getattr(L, fn).argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_int),
                                       ctypes.c_void_p, ctypes.c_void_p]
        L.orc_jitter.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [ctypes.c_uint64, _dp]
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _ip, _ip,
                                 ctypes.c_int, _dp, ctypes.c_double, ctypes.c_int]
        L.orc_create.restype = vp
        L.orc_create_mixed.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _ip, _ip, _ip, ctypes.c_int, _dp,
                                       ctypes.c_double, ctypes.c_int]
        L.orc_create_mixed.restype = vp
        L.orc_nodal_factors.argtypes = [vp] + [ctypes.c_void_p] * 4
        L.orc_nodal_factors.restype = ctypes.c_int
        L.orc_set_element_materials.argtypes = [vp, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_set_element_materials.restype = ctypes.c_int
        L.orc_elem_num_ip.argtypes = [vp, ctypes.c_int]
        L.orc_elem_num_ip.restype = ctypes.c_int
        L.orc_destroy.argtypes = [vp]
        for name in ("orc_incomp_method", "orc_num_active", "orc_nnzb"):
            getattr(L, name).argtypes = [vp]
            getattr(L, name).restype = ctypes.c_int
        L.orc_solve_index.argtypes = [vp, _ip]
        L.orc_pattern.argtypes = [vp, _ip, _ip]
        L.orc_masses.argtypes = [vp, _dp]
        L.orc_rest_volumes.argtypes = [vp, _dp]
        L.orc_crs.argtypes = [vp, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.orc_crs.restype = ctypes.c_int
        L.orc_update_stress_stiffness.argtypes = [vp, _dp, _dp, _dp]
        L.orc_update_stress_stiffness.restype = ctypes.c_int
        L.orc_nodal_pressures.argtypes = [vp, _dp]
        L.orc_be_step.argtypes = [vp, ctypes.c_double, _dp, ctypes.c_void_p, _dp, _dp, ctypes.c_int,
                                  ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_double)]
        L.orc_be_step.restype = ctypes.c_int
        L.orc_material_eval.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_double, _dp, _dp]
        L.orc_material_stiffness_block.argtypes = [_dp, _dp, ctypes.c_void_p, _dp, ctypes.c_double, _dp]
        L.orc_linear_C.argtypes = [ctypes.c_double, ctypes.c_double, _dp]
        L.orc_polar.argtypes = [_dp, _dp]
        L.orc_cbe_step.argtypes = [vp, ctypes.c_double, _dp, ctypes.c_void_p, _dp, _dp, ctypes.c_int, _ip, _dp, _dp]
        L.orc_cbe_step.restype = ctypes.c_int
        L.orc_cbe_step_points.argtypes = [vp, ctypes.c_double, _dp, ctypes.c_void_p, _dp, _dp, ctypes.c_int, _ip,
                                          _ip, _dp, _dp]
        L.orc_cbe_step_points.restype = ctypes.c_int
        L.orc_num_ip.argtypes = [vp]
        L.orc_num_ip.restype = ctypes.c_int
        L.orc_ip_data.argtypes = [vp, _dp, ctypes.c_int, ctypes.c_int, _dp, ctypes.POINTER(ctypes.c_double), _dp, _dp]
        L.orc_ip_data.restype = ctypes.c_int
        _lib = L
    return _lib


def set_threads(n: int) -> int:
    return lib().orc_num_threads(int(n))


def grid(elem_type: int, widths, cells, jitter: float = 0.0, seed: int = 0):
    """FemFactory.createTetGrid / createHexGrid plus seeded interior jitter."""
    L = lib()
    nx, ny, nz = (int(c) for c in cells)
    nn, ne = ctypes.c_int(), ctypes.c_int()
    L.orc_grid_dims(elem_type, nx, ny, nz, ctypes.byref(nn), ctypes.byref(ne))
    nen = ELEM_NODES[elem_type]
    xyz = np.zeros(3 * nn.value)
    conn = np.zeros(nen * ne.value, dtype=np.int32)
    L.orc_create_grid(elem_type, float(widths[0]), float(widths[1]), float(widths[2]), nx, ny, nz, xyz, conn)
    if jitter:
        L.orc_jitter(nx, ny, nz, float(widths[0]), float(widths[1]), float(widths[2]), float(jitter),
                     ctypes.c_uint64(seed), xyz)
    return xyz.reshape(-1, 3), conn.reshape(-1, nen)


def quadratic_tets(xyz, conn):
    """FemFactory.createQuadraticModel of a linear tet mesh."""
    L = lib()
    x = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
    c = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1)
    n = ctypes.c_int()
    L.orc_quadratic_tets(x.size // 3, x, c.size // 4, c, ctypes.byref(n), None, None)
    ox = np.zeros(3 * n.value)
    oc = np.zeros(10 * (c.size // 4), dtype=np.int32)
    L.orc_quadratic_tets(x.size // 3, x, c.size // 4, c, ctypes.byref(n), ox.ctypes.data, oc.ctypes.data)
    return ox.reshape(-1, 3), oc.reshape(-1, 10)


class OracleModel:
    """One FEM model inside the oracle."""

    def __init__(self, elem_type, rest, conn, fixed, mat_kind, mat_params, density,
                 incomp=INCOMP_AUTO):
        """elem_type: one type for every element (conn: E x nen), or a
        sequence with each element's type (conn: the elements' nodes
        concatenated) for a mesh that mixes element types."""
        self.L = lib()
        self.rest = np.ascontiguousarray(rest, dtype=np.float64).reshape(-1)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1)
        self.N = self.rest.size // 3
        fx = np.ascontiguousarray(fixed, dtype=np.int32)
        mp = np.zeros(8)
        mp[: len(mat_params)] = mat_params
        if np.ndim(elem_type) == 0:
            self.elem_type = int(elem_type)
            self.types = None
            self.E = self.conn.size // ELEM_NODES[self.elem_type]
            self.h = self.L.orc_create(self.elem_type, self.N, self.rest, self.E, self.conn, fx, mat_kind, mp,
                                       float(density), incomp)
        else:
            self.types = np.ascontiguousarray(elem_type, dtype=np.int32)
            self.elem_type = int(self.types[0])
            self.E = self.types.size
            assert self.conn.size == sum(ELEM_NODES[int(t)] for t in self.types)
            self.h = self.L.orc_create_mixed(self.N, self.rest, self.E, self.types, self.conn, fx, mat_kind, mp,
                                             float(density), incomp)
        if not self.h:
            raise ValueError("the oracle refuses this model (unknown element type)")
        self.nact = self.L.orc_num_active(self.h)
        self.nnzb = self.L.orc_nnzb(self.h)
        self.incomp = self.L.orc_incomp_method(self.h)

    def nodal_factors(self):
        """The NODAL terms of the last update_stress_stiffness: (ptr, idx, kp,
        div) -- each node's sorted direct neighbours, kp and divBlk row."""
        q = self.L.orc_nodal_factors(self.h, None, None, None, None)
        if q < 0:
            raise ValueError("no NODAL terms (model not NODAL or not updated)")
        ptr = np.zeros(self.N + 1, dtype=np.int32)
        idx = np.zeros(q, dtype=np.int32)
        kp = np.zeros(self.N)
        div = np.zeros((q, 3))
        self.L.orc_nodal_factors(self.h, ptr.ctypes.data, idx.ctypes.data, kp.ctypes.data, div.ctypes.data)
        return ptr, idx, kp, div

    def set_element_materials(self, materials):
        """materials: one entry per element, None for the model's material or
        (kind, params) for the element's own (FemElement.setMaterial); None
        instead of the list restores the model's material everywhere.  Raises
        ValueError for NODAL soft incompressibility with an element of a
        compressible material."""
        if materials is None:
            st = self.L.orc_set_element_materials(self.h, None, None)
        else:
            assert len(materials) == self.E
            kinds = np.full(self.E, -1, dtype=np.int32)
            prm = np.zeros((self.E, 8))
            for e, m in enumerate(materials):
                if m is not None:
                    kinds[e] = m[0]
                    prm[e, : len(m[1])] = m[1]
            st = self.L.orc_set_element_materials(self.h, kinds.ctypes.data, prm.ctypes.data)
        self.nnzb = self.L.orc_nnzb(self.h)
        self.incomp = self.L.orc_incomp_method(self.h)
        if st != 0:
            raise ValueError("NODAL soft incompressibility with elements of compressible materials")

    def __del__(self):
        try:
            if getattr(self, "h", None):
                self.L.orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def solve_index(self):
        out = np.zeros(self.N, dtype=np.int32)
        self.L.orc_solve_index(self.h, out)
        return out

    def pattern(self):
        rp = np.zeros(self.nact + 1, dtype=np.int32)
        col = np.zeros(self.nnzb, dtype=np.int32)
        self.L.orc_pattern(self.h, rp, col)
        return rp, col

    def masses(self):
        out = np.zeros(self.N)
        self.L.orc_masses(self.h, out)
        return out

    def rest_volumes(self):
        out = np.zeros(self.E)
        self.L.orc_rest_volumes(self.h, out)
        return out

    def crs(self, partition=0):
        nnz = self.L.orc_crs(self.h, partition, None, None, None)
        ro = np.zeros(3 * self.nact + 1, dtype=np.int32)
        ci = np.zeros(nnz, dtype=np.int32)
        sl = np.zeros(9 * self.nnzb, dtype=np.int32)
        self.L.orc_crs(self.h, partition, ro.ctypes.data, ci.ctypes.data, sl.ctypes.data)
        return ro, ci, sl

    def update_stress_stiffness(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        f = np.zeros(3 * self.N)
        K = np.zeros(9 * self.nnzb)
        ninv = self.L.orc_update_stress_stiffness(self.h, x, f, K)
        return f.reshape(-1, 3), K.reshape(-1, 3, 3), ninv

    def cbe_step_points(self, h, x, v, ptr, nodes, weights, targets, alpha=2.0, beta=0.0, gravity=(0, 0, 0),
                        fext=None):
        """One ConstrainedBackwardEuler step with LinearPointConstraints
        (constraint c: sum of weights[q] * x[nodes[q]] over q in
        [ptr[c], ptr[c+1]) held at targets[c]); dense KKT velocity solve and
        GlobalMass position correction; x, v (N,3) updated in place.
        Returns the status (0 ok)."""
        xf = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        vf = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        prm = np.array([alpha, beta, *gravity], dtype=np.float64)
        fe = None if fext is None else np.ascontiguousarray(fext, dtype=np.float64).reshape(-1)
        pt = np.ascontiguousarray(ptr, dtype=np.int32)
        nd = np.ascontiguousarray(nodes, dtype=np.int32)
        wt = np.ascontiguousarray(weights, dtype=np.float64)
        tg = np.ascontiguousarray(targets, dtype=np.float64).reshape(-1)
        st = self.L.orc_cbe_step_points(self.h, float(h), prm, None if fe is None else fe.ctypes.data, xf, vf,
                                        int(pt.size - 1), pt, nd, wt, tg)
        x.reshape(-1)[:] = xf
        v.reshape(-1)[:] = vf
        return st

    def cbe_step(self, h, x, v, nodes, normals, offsets, alpha=2.0, beta=0.0, gravity=(0, 0, 0), fext=None):
        """One ConstrainedBackwardEuler step with particle-plane constraints
        (dense KKT solve, GlobalMass position correction); x, v (N,3) are
        updated in place.  Returns the status (0 ok)."""
        xf = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        vf = np.ascontiguousarray(v, dtype=np.float64).reshape(-1)
        prm = np.array([alpha, beta, *gravity], dtype=np.float64)
        fe = None if fext is None else np.ascontiguousarray(fext, dtype=np.float64).reshape(-1)
        nd = np.ascontiguousarray(nodes, dtype=np.int32).reshape(-1)
        nr = np.ascontiguousarray(normals, dtype=np.float64).reshape(-1)
        of = np.ascontiguousarray(offsets, dtype=np.float64).reshape(-1)
        st = self.L.orc_cbe_step(self.h, float(h), prm, None if fe is None else fe.ctypes.data, xf, vf,
                                 int(nd.size), nd, nr, of)
        x.reshape(-1)[:] = xf
        v.reshape(-1)[:] = vf
        return st

    def num_ip(self, e=None):
        """Integration points of element e (default: of the first element)."""
        return self.L.orc_num_ip(self.h) if e is None else self.L.orc_elem_num_ip(self.h, int(e))

    def ip_data(self, x, e, k):
        """(GNx (nen,3), dv, sig (6), D (6,6)) of integration point k of
        element e at positions x (non-linear materials)."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        nen = ELEM_NODES[self.elem_type if self.types is None else int(self.types[e])]
        g = np.zeros(3 * nen)
        dv = ctypes.c_double()
        sig = np.zeros(6)
        D = np.zeros(36)
        if self.L.orc_ip_data(self.h, x, int(e), int(k), g, ctypes.byref(dv), sig, D) != nen:
            raise ValueError("no integration-point data for this element/point")
        return g.reshape(nen, 3), dv.value, sig, D.reshape(6, 6)

    def nodal_pressures(self):
        out = np.zeros(self.N)
        self.L.orc_nodal_pressures(self.h, out)
        return out

    def be_step(self, h, x, v, alpha=2.0, beta=0.0, gravity=(0, 0, 0), fext=None, solver=0,
                tol=1e-14, maxit=100000):
        """One BackwardEuler step; x and v (N,3) float64 arrays updated in place."""
        prm = np.array([alpha, beta, *gravity], dtype=np.float64)
        it = ctypes.c_int()
        rr = ctypes.c_double()
        fe = None
        if fext is not None:
            fe = np.ascontiguousarray(fext, dtype=np.float64).reshape(-1)
        st = self.L.orc_be_step(self.h, float(h), prm, fe.ctypes.data if fe is not None else None,
                                x.reshape(-1), v.reshape(-1), int(solver), float(tol), int(maxit),
                                ctypes.byref(it), ctypes.byref(rr))
        return st, it.value, rr.value


def material_eval(mat_kind, params, F, pressure=0.0):
    mp = np.zeros(8)
    mp[: len(params)] = params
    sig = np.zeros(6)
    D = np.zeros(36)
    lib().orc_material_eval(mat_kind, mp, np.ascontiguousarray(F, dtype=np.float64).reshape(-1),
                            float(pressure), sig, D)
    return sig, D.reshape(6, 6)


def material_stiffness_block(gi, D, gj, dv, sig=None):
    K = np.zeros(9)
    s = None if sig is None else np.ascontiguousarray(sig, dtype=np.float64)
    lib().orc_material_stiffness_block(np.asarray(gi, dtype=np.float64), np.ascontiguousarray(D, dtype=np.float64).reshape(-1),
                                       s.ctypes.data if s is not None else None,
                                       np.asarray(gj, dtype=np.float64), float(dv), K)
    return K.reshape(3, 3)


def linear_C(E, nu):
    D = np.zeros(36)
    lib().orc_linear_C(float(E), float(nu), D)
    return D.reshape(6, 6)


def polar(F):
    R = np.zeros(9)
    lib().orc_polar(np.ascontiguousarray(F, dtype=np.float64).reshape(-1), R)
    return R.reshape(3, 3)


def reduce_attachments(rowptr, col, K, act_node, n_nodes, n_frames, nodes, frames, H):
    """Master-slave reduction of a stiffness assembled over free and attached
    nodes (the extended system: rowptr/col/K over block rows whose nodes are
    act_node) onto the free nodes followed by two block rows per frame
    (translation, rotation): every block K_ij goes to T_i K_ij T_j^T, T = I
    for a free node and the attachment's 6x3 master block H for an attached
    one (scatterReduced3Block, cudssBridgeKernels.cu:325-365;
    FemModel3d.getGpuNodeReduction, FemModel3d.java:4356-4387).  Blocks of a
    reduced block are summed in extended-block order.  Returns the reduced
    rowptr, col, blocks (nnzb, 3, 3) and the per-node reduced solve index
    (-1 for fixed and attached nodes)."""
    act_node = np.asarray(act_node)
    R = act_node.size
    att_of_node = {int(n): k for k, n in enumerate(nodes)}
    att_row = np.array([att_of_node.get(int(n), -1) for n in act_node])
    red_of_row = np.full(R, -1)
    n_free = 0
    for r in range(R):
        if att_row[r] < 0:
            red_of_row[r] = n_free
            n_free += 1
    Hb = np.asarray(H, dtype=np.float64).reshape(-1, 6, 3)

    def targets(r):
        k = att_row[r]
        if k < 0:
            return [(int(red_of_row[r]), np.eye(3))]
        f = int(frames[k])
        return [(n_free + 2 * f, Hb[k, 0:3]), (n_free + 2 * f + 1, Hb[k, 3:6])]

    n_red = n_free + 2 * n_frames
    rows = [dict() for _ in range(n_red)]
    Kb = np.asarray(K).reshape(-1, 3, 3)
    for ri in range(R):
        for p in range(rowptr[ri], rowptr[ri + 1]):
            rj = col[p]
            for I, L in targets(ri):
                T = L @ Kb[p]
                for J, Rm in targets(rj):
                    blk = T @ Rm.T
                    acc = rows[I].get(J)
                    rows[I][J] = blk if acc is None else acc + blk
    rp = np.zeros(n_red + 1, dtype=np.int32)
    cols, blocks = [], []
    for I in range(n_red):
        for J in sorted(rows[I]):
            cols.append(J)
            blocks.append(rows[I][J])
        rp[I + 1] = len(cols)
    sidx = np.full(n_nodes, -1, dtype=np.int32)
    for r in range(R):
        if red_of_row[r] >= 0:
            sidx[act_node[r]] = red_of_row[r]
    return rp, np.array(cols, dtype=np.int32), np.array(blocks).reshape(-1, 3, 3), sidx


def mixed_grid(widths, cells, jitter=0.0, seed=0, split=(1 / 3, 2 / 3), kinds=(ELEM_HEX, ELEM_WEDGE, ELEM_PYRAMID)):
    """A structured grid whose cells are hexes, wedges or pyramids by the x
    position of the cell (FemFactory's hex, wedge and pyramid grids share
    their node lattice): cells left of split[0] of the length take kinds[0],
    cells up to split[1] kinds[1], the rest kinds[2].  Returns the nodes, the
    per-element types and the concatenated connectivity (element order: the
    first kind's elements, then the second's, then the third's, each in its
    grid's order)."""
    xyz = None
    types, conn = [], []
    x0 = -widths[0] / 2
    bounds = [x0 + split[0] * widths[0], x0 + split[1] * widths[0]]
    for idx, kind in enumerate(kinds):
        g, c = grid(kind, widths, cells, jitter, seed)
        if xyz is None:
            xyz = g
        cx = g[c, 0].mean(axis=1)
        lo = -np.inf if idx == 0 else bounds[idx - 1]
        hi = np.inf if idx == 2 else bounds[idx]
        sel = (cx >= lo) & (cx < hi)
        types += [kind] * int(sel.sum())
        conn.append(c[sel].reshape(-1))
    return xyz, np.array(types, dtype=np.int32), np.concatenate(conn).astype(np.int32)
