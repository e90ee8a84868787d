"""The allocation-free PCG entry point (b200fem_pcg_solve_noalloc) against
the engine's own PCG (b200fem_pcg_solve) on the same solve matrix.

The no-alloc entry point serves callers that cannot allocate device memory
(their device memory belongs to another allocator or pool, or they forbid
allocation after start-up): they pass device buffers for the matrix, b and
x, and the solver's working vectors come from a static device array.  This
file is collected last so that a failing run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12        # PCG tolerance of both solves
MATCH = 1e-9       # relative agreement required (as in the engine's own PCG test)


def test_noalloc_pcg_matches_engine_pcg(b200):
    import torch

    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200 import workloads as W
    from artisynth_core_b200.femmodel import MechSystemSolver, NeoHookeanMaterial

    wl = W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45), cells=(8, 3, 3))
    wl.build_mesh()
    m = wl.model()
    ms = MechSystemSolver(m, tol=TOL)
    x0, _ = m.getState()
    ms.backwardEuler(wl.h, 1)             # the engine's solve matrix S(x0)
    _, K = m.updateStressAndStiffness(x0)  # stiffness at the same x0 (S untouched)
    rp, col = m.getBlockPattern()
    sidx = m.getSolveIndices()
    mass = m.getNodeMasses()
    n_rows = rp.size - 1
    h, al, be = wl.h, wl.mass_damping, wl.stiffness_damping
    S = (h * h + h * be) * K
    act = np.zeros(n_rows, dtype=np.int64)
    act[sidx[sidx >= 0]] = np.nonzero(sidx >= 0)[0]
    for r in range(n_rows):
        p = rp[r] + int(np.searchsorted(col[rp[r]:rp[r + 1]], r))
        S[p] += (1.0 + h * al) * mass[act[r]] * np.eye(3)

    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp.astype(np.int32)).to(dev)
    d_col = torch.from_numpy(col.astype(np.int32)).to(dev)
    d_vals = torch.from_numpy(np.ascontiguousarray(S.reshape(-1))).to(dev)
    lib = L.lib()
    rng = np.random.default_rng(11)
    for call in range(2):  # two calls in a row share the static scratch
        b = rng.standard_normal(3 * n_rows)
        x_ref, st = ms.pcg(b, tol=TOL, max_iter=5000)
        d_b = torch.from_numpy(b).to(dev)
        d_x = torch.zeros(3 * n_rows, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        it = ctypes.c_int()
        rr = ctypes.c_double()
        status = lib.b200fem_pcg_solve_noalloc(n_rows, d_rp.data_ptr(), d_col.data_ptr(), d_vals.data_ptr(),
                                               d_b.data_ptr(), d_x.data_ptr(), TOL, 5000, None,
                                               ctypes.byref(it), ctypes.byref(rr))
        assert status == L.OK, lib.b200fem_last_error(None)
        x = d_x.cpu().numpy()
        err = np.abs(x - x_ref).max() / np.abs(x_ref).max()
        assert err <= MATCH, (call, err)
        assert rr.value <= TOL and it.value > 0


def test_noalloc_rejects_oversize(b200):
    from artisynth_core_b200 import _lib as L

    lib = L.lib()
    it = ctypes.c_int()
    rr = ctypes.c_double()
    status = lib.b200fem_pcg_solve_noalloc(8193, 1, 1, 1, 1, 1, 1e-10, 10, None,
                                           ctypes.byref(it), ctypes.byref(rr))
    assert status == L.ERR_BUDGET
    assert b"B200FEM_NOALLOC_MAX_ROWS" in lib.b200fem_last_error(None)
