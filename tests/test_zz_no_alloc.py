"""The allocation-free PCG entry point (b200fem_pcg_solve_noalloc) against
the engine's own PCG (b200fem_pcg_solve) on the same solve matrix, and
against the matrix itself (the residual of the result, formed in float64 by
numpy).

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
RESID = 1e-11      # ||S x - b|| / ||b|| of the result, formed on the host


def _bsr_matvec(rp, col, vals, x):
    n = rp.size - 1
    blocks = vals.reshape(-1, 3, 3)
    xr = x.reshape(n, 3)
    y = np.zeros((n, 3))
    rows = np.repeat(np.arange(n), np.diff(rp))
    np.add.at(y, rows, np.einsum("kij,kj->ki", blocks, xr[col]))
    return y.reshape(-1)


def _solve_matrix():
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
    return ms, rp.astype(np.int32), col.astype(np.int32), np.ascontiguousarray(S.reshape(-1))


def _call(lib, n_rows, d_rp, d_col, d_vals, d_b, d_x, tol, max_iter):
    import torch

    torch.cuda.synchronize()
    it = ctypes.c_int()
    rr = ctypes.c_double()
    status = lib.b200fem_pcg_solve_noalloc(n_rows, d_rp.data_ptr(), d_col.data_ptr(), d_vals.data_ptr(),
                                           d_b.data_ptr(), d_x.data_ptr(), tol, max_iter, None,
                                           ctypes.byref(it), ctypes.byref(rr))
    return status, it.value, rr.value


def test_noalloc_pcg_matches_engine_pcg(b200):
    import torch

    from artisynth_core_b200 import _lib as L

    ms, rp, col, S = _solve_matrix()
    n_rows = rp.size - 1
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_vals = torch.from_numpy(S).to(dev)
    lib = L.lib()
    rng = np.random.default_rng(11)
    x_prev = None
    for call in range(3):  # calls in a row share the static scratch
        b = rng.standard_normal(3 * n_rows)
        # the third call starts from a nonzero guess: the previous solution
        # plus noise (x is the initial guess on entry)
        x0 = np.zeros_like(b) if call < 2 else x_prev + 1e-3 * rng.standard_normal(b.size)
        x_ref, st = ms.pcg(b, x0=x0, tol=TOL, max_iter=5000)
        d_b = torch.from_numpy(b).to(dev)
        d_x = torch.from_numpy(x0.copy()).to(dev)
        status, it, rr = _call(lib, n_rows, d_rp, d_col, d_vals, d_b, d_x, TOL, 5000)
        assert status == L.OK, lib.b200fem_last_error(None)
        x = d_x.cpu().numpy()
        err = np.abs(x - x_ref).max() / np.abs(x_ref).max()
        assert err <= MATCH, (call, err)
        assert rr <= TOL and it > 0
        res = np.linalg.norm(_bsr_matvec(rp, col, S, x) - b) / np.linalg.norm(b)
        assert res <= RESID, (call, res)
        x_prev = x


def test_noalloc_no_converge_then_recovers(b200):
    """Two iterations at a tight tolerance run out (ERR_NO_CONVERGE, x holds
    an iterate), and the next full call on the same scratch still matches."""
    import torch

    from artisynth_core_b200 import _lib as L

    ms, rp, col, S = _solve_matrix()
    n_rows = rp.size - 1
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp).to(dev)
    d_col = torch.from_numpy(col).to(dev)
    d_vals = torch.from_numpy(S).to(dev)
    lib = L.lib()
    b = np.random.default_rng(5).standard_normal(3 * n_rows)
    d_b = torch.from_numpy(b).to(dev)
    d_x = torch.zeros(3 * n_rows, dtype=torch.float64, device=dev)
    status, it, rr = _call(lib, n_rows, d_rp, d_col, d_vals, d_b, d_x, 1e-14, 2)
    assert status == L.ERR_NO_CONVERGE, (status, lib.b200fem_last_error(None))
    assert np.all(np.isfinite(d_x.cpu().numpy()))
    d_x.zero_()
    status, it, rr = _call(lib, n_rows, d_rp, d_col, d_vals, d_b, d_x, TOL, 5000)
    assert status == L.OK, lib.b200fem_last_error(None)
    x_ref, _ = ms.pcg(b, tol=TOL, max_iter=5000)
    x = d_x.cpu().numpy()
    assert np.abs(x - x_ref).max() / np.abs(x_ref).max() <= MATCH
    res = np.linalg.norm(_bsr_matvec(rp, col, S, x) - b) / np.linalg.norm(b)
    assert res <= RESID


def test_noalloc_rejects_missing_diagonal(b200):
    """A row (neither the last nor empty) without its diagonal block is
    refused before the solve reads any block."""
    import torch

    from artisynth_core_b200 import _lib as L

    _, rp, col, S = _solve_matrix()
    n_rows = rp.size - 1
    r = n_rows // 2
    keep = np.ones(col.size, dtype=bool)
    p = rp[r] + int(np.searchsorted(col[rp[r]:rp[r + 1]], r))
    assert col[p] == r and rp[r + 1] - rp[r] > 1
    keep[p] = False
    col2 = col[keep]
    S2 = S.reshape(-1, 9)[keep].reshape(-1)
    rp2 = rp.copy()
    rp2[r + 1:] -= 1
    dev = torch.device("cuda:0")
    d_rp = torch.from_numpy(rp2).to(dev)
    d_col = torch.from_numpy(np.ascontiguousarray(col2)).to(dev)
    d_vals = torch.from_numpy(np.ascontiguousarray(S2)).to(dev)
    d_b = torch.ones(3 * n_rows, dtype=torch.float64, device=dev)
    d_x = torch.zeros(3 * n_rows, dtype=torch.float64, device=dev)
    lib = L.lib()
    status, _, _ = _call(lib, n_rows, d_rp, d_col, d_vals, d_b, d_x, TOL, 100)
    assert status == L.ERR_INVALID_ARG
    assert b"diagonal" in lib.b200fem_last_error(None)
    assert not d_x.any().item()  # the solve never ran


def test_noalloc_rejects_bad_sizes(b200):
    from artisynth_core_b200 import _lib as L

    lib = L.lib()
    it = ctypes.c_int()
    rr = ctypes.c_double()
    status = lib.b200fem_pcg_solve_noalloc(8193, 1, 1, 1, 1, 1, 1e-10, 10, None,
                                           ctypes.byref(it), ctypes.byref(rr))
    assert status == L.ERR_BUDGET
    assert b"B200FEM_NOALLOC_MAX_ROWS" in lib.b200fem_last_error(None)
    for n_rows, max_iter in ((0, 10), (10, 0), (-3, 10)):
        status = lib.b200fem_pcg_solve_noalloc(n_rows, 1, 1, 1, 1, 1, 1e-10, max_iter, None,
                                               ctypes.byref(it), ctypes.byref(rr))
        assert status == L.ERR_INVALID_ARG, (n_rows, max_iter, status)
