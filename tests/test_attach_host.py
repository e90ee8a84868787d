"""The oracle's master-slave reduction (oracle.reduce_attachments) against
the dense product P^T K P, on the CPU: P maps the reduced velocities (free
nodes, then a 6-vector per frame) to the extended ones (free and attached
nodes), v_s = H_s^T [v_F; w_F] for an attached node."""
import numpy as np

from helpers import deformed
from test_gpu_attach import attachments


def test_reduction_equals_dense_ptkp(oracle):
    xyz, conn = oracle.grid(0, (1.0, 0.4, 0.4), (5, 2, 2), jitter=0.04, seed=3)
    fixed = (xyz[:, 0] <= -0.5 + 1e-9).astype(np.int32)
    om = oracle.OracleModel(0, xyz, conn, fixed, 1, [5e4, 0.33], 1000.0)
    x = deformed(xyz, seed=2)
    _, K, _ = om.update_stress_stiffness(x)
    rp, col = om.pattern()
    sidx = om.solve_index()
    act = np.argsort(np.where(sidx >= 0, sidx, 1 << 30))[: om.nact]
    n_frames, nodes, frames, H = attachments(xyz, x)
    rrp, rcol, rK, rsidx = oracle.reduce_attachments(rp, col, K, act, len(xyz), n_frames, nodes, frames, H)
    R = om.nact
    Kd = np.zeros((3 * R, 3 * R))
    for r in range(R):
        for p in range(rp[r], rp[r + 1]):
            Kd[3 * r:3 * r + 3, 3 * col[p]:3 * col[p] + 3] = K[p]
    n_free = int((rsidx >= 0).sum())
    nred = 3 * n_free + 6 * n_frames
    P = np.zeros((3 * R, nred))
    att = {int(n): k for k, n in enumerate(nodes)}
    for r in range(R):
        n = act[r]
        if n in att:
            k = att[n]
            f = frames[k]
            P[3 * r:3 * r + 3, 3 * n_free + 6 * f:3 * n_free + 6 * f + 6] = H[k].T
        else:
            P[3 * r:3 * r + 3, 3 * rsidx[n]:3 * rsidx[n] + 3] = np.eye(3)
    Kr = P.T @ Kd @ P
    Rd = np.zeros_like(Kr)
    for r in range(nred // 3):
        for p in range(rrp[r], rrp[r + 1]):
            Rd[3 * r:3 * r + 3, 3 * rcol[p]:3 * rcol[p] + 3] = rK[p]
    assert np.abs(Rd - Kr).max() <= 1e-12 * np.abs(Kr).max()
    assert np.abs(Rd - Rd.T).max() <= 1e-12 * np.abs(Rd).max()
    # every frame's rows couple to themselves (a 6x6 block of 2 x 2 blocks)
    for f in range(n_frames):
        r0 = n_free + 2 * f
        for r in (r0, r0 + 1):
            assert r0 in rcol[rrp[r]:rrp[r + 1]] and r0 + 1 in rcol[rrp[r]:rrp[r + 1]]
