"""FEM nodes attached to active frames (PointFrameAttachment): the reduced
stiffness P^T K P of b200fem_update_stress_stiffness.

* the reduced pattern, CRS indices, slot map and solve indices bit-exact
  with the oracle's reduction (oracle.reduce_attachments), and the reduced
  blocks within the parity bar (1e-10 of the largest entry);
* the reference's own element kernel with its master-slave scatter
  (addMaterialStiffness3Element_launch with per-node dimensions and
  transforms, cudssBridgeKernels.cu:381-449 and scatterReduced3Block
  :325-365), fed the oracle's integration-point data, gives the same scalar
  CRS values;
* BackwardEuler steps of a model with attachments are refused.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import (MechSystemSolver, MooneyRivlinMaterial, NeoHookeanMaterial,
                                          StVenantKirchoffMaterial)

from helpers import deformed, oracle_model, rel_err


def attachments(rest, x):
    """Two frames: the x-max face of the beam on frame 0 (an end cap) and
    the top nodes of the middle cross-section on frame 1.  H = [I; [r]x]
    with r the node's offset from its frame's origin at positions x (the
    master block of a point on a frame whose velocity is the world twist
    [v; w]: v_point = v + w x r)."""
    xmax = rest[:, 0].max()
    cap = np.nonzero(rest[:, 0] >= xmax - 1e-9)[0]
    on_top = rest[:, 2] >= rest[:, 2].max() - 1e-9  # boundary nodes are not jittered
    xs = np.unique(np.round(rest[on_top, 0], 6))
    mid = xs[len(xs) // 2]
    top = np.nonzero((np.abs(rest[:, 0] - mid) < 1e-6) & on_top)[0]
    nodes = np.concatenate([cap, top]).astype(np.int32)
    frames = np.concatenate([np.zeros(cap.size, np.int32), np.ones(top.size, np.int32)])
    origin = [x[cap].mean(axis=0), x[top].mean(axis=0)]
    H = np.zeros((nodes.size, 6, 3))
    for k, n in enumerate(nodes):
        r = x[n] - origin[frames[k]]
        H[k, 0:3] = np.eye(3)
        H[k, 3:6] = np.array([[0, -r[2], r[1]], [r[2], 0, -r[0]], [-r[1], r[0], 0]])
    return 2, nodes, frames, H


def _case(name):
    return {
        "neohookean_tet": lambda: W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33), cells=(5, 2, 2)),
        "neohookean_hex": lambda: W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45), cells=(5, 2, 2)),
        "stvk_wedge": lambda: W.small_wedge_beam(StVenantKirchoffMaterial(5e4, 0.3), cells=(5, 2, 2)),
        "mooneyrivlin_hex_element": lambda: W.small_hex_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370),
                                                             cells=(5, 2, 2)),
    }[name]()


def _reduced_oracle(oracle, wl, x, att):
    om = oracle_model(oracle, wl)
    _, K, _ = om.update_stress_stiffness(x)
    rp, col = om.pattern()
    sidx = om.solve_index()
    act = np.argsort(np.where(sidx >= 0, sidx, 1 << 30))[: om.nact]
    n_frames, nodes, frames, H = att
    return om, oracle.reduce_attachments(rp, col, K, act, len(wl.rest), n_frames, nodes, frames, H)


def _crs(rp, col, blocks):
    """Full-partition scalar CRS (row offsets, columns, values)."""
    ro, ci, vals = [0], [], []
    for r in range(rp.size - 1):
        for i in range(3):
            for p in range(rp[r], rp[r + 1]):
                for c in range(3):
                    ci.append(3 * col[p] + c)
                    vals.append(blocks[p][i, c])
            ro.append(len(ci))
    return np.array(ro), np.array(ci), np.array(vals)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["neohookean_tet", "neohookean_hex", "stvk_wedge", "mooneyrivlin_hex_element"])
def test_reduced_stiffness_vs_oracle(b200, oracle, name):
    wl = _case(name)
    wl.build_mesh()
    x = deformed(wl.rest, seed=5)
    att = attachments(wl.rest, x)
    m = wl.model()
    m.setFrameAttachments(*att)
    f, K, crs = m.updateStressAndStiffness(x, want_crs=True)
    om, (rrp, rcol, rK, rsidx) = _reduced_oracle(oracle, wl, x, att)
    rp, col = m.getBlockPattern()
    assert np.array_equal(rp, rrp) and np.array_equal(col, rcol)
    assert np.array_equal(m.getSolveIndices(), rsidx)
    assert m.sizes()["n_active"] == rp.size - 1
    assert rel_err(K, rK) <= 1e-10, rel_err(K, rK)
    ro, ci = m.getCRSIndices(L.PART_FULL)
    oro, oci, ovals = _crs(rrp, rcol, rK)
    assert np.array_equal(ro, oro) and np.array_equal(ci, oci)
    assert rel_err(crs, ovals) <= 1e-10
    slots = m.createCrsBlockSlotMap(L.PART_FULL)
    assert np.array_equal(crs[slots], K.reshape(-1))
    # the forces stay per node (the reduction of forces belongs to the step)
    of, _, _ = om.update_stress_stiffness(x)
    assert rel_err(f, of) <= 1e-10
    with pytest.raises(L.B200FemError) as ei:
        MechSystemSolver(m, tol=1e-10).backwardEuler(wl.h, 1)
    assert ei.value.status == L.ERR_UNSUPPORTED


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["neohookean_tet", "neohookean_hex"])
def test_reduced_stiffness_vs_reference_kernel(b200, oracle, name):
    """addMaterialStiffness3Element_launch (one CTA per element, FP64
    atomics) with nodeDims 3 / 6 and nodeTransforms I / H, fed the oracle's
    point data, against the engine's reduced CRS values."""
    import torch
    from oracle import oracle as O

    R = O.ref_kernels()
    if R is None:
        pytest.skip("reference kernels not built (make -C oracle ref needs the reference tree)")
    wl = _case(name)
    wl.build_mesh()
    x = deformed(wl.rest, seed=5)
    att = attachments(wl.rest, x)
    n_frames, nodes, frames, H = att
    m = wl.model()
    m.setFrameAttachments(*att)
    _, _, crs = m.updateStressAndStiffness(x, want_crs=True)
    slots_red = m.createCrsBlockSlotMap(L.PART_FULL)
    rp, col = m.getBlockPattern()
    rsidx = m.getSolveIndices()
    n_free = int((rsidx >= 0).sum())
    om = oracle_model(oracle, wl)
    att_of = {int(n): k for k, n in enumerate(nodes)}

    def target(n):
        """reduced block rows of node n (one free, two for a frame), or None"""
        if n in att_of:
            f = int(frames[att_of[n]])
            return [n_free + 2 * f, n_free + 2 * f + 1]
        return [int(rsidx[n])] if rsidx[n] >= 0 else None

    def slot(I, J, i, c):
        p = rp[I] + int(np.searchsorted(col[rp[I]:rp[I + 1]], J))
        assert col[p] == J
        return slots_red[9 * p + 3 * i + c]

    ne, nen = wl.conn.shape
    nip = om.num_ip()
    counts, noffs, poffs, ioffs, goffs = [], [], [0], [0], []
    pairs, bslots, dims, trans, grads, Ds, sigs, dvs = [], [], [], [], [], [], [], []
    for e in range(ne):
        nd = wl.conn[e]
        counts.append(nen)
        noffs.append(len(dims))
        goffs.append(len(grads) // 3)
        for a in range(nen):
            n = int(nd[a])
            if n in att_of:
                dims.append(6)
                trans.extend(H[att_of[n]].reshape(-1))
            else:
                dims.append(3)
                trans.extend(np.concatenate([np.eye(3).reshape(-1), np.zeros(9)]))
        npair = 0
        for a in range(nen):
            Ta = target(int(nd[a]))
            if Ta is None:
                continue
            for b in range(nen):
                Tb = target(int(nd[b]))
                if Tb is None:
                    continue
                pairs.extend([a, b])
                s36 = np.full(36, -1, dtype=np.int64)
                rd, cd = 3 * len(Ta), 3 * len(Tb)
                for r in range(rd):
                    for c in range(cd):
                        s36[r * cd + c] = slot(Ta[r // 3], Tb[c // 3], r % 3, c % 3)
                bslots.extend(s36)
                npair += 1
        poffs.append(poffs[-1] + npair)
        for k in range(nip):
            g, dv, sig, D = om.ip_data(x, e, k)
            grads.extend(g.reshape(-1))
            Ds.extend(D.reshape(-1))
            sigs.extend(sig)
            dvs.append(dv)
        ioffs.append(ioffs[-1] + nip)
    iarr = lambda v: np.ascontiguousarray(np.array(v, dtype=np.int32))
    darr = lambda v: np.ascontiguousarray(np.array(v, dtype=np.float64))
    arrs_i = [iarr(counts), iarr(noffs), iarr(poffs), iarr(ioffs), iarr(goffs), iarr(pairs), iarr(bslots), iarr(dims)]
    arrs_d = [darr(trans), darr(grads), darr(Ds), darr(sigs), darr(dvs)]
    nnz = crs.size
    # every index the kernel follows stays inside its array: checked before the launch
    bs = arrs_i[6]
    assert bs.size == 36 * (arrs_i[5].size // 2) and bs.max() < nnz
    assert arrs_d[0].size == 18 * arrs_i[7].size and arrs_d[1].size == 3 * ne * nip * nen
    assert arrs_d[2].size == 36 * ne * nip and arrs_d[4].size == ne * nip
    dev = torch.device("cuda:0")
    t = [torch.from_numpy(a).to(dev) for a in arrs_i + arrs_d]
    out = torch.zeros(nnz, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    R.addMaterialStiffness3Element_launch(ne, *(a.data_ptr() for a in t), 1.0, out.data_ptr(), stream)
    torch.cuda.synchronize()
    ref = out.cpu().numpy()
    assert rel_err(crs, ref) <= 1e-10, rel_err(crs, ref)
