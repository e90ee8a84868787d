"""The reference's own device assembly kernel as a second checker.

The reference's device assembly (FemModel3d.addMaterialStiffness3CrsValue-
Contributions, FemModel3d.java:4613-4936) hands one descriptor per block
contribution to addMaterialStiffness3Kernel (cudssBridgeKernels.cu:164-242):
the current shape gradients g_i, g_j and dv of one integration point, the
material tangent D (6x6) and Cauchy stress sigma there, and the nine CRS value
slots of block (i, j).  The kernel forms B_i^T D B_j dv + (g_i . sigma g_j) dv I
and adds it into the CRS values (FP64 atomics).

That kernel, compiled from the reference source into oracle/_ref/ (`make -C
oracle ref`), is fed the oracle's integration-point data for every (element,
point, node pair) of NeoHookean tet, hex, wedge and pyramid and
StVenantKirchhoff hex and pyramid beams at deformed positions.  Its
CRS values must equal
* the engine's full-partition CRS export (b200fem_update_stress_stiffness)
  within the parity bar, 1e-10 of the largest entry, and
* the oracle's own assembly within 1e-12 (same arithmetic, summation order
  differs through the atomics).
For MooneyRivlin hex and wedge beams whose AUTO soft incompressibility
resolves to ELEMENT, the descriptors carry the element pressure and the reference's
addDilationalStiffness3ElementKernel (:658-723) adds Rinv c_i c_j^T from the
element constraint vectors.
This pins the element-tangent assembly (FemUtilities.addMaterialStiffness /
addGeometricStiffness, FemUtilities.java:78-144) to the reference's code,
not only to its restatement.

The linear rest stiffness goes through addLinearElasticStiffness3ElementKernel
(cudssBridgeKernels.cu:470-516), which builds D from (E, nu) itself
(fillLinearElasticD) and sums B_i^T D B_j dv over the integration points of
each element's node pairs, from rest shape gradients and dv: it must equal the
engine's stiffness of a non-corotated LinearMaterial (K = K0 at any position)
within 1e-10.
"""
import numpy as np
import pytest

from artisynth_core_b200.femmodel import (LinearMaterial, MooneyRivlinMaterial, NeoHookeanMaterial,
                                          StVenantKirchoffMaterial)
from artisynth_core_b200 import workloads as W
from oracle import oracle as O

from helpers import deformed, oracle_model, rel_err

pytestmark = pytest.mark.gpu


def _ref_lib():
    R = O.ref_kernels()
    if R is None:
        pytest.skip("reference kernels not built (make -C oracle ref needs the reference tree)")
    return R


def _descriptors(om, wl, x):
    """Per block contribution: slots (9), g_i, g_j, D (36), sigma (6), dv."""
    sidx = om.solve_index()
    rp, col = om.pattern()
    _, _, slots = om.crs(0)
    nen = wl.conn.shape[1]
    S, GI, GJ, DD, SG, DV = [], [], [], [], [], []
    for e in range(wl.conn.shape[0]):
        for k in range(om.num_ip()):
            g, dv, sig, D = om.ip_data(x, e, k)
            for a in range(nen):
                ra = sidx[wl.conn[e, a]]
                if ra < 0:
                    continue
                for b in range(nen):
                    rb = sidx[wl.conn[e, b]]
                    if rb < 0:
                        continue
                    p = rp[ra] + int(np.searchsorted(col[rp[ra]:rp[ra + 1]], rb))
                    assert col[p] == rb
                    S.append(slots[9 * p:9 * p + 9])
                    GI.append(g[a])
                    GJ.append(g[b])
                    DD.append(D.reshape(-1))
                    SG.append(sig)
                    DV.append(dv)
    return (np.ascontiguousarray(np.array(S, dtype=np.int32).reshape(-1)),
            np.ascontiguousarray(np.array(GI).reshape(-1)), np.ascontiguousarray(np.array(GJ).reshape(-1)),
            np.ascontiguousarray(np.array(DD).reshape(-1)), np.ascontiguousarray(np.array(SG).reshape(-1)),
            np.ascontiguousarray(np.array(DV)))


def _reference_crs(R, desc, nnz, dilational=None):
    import torch
    slots, gi, gj, D, sig, dv = desc
    nb = dv.size
    # every array the kernel indexes is sized for nb blocks, and every slot
    # lies inside the CRS value array: checked before the launch
    assert slots.size == 9 * nb and gi.size == 3 * nb and gj.size == 3 * nb
    assert D.size == 36 * nb and sig.size == 6 * nb
    assert slots.min() >= 0 and slots.max() < nnz
    dev = torch.device("cuda:0")
    t = [torch.from_numpy(a).to(dev) for a in (slots, gi, gj, D, sig, dv)]
    crs = torch.zeros(nnz, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    R.addMaterialStiffness3_launch(nb, *(a.data_ptr() for a in t), 1.0, crs.data_ptr(), stream)
    torch.cuda.synchronize()
    if dilational is not None:
        _add_reference_dilational(R, dilational, crs, nnz)
    return crs.cpu().numpy()


def _dilational_arrays(om, wl, x):
    """Arrays of addDilationalStiffness3Element_launch for ELEMENT soft
    incompressibility with one pressure value per element: constraint
    vectors c_i = sum_k GNx_i dv (FemUtilities.addToIncompressConstraints)
    and Rinv = effectiveModulus(kappa, V/V0) / V0 (computePressuresAndRinv,
    FemModel3d.java:2517-2591); every node free (dimension 3, identity
    transform, the block's nine slots first in its 36-slot record)."""
    sidx = om.solve_index()
    rp, col = om.pattern()
    _, _, slots = om.crs(0)
    ne, nen = wl.conn.shape
    mat = wl.material
    V0 = om.rest_volumes()
    cons = np.zeros((ne, nen, 3))
    rinv = np.zeros(ne)
    pair_off = [0]
    pairs, bslots = [], []
    for e in range(ne):
        V = 0.0
        for k in range(om.num_ip()):
            g, dv, _, _ = om.ip_data(x, e, k)
            cons[e] += g * dv
            V += dv
        J = V / V0[e]
        keff = mat.kappa if mat.bulk_potential == 0 else mat.kappa * (1 - np.log(J)) / (J * J)
        rinv[e] = keff / V0[e]
        for a in range(nen):
            ra = sidx[wl.conn[e, a]]
            if ra < 0:
                continue
            for b in range(nen):
                rb = sidx[wl.conn[e, b]]
                if rb < 0:
                    continue
                p = rp[ra] + int(np.searchsorted(col[rp[ra]:rp[ra + 1]], rb))
                assert col[p] == rb
                pairs.append((a, b))
                rec = np.full(36, -1, dtype=np.int32)
                rec[:9] = slots[9 * p:9 * p + 9]
                bslots.append(rec)
        pair_off.append(len(pairs))
    eye = np.zeros(18)
    eye[[0, 4, 8]] = 1.0
    return dict(counts=np.full(ne, nen, dtype=np.int32), node_off=np.arange(ne, dtype=np.int32) * nen,
                pcount=np.ones(ne, dtype=np.int32), pair_off=np.array(pair_off, dtype=np.int32),
                cons_off=np.arange(ne, dtype=np.int32) * nen, rinv_off=np.arange(ne, dtype=np.int32),
                pairs=np.array(pairs, dtype=np.int32).reshape(-1), slots=np.array(bslots, dtype=np.int32).reshape(-1),
                dims=np.full(ne * nen, 3, dtype=np.int32), transforms=np.tile(eye, ne * nen),
                cons=cons.reshape(-1), rinv=rinv)


def _add_reference_dilational(R, arr, crs_dev, nnz):
    import torch
    ne = arr["counts"].size
    npair = arr["pair_off"][-1]
    # the kernel's indexing, checked before the launch
    assert arr["pairs"].size == 2 * npair and arr["slots"].size == 36 * npair
    assert arr["slots"][arr["slots"] >= 0].max() < nnz
    assert arr["dims"].size == arr["cons"].size // 3 == ne * arr["counts"][0]
    assert arr["transforms"].size == 18 * arr["dims"].size and arr["rinv"].size == ne
    dev = torch.device("cuda:0")
    order = ("counts", "node_off", "pcount", "pair_off", "cons_off", "rinv_off", "pairs", "slots", "dims",
             "transforms", "cons", "rinv")
    t = [torch.from_numpy(np.ascontiguousarray(arr[k])).to(dev) for k in order]
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    R.addDilationalStiffness3Element_launch(ne, *(a.data_ptr() for a in t), 1.0, crs_dev.data_ptr(), stream)
    torch.cuda.synchronize()


@pytest.mark.parametrize("case", ["neohookean_tet", "neohookean_hex", "stvk_hex", "mooneyrivlin_hex_element",
                                  "neohookean_wedge", "neohookean_pyramid", "stvk_pyramid",
                                  "mooneyrivlin_wedge_element", "neohookean_quadtet",
                                  "mooneyrivlin_quadtet_element", "neohookean_quadhex"])
def test_reference_kernel_assembles_engine_stiffness(b200, oracle, case):
    R = _ref_lib()
    if case == "neohookean_tet":
        wl = W.small_tet_beam(NeoHookeanMaterial(5e4, 0.33))
    elif case == "neohookean_hex":
        wl = W.small_hex_beam(NeoHookeanMaterial(5e4, 0.45))
    elif case == "stvk_hex":
        wl = W.small_hex_beam(StVenantKirchoffMaterial(5e4, 0.3))
    elif case == "neohookean_wedge":
        wl = W.small_wedge_beam(NeoHookeanMaterial(5e4, 0.45))
    elif case == "neohookean_pyramid":
        wl = W.small_pyramid_beam(NeoHookeanMaterial(5e4, 0.45))
    elif case == "stvk_pyramid":
        wl = W.small_pyramid_beam(StVenantKirchoffMaterial(5e4, 0.3))
    elif case == "neohookean_quadhex":
        wl = W.small_quadhex_beam(NeoHookeanMaterial(5e4, 0.45))
    elif case == "neohookean_quadtet":
        wl = W.small_quadtet_beam(NeoHookeanMaterial(5e4, 0.45))
    elif case == "mooneyrivlin_quadtet_element":
        wl = W.small_quadtet_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370))
    elif case == "mooneyrivlin_wedge_element":
        # AUTO resolves to ELEMENT: 32 wedges <= 36 active nodes
        wl = W.small_wedge_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370))
    else:
        wl = W.small_hex_beam(MooneyRivlinMaterial(1037, 120, 0, 486, 0, 10370))
    wl.build_mesh()
    om = oracle_model(oracle, wl)
    x = deformed(wl.rest, seed=5)
    _, oK, ninv = om.update_stress_stiffness(x)
    assert ninv == 0
    m = wl.model()
    _, K, crs = m.updateStressAndStiffness(x, want_crs=True)
    dil = _dilational_arrays(om, wl, x) if om.incomp == O.INCOMP_ELEMENT else None
    ref = _reference_crs(R, _descriptors(om, wl, x), crs.size, dil)
    _, _, slots = om.crs(0)
    ocrs = np.zeros(crs.size)
    ocrs[slots] = oK.reshape(-1)
    assert rel_err(ocrs, ref) <= 1e-12, rel_err(ocrs, ref)
    assert rel_err(crs, ref) <= 1e-10, rel_err(crs, ref)


def _linear_element_arrays(om_geom, wl, E, nu):
    """Per-element arrays of addLinearElasticStiffness3Element_launch from the
    rest kinematics (shape gradients, dv) of the oracle model om_geom."""
    sidx = om_geom.solve_index()
    rp, col = om_geom.pattern()
    _, _, slots = om_geom.crs(0)
    ne, nen = wl.conn.shape
    nip = om_geom.num_ip()
    counts = np.full(ne, nen, dtype=np.int32)
    pair_off = [0]
    pairs, bslots = [], []
    grads = np.zeros((ne, nip, nen, 3))
    dvs = np.zeros((ne, nip))
    for e in range(ne):
        for k in range(nip):
            g, dv, _, _ = om_geom.ip_data(wl.rest, e, k)
            grads[e, k] = g
            dvs[e, k] = dv
        for a in range(nen):
            ra = sidx[wl.conn[e, a]]
            if ra < 0:
                continue
            for b in range(nen):
                rb = sidx[wl.conn[e, b]]
                if rb < 0:
                    continue
                p = rp[ra] + int(np.searchsorted(col[rp[ra]:rp[ra + 1]], rb))
                assert col[p] == rb
                pairs.append((a, b))
                bslots.append(slots[9 * p:9 * p + 9])
        pair_off.append(len(pairs))
    ip_off = np.arange(ne + 1, dtype=np.int32) * nip
    grad_off = np.arange(ne, dtype=np.int32) * nip * nen
    params = np.tile(np.array([E, nu]), ne)
    return (counts, np.array(pair_off, dtype=np.int32), ip_off, grad_off,
            np.array(pairs, dtype=np.int32).reshape(-1), np.array(bslots, dtype=np.int32).reshape(-1),
            params, grads.reshape(-1), dvs.reshape(-1))


@pytest.mark.parametrize("case", ["tet", "hex", "wedge", "pyramid", "quadtet", "quadhex"])
def test_reference_kernel_assembles_linear_rest_stiffness(b200, oracle, case):
    import torch
    R = _ref_lib()
    E, nu = 5e4, 0.33
    beam = {"tet": W.small_tet_beam, "hex": W.small_hex_beam, "wedge": W.small_wedge_beam,
            "pyramid": W.small_pyramid_beam, "quadtet": W.small_quadtet_beam,
            "quadhex": W.small_quadhex_beam}[case]
    wl = beam(LinearMaterial(E, nu, False))
    geom = beam(NeoHookeanMaterial(E, nu))
    wl.build_mesh()
    geom.build_mesh()
    assert np.array_equal(wl.rest, geom.rest) and np.array_equal(wl.conn, geom.conn)
    om_geom = oracle_model(oracle, geom)
    arrs = _linear_element_arrays(om_geom, wl, E, nu)
    counts, pair_off, ip_off, grad_off, pairs, bslots, params, grads, dvs = arrs
    m = wl.model()
    _, K, crs = m.updateStressAndStiffness(deformed(wl.rest, seed=5), want_crs=True)
    ne, nen = wl.conn.shape
    nip = om_geom.num_ip()
    # the kernel's indexing, checked before the launch: pair lists, local
    # node indices, gradient and dv offsets, CRS slots
    assert pair_off[-1] * 2 == pairs.size and pair_off[-1] * 9 == bslots.size
    assert pairs.min() >= 0 and pairs.max() < nen
    assert grads.size == 3 * ne * nip * nen and dvs.size == ne * nip and ip_off[-1] == dvs.size
    assert bslots.min() >= 0 and bslots.max() < crs.size
    dev = torch.device("cuda:0")
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev)
         for a in (counts, pair_off, ip_off, grad_off, pairs, bslots, params, grads, dvs)]
    out = torch.zeros(crs.size, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream(dev).cuda_stream
    R.addLinearElasticStiffness3Element_launch(ne, *(a.data_ptr() for a in t), 1.0, out.data_ptr(), stream)
    torch.cuda.synchronize()
    ref = out.cpu().numpy()
    assert rel_err(crs, ref) <= 1e-10, rel_err(crs, ref)
