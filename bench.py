"""Benchmark: BackwardEuler steps/s of the NeoHookean hex beam (40x10x10
hexes, 8 Gauss points, 4,961 nodes, 14,520 active DOF, PCG to 1e-10) on
B200, next to the CPU oracle on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

One step = one BackwardEuler step (element kernel, block gather, RHS, PCG,
state update) on device-resident state.  The model's working set (~30 MB)
fits in L2, so a 256 MB buffer is written between timed steps to flush L2.
Multi-GPU runs are independent replicas (one model per rank, weak scaling):
the path has no cross-model exchange.

On one GPU the line also carries the two other forms of the path:
  "batched" -- 256 uneven NeoHookean tet beams in one pack (mixed FP32/FP64,
               20 steps), model-steps/s next to the plain FP64 drop-in
               stepping the models one at a time, and the position error
               against that FP64 run;
  "served"  -- a Poisson stream of 10-step requests (2000/s, 60 s) over a
               pool of 512 beams with continuous batching and a 60 GB
               device-memory budget: p50/p99 latency, throughput, error.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FEM BackwardEuler steps/s"
UNIT = "steps/s"


def algorithmic_bytes(wl, nnzb, n_active):
    """Bytes per unit of work (per launch) used for the roofline.

    assembly (element + gather + RHS kernels), one BackwardEuler system:
      24 N (x read) + 4 nen E (connectivity) + 72 nip E (rest invJ0)
      + 4 nen^2 E (scatter map) + 72 nnzb (S written) + 24 N (f / b)
    PCG iteration:
      76 nnzb (S + block column) + 4 (Na + 1) (row offsets)
      + 24 Na (x) + 24 Na (y) + 72 Na (block-Jacobi inverse) + 9 * 24 Na
    """
    N = wl.rest.shape[0]
    E = wl.conn.shape[0]
    nen = wl.conn.shape[1]
    nip = 8 if nen == 8 else 1
    asm = 24 * N + 4 * nen * E + 72 * nip * E + 4 * nen * nen * E + 72 * nnzb + 24 * N
    it = 76 * nnzb + 4 * (n_active + 1) + 48 * n_active + 72 * n_active + 9 * 24 * n_active
    return asm, it


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.index)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(n):
    if n <= 1 or "RANK" not in os.environ:
        return None, 0, 1, 0
    import datetime

    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist, dist.get_rank(), dist.get_world_size(), local


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def oracle_mesher(elem_type, widths, cells, jitter, seed):
    """The oracle's own grid factory and jitter (bit-identical to the
    library's): the CPU legs build their meshes without loading the
    library."""
    from oracle import oracle as O
    O.build()
    return O.grid(elem_type, widths, cells, jitter, seed)


def cpu_info():
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def cpu_oracle_protocol(wl, threads, runs=5, warmup=3, budget_s=8.0, max_k=50):
    """Times the CPU oracle (FP64 restatement of the Java path; Jacobi-PCG to
    the workload tolerance) on `threads` host threads: `warmup` untimed
    steps, then `runs` timed runs of k consecutive BackwardEuler steps (k
    sized from the warm-up so that the runs take about budget_s together);
    returns the median steps/s over the runs, the runs, k and the threads
    used."""
    from oracle import oracle as O
    O.build()
    used = O.set_threads(threads)
    om = O.OracleModel(wl.elem_type, wl.rest, wl.conn, wl.fixed, wl.material.kind, wl.material.params(),
                       wl.density)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    fext = wl.fext if wl.traction is not None else None

    def step():
        st, _, _ = om.be_step(wl.h, x, v, alpha=wl.mass_damping, beta=wl.stiffness_damping, gravity=wl.gravity,
                              fext=fext, tol=wl.tol)
        return st

    t0 = time.perf_counter()
    for _ in range(warmup):
        step()
    tw = (time.perf_counter() - t0) / max(warmup, 1)
    k = int(max(1, min(max_k, budget_s / runs / max(tw, 1e-6))))
    rates = []
    for _ in range(runs):
        t0 = time.perf_counter()
        for _ in range(k):
            step()
        rates.append(k / (time.perf_counter() - t0))
    del om
    return statistics.median(rates), rates, k, used


def cpu_baseline_entry(wl, label, budget_s=8.0, runs=5, warmup=3):
    """Both CPU variants of the baseline protocol: single thread (the Java
    loop order) and OpenMP on every host core; `value` is the all-cores
    median."""
    allc = os.cpu_count() or 1
    v1, r1, k1, _ = cpu_oracle_protocol(wl, 1, runs=runs, warmup=warmup, budget_s=budget_s)
    va, ra, ka, used = cpu_oracle_protocol(wl, allc, runs=runs, warmup=warmup, budget_s=budget_s)
    out = {"value": va, "unit": UNIT, "cores": used, "kind": "port",
           "sample": f"median of {runs} runs of {ka} consecutive BackwardEuler steps of the {label} after "
                     f"{warmup} warm-up steps (FP64 oracle, Jacobi-PCG {wl.tol:g}, OpenMP on {used} threads)",
           "runs": ra,
           "single_thread": {"value": v1, "unit": UNIT, "cores": 1, "runs": r1,
                             "sample": f"median of {runs} runs of {k1} steps after {warmup} warm-up steps"}}
    out.update(cpu_info())
    return out


def run_reference(args):
    dist, rank, world, local = dist_setup(args.gpus)
    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return
    from artisynth_core_b200 import workloads as W
    wl = W.neohookean_hex_beam().build_mesh(mesher=oracle_mesher)
    threads = os.cpu_count() or 1
    from oracle import oracle as O
    O.build()
    used = O.set_threads(threads)
    om = O.OracleModel(wl.elem_type, wl.rest, wl.conn, wl.fixed, wl.material.kind, wl.material.params(),
                       wl.density)
    x = wl.rest.copy()
    v = np.zeros_like(x)
    for _ in range(args.warmup):
        om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, fext=wl.fext, tol=wl.tol)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        om.be_step(wl.h, x, v, alpha=wl.mass_damping, gravity=wl.gravity, fext=wl.fext, tol=wl.tol)
    dt = time.perf_counter() - t0
    val = args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": dict(wl.describe(), solver="Jacobi-PCG 1e-10"),
        "cpu_baseline": dict({"value": val, "unit": UNIT, "cores": used, "kind": "port",
                              "sample": f"{args.steps} consecutive BackwardEuler steps of the 40x10x10 hex beam "
                                        f"after {args.warmup} warm-up steps (FP64 oracle, Jacobi-PCG 1e-10, "
                                        f"OpenMP on {used} threads)"}, **cpu_info()),
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    try:
        line["reference_device_kernel"] = time_reference_kernel(O, om, wl, x)
    except Exception as exc:  # no GPU, or the reference kernels were not built
        line["reference_device_kernel"] = {"unavailable": f"{type(exc).__name__}: {exc}"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def time_reference_kernel(O, om, wl, x, warmup=3, launches=20):
    """The reference's own device assembly of the stiffness,
    addMaterialStiffness3Element_launch (cudssBridgeKernels.cu:381-449:
    one CTA per element, FP64 atomicAdd of B_i^T D B_j dv + (g_i . sigma g_j)
    dv I into the CRS values), built from the reference source into
    oracle/_ref, timed with CUDA events on the hex beam at the positions x.
    Its per-point D, sigma, shape gradients and dv come from the host (here
    the oracle), as the reference's Java path hands them over: the kernel time
    covers the block products and the scatter only."""
    import torch
    R = O.ref_kernels()
    if R is None or not torch.cuda.is_available():
        raise RuntimeError("reference kernels not built or no CUDA device")
    ne, nen = wl.conn.shape
    nip = om.num_ip()
    sidx = om.solve_index()
    rp, col = om.pattern()
    _, _, slots = om.crs(0)
    nrow = rp.size - 1
    blk_row = np.repeat(np.arange(nrow), np.diff(rp))
    keys = blk_row.astype(np.int64) * nrow + col
    grads = np.zeros((ne, nip, nen, 3))
    Ds = np.zeros((ne, nip, 36))
    sigs = np.zeros((ne, nip, 6))
    dvs = np.zeros((ne, nip))
    for e in range(ne):
        for k in range(nip):
            g, dv, sig, D = om.ip_data(x, e, k)
            grads[e, k] = g
            Ds[e, k] = D.reshape(-1)
            sigs[e, k] = sig
            dvs[e, k] = dv
    a_idx, b_idx = np.meshgrid(np.arange(nen), np.arange(nen), indexing="ij")
    pairs_e, pairs_a, pairs_b = [], [], []
    for e in range(ne):
        ra, rb = sidx[wl.conn[e, a_idx]], sidx[wl.conn[e, b_idx]]
        ok = (ra >= 0) & (rb >= 0)
        pairs_e.append(np.full(ok.sum(), e))
        pairs_a.append(a_idx[ok])
        pairs_b.append(b_idx[ok])
    pe, pa, pb = (np.concatenate(v) for v in (pairs_e, pairs_a, pairs_b))
    ra = sidx[wl.conn[pe, pa]].astype(np.int64)
    rb = sidx[wl.conn[pe, pb]].astype(np.int64)
    blk = np.searchsorted(keys, ra * nrow + rb)
    assert np.all(keys[blk] == ra * nrow + rb)
    bslots = np.full((pe.size, 36), -1, dtype=np.int32)
    bslots[:, :9] = np.asarray(slots, dtype=np.int32).reshape(-1, 9)[blk]
    poffs = np.concatenate([[0], np.cumsum(np.bincount(pe, minlength=ne))]).astype(np.int32)
    ints = [np.full(ne, nen, np.int32), (np.arange(ne) * nen).astype(np.int32), poffs,
            (np.arange(ne + 1) * nip).astype(np.int32), (np.arange(ne) * nip * nen).astype(np.int32),
            np.stack([pa, pb], axis=1).astype(np.int32).reshape(-1), bslots.reshape(-1),
            np.full(ne * nen, 3, np.int32)]
    eye18 = np.tile(np.concatenate([np.eye(3).reshape(-1), np.zeros(9)]), ne * nen)
    dbls = [eye18, grads.reshape(-1), Ds.reshape(-1), sigs.reshape(-1), dvs.reshape(-1)]
    nnz = int(np.asarray(slots).max()) + 1
    dev = torch.device("cuda:0")
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in ints + dbls]
    out = torch.zeros(nnz, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    total = 0.0
    for i in range(warmup + launches):
        out.zero_()
        ev0.record(stream)
        R.addMaterialStiffness3Element_launch(ne, *(a.data_ptr() for a in t), 1.0, out.data_ptr(),
                                              stream.cuda_stream)
        ev1.record(stream)
        torch.cuda.synchronize()
        if i >= warmup:
            total += ev0.elapsed_time(ev1)
    return {"kernel": "addMaterialStiffness3Element_launch (reference source, FP64 atomics)",
            "workload": "neohookean_hex_beam_40x10x10 stiffness at the last stepped positions",
            "ms_per_launch": total / launches, "launches": launches, "pairs": int(pe.size),
            "includes": "block products and CRS scatter; D, sigma, gradients and dv precomputed on the host"}


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))


def _fp64_alone(w, steps, tol, dev):
    """Positions of a model after `steps` steps of the plain FP64 drop-in."""
    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200.femmodel import MechSystemSolver
    m = w.model(precision=L.PREC_FP64, device=dev)
    MechSystemSolver(m, tol=tol, max_iter=20000).backwardEuler(w.h, steps)
    x, _ = m.getState()
    m._invalidate()
    return x


def run_batched(dev, steps=20, tol=1e-10, sample_every=4, tune=True, layout=None):
    """Batched uneven models: 256 NeoHookean tet beams in one pack (mixed
    FP32/FP64), `steps` BackwardEuler steps; next to the plain FP64 drop-in
    stepping the models one at a time (every `sample_every`-th model).
    `layout`: build-time options fixed for the pack (e.g. the PCG split or
    the tet assembly path, to compare the alternatives)."""
    import torch
    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200 import workloads as W
    from artisynth_core_b200.femmodel import FemPack, MechSystemSolver
    from artisynth_core_b200 import autotune
    import tempfile
    bs = W.batched_beams()
    for b in bs:
        b.build_mesh()
    models = [b.model(device=dev) for b in bs]

    def make(opts):
        p = FemPack(models, precision=L.PREC_MIXED, device=dev, options={**(layout or {}), **opts})
        p.engine()
        return p

    t0 = time.perf_counter()
    if tune:
        # a fresh cache: the tuning cost is part of what is reported
        with tempfile.TemporaryDirectory() as td:
            pack, tuned, _ = autotune.tune_pack(make, models, L.PREC_MIXED, bs[0].h, tol,
                                                cache=autotune.TuneCache(os.path.join(td, "tune.json")))
    else:
        pack, tuned = make({}), {}
    build_s = time.perf_counter() - t0
    torch.cuda.synchronize()
    asm = pcg = 0.0
    its = []
    t0 = time.perf_counter()
    for _ in range(steps):
        pack.backwardEuler(bs[0].h, 1, tol=tol)
        a, p = pack.lastTiming()
        asm += a
        pcg += p
        its.append(pack.stats.iterations)
    wall = time.perf_counter() - t0
    it_m, _ = pack.modelStats()
    xs = [x for x, _ in pack.getStates()]
    pack_lanes, pack_tile = pack.option(L.OPT_ROW_LANES), pack.option(L.OPT_ELEM_TILE)
    split = pack.option(L.OPT_PCG_SPLIT)
    fused = pack.option(L.OPT_FUSED_ASSEMBLY) == 1
    node_rows = pack.option(L.OPT_TET_ASSEMBLY) == 0
    nbytes = pack.deviceBytes()
    import ctypes
    na, nb = ctypes.c_int(), ctypes.c_int()
    pack.engine().call("b200fem_get_sizes", ctypes.byref(na), ctypes.byref(nb), None, None)
    pack.close()
    # algorithmic assembly bytes of one pack step (element data at the stored
    # precision: f32 rest data and S in the mixed form)
    N = sum(b.rest.shape[0] for b in bs)
    E = sum(b.conn.shape[0] for b in bs)
    nen, nip = 4, 1
    asm_bytes = 24 * N + 4 * nen * E + 36 * nip * E + 4 * nen * nen * E + 36 * nb.value + 24 * N
    peak, kind = peaks()
    asm_gbs = asm_bytes / (asm / steps * 1e-3) / 1e9
    # the same pack with one refinement sweep against the FP64 operator
    rpack = make({L.OPT_ROW_LANES: pack_lanes, L.OPT_ELEM_TILE: pack_tile, L.OPT_REFINE: 1})
    rpack.backwardEuler(bs[0].h, 1, tol=tol)  # capture
    rpack.setStates([b.rest for b in bs], [np.zeros_like(b.rest) for b in bs])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rsolve = 0.0
    for _ in range(steps):
        rpack.backwardEuler(bs[0].h, 1, tol=tol)
        rsolve += rpack.lastTiming()[1]
    rwall = time.perf_counter() - t0
    rxs = [x for x, _ in rpack.getStates()]
    rpack.close()
    # plain FP64 drop-in, one model at a time, on a sample
    sample = list(range(0, len(bs), sample_every))
    t_single = 0.0
    err = derr = rerr = rderr = 0.0
    for i in sample:
        b = bs[i]
        m = b.model(precision=L.PREC_FP64, device=dev)
        ms = MechSystemSolver(m, tol=1e-10, max_iter=20000)
        m.engine()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ms.backwardEuler(b.h, steps)
        t_single += time.perf_counter() - t1
        x, _ = m.getState()
        m._invalidate()
        err = max(err, _rel(xs[i], x))
        derr = max(derr, _rel(xs[i] - b.rest, x - b.rest))
        rerr = max(rerr, _rel(rxs[i], x))
        rderr = max(rderr, _rel(rxs[i] - b.rest, x - b.rest))
    single = len(sample) * steps / t_single
    n = len(bs)
    return {
        "workload": "256 uneven NeoHookean tet beams (n 4-60, m 2-8, seed 3), 20 steps h=0.01",
        "models": n, "tets": int(sum(b.conn.shape[0] for b in bs)), "steps": steps, "tol": tol,
        "precision": "mixed FP32 element/SpMV, FP64 vectors", "pcg_split": {1: "contiguous", 2: "strided", 3: "cluster"}.get(split, str(split)),
        "device_bytes": nbytes, "build_and_tune_s": build_s,
        "tuned": {k: v for k, v in tuned.items() if not k.endswith("_ms") and not k.endswith("_it")},
        "model_steps_per_s": n * steps / wall, "device_ms_per_step": (asm + pcg) / steps,
        "assembly_ms_per_step": asm / steps, "pcg_ms_per_step": pcg / steps,
        "assembly": {"path": "fused row-chunk" if fused else "node rows" if node_rows else "element kernel + gather",
                     "algorithmic_bytes": asm_bytes, "achieved_gbs": asm_gbs, "peak_gbs": peak,
                     "frac": asm_gbs / peak, "peak_kind": kind, "nnzb": nb.value},
        "element_updates_per_s": sum(b.conn.shape[0] for b in bs) * steps / wall,
        "pcg_iterations": {"max_per_step_mean": float(np.mean(its)), "model_median": float(np.median(it_m)),
                           "model_p90": float(np.percentile(it_m, 90))},
        "plain_fp64_single_model_steps_per_s": single,
        "speedup_vs_plain_fp64": n * steps / wall / single,
        "plain_fp64_sample": f"{len(sample)} of {n} models (every {sample_every}th), {steps} steps each",
        "max_rel_position_error_vs_fp64": err,
        "max_rel_displacement_error_vs_fp64": derr,
        "refined_1_sweep": {"model_steps_per_s": n * steps / rwall, "solve_ms_per_step": rsolve / steps,
                            "max_rel_position_error_vs_fp64": rerr,
                            "max_rel_displacement_error_vs_fp64": rderr},
    }


def block_bytes(N, E, nnzb, n_active, s_bytes=72, rest_bytes=72, factored=None):
    """Algorithmic bytes of the MooneyRivlin block (4-node tets, one point):
    assembly 24 N (x) + 16 E (connectivity) + rest_bytes E (invJ0) + 64 E
    (scatter map) + s_bytes nnzb (S written, the NODAL 2-ring included) +
    24 N (f / b); PCG iteration (s_bytes + 4) nnzb (S and block columns) +
    4 (Na + 1) + 48 Na + 72 Na + 9 * 24 Na.  Factored NODAL solve matrix
    (factored = (direct blocks nnzb1, divBlk slots of the active nodes)):
    S1 (nnzb1 blocks) and divBlk (24 per slot) written instead of the 2-ring
    S; per iteration S1 and its columns, divBlk once, the rows' (node, slot)
    entries (8 each, one per direct block), the slots' rows (4) and t (8 per
    active node) in place of the 2-ring S."""
    vec = 4 * (n_active + 1) + 48 * n_active + 72 * n_active + 9 * 24 * n_active
    if factored is not None:
        nnzb1, slots = factored
        asm = 24 * N + 16 * E + rest_bytes * E + 64 * E + s_bytes * nnzb1 + 24 * slots + 24 * N
        it = (s_bytes + 4) * nnzb1 + 24 * slots + 8 * nnzb1 + 4 * slots + 8 * n_active + vec
        return asm, it
    asm = 24 * N + 16 * E + rest_bytes * E + 64 * E + s_bytes * nnzb + 24 * N
    it = (s_bytes + 4) * nnzb + vec
    return asm, it


def direct_counts(conn, fixed):
    """Blocks between active nodes that share an element (self included),
    and the neighbour slots (nodes sharing an element, self included) of the
    active nodes."""
    c = np.asarray(conn, dtype=np.int64)
    N = int(c.max()) + 1
    k = c.shape[1]
    a = np.repeat(c, k, axis=1).reshape(-1)
    b = np.tile(c, (1, k)).reshape(-1)
    key = np.unique(a * N + b)
    ia, ib = key // N, key % N
    act = np.asarray(fixed).reshape(-1) == 0
    return int(np.count_nonzero(act[ia] & act[ib])), int(np.count_nonzero(act[ia]))


def run_block(dev, steps=50, tol=1e-10, cpu=True, factored=0, row_lanes=0, resident=0):
    """The MooneyRivlin tet block (60x30x30 cells of a 0.3x0.15x0.15 m block,
    270,000 tets, 58,621 nodes; AUTO soft incompressibility resolves to NODAL:
    3,935,980 blocks), `steps` BackwardEuler steps from rest in the plain
    FP64 form and in the mixed form, on device-resident state (S alone is
    283 MB, above the 126 MB L2, so nothing is flushed); the mixed form's
    position error against the FP64 run after the same steps.  factored:
    B200FEM_OPT_NODAL_FACTORED (0 auto: the factored solve matrix, S1 51 MB
    f64 with divBlk 21 MB, near the L2 size, so L2 is flushed between steps;
    1 the assembled 2-ring S, 283 MB f64)."""
    import ctypes
    import torch
    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200 import workloads as W
    from artisynth_core_b200.femmodel import MechSystemSolver
    wl = W.mooneyrivlin_tet_block().build_mesh()
    peak, kind = peaks()
    out = {"workload": "mooneyrivlin_tet_block_60x30x30 (270,000 tets, NODAL incompressibility, gravity, "
                       f"z-min fixed), {steps} steps h=0.01 from rest, PCG {tol:g}",
           "steps": steps, "tol": tol, "l2": "flushed between steps (256 MB write)"}
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")
    counts = direct_counts(wl.conn, wl.fixed)
    xs = {}
    for prec, name in ((L.PREC_FP64, "fp64"), (L.PREC_MIXED, "mixed")):
        m = wl.model(precision=prec, device=dev)
        m.options = {L.OPT_NODAL_FACTORED: factored, L.OPT_ROW_LANES: row_lanes, L.OPT_PCG_RESIDENT: resident}
        ms = MechSystemSolver(m, tol=tol, max_iter=20000)
        t0 = time.perf_counter()
        m.engine()
        sz = m.sizes()
        ms.backwardEuler(wl.h, 1)  # captures the step graph
        m.setState(wl.rest, np.zeros_like(wl.rest))
        build_s = time.perf_counter() - t0
        torch.cuda.synchronize()
        asm = pcg = 0.0
        its = []
        fv = ctypes.c_int()
        m.engine().call("b200fem_get_option", L.OPT_NODAL_FACTORED, ctypes.byref(fv))
        wall = 0.0
        for _ in range(steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            ms.backwardEuler(wl.h, 1)
            a, p = ms.lastTiming()
            wall += time.perf_counter() - t0
            asm += a
            pcg += p
            its.append(ms.stats.iterations)
        xs[name], _ = m.getState()
        m._invalidate()
        sb = 72 if name == "fp64" else 36
        asm_b, it_b = block_bytes(wl.rest.shape[0], wl.conn.shape[0], sz["nnzb"], sz["n_active"], s_bytes=sb,
                                  rest_bytes=72 if name == "fp64" else 36,
                                  factored=counts if fv.value == 2 else None)
        mean_it = float(np.mean(its))
        asm_gbs = asm_b / (asm / steps * 1e-3) / 1e9
        pcg_gbs = it_b * (mean_it + 2) / (pcg / steps * 1e-3) / 1e9
        out[name] = {"steps_per_s": steps / wall, "device_ms_per_step": (asm + pcg) / steps,
                     "solve_matrix": "factored (S1 + divBlk)" if fv.value == 2 else "assembled (2-ring S)",
                     "assembly_ms_per_step": asm / steps, "pcg_ms_per_step": pcg / steps,
                     "pcg_iterations_mean": mean_it, "build_s": build_s,
                     "element_updates_per_s": wl.conn.shape[0] * steps / wall,
                     "assembly_roofline": {"algorithmic_bytes": asm_b, "achieved_gbs": asm_gbs, "peak_gbs": peak,
                                           "frac": asm_gbs / peak, "peak_kind": kind},
                     "pcg_roofline": {"bytes_per_iteration": it_b, "achieved_gbs": pcg_gbs, "peak_gbs": peak,
                                      "frac": pcg_gbs / peak, "peak_kind": kind}}
        out["nnzb"] = sz["nnzb"]
        out["active_dof"] = 3 * sz["n_active"]
    out["mixed_max_rel_position_error_vs_fp64"] = _rel(xs["mixed"], xs["fp64"])
    out["mixed_max_rel_displacement_error_vs_fp64"] = _rel(xs["mixed"] - wl.rest, xs["fp64"] - wl.rest)
    if cpu:
        # the oracle on every host core: a bounded sample of the same run
        # (one warm-up step, then the median of 5 single-step runs)
        cw = W.mooneyrivlin_tet_block().build_mesh(mesher=oracle_mesher)
        v, runs, k, used = cpu_oracle_protocol(cw, os.cpu_count() or 1, runs=5, warmup=1, budget_s=1e-3, max_k=1)
        out["cpu_baseline"] = dict({"value": v, "unit": UNIT, "cores": used, "kind": "port", "runs": runs,
                                    "sample": f"median of 5 single BackwardEuler steps after 1 warm-up step "
                                              f"(FP64 oracle, Jacobi-PCG {cw.tol:g}, OpenMP on {used} threads)"},
                                   **cpu_info())
    return out


def run_served(dev, seconds=60.0, pool_size=512, rate=2000.0, steps_per_request=10, tol=1e-6,
               drain_s=30.0, err_sample=16, plain_sample=32):
    """Served stream: Poisson arrivals (seed 4) of 10-step requests on models
    of the config-4 distribution with 10% large (n 80-120) beams, 60 GB
    device-memory budget, continuous batching."""
    from artisynth_core_b200 import workloads as W
    from artisynth_core_b200.serve import NativeServer, poisson_arrivals, run_stream_native
    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200.femmodel import FemPack
    import tempfile
    from artisynth_core_b200 import autotune
    pool = W.batched_beams(count=pool_size, seed=4, large_frac=0.1)
    for w in pool:
        w.build_mesh()
    # the layout options for the server's packs: tuned once on a probe pack of
    # the pool's first models (fresh cache, the cost is part of preload_s)
    t0 = time.perf_counter()
    probe_models = [w.model(device=dev) for w in pool[:256]]

    def make(opts):
        p = FemPack(probe_models, precision=L.PREC_MIXED, device=dev, options=opts)
        p.engine()
        return p

    with tempfile.TemporaryDirectory() as td:
        probe, tuned, _ = autotune.tune_pack(make, probe_models, L.PREC_MIXED, pool[0].h, tol,
                                             cache=autotune.TuneCache(os.path.join(td, "tune.json")),
                                             piece_rows=False)
    probe.close()
    srv = NativeServer(pool, budget=60e9, tol=tol, device=dev,
                       options={L.OPT_ROW_LANES: tuned["row_lanes"], L.OPT_ELEM_TILE: tuned["elem_tile"]})
    srv.preload()
    preload_s = time.perf_counter() - t0
    arrivals = poisson_arrivals(rate, seconds, pool_size, seed=4)
    out = run_stream_native(srv, arrivals, steps_per_request, drain_s=drain_s)
    # accuracy: served models against the plain FP64 drop-in for the same steps
    times, models = arrivals
    steps_of = {}
    for m in models[: out["requests"]]:
        steps_of[int(m)] = steps_of.get(int(m), 0) + steps_per_request
    checked = sorted(steps_of)[:err_sample] if out["incomplete"] == 0 else []
    err = derr = 0.0
    for m in checked:
        x, _ = srv.state(m)
        xr = _fp64_alone(pool[m], steps_of[m], 1e-10, dev)
        err = max(err, _rel(x, xr))
        derr = max(derr, _rel(x - pool[m].rest, xr - pool[m].rest))
    srv.close()
    # saturation: the same pool and server setup with arrivals at ten times the
    # offered rate for 10 s -- the completed model steps per second of wall
    # time is what the server sustains
    opts = {L.OPT_ROW_LANES: tuned["row_lanes"], L.OPT_ELEM_TILE: tuned["elem_tile"]}
    sat_srv = NativeServer(pool, budget=60e9, tol=tol, device=dev, options=opts)
    sat_srv.preload()
    sat = run_stream_native(sat_srv, poisson_arrivals(rate * 10, 10.0, pool_size, seed=5), steps_per_request,
                            drain_s=10.0)
    sat_srv.close()
    # admission under budget pressure: packs of 64 models and a 1 GB budget
    # (the pool needs about 3.5 GB), so idle packs are evicted and models
    # re-admitted from their host-saved states while the stream runs
    pr_srv = NativeServer(pool, budget=1e9, tol=tol, device=dev, pack_models=64, options=opts)
    pres = run_stream_native(pr_srv, poisson_arrivals(rate, 10.0, pool_size, seed=6), steps_per_request,
                             drain_s=20.0)
    pr_srv.close()
    # the plain FP64 drop-in on the same distribution, one model at a time
    import torch
    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200.femmodel import MechSystemSolver
    t_plain, n_plain = 0.0, 0
    for i in range(0, pool_size, max(1, pool_size // plain_sample)):
        w = pool[i]
        mdl = w.model(precision=L.PREC_FP64, device=dev)
        ms = MechSystemSolver(mdl, tol=1e-10, max_iter=20000)
        mdl.engine()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        ms.backwardEuler(w.h, steps_per_request)
        t_plain += time.perf_counter() - t1
        n_plain += steps_per_request
        mdl._invalidate()
    plain = n_plain / t_plain
    out.update({
        "workload": f"Poisson {rate:.0f} req/s (seed 4) for {seconds:.0f} s, {steps_per_request} steps/request, "
                    f"pool of {pool_size} beams (config-4 distribution, 10% n 80-120)",
        "pool_tets": int(sum(w.conn.shape[0] for w in pool)), "tol": tol, "budget_bytes": 60e9,
        "preload_and_tune_s": preload_s, "offered_model_steps_per_s": rate * steps_per_request,
        "tuned": {"row_lanes": tuned["row_lanes"], "elem_tile": tuned["elem_tile"]},
        "max_rel_position_error_vs_fp64": err, "max_rel_displacement_error_vs_fp64": derr,
        "error_sample_models": len(checked),
        "plain_fp64_single_model_steps_per_s": plain,
        "speedup_vs_plain_fp64": out["model_steps_per_s"] / plain,
        "plain_fp64_sample": f"{n_plain // steps_per_request} pool models, {steps_per_request} steps each, PCG 1e-10",
        "saturation": dict({"offered_requests_per_s": rate * 10, "seconds": 10.0}, **sat),
        "budget_pressure": dict({"budget_bytes": 1e9, "pack_models": 64, "offered_requests_per_s": rate,
                                 "seconds": 10.0}, **pres),
    })
    return out


def run_batched_sharded(dist, rank, world, dev, steps=20, tol=1e-10):
    """The batched leg on `world` GPUs: the 256 models dealt to ranks by LPT
    on their element counts (strong scaling: the total work is fixed), one
    tuned pack per rank, no collective on the data path; time = the slowest
    rank's."""
    import tempfile
    import torch
    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200 import autotune, shard
    from artisynth_core_b200 import workloads as W
    from artisynth_core_b200.femmodel import FemPack
    bs = W.batched_beams()
    for b in bs:
        b.build_mesh()
    mine = shard.lpt_partition([b.conn.shape[0] for b in bs], world)[rank]
    local = [bs[i] for i in mine]
    models = [b.model(device=dev) for b in local]

    def make(opts):
        p = FemPack(models, precision=L.PREC_MIXED, device=dev, options=opts)
        p.engine()
        return p

    with tempfile.TemporaryDirectory() as td:
        pack, tuned, _ = autotune.tune_pack(make, models, L.PREC_MIXED, bs[0].h, tol,
                                            cache=autotune.TuneCache(os.path.join(td, "tune.json")))
    dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        pack.backwardEuler(bs[0].h, 1, tol=tol)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    pack.close()
    slowest = shard.max_over_ranks(dist, wall)
    per_rank = shard.gather_to_root(dist, {"models": len(mine), "tets": int(sum(b.conn.shape[0] for b in local)),
                                           "wall_s": wall})
    if rank != 0:
        return None
    return {"workload": "256 uneven NeoHookean tet beams (seed 3), 20 steps, dealt to ranks by LPT on elements",
            "ranks": world, "scaling": "strong", "steps": steps, "tol": tol,
            "model_steps_per_s": len(bs) * steps / slowest, "per_rank": per_rank}


def run_served_sharded(dist, rank, world, dev, seconds=60.0, pool_size=512, rate=2000.0, steps_per_request=10,
                       tol=1e-6, drain_s=30.0):
    """The served leg on `world` GPUs: pool models dealt to ranks by LPT;
    every rank replays the same arrival stream and serves the requests for
    its own models; latencies gathered to rank 0."""
    import tempfile
    import numpy as np
    from artisynth_core_b200 import autotune, shard
    from artisynth_core_b200 import workloads as W
    from artisynth_core_b200.serve import FemServer, poisson_arrivals, run_stream
    pool = W.batched_beams(count=pool_size, seed=4, large_frac=0.1)
    for w in pool:
        w.build_mesh()
    mine = shard.lpt_partition([w.conn.shape[0] for w in pool], world)[rank]
    local_of = {m: i for i, m in enumerate(mine)}
    td = tempfile.TemporaryDirectory()
    srv = FemServer([pool[m] for m in mine], budget=60e9, tol=tol, device=dev, autotune=True,
                    tune_cache=autotune.TuneCache(os.path.join(td.name, "tune.json")))
    srv.preload()
    times, models = poisson_arrivals(rate, seconds, pool_size, seed=4)
    keep = np.array([int(m) in local_of for m in models], dtype=bool)
    arr = (times[keep], np.array([local_of[int(m)] for m in models[keep]], dtype=np.int64))
    dist.barrier()
    out = run_stream(srv, arr, steps_per_request, drain_s=drain_s)
    lat = [r.latency * 1e3 for r in srv.done]
    srv.close()
    td.cleanup()
    gathered = shard.gather_to_root(dist, {"lat": lat, "out": out})
    if rank != 0:
        return None
    alllat = np.concatenate([np.asarray(g["lat"]) for g in gathered]) if gathered else np.zeros(0)
    wall = max(g["out"]["wall_s"] for g in gathered)
    steps = sum(g["out"]["model_steps_per_s"] * g["out"]["wall_s"] for g in gathered)
    return {"workload": f"Poisson {rate:.0f} req/s (seed 4), {seconds:.0f} s, pool of {pool_size} dealt to ranks by LPT",
            "ranks": world, "requests": int(sum(g["out"]["requests"] for g in gathered)),
            "completed": int(len(alllat)), "incomplete": int(sum(g["out"]["incomplete"] for g in gathered)),
            "p50_ms": float(np.percentile(alllat, 50)) if len(alllat) else None,
            "p99_ms": float(np.percentile(alllat, 99)) if len(alllat) else None,
            "model_steps_per_s": steps / wall, "tol": tol}


def run_b200(args):
    import torch
    dist, rank, world, local = dist_setup(args.gpus)
    dev = local if dist is not None else 0
    torch.cuda.set_device(dev)
    from artisynth_core_b200 import _lib as L
    from artisynth_core_b200 import workloads as W
    from artisynth_core_b200.femmodel import MechSystemSolver

    wl = W.neohookean_hex_beam().build_mesh()
    m = wl.model(device=dev)
    sz = m.sizes()
    ms = MechSystemSolver(m, tol=wl.tol, max_iter=20000)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")

    for _ in range(args.warmup):
        ms.backwardEuler(wl.h, 1)
    # ---- timed region: device-resident state, L2 flushed between steps
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    asm_ms, pcg_ms, iters = 0.0, 0.0, []
    with ClockSampler(dev) as clk:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ms.backwardEuler(wl.h, 1)
            a, s = ms.lastTiming()
            asm_ms += a
            pcg_ms += s
            iters.append(ms.stats.iterations)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    step_ms = (asm_ms + pcg_ms) / args.steps
    t = torch.tensor([step_ms], dtype=torch.float64, device=f"cuda:{dev}")
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    step_ms_max = float(t.item())
    value = world * 1e3 / step_ms_max

    # ---- the drop-in FemModel3d.updateStressAndStiffness on the same beam
    # (element kernel, FP64 stiffness gather, forces): device time per call,
    # beside the reference's own device stiffness kernel timed by the
    # reference arm on this mesh
    xs_now, _ = m.getState()
    uss = []
    for i in range(3 + 20):
        m.updateStressAndStiffness(xs_now)
        if i >= 3:
            uss.append(ms.lastTiming()[0])
    uss_ms = float(np.mean(uss))
    # ---- end to end through the C ABI with host buffers: every step,
    # b200fem_backward_euler_step_host copies x, v in from pinned host memory,
    # steps, and copies the new x, v back (one synchronisation per call)
    xs, vs = m.getState()
    x_h = torch.empty(xs.size, dtype=torch.float64, pin_memory=True).numpy()
    v_h = torch.empty(vs.size, dtype=torch.float64, pin_memory=True).numpy()
    x_h[:] = xs.reshape(-1)
    v_h[:] = vs.reshape(-1)
    e2e_steps = max(3, args.steps)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ms.backwardEulerHost(wl.h, x_h, v_h)
    t1 = time.perf_counter()
    e2e_ms = torch.tensor([1e3 * (t1 - t0) / e2e_steps], dtype=torch.float64, device=f"cuda:{dev}")
    if dist is not None:
        dist.all_reduce(e2e_ms, op=dist.ReduceOp.MAX)
    e2e_val = world * 1e3 / float(e2e_ms.item())
    state_bytes = 2 * 3 * wl.rest.shape[0] * 8

    # multi-GPU forms of the batched and served legs (every rank takes part)
    batched_sharded = served_sharded = None
    if world > 1 and not args.no_batched:
        batched_sharded = run_batched_sharded(dist, rank, world, dev, steps=args.batch_steps, tol=args.batch_tol)
    if world > 1 and args.served_seconds > 0:
        served_sharded = run_served_sharded(dist, rank, world, dev, seconds=args.served_seconds, tol=args.served_tol)

    if rank == 0:
        asm_b, it_b = algorithmic_bytes(wl, sz["nnzb"], sz["n_active"])
        mean_it = float(np.mean(iters))
        pcg_bytes = it_b * (mean_it + 2)  # iterations + the initial and final SpMV
        asm_gbs = asm_b / (asm_ms / args.steps * 1e-3) / 1e9
        pcg_gbs = pcg_bytes / (pcg_ms / args.steps * 1e-3) / 1e9
        peak, kind = peaks()
        dominant = "pcg_kernel" if pcg_ms >= asm_ms else "assembly (elem + gather + rows)"
        achieved = pcg_gbs if pcg_ms >= asm_ms else asm_gbs
        traffic = None
        prof = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(prof):
            try:
                traffic = json.load(open(prof)).get("pcg_kernel" if pcg_ms >= asm_ms else "assembly")
            except Exception:
                traffic = None
        batched = served = None
        if world > 1 and not args.no_batched:
            batched = batched_sharded
        if world > 1 and args.served_seconds > 0:
            served = served_sharded
        if world == 1 and not args.no_batched:
            with ClockSampler(dev) as c:
                batched = run_batched(dev, steps=args.batch_steps, tol=args.batch_tol, tune=not args.no_tune)
            batched["clocks"] = c.summary()
        if world == 1 and args.served_seconds > 0:
            with ClockSampler(dev) as c:
                served = run_served(dev, seconds=args.served_seconds, tol=args.served_tol)
            served["clocks"] = c.summary()
        block = None
        if world == 1 and not args.no_block:
            with ClockSampler(dev) as c:
                block = run_block(dev, steps=args.block_steps, cpu=not args.no_cpu, factored=args.nodal_factored,
                                  row_lanes=args.block_row_lanes, resident=args.block_resident)
            block["clocks"] = c.summary()
        cpu = None
        if not args.no_cpu and world == 1:
            cpu = cpu_baseline_entry(wl, "40x10x10 hex beam", budget_s=args.cpu_budget)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms_max, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(wl.describe(), parallelism=f"replicas{world}", l2="flushed between steps (256 MB write)",
                           tol=wl.tol, nnzb=sz["nnzb"], active_dof=3 * sz["n_active"]),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                    "d2h_bytes_per_step": state_bytes},
            # per timed step: status reset, element kernel, block gather, RHS rows,
            # PCG, and the status record the call reads back
            "gpu_launches": 6 * args.steps,
            "phases_ms_per_step": {"assembly": asm_ms / args.steps, "pcg": pcg_ms / args.steps,
                                   "pcg_iterations": mean_it},
            "update_stress_stiffness_ms": {"value": uss_ms, "what": "b200fem_update_stress_stiffness device time "
                                           "(element kernel computing F, sigma, D and blocks, FP64 stiffness "
                                           "gather, nodal forces) on the hex beam"},
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": kind, "traffic": traffic,
                         "bytes_per_launch": pcg_bytes if pcg_ms >= asm_ms else asm_b,
                         "assembly_gbs": asm_gbs, "pcg_gbs": pcg_gbs},
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            "block": block,
            "batched": batched,
            "served": served,
        }
        print(json.dumps(line), flush=True)
    m._invalidate()
    if dist is not None:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=8.0, help="seconds per CPU-baseline variant")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-pack leg")
    ap.add_argument("--no-block", action="store_true", help="skip the MooneyRivlin block leg")
    ap.add_argument("--block-steps", type=int, default=50)
    ap.add_argument("--only", choices=["batched", "block"], default=None,
                    help="run only this leg (for profiling): prints its JSON object")
    ap.add_argument("--batch-steps", type=int, default=20)
    ap.add_argument("--no-tune", action="store_true", help="batched leg without the autotuner")
    ap.add_argument("--pcg-split", type=int, default=0, choices=[0, 1, 2, 3],
                    help="batched leg: B200FEM_OPT_PCG_SPLIT (0 auto, 2 strided, 3 cluster)")
    ap.add_argument("--tet-assembly", type=int, default=1, choices=[0, 1],
                    help="batched leg: B200FEM_OPT_TET_ASSEMBLY (0 node rows, 1 element kernel + gather)")
    ap.add_argument("--nodal-factored", type=int, default=0, choices=[0, 1, 2],
                    help="block leg: B200FEM_OPT_NODAL_FACTORED (0 auto, 1 assembled 2-ring S, 2 factored)")
    ap.add_argument("--block-row-lanes", type=int, default=0, choices=[0, 4, 8, 16, 32],
                    help="block leg: B200FEM_OPT_ROW_LANES (0 auto)")
    ap.add_argument("--block-resident", type=int, default=0, choices=[0, 1, 2],
                    help="block leg: B200FEM_OPT_PCG_RESIDENT (0 auto)")
    ap.add_argument("--served-seconds", type=float, default=60.0, help="length of the served stream (0: skip)")
    ap.add_argument("--batch-tol", type=float, default=1e-10, help="PCG tolerance of the batched leg")
    ap.add_argument("--served-tol", type=float, default=1e-6,
                    help="PCG tolerance of the served leg (the loosest that keeps positions within 1e-6 of FP64)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.only == "batched":
        import torch
        torch.cuda.set_device(0)
        from artisynth_core_b200 import _lib as L
        layout = {L.OPT_TET_ASSEMBLY: args.tet_assembly}
        if args.pcg_split:
            layout[L.OPT_PCG_SPLIT] = args.pcg_split
        print(json.dumps(run_batched(0, steps=args.batch_steps, tol=args.batch_tol, sample_every=64,
                                     tune=not args.no_tune, layout=layout)), flush=True)
    elif args.only == "block":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_block(0, steps=args.block_steps, cpu=not args.no_cpu, factored=args.nodal_factored,
                                   row_lanes=args.block_row_lanes, resident=args.block_resident)), flush=True)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
