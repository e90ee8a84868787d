"""Served stream: continuous batching of BackwardEuler step requests.

A request asks for `steps` BackwardEuler steps of one model of a pool.  The
server keeps every admitted model resident on the device -- positions,
velocities, solve pattern, scatter map and preconditioner live in the
device arrays of a pack (:class:`FemPack`) -- and advances the models in
*ticks*: one tick runs one BackwardEuler step of every resident model that
has work, all models of a pack in the same kernel launches (the pack's
active mask leaves idle models out of assembly, PCG and the state update).
Requests that arrive while others are on the GPU join at the next tick:
their model steps alongside the models already in flight (continuous
batching), and a model's queued requests run back to back.

Admission is against a device-memory budget: models that are not resident
are admitted in batches as a new pack when its estimated size fits; when it
does not, packs whose models have no work are evicted (least recently used
first) after their states are copied to the host, and a re-admitted model
continues from its saved state.

The reference has no counterpart (ArtiSynth steps one MechModel per
scheduler); the results of each request equal those of its model stepped
alone through :class:`MechSystemSolver`, to rounding.
"""
from __future__ import annotations

import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .femmodel import FemPack


@dataclass
class Request:
    rid: int
    model: int
    steps: int
    t_arrive: float
    remaining: int = 0
    t_start: float | None = None
    t_done: float | None = None
    error: str | None = None   # set when the request cannot be served

    @property
    def latency(self):
        return None if self.t_done is None else self.t_done - self.t_arrive


@dataclass
class _Slot:
    pack: FemPack
    models: list            # pool indices, in pack order
    mask: np.ndarray = None
    last_used: float = 0.0
    bytes: int = 0


@dataclass
class ServerStats:
    ticks: int = 0
    model_steps: int = 0
    slot_steps: int = 0
    builds: int = 0
    evictions: int = 0
    peak_bytes: int = 0
    build_s: float = 0.0
    step_s: float = 0.0
    pcg_ms: float = 0.0
    asm_ms: float = 0.0
    max_iterations: int = 0
    iterations: list = field(default_factory=list)


class FemServer:
    """Continuous-batching server over a pool of models.

    workloads   -- the pool (:class:`workloads.Workload`, meshes built lazily)
    budget      -- device-memory budget in bytes for all resident packs
    pack_models -- most models admitted into one pack
    """

    def __init__(self, workloads, budget=60e9, precision=L.PREC_MIXED, pack_models=256, tol=1e-10,
                 max_iter=20000, device=0, clock=time.perf_counter, autotune=False, tune_cache=None):
        self.pool = list(workloads)
        self.budget = float(budget)
        self.precision = precision
        self.pack_models = int(pack_models)
        self.tol = tol
        self.max_iter = max_iter
        self.device = device
        self.clock = clock
        self.autotune = autotune        # tune each new pack's run-time layout options
        self.tune_cache = tune_cache
        self.slots: list[_Slot] = []
        self.where = {}                  # model -> (slot, index in pack)
        self.saved = {}                  # model -> (x, v) of an evicted model
        self.queues = {}                 # model -> deque of Requests
        self.waiting = deque()           # models with work that are not resident
        self.done: list[Request] = []
        self.failed: list[Request] = []
        self.stats = ServerStats()
        # admission estimate: bytes = pack_overhead + bytes_per_elem * elements,
        # fitted to the packs built so far
        self.bytes_per_elem = 4096.0
        self.pack_overhead = 0.0
        self._sizes = []                 # (elements, bytes) of every build
        self._rid = 0
        h = {w.h for w in self.pool}
        if len(h) != 1:
            raise ValueError("one step size for the pool")
        self.h = h.pop()

    # ---- requests ---------------------------------------------------------
    def submit(self, model: int, steps: int, t_arrive: float | None = None) -> Request:
        if not 0 <= model < len(self.pool):
            raise ValueError("unknown model")
        r = Request(self._rid, model, int(steps), self.clock() if t_arrive is None else t_arrive, int(steps))
        self._rid += 1
        q = self.queues.setdefault(model, deque())
        q.append(r)
        if model not in self.where and model not in self.waiting:
            self.waiting.append(model)
        return r

    def preload(self, models=None):
        """Admit models before their first request (as far as the budget
        allows), so that the stream starts with them resident."""
        for m in range(len(self.pool)) if models is None else models:
            if m not in self.where and m not in self.waiting:
                self.waiting.append(m)
        self._admit()

    def pending(self) -> int:
        return sum(len(q) for q in self.queues.values())

    def resident_bytes(self) -> int:
        return sum(s.bytes for s in self.slots)

    # ---- admission --------------------------------------------------------
    def _elems(self, model: int) -> int:
        w = self.pool[model]
        if w.conn is None:
            w.build_mesh()
        return w.conn.shape[0]

    def _estimate(self, model: int) -> float:
        return self.bytes_per_elem * self._elems(model)

    def _calibrate(self, elems: int, nbytes: int):
        self._sizes.append((elems, nbytes))
        e = np.array([a for a, _ in self._sizes], dtype=float)
        b = np.array([c for _, c in self._sizes], dtype=float)
        if len(set(e.tolist())) >= 2:
            slope, icpt = np.polyfit(e, b, 1)
            if slope > 0:
                self.bytes_per_elem = float(slope) * 1.02
                self.pack_overhead = max(0.0, float(icpt)) * 1.02
                worst = float(np.max(b - (self.pack_overhead + self.bytes_per_elem * e)))
                self.pack_overhead += max(0.0, worst)  # cover every pack seen
                return
        self.bytes_per_elem = max(self.bytes_per_elem, nbytes / max(1, elems))

    def _evict_idle(self, need: float) -> bool:
        idle = [s for s in self.slots if not any(self.queues.get(m) for m in s.models)]
        idle.sort(key=lambda s: s.last_used)
        freed = False
        for s in idle:
            if self.resident_bytes() + need <= self.budget:
                break
            for m, (x, v) in zip(s.models, s.pack.getStates()):
                self.saved[m] = (x.copy(), v.copy())
                del self.where[m]
            s.pack.close()
            self.slots.remove(s)
            self.stats.evictions += 1
            freed = True
        return freed

    def _admit(self):
        while self.waiting:
            batch, est = [], self.pack_overhead
            for m in list(self.waiting)[: self.pack_models]:
                e = self._estimate(m)
                if batch and self.resident_bytes() + est + e > self.budget:
                    break
                batch.append(m)
                est += e
            if self.resident_bytes() + est > self.budget:
                self._evict_idle(est)
            while batch and self.resident_bytes() + est > self.budget:
                est -= self._estimate(batch.pop())
            if not batch:
                if any(any(self.queues.get(m) for m in s.models) for s in self.slots):
                    return  # no room until work finishes and packs turn idle
                # nothing else can make room: try the first model by its real size
                batch = [self.waiting[0]]
            t0 = self.clock()
            models = [self.pool[m].model(precision=self.precision, device=self.device) for m in batch]
            if self.autotune:
                from . import autotune as at

                def make(opts):
                    p = FemPack(models, precision=self.precision, device=self.device, options=opts)
                    p.engine()
                    return p

                pack, _, _ = at.tune_pack(make, models, self.precision, self.h, self.tol,
                                          cache=self.tune_cache or at.TuneCache(), piece_rows=False)
            else:
                pack = FemPack(models, precision=self.precision, device=self.device)
                pack.engine()
            if any(m in self.saved for m in batch):
                xs, vs = [], []
                for i, m in enumerate(batch):
                    if m in self.saved:
                        x, v = self.saved.pop(m)
                    else:
                        w = self.pool[m]
                        x, v = w.rest, np.zeros_like(w.rest)
                    xs.append(x)
                    vs.append(v)
                pack.setStates(xs, vs)
            nb = pack.deviceBytes()
            self._calibrate(sum(self._elems(m) for m in batch), nb)
            slot = _Slot(pack, batch, np.zeros(len(batch), dtype=np.int32), self.clock(), nb)
            self.slots.append(slot)
            for i, m in enumerate(batch):
                self.where[m] = (slot, i)
                self.waiting.remove(m)
            if self.resident_bytes() > self.budget:
                # the estimate fell short: make room with idle packs
                self._evict_idle(0.0)
            if nb > self.budget:
                # larger than the whole budget: its requests cannot be served
                self.slots.remove(slot)
                pack.close()
                for m in batch:
                    del self.where[m]
                    for r in self.queues.pop(m, ()):
                        r.error = "model larger than the device-memory budget"
                        self.failed.append(r)
            self.stats.builds += 1
            self.stats.build_s += self.clock() - t0
            self.stats.peak_bytes = max(self.stats.peak_bytes, self.resident_bytes())

    # ---- one tick ---------------------------------------------------------
    def tick(self) -> int:
        """Admit what fits, then one BackwardEuler step of every resident
        model with work.  Returns the number of model steps taken."""
        self._admit()
        taken = 0
        for s in list(self.slots):
            mask = np.array([1 if self.queues.get(m) else 0 for m in s.models], dtype=np.int32)
            if not mask.any():
                continue
            if not np.array_equal(mask, s.mask):
                s.pack.setActive(None if mask.all() else mask)
                s.mask = mask
            t0 = self.clock()
            for i in np.nonzero(mask)[0]:
                r = self.queues[s.models[i]][0]
                if r.t_start is None:
                    r.t_start = t0
            s.pack.backwardEuler(self.h, 1, tol=self.tol, max_iter=self.max_iter)
            t1 = self.clock()
            a, p = s.pack.lastTiming()
            self.stats.asm_ms += a
            self.stats.pcg_ms += p
            self.stats.step_s += t1 - t0
            self.stats.slot_steps += 1
            self.stats.max_iterations = max(self.stats.max_iterations, s.pack.stats.iterations)
            s.last_used = t1
            for i in np.nonzero(mask)[0]:
                m = s.models[i]
                q = self.queues[m]
                r = q[0]
                r.remaining -= 1
                if r.remaining == 0:
                    r.t_done = t1
                    self.done.append(r)
                    q.popleft()
                taken += 1
        self.stats.ticks += 1
        self.stats.model_steps += taken
        return taken

    # ---- results ----------------------------------------------------------
    def state(self, model: int):
        """(x, v) of a model: from its pack when resident, else as saved."""
        if model in self.where:
            s, i = self.where[model]
            return s.pack.getStates()[i]
        if model in self.saved:
            return self.saved[model]
        w = self.pool[model]
        return w.rest, np.zeros_like(w.rest)

    def close(self):
        for s in self.slots:
            s.pack.close()
        self.slots.clear()
        self.where.clear()


def poisson_arrivals(rate: float, duration: float, n_models: int, seed: int = 4):
    """Arrival times (s) of a Poisson stream and the model of each request
    (uniform over the pool)."""
    rng = np.random.default_rng(seed)
    n = int(rate * duration * 1.5) + 16
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t = t[t < duration]
    models = rng.integers(0, n_models, size=t.shape[0])
    return t, models


def run_stream(server: FemServer, arrivals, steps_per_request: int = 10, drain_s: float = 30.0):
    """Replay an arrival stream against the wall clock: requests are released
    when their arrival time has passed and the server ticks continuously.
    Returns a summary dict (latencies in ms)."""
    times, models = arrivals
    t0 = server.clock()
    nxt = 0
    duration = float(times[-1]) if len(times) else 0.0
    reqs = []
    while True:
        now = server.clock() - t0
        while nxt < len(times) and times[nxt] <= now:
            reqs.append(server.submit(int(models[nxt]), steps_per_request, t0 + float(times[nxt])))
            nxt += 1
        if nxt >= len(times) and server.pending() == 0:
            break
        if now > duration + drain_s:
            break
        if server.pending() == 0:
            time.sleep(min(0.0005, max(0.0, float(times[nxt]) - now)))
            continue
        server.tick()
    wall = server.clock() - t0
    lat = np.array([r.latency for r in reqs if r.t_done is not None]) * 1e3
    done = len(lat)
    st = server.stats
    return {
        "requests": len(reqs),
        "completed": done,
        "incomplete": len(reqs) - done,
        "wall_s": wall,
        "p50_ms": float(np.percentile(lat, 50)) if done else None,
        "p99_ms": float(np.percentile(lat, 99)) if done else None,
        "mean_ms": float(lat.mean()) if done else None,
        "requests_per_s": done / wall if wall > 0 else 0.0,
        "model_steps_per_s": st.model_steps / wall if wall > 0 else 0.0,
        "ticks": st.ticks,
        "slot_steps": st.slot_steps,
        "models_per_slot_step": st.model_steps / max(1, st.slot_steps),
        "builds": st.builds,
        "evictions": st.evictions,
        "peak_bytes": st.peak_bytes,
        "build_s": st.build_s,
        "gpu_step_s": st.step_s,
        "max_iterations": st.max_iterations,
    }


class NativeServer:
    """The same served form run by the library's native server
    (b200fem_server_*, the entry points a Java host binds): admission,
    eviction, ticks and request bookkeeping in C++; this class only forwards.
    `options` (B200FEM_OPT_* -> value) apply to every pack it builds."""

    def __init__(self, workloads, budget=60e9, precision=L.PREC_MIXED, pack_models=256, tol=1e-10,
                 max_iter=20000, device=0, options=None):
        import ctypes
        self._c = ctypes
        self.pool = list(workloads)
        w0 = self.pool[0]
        p = L.StepParams()
        p.h = w0.h
        p.alpha_m = w0.mass_damping
        p.beta_k = w0.stiffness_damping
        for i in range(3):
            p.gravity[i] = w0.gravity[i]
        p.tol = tol
        p.max_iter = max_iter
        cfg = L.Config()
        cfg.device = device
        cfg.precision = precision
        self._lib = L.lib()
        self.h = self._lib.b200fem_server_create(ctypes.byref(cfg), float(budget), int(pack_models), ctypes.byref(p))
        if not self.h:
            raise L.B200FemError(L.ERR_INVALID_ARG, "b200fem_server_create failed")
        for k, v in (options or {}).items():
            self._call("b200fem_server_set_option", int(k), int(v))
        for w in self.pool:
            if w.conn is None:
                w.build_mesh()
            m = w.model(precision=precision, device=device)
            prm = np.zeros(8)
            pp = m.material.params()
            prm[: len(pp)] = pp
            fext = None if m.fext is None else np.ascontiguousarray(m.fext.reshape(-1))
            idx = ctypes.c_int()
            self._call("b200fem_server_add_model", m.elem_type, m.numNodes(),
                       L.dptr(np.ascontiguousarray(m.rest.reshape(-1))), m.numElements(),
                       L.iptr(np.ascontiguousarray(m.conn.reshape(-1))), L.iptr(m.fixed), m.material.kind,
                       L.dptr(prm), m.density, m.soft_incomp, L.dptr(fext), ctypes.byref(idx))

    def _call(self, name, *args):
        st = getattr(self._lib, name)(self.h, *args)
        if st != 0:
            raise L.B200FemError(st, (self._lib.b200fem_server_last_error(self.h) or b"").decode(errors="replace"))
        return st

    def clock(self) -> float:
        return self._lib.b200fem_server_clock(self.h)

    def submit(self, model: int, steps: int, t_arrive: float = -1.0) -> int:
        rid = self._c.c_int()
        self._call("b200fem_server_submit", int(model), int(steps), float(t_arrive), self._c.byref(rid))
        return rid.value

    def preload(self):
        self._call("b200fem_server_preload")

    def tick(self) -> int:
        n = self._c.c_int()
        self._call("b200fem_server_tick", self._c.byref(n))
        return n.value

    def poll(self, rid: int):
        st, lat = self._c.c_int(), self._c.c_double()
        self._call("b200fem_server_poll", int(rid), self._c.byref(st), self._c.byref(lat))
        return st.value, lat.value

    def state(self, model: int):
        n = self.pool[model].rest.shape[0]
        x, v = np.zeros(3 * n), np.zeros(3 * n)
        self._call("b200fem_server_get_state", int(model), L.dptr(x), L.dptr(v))
        return x.reshape(-1, 3), v.reshape(-1, 3)

    def stats(self) -> dict:
        s = L.ServerStats()
        self._call("b200fem_server_get_stats", self._c.byref(s))
        return {k: getattr(s, k) for k, _ in L.ServerStats._fields_}

    def pending(self) -> int:
        return self.stats()["pending"]

    def close(self):
        if self.h:
            self._lib.b200fem_server_destroy(self.h)
            self.h = None


def run_stream_native(server: NativeServer, arrivals, steps_per_request: int = 10, drain_s: float = 30.0):
    """run_stream for the native server: requests are submitted with their
    scheduled arrival time on the server clock; latencies come from it."""
    times, models = arrivals
    t0 = server.clock()
    nxt = 0
    duration = float(times[-1]) if len(times) else 0.0
    rids = []
    pending = 0
    while True:
        now = server.clock() - t0
        while nxt < len(times) and times[nxt] <= now:
            rids.append(server.submit(int(models[nxt]), steps_per_request, t0 + float(times[nxt])))
            nxt += 1
            pending += 1
        if nxt >= len(times) and server.pending() == 0:
            break
        if now > duration + drain_s:
            break
        if server.pending() == 0:
            time.sleep(min(0.0005, max(0.0, float(times[nxt]) - now)))
            continue
        server.tick()
    wall = server.clock() - t0
    lat = []
    for r in rids:
        st, l = server.poll(r)
        if st == 2:
            lat.append(l * 1e3)
    lat = np.array(lat)
    s = server.stats()
    done = len(lat)
    return {
        "requests": len(rids), "completed": done, "incomplete": len(rids) - done, "wall_s": wall,
        "p50_ms": float(np.percentile(lat, 50)) if done else None,
        "p99_ms": float(np.percentile(lat, 99)) if done else None,
        "mean_ms": float(lat.mean()) if done else None,
        "requests_per_s": done / wall if wall > 0 else 0.0,
        "model_steps_per_s": s["model_steps"] / wall if wall > 0 else 0.0,
        "ticks": s["ticks"], "slot_steps": s["slot_steps"], "builds": s["builds"], "evictions": s["evictions"],
        "peak_bytes": s["peak_bytes"], "server": "native",
    }
