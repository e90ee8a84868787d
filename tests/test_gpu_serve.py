"""Served stream on the GPU: continuous batching over resident packs.

* a request's result equals its model stepped alone (1e-9 at PCG 1e-12:
  only the dot-product partition differs), whether it ran alone or in the
  mix, including models admitted while others were in flight and models
  evicted under the memory budget and re-admitted from their saved state;
* a short Poisson stream completes and reports latency percentiles.
"""
import numpy as np
import pytest

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import workloads as W
from artisynth_core_b200.femmodel import MechSystemSolver
from artisynth_core_b200.serve import FemServer, poisson_arrivals, run_stream

from helpers import rel_err

pytestmark = [pytest.mark.gpu, pytest.mark.timeout(600)]


def drain(srv, limit=10000):
    for _ in range(limit):
        if not srv.pending():
            return
        srv.tick()
    raise AssertionError("requests still pending after %d ticks" % limit)


def _pool(count=8, seed=4):
    ws = W.batched_beams(count=count, seed=seed, large_frac=0.1)
    for w in ws:
        w.cells = (min(w.cells[0], 10), w.cells[1], w.cells[2])
        w.widths = (w.cells[0] * 0.05, w.widths[1], w.widths[2])
        w.build_mesh()
    return ws


def _alone(w, steps, precision):
    m = w.model(precision=precision)
    MechSystemSolver(m, tol=1e-12).backwardEuler(w.h, steps)
    x, _ = m.getState()
    m._invalidate()
    return x


@pytest.mark.parametrize("precision", [L.PREC_MIXED, L.PREC_FP64])
def test_results_same_alone_and_in_the_mix(b200, precision):
    pool = _pool()
    srv = FemServer(pool, precision=precision, tol=1e-12, pack_models=4)
    steps = {m: 0 for m in range(len(pool))}

    def submit(m, k):
        srv.submit(m, k)
        steps[m] += k

    # a first wave, then requests arriving while those are on the GPU
    for m in (0, 1, 2):
        submit(m, 5)
    srv.tick()
    srv.tick()
    submit(3, 4)      # a new model joins mid-flight
    submit(0, 3)      # a second request queues behind model 0's first
    srv.tick()
    for m in (4, 5, 6, 7):
        submit(m, 2)
    drain(srv)
    assert srv.stats.builds >= 2  # later arrivals were admitted as new packs
    assert all(r.t_done is not None for r in srv.done)
    for m, w in enumerate(pool):
        x, _ = srv.state(m)
        xa = _alone(w, steps[m], precision)
        assert rel_err(x, xa) <= 1e-9, (m, rel_err(x, xa))
    srv.close()


def test_budget_evicts_idle_packs_and_restores_state(b200):
    pool = _pool(count=6, seed=8)
    probe = FemServer(pool[:2], tol=1e-12, pack_models=2)
    for m in (0, 1):
        probe.submit(m, 1)
    probe.tick()
    per_elem = probe.resident_bytes() / sum(w.conn.shape[0] for w in pool[:2])
    probe.close()
    # room for the biggest model and a small one at a time
    biggest = max(w.conn.shape[0] for w in pool) * per_elem
    assert sum(w.conn.shape[0] for w in pool) * per_elem > 1.5 * biggest
    srv = FemServer(pool, budget=1.3 * biggest, tol=1e-12, pack_models=2)
    steps = {m: 0 for m in range(len(pool))}
    for rnd in range(2):
        for m in range(len(pool)):
            srv.submit(m, 2)
            steps[m] += 2
            drain(srv)
    assert srv.stats.evictions > 0 and not srv.failed
    assert srv.stats.peak_bytes <= 1.25 * srv.budget  # at most an estimate's error over
    for m, w in enumerate(pool):
        x, _ = srv.state(m)
        assert rel_err(x, _alone(w, steps[m], L.PREC_MIXED)) <= 1e-9, m
    srv.close()


def test_short_poisson_stream(b200):
    pool = _pool(count=12, seed=4)
    srv = FemServer(pool, tol=1e-10)
    arrivals = poisson_arrivals(200.0, 0.5, len(pool), seed=4)
    out = run_stream(srv, arrivals, steps_per_request=3, drain_s=30.0)
    assert out["requests"] == len(arrivals[0]) > 0
    assert out["incomplete"] == 0
    assert 0 < out["p50_ms"] <= out["p99_ms"]
    assert out["model_steps_per_s"] > 0
    srv.close()


# ---- the native server (b200fem_server_*, what a Java host binds) --------
from artisynth_core_b200.serve import NativeServer, run_stream_native  # noqa: E402


def test_native_server_same_alone_and_in_the_mix(b200):
    pool = _pool()
    srv = NativeServer(pool, tol=1e-12, pack_models=4)
    steps = {m: 0 for m in range(len(pool))}
    rids = []

    def submit(m, k):
        rids.append(srv.submit(m, k))
        steps[m] += k

    for m in (0, 1, 2):
        submit(m, 5)
    srv.tick()
    srv.tick()
    submit(3, 4)
    submit(0, 3)
    srv.tick()
    for m in (4, 5, 6, 7):
        submit(m, 2)
    for _ in range(1000):
        if not srv.pending():
            break
        srv.tick()
    assert srv.pending() == 0
    st = srv.stats()
    assert st["builds"] >= 2 and st["completed"] == len(rids) and st["failed"] == 0
    for r in rids:
        state, lat = srv.poll(r)
        assert state == 2 and lat > 0
    for m, w in enumerate(pool):
        x, _ = srv.state(m)
        xa = _alone(w, steps[m], L.PREC_MIXED)
        assert rel_err(x, xa) <= 1e-9, (m, rel_err(x, xa))
    srv.close()


def test_native_server_budget_eviction(b200):
    pool = _pool(count=6, seed=8)
    probe = FemServer(pool[:2], tol=1e-12, pack_models=2)
    for m in (0, 1):
        probe.submit(m, 1)
    probe.tick()
    per_elem = probe.resident_bytes() / sum(w.conn.shape[0] for w in pool[:2])
    probe.close()
    biggest = max(w.conn.shape[0] for w in pool) * per_elem
    srv = NativeServer(pool, budget=1.3 * biggest, tol=1e-12, pack_models=2)
    steps = {m: 0 for m in range(len(pool))}
    for rnd in range(2):
        for m in range(len(pool)):
            srv.submit(m, 2)
            steps[m] += 2
            for _ in range(1000):
                if not srv.pending():
                    break
                srv.tick()
    st = srv.stats()
    assert st["evictions"] > 0 and st["failed"] == 0 and st["pending"] == 0
    for m, w in enumerate(pool):
        x, _ = srv.state(m)
        assert rel_err(x, _alone(w, steps[m], L.PREC_MIXED)) <= 1e-9, m
    srv.close()


def test_native_short_poisson_stream(b200):
    pool = _pool(count=12, seed=4)
    srv = NativeServer(pool, tol=1e-10, options={L.OPT_ROW_LANES: 4})
    srv.preload()
    out = run_stream_native(srv, poisson_arrivals(200.0, 0.5, len(pool), seed=4), steps_per_request=3)
    assert out["incomplete"] == 0 and out["requests"] > 0
    assert 0 < out["p50_ms"] <= out["p99_ms"]
    srv.close()
