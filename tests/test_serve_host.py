"""Host logic of the serving loop on the CPU: the server runs against a fake
pack that records the steps it is asked for, so scheduling, per-model FIFO
order, continuous batching and budget admission/eviction are checked
without a GPU."""
import numpy as np
import pytest

from artisynth_core_b200 import serve
from artisynth_core_b200 import workloads as W


class FakePack:
    BYTES_PER_ELEM = 1000
    live = []

    def __init__(self, models, precision=None, device=0, options=None):
        self.models = models
        self.x = [m.rest.copy() for m in models]
        self.v = [np.zeros_like(m.rest) for m in models]
        self.active = np.ones(len(models), dtype=bool)
        self.log = []
        self.stats = type("S", (), {"iterations": 7})()
        FakePack.live.append(self)

    def engine(self):
        return self

    def deviceBytes(self):
        return sum(m.conn.shape[0] for m in self.models) * self.BYTES_PER_ELEM

    def setActive(self, active=None):
        self.active = np.ones(len(self.models), dtype=bool) if active is None else np.asarray(active) != 0

    def setStates(self, xs, vs):
        self.x = [np.array(x) for x in xs]
        self.v = [np.array(v) for v in vs]

    def getStates(self):
        return list(zip(self.x, self.v))

    def backwardEuler(self, h, nsteps=1, tol=None, max_iter=None):
        self.log.append(self.active.copy())
        for i in np.nonzero(self.active)[0]:
            self.v[i] = self.v[i] + 1.0  # one "step": v counts the steps taken
            self.x[i] = self.x[i] + h * self.v[i]

    def lastTiming(self):
        return 0.1, 0.2

    def close(self):
        FakePack.live.remove(self)


@pytest.fixture
def pool(monkeypatch):
    monkeypatch.setattr(serve, "FemPack", FakePack)
    FakePack.live = []
    ws = W.batched_beams(count=6, seed=4)
    for w in ws:
        w.cells = (4, 2, 2)
        w.widths = (0.2, 0.1, 0.1)
        w.build_mesh()
    return ws


def drain(srv, limit=1000):
    for _ in range(limit):
        if not srv.pending():
            return
        srv.tick()
    raise AssertionError("requests still pending")


def steps_taken(srv, m):
    return int(round(srv.state(m)[1][0, 0]))


def test_fifo_and_continuous_batching(pool):
    srv = serve.FemServer(pool, pack_models=3)
    srv.submit(0, 3)
    srv.submit(1, 1)
    srv.tick()
    assert srv.stats.builds == 1
    srv.submit(0, 2)   # queues behind model 0's first request
    srv.submit(2, 2)   # same pack (admitted with the next batch)
    srv.submit(4, 1)   # a new pack while the first is in flight
    drain(srv)
    assert [steps_taken(srv, m) for m in range(6)] == [5, 1, 2, 0, 1, 0]
    r0 = [r for r in srv.done if r.model == 0]
    assert r0[0].t_done <= r0[1].t_start  # FIFO per model
    # idle models are masked out of a pack step, busy ones step together
    first = FakePack.live[0]
    assert first.log[0].tolist() == [True, True]
    assert any(a.sum() == 1 for a in first.log)


def test_budget_admission_and_eviction(pool):
    per = max(w.conn.shape[0] for w in pool) * FakePack.BYTES_PER_ELEM
    srv = serve.FemServer(pool, budget=2.5 * per, pack_models=1)
    srv.bytes_per_elem = FakePack.BYTES_PER_ELEM
    for m in range(6):
        srv.submit(m, 2)
    for _ in range(1000):
        if not srv.pending():
            break
        srv.tick()
        assert srv.resident_bytes() <= srv.budget
    assert srv.stats.evictions >= 3
    srv.submit(0, 1)  # an evicted model continues from its saved state
    drain(srv)
    assert [steps_taken(srv, m) for m in range(6)] == [3, 2, 2, 2, 2, 2]


def test_poisson_arrivals_deterministic():
    t1, m1 = serve.poisson_arrivals(2000.0, 1.0, 256, seed=4)
    t2, m2 = serve.poisson_arrivals(2000.0, 1.0, 256, seed=4)
    assert np.array_equal(t1, t2) and np.array_equal(m1, m2)
    assert np.all(np.diff(t1) > 0) and t1[-1] < 1.0
    assert 1800 < len(t1) < 2200 and m1.min() >= 0 and m1.max() < 256


def test_model_larger_than_budget_is_rejected(pool):
    srv = serve.FemServer(pool, budget=10 * FakePack.BYTES_PER_ELEM, pack_models=1)
    srv.bytes_per_elem = 1.0  # an estimate that lets it be tried
    r = srv.submit(2, 3)
    drain(srv)
    assert r.error and r in srv.failed and not srv.slots
