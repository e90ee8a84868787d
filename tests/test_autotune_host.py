"""Autotuner logic on the CPU, against a fake pack whose step times depend
on the layout options: it must pick the fastest setting of each option,
leave the models' state as it found it, and serve the choice from the cache
for a pack of the same shape."""
import numpy as np

from artisynth_core_b200 import _lib as L
from artisynth_core_b200 import autotune
from artisynth_core_b200 import workloads as W


class FakePack:
    built = 0

    def __init__(self, models, options):
        FakePack.built += 1
        self.models = models
        self.opts = {L.OPT_ROW_LANES: 16, L.OPT_ELEM_TILE: 1, L.OPT_PIECE_ROWS: 64}
        self.opts.update(options)
        self.x = [m.rest.copy() for m in models]
        self.v = [np.zeros_like(m.rest) for m in models]
        self.stats = type("S", (), {"iterations": 10})()
        self.closed = False

    def option(self, key):
        return L.SPLIT_STRIDED if key == L.OPT_PCG_SPLIT else self.opts[key]

    def setOption(self, key, value):
        self.opts[key] = value

    def getStates(self):
        return [(x.copy(), v.copy()) for x, v in zip(self.x, self.v)]

    def setStates(self, xs, vs):
        self.x = [np.array(x) for x in xs]
        self.v = [np.array(v) for v in vs]

    def backwardEuler(self, h, n=1, tol=None):
        for v in self.v:
            v += 1.0

    def lastTiming(self):
        lanes = self.opts[L.OPT_ROW_LANES]
        pcg = {4: 3.0, 8: 2.0, 16: 4.0, 32: 5.0}[lanes] * (1.0 if self.opts[L.OPT_PIECE_ROWS] == 32 else 1.5)
        asm = {0: 1.5, 1: 2.0, 2: 1.0}[self.opts[L.OPT_ELEM_TILE]]
        return asm, pcg * self.stats.iterations

    def close(self):
        self.closed = True


def models():
    ws = W.batched_beams(count=3, seed=1)
    out = []
    for w in ws:
        w.cells = (4, 2, 2)
        w.widths = (0.2, 0.1, 0.1)
        out.append(w.build_mesh().model())
    return out


def test_picks_fastest_and_restores_state(tmp_path):
    ms = models()
    cache = autotune.TuneCache(str(tmp_path / "tune.json"))
    FakePack.built = 0
    pack, res, hit = autotune.tune_pack(lambda o: FakePack(ms, o), ms, L.PREC_MIXED, 0.01, 1e-6, cache=cache)
    assert not hit
    assert res["row_lanes"] == 8 and res["elem_tile"] == 2 and res["piece_rows"] == 32
    assert pack.opts[L.OPT_ROW_LANES] == 8 and pack.opts[L.OPT_ELEM_TILE] == 2
    assert pack.opts[L.OPT_PIECE_ROWS] == 32
    for x, v in pack.getStates():
        assert np.all(v == 0)  # tuning steps did not advance the models
    # same shape: served from the cache, one build
    FakePack.built = 0
    pack2, res2, hit2 = autotune.tune_pack(lambda o: FakePack(ms, o), ms, L.PREC_MIXED, 0.01, 1e-6,
                                           cache=autotune.TuneCache(str(tmp_path / "tune.json")))
    assert hit2 and FakePack.built == 1
    assert pack2.opts[L.OPT_ROW_LANES] == 8 and pack2.opts[L.OPT_PIECE_ROWS] == 32


def test_shape_key_separates_precision_and_size():
    ms = models()
    k1 = autotune.shape_key(ms, L.PREC_MIXED)
    assert k1 == autotune.shape_key(ms, L.PREC_MIXED)
    assert k1 != autotune.shape_key(ms, L.PREC_FP64)
    assert k1 != autotune.shape_key(ms * 8, L.PREC_MIXED)
