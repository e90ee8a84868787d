"""Autotuner for the layout options of a pack (B200FEM_OPT_*).

What it chooses, by timing real BackwardEuler steps on the device:
  * ROW_LANES  -- lanes per block row in the PCG SpMV (4, 8, 16, 32): the
                  trade between rows in flight per warp and blocks per lane;
  * ELEM_TILE  -- the non-linear element kernel: one thread per tetrahedron,
                  or the shared-memory staged kernel with its large or half tile;
  * PIECE_ROWS -- (packs with the strided split) rows per piece, i.e. how
                  finely the models are dealt over the CTAs, which sets the
                  PCG schedule of the pack.
ROW_LANES and ELEM_TILE change on the built pack; PIECE_ROWS needs a build
per candidate.  The tuning steps run on a copy of the state that is put back
afterwards, so tuning leaves the models where they were.

Results are cached by the shape of the pack -- element type and material
mix, precision, model count and size buckets -- in a JSON file
($B200FEM_TUNE_CACHE, default ~/.cache/artisynth_core_b200/tune.json), so a
pack of the same shape later starts tuned.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import _lib as L

LANES = (4, 8, 16, 32)
TILES = (0, 1, 2)
PIECE_ROWS = (32, 64, 128)


def cache_path() -> str:
    return os.environ.get("B200FEM_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "artisynth_core_b200", "tune.json"))


def shape_key(models, precision) -> str:
    """Key of a pack's shape: what the best layout depends on."""
    kinds = sorted({(m.elem_type, m.material.kind, int(getattr(m, "soft_incomp", 0))) for m in models})
    elems = sum(m.numElements() for m in models)
    nodes = sum(m.numNodes() for m in models)
    b = lambda v: int(round(math.log2(max(v, 1))))
    return json.dumps({"kinds": kinds, "prec": int(precision), "models": b(len(models)),
                       "elems": b(elems), "nodes_per_elem": round(nodes / max(elems, 1), 1)})


class TuneCache:
    def __init__(self, path: str | None = None):
        self.path = path or cache_path()
        self.data = {}
        if os.path.exists(self.path):
            try:
                self.data = json.load(open(self.path))
            except (OSError, ValueError):
                self.data = {}

    def get(self, key):
        return self.data.get(key)

    def put(self, key, value):
        self.data[key] = value
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            tmp = self.path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.data, f, indent=1, sort_keys=True)
            os.replace(tmp, self.path)
        except OSError:
            pass  # a read-only home only costs re-tuning


def _time_steps(pack, h, tol, reps):
    """Device times (assembly ms, PCG ms per iteration) of `reps` steps."""
    asm, pcg = [], []
    for _ in range(reps):
        pack.backwardEuler(h, 1, tol=tol)
        a, p = pack.lastTiming()
        asm.append(a)
        pcg.append(p / max(1, pack.stats.iterations))
    return min(asm), min(pcg)


def tune_runtime(pack, h, tol, reps=2):
    """Choose ROW_LANES and ELEM_TILE on a built pack; sets them and returns
    {"row_lanes", "elem_tile", "timings"}."""
    saved = pack.getStates()
    xs, vs = [x.copy() for x, _ in saved], [v.copy() for _, v in saved]
    pack.backwardEuler(h, 1, tol=tol)  # warm-up (graph capture)
    timings = {}
    best_lanes, best_pcg = None, math.inf
    for lanes in LANES:
        pack.setOption(L.OPT_ROW_LANES, lanes)
        pack.setStates(xs, vs)
        pack.backwardEuler(h, 1, tol=tol)
        _, p = _time_steps(pack, h, tol, reps)
        timings[f"lanes{lanes}_pcg_ms_per_it"] = p
        if p < best_pcg:
            best_lanes, best_pcg = lanes, p
    pack.setOption(L.OPT_ROW_LANES, best_lanes)
    best_tile, best_asm = None, math.inf
    for tile in TILES:
        pack.setOption(L.OPT_ELEM_TILE, tile)
        pack.setStates(xs, vs)
        pack.backwardEuler(h, 1, tol=tol)
        a, _ = _time_steps(pack, h, tol, reps)
        timings[f"tile{tile}_asm_ms"] = a
        if a < best_asm:
            best_tile, best_asm = tile, a
    pack.setOption(L.OPT_ELEM_TILE, best_tile)
    pack.setStates(xs, vs)
    return {"row_lanes": best_lanes, "elem_tile": best_tile, "timings": timings}


def tune_pack(make_pack, models, precision, h, tol, cache: TuneCache | None = None, piece_rows=True, reps=2):
    """Options for a pack of `models`: from the cache, else by timing.

    make_pack(options) -> a FemPack built with those build-time options.
    Returns (pack, options, from_cache): the pack built with the chosen
    options and already set to the chosen run-time ones."""
    cache = cache or TuneCache()
    key = shape_key(models, precision)
    hit = cache.get(key)
    if hit is not None:
        opts = {L.OPT_ROW_LANES: hit["row_lanes"], L.OPT_ELEM_TILE: hit["elem_tile"]}
        if hit.get("piece_rows"):
            opts[L.OPT_PIECE_ROWS] = hit["piece_rows"]
        return make_pack(opts), hit, True
    result = {}
    pack = make_pack({})
    strided = pack.option(L.OPT_PCG_SPLIT) == L.SPLIT_STRIDED
    if piece_rows and strided:
        best, best_t = None, math.inf
        for pr in PIECE_ROWS:
            cand = pack if pr == 64 else make_pack({L.OPT_PIECE_ROWS: pr})
            saved = cand.getStates()
            cand.backwardEuler(h, 1, tol=tol)
            _, p = _time_steps(cand, h, tol, reps)
            cand.setStates([x for x, _ in saved], [v for _, v in saved])
            result[f"piece{pr}_pcg_ms_per_it"] = p
            if p < best_t:
                if best is not None and best is not pack:
                    best.close()
                best, best_t = cand, p
                result["piece_rows"] = pr
            elif cand is not pack:
                cand.close()
        if best is not pack:
            pack.close()
        pack = best
    rt = tune_runtime(pack, h, tol, reps)
    result.update(rt["timings"])
    result["row_lanes"], result["elem_tile"] = rt["row_lanes"], rt["elem_tile"]
    cache.put(key, result)
    return pack, result, False
