"""The C-ABI library loads and exports every entry point declared in
include/b200fem.h; the host-only mesh factory matches the oracle bit for
bit; without a device, handle creation fails with a status instead of
falling back to the CPU."""
import ctypes

import numpy as np
import pytest

from conftest import HAVE_GPU


def test_exports_every_declared_symbol(b200):
    L = b200.lib()
    names = b200._lib.header_symbols()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


@pytest.mark.parametrize("etype,cells,widths,jit,seed", [
    (0, (10, 2, 2), (1.0, 0.2, 0.2), 0.05, 0),
    (1, (40, 10, 10), (1.0, 0.25, 0.25), 0.03, 1),
    (0, (7, 3, 2), (0.3, 0.15, 0.15), 0.05, 2),
    (1, (1, 1, 1), (1.0, 0.8, 0.6), 0.0, 0),
])
def test_grid_factory_matches_oracle(b200, oracle, etype, cells, widths, jit, seed):
    x, c = b200.create_grid(etype, *widths, *cells)
    if jit:
        x = b200.jitter_grid(x, *cells, *widths, jit, seed)
    ox, oc = oracle.grid(etype, widths, cells, jit, seed)
    assert np.array_equal(x, ox) and np.array_equal(c, oc)


def test_grid_factory_rejects_bad_sizes(b200):
    with pytest.raises(b200.B200FemError) as ei:
        b200.create_grid(0, 1.0, 1.0, 1.0, 0, 1, 1)
    assert ei.value.status == b200._lib.ERR_INVALID_ARG


@pytest.mark.skipif(HAVE_GPU, reason="checks the no-device failure path")
def test_create_without_device_fails_loudly(b200):
    L = b200.lib()
    cfg = b200._lib.Config(0, 0)
    h = L.b200fem_create(ctypes.byref(cfg))
    assert not h
    assert b"CUDA" in L.b200fem_last_error(None) or b"device" in L.b200fem_last_error(None)
    assert L.b200fem_destroy(None) == 0
