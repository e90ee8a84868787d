"""Shared helpers of the parity tests: build the same model in the oracle
and in the engine, and deformed states that exercise every term."""
import numpy as np

from artisynth_core_b200 import _lib as L


def oracle_model(O, wl):
    if wl.rest is None:
        wl.build_mesh()
    m = wl.material
    return O.OracleModel(wl.elem_type, wl.rest, wl.conn, wl.fixed, m.kind, m.params(), wl.density,
                         getattr(wl, "incomp", L.INCOMP_AUTO))


def deformed(rest, seed=3, rot_deg=25.0, bend=0.05, noise=0.002):
    """Rigid rotation + bending + small random perturbation of the rest
    positions (keeps every element well shaped)."""
    rng = np.random.default_rng(seed)
    x = rest.copy()
    xs = x[:, 0] - x[:, 0].min()
    x[:, 2] += bend * xs ** 2
    x += noise * rng.standard_normal(x.shape) * (np.ptp(rest, axis=0).min() / 10)
    t = np.deg2rad(rot_deg)
    R = np.array([[np.cos(t), 0, np.sin(t)], [0, 1, 0], [-np.sin(t), 0, np.cos(t)]])
    a = np.deg2rad(10.0)
    R2 = np.array([[np.cos(a), -np.sin(a), 0], [np.sin(a), np.cos(a), 0], [0, 0, 1]])
    return x @ (R2 @ R).T


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale
