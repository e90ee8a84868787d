"""Synthetic workloads of the benchmark: structured grids from
``FemFactory.createTetGrid/createHexGrid`` with seeded interior jitter.

Reference defaults that the workloads state explicitly:
* ``LinearMaterial(E, nu)`` is corotated (LinearMaterial.java:53-55);
* massDamping 2, stiffnessDamping 0 (FemModel.java:303-304);
* grids are centred at the origin, so "the x = 0 face" of a beam is the
  x = -wx/2 face (FemFactory.java:53-78);
* MooneyRivlin with soft incompressibility AUTO resolves to NODAL when there
  are more elements than active nodes (FemModel3d.java:462-481).
* The reference has no surface-traction load; the hex beam's traction is
  applied as consistent nodal forces on the flat x-max face, in -z.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .femmodel import (FemModel3d, LinearMaterial, MooneyRivlinMaterial, NeoHookeanMaterial,
                       create_grid, jitter_grid)


@dataclass
class Workload:
    name: str
    elem_type: int
    cells: tuple
    widths: tuple
    jitter: float
    seed: int
    material: object
    density: float
    fix: str  # 'xmin' or 'zmin'
    gravity: tuple
    h: float
    steps: int
    tol: float = 1e-10
    traction: tuple | None = None  # traction vector on the x-max face
    mass_damping: float = 2.0
    stiffness_damping: float = 0.0
    rest: np.ndarray = field(default=None, repr=False)
    conn: np.ndarray = field(default=None, repr=False)
    fixed: np.ndarray = field(default=None, repr=False)
    fext: np.ndarray = field(default=None, repr=False)

    def build_mesh(self, mesher=None):
        """Grid, jitter, fixed nodes and external forces.  `mesher(elem_type,
        widths, cells, jitter, seed) -> (xyz, conn)` replaces the library's
        grid factory (a caller that must not load the library, such as a CPU
        baseline, passes a generator of its own that makes the same mesh)."""
        nx, ny, nz = self.cells
        wx, wy, wz = self.widths
        if mesher is not None:
            xyz, conn = mesher(self.elem_type, self.widths, self.cells, self.jitter, self.seed)
        else:
            xyz, conn = create_grid(self.elem_type, wx, wy, wz, nx, ny, nz)
            if self.jitter:
                xyz = jitter_grid(xyz, nx, ny, nz, wx, wy, wz, self.jitter, self.seed)
        self.rest, self.conn = xyz, conn
        if self.fix == "xmin":
            self.fixed = (xyz[:, 0] <= -wx / 2 + 1e-9).astype(np.int32)
        else:
            self.fixed = (xyz[:, 2] <= -wz / 2 + 1e-9).astype(np.int32)
        self.fext = np.zeros_like(xyz)
        if self.traction is not None:
            # consistent nodal forces of a uniform traction on the flat,
            # rectangular faces of the x-max boundary: area/4 per corner
            area = (wy / ny) * (wz / nz)
            t = np.asarray(self.traction, dtype=np.float64)
            idx = np.arange(xyz.shape[0])
            i = idx % (nx + 1)
            j = (idx // (nx + 1)) % (ny + 1)
            k = idx // ((nx + 1) * (ny + 1))
            on = i == nx
            cj = np.where((j == 0) | (j == ny), 1, 2)
            ck = np.where((k == 0) | (k == nz), 1, 2)
            w = np.where(on, cj * ck, 0) * (area / 4)
            self.fext = w[:, None] * t[None, :]
        return self

    def model(self, precision=L.PREC_FP64, device=0) -> FemModel3d:
        if self.rest is None:
            self.build_mesh()
        m = FemModel3d()
        m.setMesh(self.elem_type, self.rest, self.conn, self.fixed)
        m.setMaterial(self.material)
        m.setDensity(self.density)
        m.setMassDamping(self.mass_damping)
        m.setStiffnessDamping(self.stiffness_damping)
        m.setGravity(np.array(self.gravity, dtype=np.float64))
        m.precision = precision
        m.device = device
        if self.traction is not None:
            m.setExternalForces(self.fext)
        return m

    def describe(self):
        return {"workload": self.name, "elem": "tet" if self.elem_type == L.ELEM_TET else "hex",
                "cells": list(self.cells), "widths": list(self.widths), "steps": self.steps, "h": self.h}


def linear_tet_beam() -> Workload:
    """10x2x2 cells of a 1.0x0.2x0.2 m beam, 5 tets per cell (200 tets, 99
    nodes), jitter 5% (seed 0), corotated LinearMaterial(1e5, 0.33), density
    1000, x-min face fixed, gravity -9.81 z, 100 steps of h = 0.01."""
    return Workload("linear_tet_beam_10x2x2", L.ELEM_TET, (10, 2, 2), (1.0, 0.2, 0.2), 0.05, 0,
                    LinearMaterial(1e5, 0.33, True), 1000.0, "xmin", (0.0, 0.0, -9.81), 0.01, 100,
                    tol=1e-13)


def neohookean_hex_beam() -> Workload:
    """40x10x10 hexes (8 Gauss points) over a 1.0x0.25x0.25 m beam (4,000
    hexes, 4,961 nodes), jitter 3% (seed 1), NeoHookean(5e4, 0.45), density
    1000, x-min face fixed, 10 N/m^2 traction on the x-max face, 200 steps
    of h = 0.005, PCG to 1e-10 relative residual."""
    return Workload("neohookean_hex_beam_40x10x10", L.ELEM_HEX, (40, 10, 10), (1.0, 0.25, 0.25), 0.03, 1,
                    NeoHookeanMaterial(5e4, 0.45), 1000.0, "xmin", (0.0, 0.0, 0.0), 0.005, 200,
                    tol=1e-10, traction=(0.0, 0.0, -10.0))


def mooneyrivlin_tet_block() -> Workload:
    """60x30x30 cells of a 0.3x0.15x0.15 m block, 5 tets per cell (270,000
    tets, 58,621 nodes), jitter 5% (seed 2), MooneyRivlin(c10=1000,
    c01=500, kappa=1e5), density 1050, z-min face fixed, gravity, 50 steps of
    h = 0.01."""
    return Workload("mooneyrivlin_tet_block_60x30x30", L.ELEM_TET, (60, 30, 30), (0.3, 0.15, 0.15), 0.05, 2,
                    MooneyRivlinMaterial(1000.0, 500.0, 0.0, 0.0, 0.0, 1e5), 1050.0, "zmin",
                    (0.0, 0.0, -9.81), 0.01, 50, tol=1e-10)


def small_tet_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.05, seed=7,
                   gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    """Small beams in the shapes of the reference's own equivalence tests
    (FemModel3dTest.runNonlinearBeamStep, FemModel3dTest.java:970-1055)."""
    return Workload("small_tet_beam", L.ELEM_TET, cells, widths, jitter, seed, material, 1000.0, "xmin",
                    gravity, h, steps, tol=1e-13)


def small_hex_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.03, seed=11,
                   gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    return Workload("small_hex_beam", L.ELEM_HEX, cells, widths, jitter, seed, material, 1000.0, "xmin",
                    gravity, h, steps, tol=1e-13)


def small_wedge_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.03, seed=13,
                     gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    """Small beam of wedges (FemFactory.createWedgeGrid: two per cell)."""
    return Workload("small_wedge_beam", L.ELEM_WEDGE, cells, widths, jitter, seed, material, 1000.0, "xmin",
                    gravity, h, steps, tol=1e-13)


def small_pyramid_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.03, seed=17,
                       gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    """Small beam of pyramids (FemFactory.createPyramidGrid: three per cell)."""
    return Workload("small_pyramid_beam", L.ELEM_PYRAMID, cells, widths, jitter, seed, material, 1000.0, "xmin",
                    gravity, h, steps, tol=1e-13)


def small_quadtet_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.03, seed=19,
                       gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    """Small beam of quadratic tets (FemFactory.createQuadtetGrid: the tet
    grid with shared edge nodes; the jitter moves the lattice nodes only, so
    edges bend slightly)."""
    return Workload("small_quadtet_beam", L.ELEM_QUADTET, cells, widths, jitter, seed, material, 1000.0, "xmin",
                    gravity, h, steps, tol=1e-13)


def small_quadhex_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.03, seed=23,
                       gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    """Small beam of quadratic hexes (FemFactory.createQuadhexGrid)."""
    return Workload("small_quadhex_beam", L.ELEM_QUADHEX, cells, widths, jitter, seed, material, 1000.0, "xmin",
                    gravity, h, steps, tol=1e-13)


def small_quadwedge_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.03, seed=29,
                         gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    """Small beam of quadratic wedges (FemFactory.createQuadwedgeGrid)."""
    return Workload("small_quadwedge_beam", L.ELEM_QUADWEDGE, cells, widths, jitter, seed, material, 1000.0, "xmin",
                    gravity, h, steps, tol=1e-13)


def small_quadpyramid_beam(material, cells=(4, 2, 2), widths=(1.0, 0.4, 0.4), jitter=0.03, seed=31,
                           gravity=(0.0, 0.0, -9.81), h=0.005, steps=10) -> Workload:
    """Small beam of quadratic pyramids (FemFactory.createQuadpyramidGrid)."""
    return Workload("small_quadpyramid_beam", L.ELEM_QUADPYRAMID, cells, widths, jitter, seed, material, 1000.0,
                    "xmin", gravity, h, steps, tol=1e-13)


def batched_beams(count=256, seed=3, cell=0.05, jitter=0.05, large_frac=0.0, large_n=(80, 120)):
    """Uneven NeoHookean tet beams: n x m x m cells of size `cell` (5 tets per
    cell), n ~ U{4..60}, m ~ U{2..8}, E log-uniform in [1e3, 1e6] Pa, nu
    uniform in [0.30, 0.49], density 1000, x-min face fixed, gravity; 20
    steps of h = 0.01.  With large_frac > 0 that fraction of the beams draws
    n ~ U{80..120} instead (the served-stream distribution)."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.integers(4, 61))
        if large_frac and rng.random() < large_frac:
            n = int(rng.integers(large_n[0], large_n[1] + 1))
        m = int(rng.integers(2, 9))
        E = float(10 ** rng.uniform(3, 6))
        nu = float(rng.uniform(0.30, 0.49))
        wl = Workload(f"beam{i}_{n}x{m}x{m}", L.ELEM_TET, (n, m, m), (n * cell, m * cell, m * cell), jitter,
                      1000 + i, NeoHookeanMaterial(E, nu), 1000.0, "xmin", (0.0, 0.0, -9.81), 0.01, 20,
                      tol=1e-10)
        out.append(wl)
    return out
