"""Seeded synthetic structures with the shapes of the benchmark workloads.

The reference benchmarks on fixture files (tests/data/*.xyz of
neighborlist-rs) and on ad-hoc molecules; the workloads below are seeded
synthetic stand-ins with the sizes, densities and cell shapes of the
benchmark configurations:

* ``isolated_cube``    -- N=1000 uniform in [0, 21.5)^3, no cell (rc 6)
* ``cluster_liquid``   -- 1112 rigid 9-atom clusters in a cubic L=46.4 box,
                           full PBC (rc 6 and 14)
* ``triclinic_uniform``-- N=20000 uniform in fractional coordinates, lengths
                           U(50,60), angles U(70,110) (rc 5/6/12 multi pass)
* ``uneven_batch``     -- 4096 systems, N ~ U{8..256}, density 0.1; half
                           isolated, half triclinic PBC with angles U(75,105)
* ``request_stream``   -- served stream: N log-uniform in [16, 1e6], 70 %
                           orthorhombic, 20 % triclinic, 10 % isolated,
                           density 0.1, rc in {5, 6, 8}

Cells are returned as ``rows`` (ASE convention: each row a lattice vector).
The library's single-system API takes ``h = rows.T`` (columns = lattice
vectors); the batched API takes the row form and transposes it.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def cell_from_parameters(a, b, c, alpha, beta, gamma):
    """Lattice rows from lengths and angles (degrees); None if not a valid cell."""
    ca, cb, cg = (math.cos(math.radians(x)) for x in (alpha, beta, gamma))
    sg = math.sin(math.radians(gamma))
    cx = cb
    cy = (ca - cb * cg) / sg
    arg = 1.0 - cx * cx - cy * cy
    if arg <= 1e-6:
        return None
    return np.array([[a, 0.0, 0.0],
                     [b * cg, b * sg, 0.0],
                     [c * cx, c * cy, c * math.sqrt(arg)]], dtype=np.float64)


def random_rotation(rng):
    """Uniformly random rotation matrix (quaternion method)."""
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def isolated_cube(n=1000, side=21.5, seed=1):
    rng = np.random.default_rng(seed)
    return rng.random((n, 3)) * side


def cluster_liquid(n_clusters=1112, per_cluster=9, box=46.4, sigma=0.8, min_sep=0.9, seed=2):
    """Rigid clusters: offsets N(0, sigma) about each centre with rejection to a
    minimum intra-cluster separation, uniformly random orientation, uniform
    centres in a cubic box.  Returns (positions, cell_rows)."""
    rng = np.random.default_rng(seed)
    # One template per cluster, drawn with rejection.
    pos = np.empty((n_clusters * per_cluster, 3), dtype=np.float64)
    for c in range(n_clusters):
        while True:
            off = rng.normal(0.0, sigma, size=(per_cluster, 3))
            d = np.linalg.norm(off[:, None, :] - off[None, :, :], axis=-1)
            d[np.diag_indices(per_cluster)] = np.inf
            if d.min() >= min_sep:
                break
        off -= off.mean(axis=0)
        centre = rng.random(3) * box
        pos[c * per_cluster:(c + 1) * per_cluster] = centre + off @ random_rotation(rng).T
    return pos, np.diag([box, box, box]).astype(np.float64)


def triclinic_uniform(n=20000, seed=3, lengths=(50.0, 60.0), angles=(70.0, 110.0)):
    rng = np.random.default_rng(seed)
    while True:
        a, b, c = rng.uniform(*lengths, size=3)
        al, be, ga = rng.uniform(*angles, size=3)
        rows = cell_from_parameters(a, b, c, al, be, ga)
        if rows is not None:
            break
    frac = rng.random((n, 3))
    return frac @ rows, rows


@dataclass
class System:
    positions: np.ndarray          # (N, 3) float64
    cell_rows: np.ndarray | None   # (3, 3) rows = lattice vectors, None = isolated
    cutoff: float = 5.0


def density_cell(n, density, rng, angle_range, ortho=False):
    """Triclinic (or orthorhombic) cell whose volume holds n atoms at `density`."""
    vol = n / density
    while True:
        if ortho:
            al = be = ga = 90.0
        else:
            al, be, ga = rng.uniform(*angle_range, size=3)
        unit = cell_from_parameters(1.0, 1.0, 1.0, al, be, ga)
        if unit is not None:
            break
    v1 = abs(np.linalg.det(unit))
    return unit * (vol / v1) ** (1.0 / 3.0)


def uneven_batch(n_systems=4096, n_range=(8, 256), density=0.1, seed=4,
                 angle_range=(75.0, 105.0)):
    """Half isolated, half triclinic PBC systems (alternating)."""
    rng = np.random.default_rng(seed)
    systems = []
    for s in range(n_systems):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        if s % 2 == 0:
            side = (n / density) ** (1.0 / 3.0)
            systems.append(System(rng.random((n, 3)) * side, None, 5.0))
        else:
            rows = density_cell(n, density, rng, angle_range)
            systems.append(System(rng.random((n, 3)) @ rows, rows, 5.0))
    return systems


def request_stream(n_requests, seed=5, n_range=(16, 1_000_000), density=0.1,
                   cutoffs=(5.0, 6.0, 8.0), max_atoms=None):
    """Served stream structures (positions, cell rows or None, cutoff)."""
    rng = np.random.default_rng(seed)
    out = []
    lo, hi = math.log(n_range[0]), math.log(n_range[1] if max_atoms is None
                                             else min(n_range[1], max_atoms))
    for _ in range(n_requests):
        n = int(round(math.exp(rng.uniform(lo, hi))))
        kind = rng.random()
        rc = float(rng.choice(cutoffs))
        if kind < 0.7:
            rows = density_cell(n, density, rng, None, ortho=True)
            out.append(System(rng.random((n, 3)) @ rows, rows, rc))
        elif kind < 0.9:
            rows = density_cell(n, density, rng, (75.0, 105.0))
            out.append(System(rng.random((n, 3)) @ rows, rows, rc))
        else:
            side = (n / density) ** (1.0 / 3.0)
            out.append(System(rng.random((n, 3)) * side, None, rc))
    return out


def concat_batch(systems):
    """positions (sum N, 3), batch int32, cells (B, 3, 3) rows (zeros = isolated)."""
    pos = np.concatenate([s.positions for s in systems], axis=0)
    batch = np.concatenate([np.full(len(s.positions), i, np.int32)
                            for i, s in enumerate(systems)])
    cells = np.zeros((len(systems), 3, 3), np.float64)
    for i, s in enumerate(systems):
        if s.cell_rows is not None:
            cells[i] = s.cell_rows
    return pos, batch, cells
