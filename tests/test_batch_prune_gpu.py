"""Candidate-chunk pruning of the batched cell-list pass: each 32-slot block
of a system's sorted atoms keeps an FP64 box, and a cell's candidate chunks
whose boxes lie beyond the cutoff are skipped.  These cases put the box test
where it is easiest to get wrong -- one-bin periodic cells whose 27 images
all hold every atom, lattice pairs at exactly the cutoff, skewed cells, and
isolated systems far from the origin -- and compare every call (the tuning
call with its recomputing emit, then the recorded count and its expansion)
with the oracle."""

import numpy as np
import pytest

from helpers import assert_same

pytestmark = pytest.mark.gpu

PBC3 = [True, True, True]


@pytest.fixture(scope="module")
def nl():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import neighborlist_rs

    return neighborlist_rs


def _concat(systems):
    pos = np.concatenate([p for p, _ in systems])
    batch = np.concatenate([np.full(len(p), i, dtype=np.int32) for i, (p, _) in enumerate(systems)])
    cells = np.stack([np.zeros((3, 3)) if c is None else c for _, c in systems])
    return pos, batch, cells


def _check(nl, oracle, systems, rc, calls=3):
    nl.batch_tuner_reset()
    pos, batch, cells = _concat(systems)
    ocells = [None if c is None else (c.T, PBC3) for _, c in systems]
    (ref,) = oracle.search_batch(pos, batch, ocells, [rc], nthreads=16)
    assert ref[0].shape[1] > 0
    for k in range(calls):
        got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=rc)
        assert_same(got, ref, f"call {k}")


def test_one_bin_lattice_pairs_at_the_cutoff(nl, oracle):
    # Cubic cells of 9.9 A (one bin at rc 5), atoms on a 2.5 A lattice: many
    # pairs lie at exactly 5.0 A (not neighbours) and their images at 4.9 A.
    g = np.arange(4) * 2.5
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    rng = np.random.default_rng(61)
    systems = []
    for s in range(96):
        cell = np.eye(3) * 9.9
        keep = rng.permutation(len(lat))[: int(rng.integers(20, 65))]
        p = lat[keep]
        if s % 3 == 1:  # a few atoms nudged by one ulp towards the cutoff
            p = np.nextafter(p, p + 1.0)
        systems.append((p, cell))
    _check(nl, oracle, systems, 5.0)


def test_one_bin_skewed_cells(nl, oracle):
    from neighborlist_rs import workloads as W

    rng = np.random.default_rng(62)
    systems = []
    for _ in range(256):
        n = int(rng.integers(8, 121))
        rows = W.density_cell(n, 0.1, rng, (60.0, 120.0))
        systems.append((rng.random((n, 3)) @ rows, rows))
    _check(nl, oracle, systems, 5.0)
    _check(nl, oracle, systems, 6.0, calls=2)


def test_isolated_cell_lists_far_from_the_origin(nl, oracle):
    # Isolated systems above the brute-force threshold take the cell list;
    # offsets of up to 1e6 A make the boxes' slack scale with the magnitude.
    rng = np.random.default_rng(63)
    systems = []
    for s in range(24):
        n = int(rng.integers(1000, 1600))
        side = (n / 0.1) ** (1.0 / 3.0)
        off = rng.uniform(-1e6, 1e6, 3) if s % 2 else np.zeros(3)
        systems.append((rng.random((n, 3)) * side + off, None))
    _check(nl, oracle, systems, 5.0, calls=2)
