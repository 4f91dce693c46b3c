"""Device-sized batched builds and their CUDA-graph replay: a batch of small
systems runs plan -> count -> scan -> emit without a host round trip (the
emit pass reads each list's total on the device), a repeated identical batch
replays a captured graph, new positions of the same shapes reuse it, and an
arena that turns out too small is grown and the emit pass rerun -- every
result equal to the oracle's."""

import ctypes

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

    neighborlist_rs._lib.nlb_graph_replays.restype = ctypes.c_int64
    return neighborlist_rs


def replays(nl):
    return int(nl._lib.nlb_graph_replays())


def test_repeated_batch_replays_a_graph(nl, oracle):
    from neighborlist_rs import workloads as W

    systems = W.uneven_batch(n_systems=1024, seed=51)
    pos, batch, cells = W.concat_batch(systems)
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    (ref,) = oracle.search_batch(pos, batch, ocells, [5.0], nthreads=16)
    r0 = replays(nl)
    for k in range(5):  # tuning call, direct calls while the arenas settle, capture, replay
        got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
        assert_same(got, ref, f"call {k}")
    assert replays(nl) - r0 >= 2
    # With the per-system offset table (a different launch sequence).
    got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0, return_offsets=True)
    assert_same(got, ref, "offsets call")
    counts = np.bincount(batch[ref[0][0]], minlength=1024)
    assert np.array_equal(got["system_offsets"], np.concatenate([[0], np.cumsum(counts)]))
    # New positions (and cells) of the same shapes reuse the graph.
    rng = np.random.default_rng(52)
    moved = pos + rng.normal(0.0, 0.05, pos.shape)
    cells2 = cells * 1.01
    ocells2 = [None if not c.any() else (c.T, PBC3) for c in cells2]
    (ref2,) = oracle.search_batch(moved, batch, ocells2, [5.0], nthreads=16)
    for k in range(3):
        assert_same(nl.build_neighborlists_batch(moved, batch, cells=cells2, cutoff=5.0), ref2,
                    f"moved call {k}")
    r1 = replays(nl)
    for k in range(2):
        assert_same(nl.build_neighborlists_batch(moved, batch, cells=cells2, cutoff=5.0), ref2,
                    f"moved replay {k}")
    assert replays(nl) - r1 == 2


def test_multi_cutoff_batch_graph_and_offsets(nl, oracle):
    from neighborlist_rs import workloads as W

    pos, batch, cells = W.concat_batch(W.uneven_batch(n_systems=600, seed=53))
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    cutoffs = [5.0, 2.5, 4.0, 3.0, 4.5]  # two passes of the batched kernels
    ref = oracle.search_batch(pos, batch, ocells, cutoffs, disjoint=True, nthreads=16)
    r0 = replays(nl)
    for k in range(4):
        got = nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=cutoffs,
                                                 disjoint=True, return_offsets=True)
        for q, rc in enumerate(cutoffs):
            assert_same(got[q], ref[q], f"call {k} rc {rc}")
            counts = np.bincount(batch[ref[q][0][0]], minlength=600) if ref[q][0].shape[1] \
                else np.zeros(600, np.int64)
            assert np.array_equal(got[q]["system_offsets"],
                                  np.concatenate([[0], np.cumsum(counts)]))
    assert replays(nl) - r0 >= 1


def test_small_arena_is_grown_and_emitted_again(nl, oracle):
    """Tiny periodic boxes at a long cutoff: hundreds of image edges per atom,
    far above the first arena's 16 per atom, so the first device-sized call
    finds its arena too small, grows it and runs the emit pass again."""
    rng = np.random.default_rng(54)
    systems_pos, batch, cells = [], [], []
    for s in range(48):
        n = int(rng.integers(8, 40))
        rows = np.diag(rng.uniform(4.0, 6.0, 3))
        systems_pos.append(rng.random((n, 3)) @ rows)
        batch.append(np.full(n, s, np.int32))
        cells.append(rows)
    pos = np.concatenate(systems_pos)
    batch = np.concatenate(batch)
    cells = np.array(cells)
    ocells = [(c.T, PBC3) for c in cells]
    (ref,) = oracle.search_batch(pos, batch, ocells, [9.0], nthreads=16)
    assert ref[0].shape[1] > 16 * pos.shape[0]
    # A fresh host thread has a fresh workspace (first arena: 16 edges per atom).
    import threading

    import torch

    errors, results = [], []

    def run():
        try:
            torch.cuda.set_device(0)
            for _ in range(4):
                results.append(nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=9.0))
        except Exception as e:  # reported below
            errors.append(e)

    t = threading.Thread(target=run)
    t.start()
    t.join()
    assert not errors, errors
    for k, got in enumerate(results):
        assert_same(got, ref, f"call {k}")
