"""Batched-kernel launch shapes and their tuner: every shape gives the
oracle's edges (sizes on both sides of each shape's split threshold), the
tuner decides each kind of batch on its first batch without changing any result,
and pinning / resetting behave."""

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

    yield neighborlist_rs
    neighborlist_rs.set_batch_shape(None)
    neighborlist_rs.batch_tuner_reset()


def spread_batch(seed=5, n_systems=40):
    """Systems from 8 to 2048 atoms (log-uniform, half periodic triclinic),
    so every shape splits some and keeps others whole."""
    from neighborlist_rs import workloads as W

    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(8), np.log(2048), n_systems)).astype(int)
    sizes[:4] = [8, 257, 513, 1025]
    systems = []
    for s, n in enumerate(sizes):
        if s % 2 == 0:
            side = (n / 0.1) ** (1.0 / 3.0)
            systems.append(W.System(rng.random((n, 3)) * side, None, 5.0))
        else:
            rows = W.density_cell(int(n), 0.1, rng, (75.0, 105.0))
            systems.append(W.System(rng.random((n, 3)) @ rows, rows, 5.0))
    return W.concat_batch(systems)


def test_every_shape_matches_oracle(nl, oracle):
    pos, batch, cells = spread_batch()
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    (ref,) = oracle.search_batch(pos, batch, ocells, [5.0], nthreads=8)
    refm = oracle.search_batch(pos, batch, ocells, [5.0, 3.0], disjoint=True, nthreads=8)
    n_shapes = nl.set_batch_shape(0)
    assert n_shapes >= 2
    try:
        for i in range(n_shapes):
            info = nl.batch_shape_info(i)
            assert info["small_threads"] in (64, 128, 256, 512) and info["chunk"] > 0
            nl.set_batch_shape(i)
            got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
            assert_same(got, ref, f"shape {i} {info}")
            gm = nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=[5.0, 3.0],
                                                    disjoint=True)
            assert_same(gm[0], refm[0], f"shape {i} disjoint rc 5")
            assert_same(gm[1], refm[1], f"shape {i} disjoint rc 3")
    finally:
        nl.set_batch_shape(None)
    with pytest.raises(ValueError):
        nl.set_batch_shape(n_shapes)
    with pytest.raises(ValueError):
        nl.batch_shape_info(-1)


def test_tuner_decides_on_first_batch_and_keeps_results(nl, oracle):
    from neighborlist_rs import workloads as W

    nl.set_batch_shape(None)
    nl.batch_tuner_reset()
    systems = W.uneven_batch(n_systems=256, seed=12)
    pos, batch, cells = W.concat_batch(systems)
    first = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    (ref,) = oracle.search_batch(pos, batch, ocells, [5.0], nthreads=8)
    assert_same(first, ref, "batch timed in every candidate shape")
    state = nl.batch_tuner_state()
    assert len(state) == 1, state
    (entry,) = state
    assert entry["cutoffs"] == 1 and entry["systems_log2"] == 8
    n_shapes = nl.set_batch_shape(None)
    assert 2 <= entry["candidates"] <= n_shapes and 0 <= entry["shape"] < n_shapes, entry
    for _ in range(3):
        got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
        assert_same(got, ref, "batch in the chosen shape")
    assert nl.batch_tuner_state() == state
    # A different kind of batch is a new entry; reset forgets both.
    nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=[5.0, 3.0])
    assert len(nl.batch_tuner_state()) == 2
    nl.batch_tuner_reset()
    assert nl.batch_tuner_state() == []
