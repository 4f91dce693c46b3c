"""The cell-list build's paths and the pruned pair tests against the oracle,
bit-exact: bins of every size class -- rank-placed bins of 1..512 atoms and
bins of more than 512 atoms sorted by one CTA each -- on sparse grids (the
one-launch search, whose candidates are pruned by the group's box) and on
dense grids (chunk boxes, the pruned three-launch count pass)."""

import numpy as np
import pytest

from helpers import assert_same

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nl():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import neighborlist_rs

    return neighborlist_rs


def check(nl, oracle, pos, box, rc, what):
    h = np.eye(3) * box
    cell = nl.PyCell(h.tolist(), [True, True, True])
    got = nl.build_neighborlists(cell, np.ascontiguousarray(pos), rc)
    ref = oracle.search_single(pos, h, [True, True, True], rc, nthreads=8)
    assert_same(got, ref, what)
    return got


def clustered(n_gas, n_blob, box, blob_edge, seed):
    """Uniform gas plus one dense blob: one bin far above the mean size."""
    rng = np.random.default_rng(seed)
    gas = rng.uniform(0.0, box, (n_gas, 3))
    blob = 0.5 * box + rng.uniform(0.0, blob_edge, (n_blob, 3))
    pos = np.concatenate([gas, blob])
    return pos[rng.permutation(pos.shape[0])]


@pytest.mark.parametrize("n_blob", [40, 300, 900, 2500])
def test_build_bin_sizes(nl, oracle, n_blob):
    # 12 bins per axis at rc 5: the blob's bin holds ~n_blob atoms (rank
    # placement up to 512, one CTA's sort above), the rest a few each.
    pos = clustered(4000, n_blob, 60.0, 1.5, seed=n_blob)
    check(nl, oracle, pos, 60.0, 5.0, f"gas 4000 + blob {n_blob}")


def test_dense_grid_chunk_boxes(nl, oracle):
    # 3 bins per axis at rc 14: chunk boxes on, bins of ~740 atoms sorted by
    # one CTA each, the count pass pruning chunks and candidates.
    rng = np.random.default_rng(11)
    pos = rng.uniform(0.0, 46.0, (20000, 3))
    check(nl, oracle, pos, 46.0, 14.0, "uniform 20000 rc 14")


@pytest.mark.parametrize("n", [32768, 40000])
def test_uniform_sizes(nl, oracle, n):
    rng = np.random.default_rng(n)
    box = (n / 0.1) ** (1.0 / 3.0)
    pos = rng.uniform(0.0, box, (n, 3))
    check(nl, oracle, pos, box, 5.0, f"uniform {n} rc 5")


def test_device_results_past_the_capacity_estimate(nl, oracle):
    """A dense blob holds far more edges than the density estimate sizes the
    arrays for: unless earlier builds of the process already grew them, the
    first launch writes nothing, the arrays grow and the search runs again --
    here with device results on a caller's stream (the call otherwise returns
    as soon as M is known)."""
    import torch

    pos = clustered(4000, 2500, 60.0, 1.5, seed=77)
    h = np.eye(3) * 60.0
    cell = nl.PyCell(h.tolist(), [True, True, True])
    d = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        r = nl.build_neighborlists_torch(cell, d, 5.0)
        got = {"edge_index": r["edge_index"].cpu().numpy(), "shift": r["shift"].cpu().numpy()}
    ref = oracle.search_single(pos, h, [True, True, True], 5.0, nthreads=8)
    assert_same(got, ref, "blob, device results")
