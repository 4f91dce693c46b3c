"""Output options (directed list, displacement vectors, distances) of the
CUDA library against the oracle: identical arrays, floats compared bit for
bit (the FP64 expression order is fixed on both sides)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nl():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import neighborlist_rs

    return neighborlist_rs


def bits_equal(a, b):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    return a.shape == b.shape and np.array_equal(a.view(np.int64), b.view(np.int64))


def systems():
    from neighborlist_rs import workloads as W

    rng = np.random.default_rng(7)
    out = []
    pos, rows = W.cluster_liquid(n_clusters=300, box=30.0, seed=3)
    out.append(("cluster liquid (cell list, FP32 band)", pos, rows.T, [True] * 3, 6.0))
    tri = np.array([[14.0, 0.0, 0.0], [3.1, 13.2, 0.0], [-2.4, 1.7, 12.5]])
    out.append(("triclinic", rng.random((900, 3)) @ tri, tri.T, [True] * 3, 5.0))
    out.append(("isolated brute force", rng.random((600, 3)) * 18.0, None, None, 5.0))
    out.append(("isolated cell list", rng.random((2500, 3)) * 30.0, None, None, 4.0))
    out.append(("mixed pbc (MIC brute force)", rng.random((300, 3)) * 20.0, np.eye(3) * 20.0,
                [True, False, True], 4.5))
    out.append(("tiny box, many images", rng.random((5, 3)) * 3.0, np.eye(3) * 3.0, [True] * 3,
                7.0))
    return out


@pytest.mark.parametrize("directed", [False, True])
def test_extras_match_oracle(nl, oracle, directed):
    for what, pos, h, pbc, rc in systems():
        cell = None if h is None else nl.PyCell(np.asarray(h).tolist(), pbc)
        got = nl.build_neighborlists_ex(cell, pos, rc, directed=directed, vectors=True,
                                        distances=True)
        half = oracle.search_single(pos, h, pbc, rc, nthreads=8)
        ei, sh, vec, dist = oracle.edge_extras(pos, h, half, directed=directed)
        assert np.array_equal(got["edge_index"], ei), what
        assert np.array_equal(got["shift"], sh), what
        assert bits_equal(got["vectors"], vec), what
        assert bits_equal(got["distances"], dist), what
        # The spec's validation rule: each shift reproduces a displacement
        # within the cutoff (up to the rounding of the two expressions).
        assert (got["distances"] < rc * (1 + 1e-12)).all(), what


def test_extras_options_independent(nl, oracle):
    what, pos, h, pbc, rc = systems()[1]
    cell = nl.PyCell(np.asarray(h).tolist(), pbc)
    plain = nl.build_neighborlists(cell, pos, rc)
    only_half = nl.build_neighborlists_ex(cell, pos, rc)
    assert set(only_half) == {"edge_index", "shift"}
    assert np.array_equal(only_half["edge_index"], plain["edge_index"])
    assert np.array_equal(only_half["shift"], plain["shift"])
    d = nl.build_neighborlists_ex(cell, pos, rc, distances=True)
    v = nl.build_neighborlists_ex(cell, pos, rc, vectors=True)
    assert set(d) == {"edge_index", "shift", "distances"}
    assert np.allclose(np.linalg.norm(v["vectors"], axis=1), d["distances"], rtol=1e-15)
    m = plain["edge_index"].shape[1]
    full = nl.build_neighborlists_ex(cell, pos, rc, directed=True)
    assert full["edge_index"].shape == (2, 2 * m)
    assert np.array_equal(full["edge_index"][:, m:], plain["edge_index"][::-1])
    assert np.array_equal(full["shift"][m:], -plain["shift"])


def test_extras_torch_matches_host(nl):
    import torch

    what, pos, h, pbc, rc = systems()[0]
    cell = nl.PyCell(np.asarray(h).tolist(), pbc)
    host = nl.build_neighborlists_ex(cell, pos, rc, directed=True, vectors=True, distances=True)
    dev = nl.build_neighborlists_torch(cell, torch.from_numpy(pos).cuda(), rc, directed=True,
                                       vectors=True, distances=True)
    torch.cuda.synchronize()
    for k in host:
        assert bits_equal(dev[k].cpu().numpy(), host[k]) if host[k].dtype == np.float64 else \
            np.array_equal(dev[k].cpu().numpy(), host[k]), k
    # No cell: vectors are plain position differences.
    p = np.random.default_rng(2).random((700, 3)) * 15.0
    r = nl.build_neighborlists_torch(None, torch.from_numpy(p).cuda(), 3.0, vectors=True)
    ei = r["edge_index"].cpu().numpy()
    assert bits_equal(r["vectors"].cpu().numpy(), p[ei[1]] - p[ei[0]])


def test_extras_empty_and_errors(nl):
    r = nl.build_neighborlists_ex(None, np.zeros((0, 3)), 5.0, directed=True, vectors=True,
                                  distances=True)
    assert r["edge_index"].shape == (2, 0) and r["vectors"].shape == (0, 3)
    assert r["distances"].shape == (0,)
    with pytest.raises(ValueError, match="Cutoff must be positive and finite"):
        nl.build_neighborlists_ex(None, np.zeros((3, 3)), 0.0)
