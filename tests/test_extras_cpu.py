"""The oracle's output options (directed list, vectors, distances) on known
answers: the reference's own shift cases and the spec's displacement rule
d_ij = r_j + S.H - r_i (spec.md:60-75)."""

import numpy as np


def test_known_shift_case_vectors(oracle):
    # tests/test_basic.py:30-68 of the reference: two atoms across the x
    # boundary of a 10 A box; the edge carries shift (-1, 0, 0).
    pos = np.array([[0.5, 5.0, 5.0], [9.5, 5.0, 5.0]])
    h = np.eye(3) * 10.0
    half = oracle.search_single(pos, h, [True] * 3, 2.0)
    assert half[0].tolist() == [[0], [1]] and half[1].tolist() == [[-1, 0, 0]]
    ei, sh, vec, dist = oracle.edge_extras(pos, h, half, directed=True)
    assert ei.tolist() == [[0, 1], [1, 0]]
    assert sh.tolist() == [[-1, 0, 0], [1, 0, 0]]
    assert vec.tolist() == [[-1.0, 0.0, 0.0], [1.0, -0.0, -0.0]]
    assert dist.tolist() == [1.0, 1.0]


def test_vectors_follow_shift_convention(oracle):
    rng = np.random.default_rng(5)
    h = np.array([[9.0, 1.5, -0.7], [0.0, 8.2, 1.1], [0.0, 0.0, 7.5]])  # columns = a, b, c
    pos = rng.random((40, 3)) @ h.T
    half = oracle.search_single(pos, h, [True] * 3, 4.0)
    ei, sh, vec, dist = oracle.edge_extras(pos, h, half)
    ref = pos[ei[1]] - pos[ei[0]] + sh @ h.T
    assert np.allclose(vec, ref, atol=1e-12)
    assert (dist < 4.0 + 1e-12).all() and np.allclose(dist, np.linalg.norm(ref, axis=1))
    full = oracle.edge_extras(pos, h, half, directed=True)
    m = ei.shape[1]
    assert np.array_equal(full[0][:, m:], ei[::-1]) and np.array_equal(full[1][m:], -sh)
    assert np.array_equal(full[2][m:], -vec) and np.array_equal(full[3][m:], dist)


def test_verlet_filter_restatement(oracle):
    """oracle.verlet_filter on known answers: for an isolated brute-force
    system (raw positions, d = r_j - r_i in both computations) filtering the
    list at rc + skin down to rc gives exactly the oracle's list at rc, in
    order; for a periodic system it gives the same pair set away from rc."""
    rng = np.random.default_rng(8)
    pos = rng.random((400, 3)) * 16.0
    wide = oracle.search_single(pos, None, None, 5.0)
    got = oracle.verlet_filter(pos, None, wide, 4.0)
    want = oracle.search_single(pos, None, None, 4.0)
    assert np.array_equal(got[0], want[0]) and np.array_equal(got[1], want[1])
    h = np.eye(3) * 14.0
    pos = rng.random((1200, 3)) * 14.0
    wide = oracle.search_single(pos, h, [True] * 3, 5.0)
    got = oracle.verlet_filter(pos, h, wide, 4.0)
    want = oracle.search_single(pos, h, [True] * 3, 4.0)
    as_set = lambda e: set(zip(e[0][0].tolist(), e[0][1].tolist(), map(tuple, e[1].tolist())))
    assert as_set(got) == as_set(want)
    # moved positions: exactly the stored pairs now inside rc, stored order kept
    moved = pos + rng.normal(0.0, 0.05, pos.shape)
    got = oracle.verlet_filter(moved, h, wide, 4.0)
    d = moved[wide[0][1]] - moved[wide[0][0]] + wide[1] @ h.T
    keep = (d * d).sum(axis=1) < 16.0
    assert np.array_equal(got[0], wide[0][:, keep]) and np.array_equal(got[1], wide[1][keep])
