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
