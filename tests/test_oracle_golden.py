"""Pins the CPU oracle to the reference's own golden vectors (no GPU).

Every expected value below is taken from a test or a printed benchmark result
of solccp/neighborlist-rs; the file:line of each source is given per test.
"""

import numpy as np
import pytest

PBC3 = [True, True, True]


def eye(s):
    return np.eye(3) * s


def n_ij(ei):
    return int((ei[0] != ei[1]).sum())


# ---------------------------------------------------------------- fixtures

FIXTURE_CASES = [
    ("isolated_100", "6.0"), ("isolated_two_clusters", "6.0"), ("isolated_1000", "6.0"),
    ("isolated_10000", "6.0"), ("ethanol_1000", "6.0"), ("ethanol_10000", "6.0"),
    ("si_bulk", "6.0"), ("isolated_100", "14.0"), ("isolated_two_clusters", "14.0"),
    ("isolated_1000", "14.0"), ("ethanol_1000", "14.0"), ("ethanol_10000", "14.0"),
    ("si_bulk", "14.0"), ("isolated_100", "30.0"), ("isolated_two_clusters", "30.0"),
    ("si_bulk", "30.0"), ("ethanol_1000", "30.0"),
]


@pytest.mark.parametrize("name,rc", FIXTURE_CASES)
def test_fixture_counts(oracle, fixtures, golden_counts, name, rc):
    """benchmarks/benchmark_grace.txt: 'Total Edges RS' and 'Unique Pairs' per
    fixture and cutoff (computed by benchmarks/comprehensive_benchmark.py:62-109:
    PBC fixtures use PyCell(cell.T), isolated ones cell=None)."""
    pos, rows = fixtures[name]
    g = golden_counts[rc][name]
    if rows is None:
        ei, sh = oracle.search_single(pos, None, None, float(rc), nthreads=8)
        assert not sh.any()
    else:
        ei, sh = oracle.search_single(pos, rows.T, PBC3, float(rc), nthreads=8)
    assert n_ij(ei) == g["edges_i_ne_j"]
    mask = ei[0] != ei[1]
    pairs = set(zip(np.minimum(ei[0], ei[1])[mask].tolist(), np.maximum(ei[0], ei[1])[mask].tolist()))
    assert len(pairs) == g["unique_pairs"]
    # half list: i < j, or i == j with a non-zero image
    assert np.all(ei[0] <= ei[1])
    assert np.all(np.any(sh[~mask] != 0, axis=1))


# ---------------------------------------------------------------- cell.rs

def test_cell_fractional_and_triclinic(oracle):
    # src/cell.rs:101-132
    inv = oracle.cell_inverse(eye(10.0))
    assert np.allclose(inv @ [5.0, 2.0, 8.0], [0.5, 0.2, 0.8])
    h = np.array([[10.0, 2.0, 1.0], [0.0, 10.0, 0.5], [0.0, 0.0, 10.0]])
    assert np.allclose(oracle.cell_inverse(h) @ [13.0, 10.5, 10.0], [1.0, 1.0, 1.0])


def test_cell_invalid(oracle):
    # src/cell.rs:134-139
    with pytest.raises(RuntimeError, match="Cell matrix is not invertible"):
        oracle.cell_inverse(np.zeros((3, 3)))


def test_cell_wrap(oracle):
    # src/cell.rs:151-176
    assert np.allclose(oracle.wrap(eye(10.0), [1, 1, 1], [15.0, -2.0, 8.0]), [5.0, 8.0, 8.0])
    assert np.allclose(oracle.wrap(eye(10.0), [1, 0, 0], [15.0, 15.0, 15.0]), [5.0, 15.0, 15.0])


def test_cell_minimum_image(oracle):
    # src/cell.rs:178-215
    s, d = oracle.minimum_image(eye(10.0), [1, 1, 1], [1.0, 1.0, 1.0], [9.0, 9.0, 9.0])
    assert list(s) == [-1, -1, -1] and np.allclose(d, [-2.0, -2.0, -2.0])
    s, d = oracle.minimum_image(eye(10.0), [1, 0, 0], [1.0, 1.0, 1.0], [9.0, 9.0, 9.0])
    assert list(s) == [-1, 0, 0] and np.allclose(d, [-2.0, 8.0, 8.0])


def test_cell_perpendicular_widths(oracle):
    # src/cell.rs:217-239
    assert np.allclose(oracle.perpendicular_widths(np.diag([10.0, 5.0, 2.0])), [10.0, 5.0, 2.0])
    h = np.array([[1.0, 1.0, 0.0], [0.0, 1.0, 0.0], [0.0, 0.0, 1.0]])
    assert np.isclose(oracle.perpendicular_widths(h)[0], 1.0 / np.sqrt(2.0))


def test_inverse_orthorhombic_bits(oracle):
    """For a diagonal H the cofactor inverse gives (H11*H22)/det etc.; check the
    exact bits of that expression, which is what the library computes too."""
    for L in (46.4, 43.98055944840695, 5.43, 57.08566943):
        h = eye(L)
        inv = oracle.cell_inverse(h)
        det = L * (L * L)
        assert inv[0, 0] == (L * L) / det


# ---------------------------------------------------------------- search.rs

def test_z_order(oracle):
    # src/search.rs:1457-1474
    z1 = oracle.zorder([0.1, 0.1, 0.1])
    z2 = oracle.zorder([0.1, 0.1, 0.11])
    z3 = oracle.zorder([0.9, 0.9, 0.9])
    assert z1 < z2 < z3
    assert oracle.zorder([1.1, -0.1, 0.5]) > 0


def test_cell_list_structure(oracle):
    # src/search.rs:1543-1569: three atoms, box 10, rc 3 -> 3x3x3 bins
    pos = np.array([[1.0, 1.0, 1.0], [9.0, 9.0, 9.0], [1.1, 1.1, 1.1]])
    nb, ns, parts, abin = oracle.cell_list(pos, eye(10.0), 3.0)
    assert list(nb) == [3, 3, 3]
    assert abin[0] == 0 and abin[2] == 0
    assert abin[1] == 2 + 3 * (2 + 3 * 2)
    # src/search.rs:1476-1521: atoms 0 and 2 are adjacent in sorted order
    loc = {int(p): s for s, p in enumerate(parts)}
    assert abs(loc[0] - loc[2]) == 1


def test_cell_list_vs_brute_force(oracle):
    # src/search.rs:1571-1600 (cell list forced by N >= brute-force threshold 0)
    pos = np.array([[1.0, 1.0, 1.0], [1.2, 1.2, 1.2], [9.8, 9.8, 9.8], [5.0, 5.0, 5.0]])
    oracle.set_thresholds(0, 300)
    try:
        ei, _ = oracle.search_single(pos, eye(10.0), PBC3, 2.0)
    finally:
        oracle.set_thresholds(1000, 300)
    exp = []
    for i in range(4):
        for j in range(i + 1, 4):
            d = pos[j] - pos[i]
            d -= 10.0 * np.round(d / 10.0)
            if (d * d).sum() < 4.0:
                exp.append((i, j))
    assert sorted(zip(ei[0].tolist(), ei[1].tolist())) == exp == [(0, 1)]
    ei2, _ = oracle.search_single(pos, eye(10.0), PBC3, 2.0)  # brute-force MIC path
    assert sorted(zip(ei2[0].tolist(), ei2[1].tolist())) == exp


def test_brute_force_reference_pairs(oracle):
    # src/search.rs:1523-1541
    pos = np.array([[1.0, 1.0, 1.0], [1.0, 3.5, 1.0], [8.5, 1.0, 1.0]])
    ei, _ = oracle.search_single(pos, eye(10.0), PBC3, 3.0)
    assert sorted(zip(ei[0].tolist(), ei[1].tolist())) == [(0, 1), (0, 2)]


def test_dense_bin(oracle):
    # src/search.rs:1884-1910: 5 atoms in one bin, rc 2 -> 10 edges
    pos = np.array([[0.1 * i, 0.1, 0.1] for i in range(5)])
    oracle.set_thresholds(0, 300)
    try:
        ei, _ = oracle.search_single(pos, eye(10.0), PBC3, 2.0)
    finally:
        oracle.set_thresholds(1000, 300)
    assert ei.shape[1] == 10


def test_large_search_radius(oracle):
    # src/search.rs:1860-1882: rc 10 in a 1 A box; 21 images per axis
    ei, sh = oracle.search_single(np.array([[0.5, 0.5, 0.5]]), eye(1.0), PBC3, 10.0)
    assert ei.shape[1] > 0
    # every lattice vector with |S| < 10 except 0, counted once per +/- pair? No:
    # self-images appear in both directions (S and -S).
    r = np.arange(-10, 11)
    S = np.stack(np.meshgrid(r, r, r, indexing="ij"), -1).reshape(-1, 3)
    expect = int(((S ** 2).sum(1) < 100).sum()) - 1
    assert ei.shape[1] == expect
    assert len({tuple(s) for s in sh.tolist()}) == expect


def test_brute_force_simd_lcg(oracle):
    # src/search.rs:1413-1455: LCG seed 42, 100 atoms, rc 2.5; i<j ascending order
    rng = 42
    vals = []
    for _ in range(300):
        rng = (rng * 6364136223846793005 + 1) % (1 << 64)
        vals.append(float(rng) / float((1 << 64) - 1))
    pos = np.array(vals).reshape(100, 3) * 10.0
    ei, sh = oracle.search_single(pos, None, None, 2.5)
    exp = [(i, j) for i in range(100) for j in range(i + 1, 100)
           if ((pos[i] - pos[j]) ** 2).sum() < 6.25]
    assert list(zip(ei[0].tolist(), ei[1].tolist())) == exp
    assert not sh.any()


@pytest.mark.parametrize("seed", range(12))
def test_random_cubic_vs_bruteforce(oracle, seed):
    """Restates the proptest of src/search.rs:1763-1791: random cubic box 10-20,
    rc 1-3, 2-50 atoms; the cell list agrees with an all-images brute force."""
    rng = np.random.default_rng(seed)
    box = rng.uniform(10, 20)
    rc = rng.uniform(1, 3)
    n = int(rng.integers(2, 51))
    pos = rng.random((n, 3)) * box
    oracle.set_thresholds(0, 300)
    try:
        ei, sh = oracle.search_single(pos, eye(box), PBC3, rc)
    finally:
        oracle.set_thresholds(1000, 300)
    got = sorted(zip(ei[0].tolist(), ei[1].tolist(), map(tuple, sh.tolist())))
    exp = []
    for i in range(n):
        for j in range(i, n):
            for S in np.array(np.meshgrid([-1, 0, 1], [-1, 0, 1], [-1, 0, 1])).T.reshape(-1, 3):
                if i == j and not S.any():
                    continue
                d = pos[j] + box * S - pos[i]
                if (d * d).sum() < rc * rc:
                    exp.append((i, j, tuple(int(x) for x in S)))
    assert got == sorted(exp)


# ---------------------------------------------------------------- single.rs / batch.rs

def test_single_basic_and_multi(oracle):
    # src/single.rs:177-211
    ei, _ = oracle.search_single(np.array([[0, 0, 0], [1.0, 0, 0]]), None, None, 1.5)
    assert ei.tolist() == [[0], [1]]
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0], [2.5, 0, 0]])
    r = oracle.search_single_multi(pos, None, None, [1.5, 3.0])
    assert r[0][0].shape[1] == 1 and r[1][0].shape[1] == 3
    pos[2, 0] = 2.1
    r = oracle.search_single_multi(pos, None, None, [1.5, 3.0], disjoint=True)
    assert r[0][0].shape[1] == 2 and r[1][0].shape[1] == 1


def test_single_force_cell_list(oracle):
    # src/single.rs:264-284 and tests/test_single_system.rs:23-44
    pos = np.array([[1.0, 1, 1], [2.0, 2, 2]])
    ei, _ = oracle.search_single(pos, eye(10.0), PBC3, 6.0)
    assert ei.shape[1] == 1
    ei, sh = oracle.search_single(np.array([[1.0, 1, 1], [9.0, 1, 1]]), eye(10.0), PBC3, 2.5)
    assert ei.tolist() == [[0], [1]] and sh.tolist() == [[-1, 0, 0]]


def test_self_images(oracle):
    # tests/test_issue_1.py:5-33: 1 atom, 5 A box, rc 6 -> 6 images, none zero
    ei, sh = oracle.search_single(np.zeros((1, 3)), eye(5.0), PBC3, 6.0)
    assert ei.shape[1] == 6
    assert sorted(map(tuple, sh.tolist())) == sorted(
        [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)])


def test_basic_shift_and_si(oracle, fixtures):
    # tests/test_basic.py:30-68 (shift (-1,0,0)) and :94-109 (Si: 16 edges)
    pos = np.array([[1.0, 1, 1], [1.5, 1, 1], [19.5, 1, 1]])
    ei, sh = oracle.search_single(pos, eye(20.0), PBC3, 2.0)
    got = {(int(i), int(j)): tuple(s) for i, j, s in zip(ei[0], ei[1], sh.tolist())}
    assert got == {(0, 1): (0, 0, 0), (0, 2): (-1, 0, 0)}
    spos, srows = fixtures["si_bulk"]
    ei, _ = oracle.search_single(spos, srows.T, PBC3, 2.5)
    assert ei.shape[1] == 16


def test_mixed_pbc(oracle):
    # tests/test_api_extensions.py:243-254: mixed PBC is honoured by the
    # brute-force MIC path (N=2), full PBC gives shift [0,0,-1]
    pos = np.array([[5.0, 5.0, 0.5], [5.0, 5.0, 9.5]])
    ei, _ = oracle.search_single(pos, eye(10.0), [True, True, False], 2.0)
    assert ei.shape[1] == 0
    ei, sh = oracle.search_single(pos, eye(10.0), PBC3, 2.0)
    assert ei.shape[1] == 1 and sh.tolist() == [[0, 0, -1]]


def test_ase_convention(oracle):
    # tests/test_ase.py:14-63: a=3, atoms at 0.1 and 2.9 -> one edge, shift [-1,0,0]
    pos = np.array([[0.1, 0.1, 0.1], [2.9, 0.1, 0.1]])
    ei, sh = oracle.search_single(pos, eye(3.0), PBC3, 1.0)
    assert ei.tolist() == [[0], [1]] and sh.tolist() == [[-1, 0, 0]]


def cu_fcc(reps, a=3.6):
    """ASE bulk('Cu', 'fcc', a) * reps: primitive rows, positions m0*a1+m1*a2+m2*a3."""
    prim = np.array([[0.0, a / 2, a / 2], [a / 2, 0.0, a / 2], [a / 2, a / 2, 0.0]])
    pos = np.array([m0 * prim[0] + m1 * prim[1] + m2 * prim[2]
                    for m0 in range(reps) for m1 in range(reps) for m2 in range(reps)])
    return pos, prim * reps


def test_disjoint_shells(oracle):
    # tests/test_disjoint.py:11-57 (Cu fcc 3x3x3; PyCell(cell) symmetric) and :60-84
    pos, rows = cu_fcc(3)
    cum = oracle.search_single_multi(pos, rows, PBC3, [3.0, 4.0, 5.0])
    dis = oracle.search_single_multi(pos, rows, PBC3, [3.0, 4.0, 5.0], disjoint=True)
    n = [r[0].shape[1] for r in cum]
    d = [r[0].shape[1] for r in dis]
    assert n[0] < n[1] < n[2]
    assert d == [n[0], n[1] - n[0], n[2] - n[1]]
    pos2, rows2 = cu_fcc(2)
    r = oracle.search_single_multi(pos2, rows2, PBC3, [5.0, 3.0], disjoint=True)
    small = oracle.search_single(pos2, rows2, PBC3, 3.0)[0].shape[1]
    total = oracle.search_single(pos2, rows2, PBC3, 5.0)[0].shape[1]
    assert r[1][0].shape[1] == small and r[0][0].shape[1] == total - small


def test_batch_reference_cases(oracle):
    # src/batch.rs:297-325, tests/test_batch_system.rs:4-50, tests/test_batch.py:5-36
    pos = np.array([[1.0, 1, 1], [1.2, 1, 1], [5.0, 5, 5], [5.2, 5, 5]])
    cells = [(eye(10.0), PBC3), (eye(10.0), PBC3)]
    (ei, _), = oracle.search_batch(pos, [0, 0, 1, 1], cells, [0.5])
    assert sorted(zip(ei[0].tolist(), ei[1].tolist())) == [(0, 1), (2, 3)]
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0], [1.0, 1, 1], [9.0, 1, 1]])
    (ei, sh), = oracle.search_batch(pos, [0, 0, 1, 1], [None, (eye(10.0), PBC3)], [2.5])
    got = {(int(i), int(j)): tuple(s) for i, j, s in zip(ei[0], ei[1], sh.tolist())}
    assert got == {(0, 1): (0, 0, 0), (2, 3): (-1, 0, 0)}
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0], [10.0, 0, 0], [11.0, 0, 0], [12.0, 0, 0]])
    (ei, _), = oracle.search_batch(pos, [0, 0, 1, 1, 1], None, [2.5])
    assert sorted(zip(ei[0].tolist(), ei[1].tolist())) == [(0, 1), (2, 3), (2, 4), (3, 4)]


def test_batch_multi_and_errors(oracle):
    # src/batch.rs:327-357, :404-421, :501-516
    pos = np.array([[1.0, 1, 1], [1.2, 1, 1], [5.0, 5, 5], [5.5, 5, 5]])
    r = oracle.search_batch(pos, [0, 0, 1, 1], [(eye(10.0), PBC3)] * 2, [0.3, 0.6])
    assert r[0][0].shape[1] == 1 and r[1][0].shape[1] == 2
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0], [2.1, 0, 0]])
    r = oracle.search_batch(pos, [0, 0, 0], [None], [1.5, 3.0], disjoint=True)
    assert r[0][0].shape[1] == 2 and r[1][0].shape[1] == 1
    with pytest.raises(RuntimeError, match="positions and batch must have the same length"):
        oracle.search_batch(np.zeros((1, 3)), [0, 1], [None], [1.0])
    with pytest.raises(RuntimeError, match="Expected at least 1 cells, but got 0"):
        oracle.search_batch(np.zeros((1, 3)), [0], [], [1.0])


def test_bug_002_batched_images(oracle):
    # tests/test_bug_002_fix.py: 2 atoms in a 5 A box, rc 6; batch == single
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0]])
    (eb, sb), = oracle.search_batch(pos, [0, 0], [(eye(5.0), PBC3)], [6.0])
    es, ss = oracle.search_single(pos, eye(5.0), PBC3, 6.0)
    assert eb.shape[1] >= 10 and (sb != 0).any(axis=1).sum() > 0
    assert np.array_equal(eb, es) and np.array_equal(sb, ss)
