"""Parity of the CUDA library (through the drop-in Python API and the C ABI)
with the CPU oracle: identical edge_index and shift arrays, element by
element and in the same order (integer index work: bit-exact)."""

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


def eye(s):
    return np.eye(3) * s


def single(nl, oracle, pos, h, rc, pbc=PBC3, what=""):
    cell = None if h is None else nl.PyCell(np.asarray(h).tolist(), pbc)
    got = nl.build_neighborlists(cell, np.ascontiguousarray(pos, dtype=np.float64), rc)
    ref = oracle.search_single(pos, h, None if h is None else pbc, rc, nthreads=8)
    assert_same(got, ref, what)
    return got


# ---------------------------------------------------------------- fixtures

@pytest.mark.parametrize("rc", [6.0, 14.0])
@pytest.mark.parametrize("name", ["isolated_100", "isolated_two_clusters", "isolated_1000",
                                  "isolated_10000", "ethanol_1000", "ethanol_10000", "si_bulk"])
def test_fixture_parity(nl, oracle, fixtures, golden_counts, name, rc):
    pos, rows = fixtures[name]
    got = single(nl, oracle, pos, None if rows is None else rows.T, rc, what=f"{name} rc {rc}")
    ei = got["edge_index"]
    assert int((ei[0] != ei[1]).sum()) == golden_counts[str(rc)][name]["edges_i_ne_j"]


# ---------------------------------------------------------------- synthetic workloads

def test_isolated_cube_1000(nl, oracle):
    from neighborlist_rs import workloads as W

    single(nl, oracle, W.isolated_cube(), None, 6.0, what="isolated cube N=1000 rc 6")


@pytest.mark.parametrize("rc", [6.0, 14.0])
def test_cluster_liquid(nl, oracle, rc):
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid()
    single(nl, oracle, pos, rows.T, rc, what=f"cluster liquid rc {rc}")


def test_triclinic_multi(nl, oracle):
    from neighborlist_rs import workloads as W

    pos, rows = W.triclinic_uniform()
    cell = nl.PyCell(rows.T.tolist())
    got = nl.build_neighborlists_multi(cell, pos, [5.0, 6.0, 12.0])
    ref = oracle.search_single_multi(pos, rows.T, PBC3, [5.0, 6.0, 12.0], nthreads=8)
    for q in range(3):
        assert_same(got[q], ref[q], f"triclinic multi cutoff {q}")


# ---------------------------------------------------------------- paths and edge cases

def test_empty_and_single_atom(nl, oracle):
    r = nl.build_neighborlists(None, np.zeros((0, 3)), 3.0)
    assert r["edge_index"].shape == (2, 0) and r["shift"].shape == (0, 3)
    single(nl, oracle, np.zeros((1, 3)), eye(5.0), 6.0, what="self images")
    single(nl, oracle, np.zeros((1, 3)), None, 6.0, what="single isolated atom")


def test_many_images_tiny_box(nl, oracle):
    # src/search.rs:1860-1882: rc 10 in a 1 A box (21 images per axis)
    single(nl, oracle, np.array([[0.5, 0.5, 0.5]]), eye(1.0), 10.0, what="rc 10 in 1 A box")
    rng = np.random.default_rng(7)
    h = np.array([[4.0, 1.0, 0.5], [0.0, 3.5, -0.8], [0.0, 0.0, 3.0]])
    pos = rng.random((40, 3)) @ h.T
    single(nl, oracle, pos, h, 7.5, what="small triclinic box, many images")


@pytest.mark.parametrize("seed", range(4))
def test_brute_force_paths(nl, oracle, seed):
    rng = np.random.default_rng(100 + seed)
    n = int(rng.integers(2, 900))
    side = (n / 0.1) ** (1 / 3)
    pos = rng.random((n, 3)) * side
    single(nl, oracle, pos, None, 5.0, what="brute isolated")
    L = max(side, 11.0)
    single(nl, oracle, pos, eye(L), 5.0, what="brute MIC")
    h = np.array([[L, 0.3 * L, 0.1 * L], [0.0, L, 0.2 * L], [0.0, 0.0, L]])
    single(nl, oracle, pos @ np.array(h).T / L, h, 4.0, what="brute MIC triclinic")
    single(nl, oracle, pos, eye(L), 5.0, pbc=[True, False, True], what="brute MIC mixed pbc")


def test_threshold_changes_dispatch(nl, oracle):
    pos = np.random.default_rng(3).random((200, 3)) * 12.0
    old = nl.get_brute_force_threshold()
    nl.set_brute_force_threshold(0)
    oracle.set_thresholds(0, 300)
    try:
        single(nl, oracle, pos, None, 3.0, what="cell list forced (isolated)")
        single(nl, oracle, pos, eye(12.0), 3.0, what="cell list forced (pbc)")
        single(nl, oracle, pos, eye(12.0), 3.0, pbc=[True, False, False], what="Q1 mixed pbc")
    finally:
        nl.set_brute_force_threshold(old)
        oracle.set_thresholds(1000, 300)


def test_duplicates_and_boundaries(nl, oracle):
    rng = np.random.default_rng(11)
    base = rng.random((600, 3)) * 20.0
    pos = np.concatenate([base, base[:300], np.zeros((50, 3)), np.full((50, 3), 20.0),
                          np.full((30, 3), -20.0), np.full((30, 3), 40.0 - 1e-12)])
    single(nl, oracle, pos, eye(20.0), 4.0, what="duplicates / boundaries / outside")
    single(nl, oracle, pos, None, 4.0, what="duplicates isolated")


def test_large_bin_merge_path(nl, oracle):
    # A single bin of 3000 atoms exercises the merge path of the bin sort.
    pos = np.random.default_rng(5).random((3000, 3)) * 8.0
    single(nl, oracle, pos, eye(8.0), 4.5, what="one 3000-atom bin")


def test_multi_cutoff_variants(nl, oracle, fixtures):
    pos, rows = fixtures["ethanol_1000"]
    cell = nl.PyCell(rows.T.tolist())
    for cs, dj in [([6.0, 3.0, 4.5], False), ([6.0, 3.0, 4.5], True), ([3.0, 3.0], True)]:
        got = nl.build_neighborlists_multi(cell, pos, cs, disjoint=dj)
        ref = oracle.search_single_multi(pos, rows.T, PBC3, cs, disjoint=dj, nthreads=8)
        for q in range(len(cs)):
            assert_same(got[q], ref[q], f"multi {cs} disjoint={dj} q={q}")
    # more than one 32-cutoff pass, with disjoint shells across the pass boundary
    cs = list(np.linspace(1.0, 7.0, 45))
    for dj in (False, True):
        got = nl.build_neighborlists_multi(cell, pos, cs, disjoint=dj)
        ref = oracle.search_single_multi(pos, rows.T, PBC3, cs, disjoint=dj, nthreads=8)
        for q in range(len(cs)):
            assert_same(got[q], ref[q], f"45 cutoffs disjoint={dj} q={q}")


@pytest.mark.parametrize("disjoint", [False, True])
def test_multi_guard_band_shell_edges(nl, oracle, disjoint):
    """Lattice pairs exactly on each cutoff of a multi-cutoff request (and one
    ulp either side): every per-cutoff FP32 pass must defer the undecidable
    pairs, including those on the inner edge of a disjoint shell."""
    a = 2.0
    g = np.arange(10) * a
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    cell = nl.PyCell(eye(20.0).tolist())
    up, dn = np.nextafter(1.0, 2.0), np.nextafter(1.0, 0.0)
    sets = [[2.0, np.sqrt(8.0), np.sqrt(12.0), 4.0],
            [2.0 * up, np.sqrt(8.0) * dn, 4.0 * up],
            [4.0, 2.0, np.sqrt(8.0)]]
    for cs in sets:
        cs = [float(c) for c in cs]
        for p in (pos, pos + 0.5):
            got = nl.build_neighborlists_multi(cell, p, cs, disjoint=disjoint)
            ref = oracle.search_single_multi(p, eye(20.0), PBC3, cs, disjoint=disjoint, nthreads=8)
            for q in range(len(cs)):
                assert_same(got[q], ref[q], f"lattice multi {cs} disjoint={disjoint} q={q}")


def test_multi_brute_and_labels(nl, oracle):
    pos = np.array([[0.0, 0, 0], [1.0, 0, 0], [2.5, 0, 0]])
    got = nl.build_neighborlists_multi(None, pos, [1.6, 3.0], labels=["s", "l"])
    ref = oracle.search_single_multi(pos, None, None, [1.6, 3.0])
    assert_same(got["s"], ref[0], "labels s")
    assert_same(got["l"], ref[1], "labels l")


def test_batch_parity(nl, oracle):
    from neighborlist_rs import workloads as W

    systems = W.uneven_batch(n_systems=96)
    pos, batch, cells = W.concat_batch(systems)
    got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    (ref,) = oracle.search_batch(pos, batch, ocells, [5.0], nthreads=8)
    assert_same(got, ref, "uneven batch")
    gm = nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=[5.0, 3.0])
    refm = oracle.search_batch(pos, batch, ocells, [5.0, 3.0], nthreads=8)
    assert_same(gm[0], refm[0], "batch multi 5")
    assert_same(gm[1], refm[1], "batch multi 3")


def test_batch_matches_singles(nl):
    """tests/test_batch.py:68-120: each system of a batch equals its single call."""
    from neighborlist_rs import workloads as W

    systems = W.uneven_batch(n_systems=12, seed=9)
    pos, batch, cells = W.concat_batch(systems)
    got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
    start = 0
    parts = []
    for s in systems:
        cell = None if s.cell_rows is None else nl.PyCell(s.cell_rows.T.tolist())
        r = nl.build_neighborlists(cell, s.positions, 5.0)
        parts.append((r["edge_index"] + start, r["shift"]))
        start += len(s.positions)
    ei = np.concatenate([p[0] for p in parts], axis=1)
    sh = np.concatenate([p[1] for p in parts], axis=0)
    assert np.array_equal(got["edge_index"], ei) and np.array_equal(got["shift"], sh)


def test_non_contiguous_inputs(nl):
    # tests/test_memory_layout.py
    rng = np.random.default_rng(0)
    pos = rng.random((100, 3)) * 10.0
    big = np.zeros((100, 4))
    big[:, :3] = pos
    a = nl.build_neighborlists(None, pos, 1.5)
    b = nl.build_neighborlists(None, big[:, :3], 1.5)
    assert np.array_equal(a["edge_index"], b["edge_index"])
    bl = np.zeros(200, np.int32)
    r = nl.build_neighborlists_batch(big[:50, :3], bl[::2][:50], None, 1.5)
    assert r["edge_index"].shape[0] == 2


def test_batch_mixed_sizes_and_many_cutoffs(nl, oracle):
    """Runs of small systems (batched kernels) around a system above the
    batched-kernel size (single-system pipeline), plus > 32 cutoffs."""
    from neighborlist_rs import workloads as W

    small = W.uneven_batch(n_systems=10, seed=41)
    rng = np.random.default_rng(42)
    big_rows = np.diag([25.0, 25.0, 25.0])
    big = W.System(rng.random((3000, 3)) @ big_rows, big_rows, 5.0)
    iso_big = W.System(rng.random((2500, 3)) * 30.0, None, 5.0)
    systems = small[:4] + [big] + small[4:7] + [iso_big] + small[7:]
    pos, batch, cells = W.concat_batch(systems)
    ocells = [None if not c.any() else (c.T, PBC3) for c in cells]
    got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
    (ref,) = oracle.search_batch(pos, batch, ocells, [5.0], nthreads=8)
    assert_same(got, ref, "mixed small/large batch")
    cs = list(np.linspace(1.5, 5.0, 35))
    for dj in (False, True):
        gm = nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=cs, disjoint=dj)
        rm = oracle.search_batch(pos, batch, ocells, cs, disjoint=dj, nthreads=8)
        for q in range(len(cs)):
            assert_same(gm[q], rm[q], f"batch 35 cutoffs disjoint={dj} q={q}")


def test_batch_system_offsets(nl):
    """The per-system offset table of a batched call: system i's edges are
    [off[i], off[i + 1]) in every list, for systems on the batched kernels and
    on the single-system pipeline alike; the edges are unchanged."""
    from neighborlist_rs import workloads as W

    small = W.uneven_batch(n_systems=40, seed=43)
    rng = np.random.default_rng(44)
    big_rows = np.diag([26.0, 26.0, 26.0])
    big = W.System(rng.random((3000, 3)) @ big_rows, big_rows, 5.0)
    systems = small[:15] + [big] + small[15:]
    pos, batch, cells = W.concat_batch(systems)
    n_sys = len(systems)
    starts = np.concatenate([[0], np.cumsum([len(s.positions) for s in systems])])

    def check(res, what):
        off = res["system_offsets"]
        src = res["edge_index"][0]
        assert off.dtype == np.int64 and off.shape == (n_sys + 1,), what
        sys_of_edge = np.searchsorted(starts, src, side="right") - 1
        want = np.concatenate([[0], np.cumsum(np.bincount(sys_of_edge, minlength=n_sys))])
        assert np.array_equal(off, want), what
        assert np.all(np.diff(sys_of_edge) >= 0), what

    plain = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0)
    got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=5.0, return_offsets=True)
    assert_same(got, (plain["edge_index"], plain["shift"]), "edges with offsets")
    check(got, "single cutoff")
    cs = [5.0, 3.0, 4.0]
    for dj in (False, True):
        pm = nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=cs, disjoint=dj)
        gm = nl.build_neighborlists_batch_multi(pos, batch, cells=cells, cutoffs=cs, disjoint=dj,
                                                return_offsets=True)
        for q in range(len(cs)):
            assert_same(gm[q], (pm[q]["edge_index"], pm[q]["shift"]), f"multi q={q} dj={dj}")
            check(gm[q], f"multi q={q} disjoint={dj}")
    empty = nl.build_neighborlists_batch(np.zeros((0, 3)), np.zeros(0, np.int32), cutoff=5.0,
                                         return_offsets=True)
    assert np.array_equal(empty["system_offsets"], [0])


def test_batch_singular_cell(nl):
    pos = np.random.default_rng(1).random((6, 3))
    batch = np.array([0, 0, 0, 1, 1, 1], np.int32)
    cells = np.zeros((2, 3, 3))
    cells[0] = np.eye(3) * 5.0
    cells[1] = [[1.0, 0, 0], [2.0, 0, 0], [0, 0, 1.0]]   # singular
    with pytest.raises(ValueError, match="Cell matrix is not invertible"):
        nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=2.0)


def test_batch_thresholds_and_self_images(nl, oracle):
    """Tiny periodic boxes (many images, nb = 1) and the brute-force threshold
    moved, inside the batched kernels."""
    from neighborlist_rs import workloads as W

    rng = np.random.default_rng(8)
    systems = []
    for s in range(40):
        n = int(rng.integers(1, 30))
        rows = W.density_cell(n, 0.1, rng, (75.0, 105.0))
        systems.append(W.System(rng.random((n, 3)) @ rows, rows, 6.0))
    pos, batch, cells = W.concat_batch(systems)
    ocells = [(c.T, PBC3) for c in cells]
    for bf in (1000, 0, 20):
        nl.set_brute_force_threshold(bf)
        oracle.set_thresholds(bf, 300)
        try:
            got = nl.build_neighborlists_batch(pos, batch, cells=cells, cutoff=6.0)
            (ref,) = oracle.search_batch(pos, batch, ocells, [6.0], nthreads=8)
            assert_same(got, ref, f"tiny boxes, brute-force threshold {bf}")
        finally:
            nl.set_brute_force_threshold(1000)
            oracle.set_thresholds(1000, 300)


@pytest.mark.parametrize("jitter", [0.0, 1e-9, 1e-6])
def test_guard_band_near_cutoff(nl, oracle, jitter):
    """Lattice pairs exactly at (or within 1e-9 / 1e-6 A of) the cutoff: the
    FP32 test must defer every undecidable pair to the exact FP64 expression."""
    a = 2.0
    g = np.arange(10) * a
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos = pos + np.random.default_rng(3).normal(0.0, jitter, pos.shape) if jitter else pos
    for rc in (2.0, np.sqrt(8.0), np.sqrt(12.0), 4.0, 2.0 * np.nextafter(1.0, 2.0)):
        single(nl, oracle, pos, eye(20.0), float(rc), what=f"lattice rc={rc!r} jitter={jitter}")
        single(nl, oracle, pos + 0.5, eye(20.0), float(rc), what=f"lattice+0.5 rc={rc!r}")
    tri = np.array([[20.0, 3.0, 1.0], [0.0, 20.0, 2.0], [0.0, 0.0, 20.0]])
    single(nl, oracle, pos @ tri.T / 20.0, tri, 2.0 * 1.0000001, what="skewed lattice")


def test_large_system_many_scan_tiles(nl, oracle):
    """200k atoms at density 0.1 (5.4 M per-(atom, cell) counts: ~1300 tiles of
    the single-pass scan), plus grid-shape changes between calls."""
    rng = np.random.default_rng(77)
    L = (200_000 / 0.1) ** (1 / 3)
    pos = rng.random((200_000, 3)) * L
    single(nl, oracle, pos, eye(L), 5.0, what="200k atoms rc 5")
    small = pos[:20_000] * 0.5
    for rc in (6.0, 3.0, 6.0):
        single(nl, oracle, small, eye(L * 0.5), rc, what=f"grid change rc {rc}")


def test_million_atoms_rc8(nl, oracle):
    """The largest served size: 1e6 atoms at rho 0.1 in a periodic box, rc 8
    (~1.1e8 edges, 3 GB of results), every edge and shift against the oracle."""
    import os

    rng = np.random.default_rng(1_000_000)
    L = (1_000_000 / 0.1) ** (1 / 3)
    pos = rng.random((1_000_000, 3)) * L
    cell = nl.PyCell(eye(L).tolist())
    got = nl.build_neighborlists(cell, pos, 8.0)
    ref = oracle.search_single(pos, eye(L), PBC3, 8.0, nthreads=os.cpu_count() or 8)
    assert got["edge_index"].shape[1] > 100_000_000
    assert_same(got, ref, "1e6 atoms rc 8")


@pytest.mark.parametrize("rc", [6.0, 14.0])
def test_repeated_calls_graph_replay(nl, oracle, rc):
    """Identical repeated builds: first direct, then captured, then replayed
    as a CUDA graph (with the hit-mask and edge arenas resized in between);
    every result must equal the oracle's."""
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid(n_clusters=400, box=33.0, seed=12)
    ref = oracle.search_single(pos, rows.T, PBC3, rc, nthreads=8)
    cell = nl.PyCell(rows.T.tolist())
    for it in range(5):
        assert_same(nl.build_neighborlists(cell, pos, rc), ref, f"call {it} rc {rc}")


def test_torch_device_api(nl, oracle):
    import torch
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid(n_clusters=300, box=30.0, seed=13)
    cell = nl.PyCell(rows.T.tolist())
    ref = oracle.search_single(pos, rows.T, PBC3, 6.0, nthreads=8)
    d = torch.from_numpy(pos).cuda()
    for it in range(3):
        r = nl.build_neighborlists_torch(cell, d, 6.0)
        assert r["edge_index"].is_cuda and r["edge_index"].dtype == torch.int64
        assert_same({"edge_index": r["edge_index"].cpu().numpy(),
                     "shift": r["shift"].cpu().numpy()}, ref, f"torch call {it}")
    r0 = nl.build_neighborlists_torch(cell, d[:0], 6.0)
    assert r0["edge_index"].shape == (2, 0)


def test_far_images_take_full_transfer(nl, oracle):
    """The count pass stores a task's image shift in three 10-bit fields
    ([-511, 511]) beside its hit masks; atoms hundreds of cells away from the
    box give larger shifts, so those tasks skip the masks and the emit pass
    recomputes their tests -- same result."""
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid(n_clusters=200, box=26.0, seed=5)
    far = pos.copy()
    far[:40] += rows[0] * 700.0 + rows[2] * -600.0   # 700 / -600 cell lengths away
    for p in (pos, far):
        got = nl.build_neighborlists(nl.PyCell(rows.T.tolist()), p, 6.0)
        ref = oracle.search_single(p, rows.T, [True] * 3, 6.0, nthreads=8)
        assert_same(got, ref, "far images" if p is far else "near")
    assert np.abs(got["shift"]).max() > 511


@pytest.mark.parametrize("rc", [8.0, 12.0])
def test_dense_system_emit_paths(nl, oracle, rc):
    """A dense liquid where a (32-atom group, stencil cell) task has a few
    hundred (rc 8) to a few thousand (rc 12) hits: the emit pass stages small
    tasks in shared memory and writes large ones lane by lane; both give the
    oracle's edges in the oracle's order."""
    rng = np.random.default_rng(17)
    box = 36.0
    pos = rng.random((20000, 3)) * box
    h = np.eye(3) * box
    got = nl.build_neighborlists(nl.PyCell(h.tolist()), pos, rc)
    ref = oracle.search_single(pos, h, PBC3, rc, nthreads=16)
    assert_same(got, ref, f"dense liquid rc {rc}")


@pytest.mark.parametrize("cell", [True, False])
def test_non_finite_positions(nl, oracle, cell):
    """NaN and infinite coordinates follow the reference's saturating casts
    (NaN -> 0) and NaN-ignoring auto-box bounds: same edges as the oracle."""
    rng = np.random.default_rng(23)
    pos = rng.random((1500, 3)) * 25.0
    pos[7] = [np.nan, 3.0, 4.0]
    pos[100] = [np.inf, 1.0, 2.0]
    pos[200, 2] = -np.inf
    pos[300] = [np.nan, np.nan, np.nan]
    h = np.eye(3) * 25.0 if cell else None
    got = nl.build_neighborlists(nl.PyCell(h.tolist()) if cell else None, pos, 5.0)
    ref = oracle.search_single(pos, h, PBC3 if cell else None, 5.0, nthreads=8)
    assert_same(got, ref, f"non-finite positions (cell={cell})")


def test_result_arrays_own_their_pinned_blocks(nl):
    """Result arrays view library-owned pinned blocks: a view outliving its
    dict keeps the block (and its values); dropped results return their
    blocks, so steady-state calls allocate no new pinned memory."""
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid(n_clusters=139, box=23.2, seed=21)
    cell = nl.PyCell(rows.T.tolist())
    first = nl.build_neighborlists(cell, pos, 6.0)
    ref_ei, ref_sh = first["edge_index"].copy(), first["shift"].copy()
    view = first["edge_index"][:, ::7]
    del first
    for _ in range(3):
        nl.build_neighborlists(cell, pos, 6.0)
    s0 = nl.pinned_stats()
    for _ in range(20):
        r = nl.build_neighborlists(cell, pos, 6.0)
        assert r["edge_index"].base is not None and not r["edge_index"].flags.owndata
        del r
    s1 = nl.pinned_stats()
    assert s1["host_alloc_calls"] == s0["host_alloc_calls"], (s0, s1)
    assert s1["cache_hits"] >= s0["cache_hits"] + 20, (s0, s1)
    assert np.array_equal(view, ref_ei[:, ::7])
    r = nl.build_neighborlists(cell, pos, 6.0)
    assert_same(r, (ref_ei, ref_sh), "after block reuse")


def test_concurrent_host_threads(nl):
    """Builds from several host threads at once (each thread has its own
    stream and workspace) give the single-threaded results."""
    import threading

    from neighborlist_rs import workloads as W

    systems = [W.cluster_liquid(n_clusters=150 + 40 * k, box=24.0 + 2 * k, seed=k)
               for k in range(6)]
    cells = [nl.PyCell(r.T.tolist()) for _, r in systems]
    expected = [nl.build_neighborlists(c, p, 6.0) for c, (p, _) in zip(cells, systems)]
    got = {}
    errors = []

    def worker(t):
        try:
            for rep in range(5):
                for k in range(len(systems)):
                    i = (k + t) % len(systems)
                    got[(t, rep, i)] = nl.build_neighborlists(cells[i], systems[i][0], 6.0)
        except Exception as e:  # reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    assert not errors, errors
    for (t, rep, i), r in got.items():
        assert_same(r, (expected[i]["edge_index"], expected[i]["shift"]), f"thread {t} rep {rep}")
