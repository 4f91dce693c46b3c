"""Verlet (skin) list manager: along seeded trajectories every update returns
exactly the pairs a fresh build at the cutoff finds (as a set of (i, j, S);
pairs within 1e-9 A of the cutoff are excluded from the comparison, as the
two computations round differently there), rebuilds happen exactly when an
atom moved more than skin / 2 or the system changed, and host and device
updates agree."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def nl():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import neighborlist_rs
    import neighborlist_rs.verlet  # noqa: F401

    return neighborlist_rs


def edge_set(res, pos, h, rc, tol=1e-9):
    """{(i, j, sx, sy, sz)} of res, without the pairs within tol of rc."""
    ei, sh = res["edge_index"], res["shift"]
    if hasattr(ei, "cpu"):
        ei, sh = ei.cpu().numpy(), sh.cpu().numpy()
    d = pos[ei[1]] - pos[ei[0]] + (0 if h is None else sh @ np.asarray(h).T)
    r = np.linalg.norm(d, axis=1) if len(d) else np.zeros(0)
    ok = np.abs(r - rc) > tol
    return {(int(a), int(b), *map(int, s)) for a, b, s, k in zip(ei[0], ei[1], sh, ok) if k}


def fresh_set(nl, cell, pos, h, rc):
    return edge_set(nl.build_neighborlists(cell, pos, rc), pos, h, rc)


def trajectory(rng, pos0, steps, step_size):
    pos = pos0.copy()
    for _ in range(steps):
        pos = pos + rng.normal(0.0, step_size, pos.shape)
        yield pos


@pytest.mark.parametrize("kind", ["periodic", "triclinic", "isolated", "small_brute"])
def test_verlet_matches_fresh_builds(nl, kind):
    from neighborlist_rs.verlet import VerletList

    rng = np.random.default_rng({"periodic": 1, "triclinic": 2, "isolated": 3,
                                 "small_brute": 4}[kind])
    if kind == "periodic":
        h = np.eye(3) * 28.0
        pos0, rc, n = rng.random((2200, 3)) * 28.0, 5.0, 2200
    elif kind == "triclinic":
        h = np.array([[24.0, 0.0, 0.0], [4.0, 22.0, 0.0], [-3.0, 2.0, 21.0]]).T
        pos0, rc = rng.random((1500, 3)) @ h.T, 4.5
    elif kind == "isolated":
        h = None
        pos0, rc = rng.random((3000, 3)) * 30.0, 4.0
    else:
        h = np.eye(3) * 12.0
        pos0, rc = rng.random((150, 3)) * 12.0, 3.0
    cell = None if h is None else nl.PyCell(h.tolist())
    skin = 1.0
    rebuilds = 0
    with VerletList(rc, skin) as vl:
        ref = pos0.copy()
        for k, pos in enumerate(trajectory(rng, pos0, 12, 0.06)):
            expect_rebuild = k == 0 or np.linalg.norm(pos - ref, axis=1).max() > skin / 2
            needs = vl.needs_rebuild(cell, pos)
            assert needs == expect_rebuild, (kind, k)
            res = vl.update(cell, pos)
            assert vl.rebuilt == expect_rebuild, (kind, k)
            if vl.rebuilt:
                ref = pos.copy()
                rebuilds += 1
            assert edge_set(res, pos, h, rc) == fresh_set(nl, cell, pos, h, rc), (kind, k)
        st = vl.stats()
    assert st["updates"] == 12 and st["rebuilds"] == rebuilds
    assert 1 <= rebuilds < 12, "the trajectory should reuse the list at least once"


def test_verlet_device_matches_host_and_system_changes(nl):
    import torch

    from neighborlist_rs.verlet import VerletList

    rng = np.random.default_rng(9)
    h = np.eye(3) * 25.0
    cell = nl.PyCell(h.tolist())
    pos = rng.random((1800, 3)) * 25.0
    with VerletList(5.0, 0.8) as a, VerletList(5.0, 0.8) as b:
        for step in range(6):
            pos = pos + rng.normal(0.0, 0.05, pos.shape)
            ha = a.update(cell, pos)
            db = b.update(cell, torch.from_numpy(pos).cuda())
            torch.cuda.synchronize()
            assert a.rebuilt == b.rebuilt
            assert np.array_equal(ha["edge_index"], db["edge_index"].cpu().numpy())
            assert np.array_equal(ha["shift"], db["shift"].cpu().numpy())
        # A new cell, a new atom count and new periodicity all force a rebuild.
        h2 = h * 1.01
        a.update(nl.PyCell(h2.tolist()), pos)
        assert a.rebuilt
        a.update(nl.PyCell(h2.tolist()), pos[:-5])
        assert a.rebuilt
        a.update(nl.PyCell(h2.tolist(), [True, False, True]), pos[:-5])
        assert a.rebuilt
        a.update(nl.PyCell(h2.tolist(), [True, False, True]), pos[:-5])
        assert not a.rebuilt
        # Re-wrapping an atom into the box moves it by a lattice vector.
        p = pos[:-5].copy()
        p[0, 0] += h2[0, 0]
        assert a.needs_rebuild(nl.PyCell(h2.tolist(), [True, False, True]), p)


def test_verlet_validation(nl):
    from neighborlist_rs.verlet import VerletList

    with pytest.raises(ValueError, match="Cutoff must be positive and finite"):
        VerletList(0.0, 1.0)
    with pytest.raises(ValueError, match="Skin must be non-negative and finite"):
        VerletList(5.0, -1.0)
    with VerletList(4.0, 0.0) as vl:  # zero skin: rebuild whenever anything moves
        p = np.random.default_rng(1).random((50, 3)) * 8.0
        r0 = vl.update(None, p)
        r1 = vl.update(None, p)
        assert not vl.rebuilt and np.array_equal(r0["edge_index"], r1["edge_index"])
        vl.update(None, p + 1e-6)
        assert vl.rebuilt
        e = vl.update(None, np.zeros((0, 3)))
        assert e["edge_index"].shape == (2, 0)


@pytest.mark.parametrize("kind", ["periodic", "triclinic", "isolated", "small_brute"])
def test_verlet_matches_oracle_restatement(nl, oracle, kind):
    """Byte for byte against the oracle: at each rebuild the oracle's half
    list at rc + skin of those positions is stored, and each update must
    return oracle.verlet_filter of the stored list with the current
    positions (same edges, same order, no pairs excluded near rc)."""
    from neighborlist_rs.verlet import VerletList

    from helpers import assert_same

    rng = np.random.default_rng({"periodic": 11, "triclinic": 12, "isolated": 13,
                                 "small_brute": 14}[kind])
    if kind == "periodic":
        h = np.eye(3) * 28.0
        pos0, rc = rng.random((2200, 3)) * 28.0, 5.0
    elif kind == "triclinic":
        h = np.array([[24.0, 0.0, 0.0], [4.0, 22.0, 0.0], [-3.0, 2.0, 21.0]]).T
        pos0, rc = rng.random((1500, 3)) @ h.T, 4.5
    elif kind == "isolated":
        h = None
        pos0, rc = rng.random((3000, 3)) * 30.0, 4.0
    else:
        h = np.eye(3) * 12.0
        pos0, rc = rng.random((150, 3)) * 12.0, 3.0
    cell = None if h is None else nl.PyCell(h.tolist())
    pbc = None if h is None else [True] * 3
    skin = 1.0
    stored = None
    reused = 0
    with VerletList(rc, skin) as vl:
        for k, pos in enumerate(trajectory(rng, pos0, 14, 0.06)):
            res = vl.update(cell, pos)
            if vl.rebuilt:
                stored = oracle.search_single(pos, h, pbc, rc + skin, nthreads=8)
            else:
                reused += 1
            want = oracle.verlet_filter(pos, h, stored, rc)
            assert_same(res, want, f"{kind} step {k}")
    assert reused >= 1


def test_verlet_device_results_are_library_blocks(nl):
    """Device updates hand over the blocks the compaction wrote (no copy):
    two blocks per update with edges, returned to the pool when the tensors
    go; the lists equal the host update's."""
    import gc

    import torch

    from neighborlist_rs import workloads as W
    from neighborlist_rs.verlet import VerletList

    pos, rows = W.cluster_liquid(n_clusters=400, box=33.0, seed=5)
    cell = nl.PyCell(rows.T.tolist())
    rng = np.random.default_rng(8)
    gc.collect()
    b0 = nl.device_blocks()
    with VerletList(6.0, 1.0) as vd, VerletList(6.0, 1.0) as vh:
        for k in range(4):
            p = pos + rng.normal(0.0, 0.02, pos.shape) * k
            rd = vd.update(cell, torch.from_numpy(p).cuda())
            rh = vh.update(cell, p)
            assert np.array_equal(rd["edge_index"].cpu().numpy(), rh["edge_index"])
            assert np.array_equal(rd["shift"].cpu().numpy(), rh["shift"])
            assert rd["edge_index"].shape[1] > 0
            b1 = nl.device_blocks()
            assert b1["handed"] - b0["handed"] >= 2 * (k + 1)
            del rd
            gc.collect()
    torch.cuda.synchronize()
    b2 = nl.device_blocks()
    assert b2["returned"] - b0["returned"] == b2["handed"] - b0["handed"]
