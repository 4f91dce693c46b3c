"""The two single-system pipelines: the one-launch kernel (count, offsets by
look-back over groups, emit) that sparse grids take by default, and the
three-launch pair-task pipeline (count, scan, emit) -- each against the
oracle on the same inputs, host and device results, repeated calls (graph
replay), a clustered system whose first edge arena is too small, multi-image
stencils up to 125 cells, and lattices with atoms on bin faces."""

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
    neighborlist_rs.set_single_pipeline(0)


def systems():
    from neighborlist_rs import workloads as W

    rng = np.random.default_rng(61)
    out = []
    pos, rows = W.cluster_liquid()
    out.append(("cluster liquid rc 6", pos, rows, 6.0))
    pos, rows = W.triclinic_uniform(n=8000, seed=62, lengths=(40.0, 44.0))
    out.append(("triclinic rc 5", pos, rows, 5.0))
    out.append(("isolated cube rc 6", W.isolated_cube(), None, 6.0))
    # small periodic box, stencil of 125 cells (two images per axis)
    rows = np.diag([9.0, 9.5, 10.0])
    out.append(("multi-image rc 7", rng.random((1100, 3)) @ rows, rows, 7.0))
    # clustered atoms in a large box: ten times the uniform-density edges
    rows = np.eye(3) * 60.0
    clustered = np.concatenate([rng.random((4000, 3)) * 12.0 + 20.0, rng.random((1000, 3)) * 60.0])
    out.append(("clustered rc 4.5", clustered, rows, 4.5))
    # lattice on bin faces (irregular atoms) and exactly-at-cutoff pairs
    g = np.arange(16) * 2.0
    lat = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    out.append(("lattice rc 4", lat, np.eye(3) * 32.0, 4.0))
    out.append(("lattice rc sqrt(8)", lat + 0.5, np.eye(3) * 32.0, float(np.sqrt(8.0))))
    return out


@pytest.mark.parametrize("mode", [0, 1])
def test_pipeline_matches_oracle(nl, oracle, mode):
    import torch

    nl.set_single_pipeline(mode)
    try:
        for what, pos, rows, rc in systems():
            cell = None if rows is None else nl.PyCell(rows.T.tolist())
            ref = oracle.search_single(pos, None if rows is None else rows.T,
                                       None if rows is None else PBC3, rc, nthreads=16)
            for k in range(3):  # direct, captured, replayed
                assert_same(nl.build_neighborlists(cell, pos, rc), ref, f"{what} mode {mode} #{k}")
            d = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
            for k in range(2):
                r = nl.build_neighborlists_torch(cell, d, rc)
                assert_same({"edge_index": r["edge_index"].cpu().numpy(),
                             "shift": r["shift"].cpu().numpy()}, ref, f"{what} mode {mode} device #{k}")
    finally:
        nl.set_single_pipeline(0)


def test_pipeline_switch_api(nl):
    assert nl.set_single_pipeline(1) == 0
    assert nl.set_single_pipeline(None) == 1
    with pytest.raises(ValueError):
        nl.set_single_pipeline(7)


def test_fresh_thread_arena_growth(nl, oracle):
    """A fresh host thread sizes its first arena from the uniform density;
    the clustered system has far more edges, so the one-launch kernel writes
    nothing, the arena grows and the launch runs again."""
    import threading

    what, pos, rows, rc = [s for s in systems() if s[0].startswith("clustered")][0]
    cell = nl.PyCell(rows.T.tolist())
    ref = oracle.search_single(pos, rows.T, PBC3, rc, nthreads=16)
    out, errors = [], []

    def run():
        try:
            import torch

            torch.cuda.set_device(0)
            out.append(nl.build_neighborlists(cell, pos, rc))
            out.append(nl.build_neighborlists(cell, pos, rc))
        except Exception as e:  # reported below
            errors.append(e)

    t = threading.Thread(target=run)
    t.start()
    t.join()
    assert not errors, errors
    for k, r in enumerate(out):
        assert_same(r, ref, f"fresh thread call {k}")
