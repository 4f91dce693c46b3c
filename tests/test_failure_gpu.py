"""Failure detection without any GPU fault.

* Device waits are bounded: the prefix scan's look-back gives up after a
  poll limit, records an error word and finishes.  The test hook
  nlb_debug_scan_stall makes one tile of the next scan withhold its
  publication (a flag that nothing sets), so the wait runs out; the build
  must report NLB_ERR_CUDA ("prefix scan gave up waiting for a tile"), the
  emit pass must write nothing, and the next builds on the same thread,
  device and workspace must be exact again (single-system fast path,
  multi-cutoff path, batched path).
* Server failure paths on the host: cancelled and abandoned tickets, a
  paused server, and a batch whose staging fails (an error code injected in
  place of a failing CUDA call), which the worker reruns one request at a
  time so that only the offending request fails.
"""

import ctypes
import time

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
    import neighborlist_rs.serving  # noqa: F401

    neighborlist_rs._lib.nlb_debug_scan_stall.argtypes = [ctypes.c_int32, ctypes.c_int32]
    return neighborlist_rs


def stall_next_scan(nl, tile=3, spins=2048):
    assert nl._lib.nlb_debug_scan_stall(tile, spins) == 0


def test_scan_hook_validates_arguments(nl):
    assert nl._lib.nlb_debug_scan_stall(-1, 10) == 1
    assert nl._lib.nlb_debug_scan_stall(0, 0) == 1


def test_single_system_scan_gives_up_and_recovers(nl, oracle):
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid()  # 10,008 atoms x 27 stencil cells: 132 scan tiles
    cell = nl.PyCell(rows.T.tolist())
    ref = oracle.search_single(pos, rows.T, PBC3, 6.0, nthreads=16)
    assert_same(nl.build_neighborlists(cell, pos, 6.0), ref, "before")
    stall_next_scan(nl)
    with pytest.raises(RuntimeError, match="prefix scan gave up waiting for a tile"):
        nl.build_neighborlists(cell, pos, 6.0)
    # Same thread, device and workspace: direct, captured and replayed builds.
    for k in range(4):
        assert_same(nl.build_neighborlists(cell, pos, 6.0), ref, f"after, call {k}")
    # The device-resident entry point (same pipeline, torch tensors out).
    import torch

    dpos = torch.from_numpy(pos).cuda()
    stall_next_scan(nl, tile=7)
    with pytest.raises(RuntimeError, match="prefix scan gave up"):
        nl.build_neighborlists_torch(cell, dpos, 6.0)
    got = nl.build_neighborlists_torch(cell, dpos, 6.0)
    assert_same({"edge_index": got["edge_index"].cpu().numpy(),
                 "shift": got["shift"].cpu().numpy()}, ref, "device after")


def test_multi_and_batched_scans_give_up_and_recover(nl, oracle):
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid()
    cell = nl.PyCell(rows.T.tolist())
    stall_next_scan(nl)
    with pytest.raises(RuntimeError, match="prefix scan gave up"):
        nl.build_neighborlists_multi(cell, pos, [5.0, 6.0])
    refm = oracle.search_single_multi(pos, rows.T, PBC3, [5.0, 6.0], nthreads=16)
    got = nl.build_neighborlists_multi(cell, pos, [5.0, 6.0])
    assert_same(got[0], refm[0], "multi rc 5 after")
    assert_same(got[1], refm[1], "multi rc 6 after")

    pb, bb, cb = W.concat_batch(W.uneven_batch(n_systems=512, seed=15))
    ocells = [None if not c.any() else (c.T, PBC3) for c in cb]
    (refb,) = oracle.search_batch(pb, bb, ocells, [5.0], nthreads=16)
    stall_next_scan(nl, tile=2)
    with pytest.raises(RuntimeError, match="prefix scan gave up"):
        nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0)
    assert_same(nl.build_neighborlists_batch(pb, bb, cells=cb, cutoff=5.0), refb, "batch after")


def small_requests(nl, n=12, seed=31):
    from neighborlist_rs import workloads as W

    out = []
    for s in W.request_stream(n, seed=seed, n_range=(16, 1500)):
        cell = None if s.cell_rows is None else nl.PyCell(s.cell_rows.T.tolist())
        out.append((cell, s.positions, s.cutoff))
    return out


def test_server_pause_and_cancel(nl):
    from neighborlist_rs.serving import Server

    reqs = small_requests(nl)
    with Server(hbm_budget_bytes=4 << 30, workers=2, max_batch=64) as srv:
        srv.pause(True)
        tickets = [srv.submit(c, p, rc) for c, p, rc in reqs]
        st = srv.stats()
        assert st["queued"] == len(reqs) and st["completed"] == 0
        srv.cancel(tickets[1])
        srv.cancel(tickets[4])
        st = srv.stats()
        assert st["queued"] == len(reqs) - 2 and st["cancelled"] == 2
        with pytest.raises(ValueError, match="unknown ticket"):
            srv.wait(tickets[1], timeout=1.0)
        srv.pause(False)
        for i, ((c, p, rc), t) in enumerate(zip(reqs, tickets)):
            if i in (1, 4):
                continue
            alone = nl.build_neighborlists(c, p, rc)
            assert_same(srv.wait(t, timeout=60.0), (alone["edge_index"], alone["shift"]),
                        f"request {i}")
        # A finished request that was never collected: cancel frees its result.
        c, p, rc = reqs[0]
        t = srv.submit(c, p, rc)
        done = srv.stats()["completed"] + 1
        for _ in range(2000):
            if srv.stats()["completed"] >= done:
                break
            time.sleep(0.005)
        srv.cancel(t)
        with pytest.raises(ValueError, match="unknown ticket"):
            srv.wait(t, timeout=1.0)
        # A device-resident result can be cancelled instead of released.
        td = srv.submit(c, p, rc, device_result=True)
        dev = srv.wait(td, timeout=60.0)
        reserved = srv.stats()["reserved_bytes"]
        assert reserved >= 28 * dev.n_edges
        srv.cancel(td)
        assert srv.stats()["reserved_bytes"] == reserved - 28 * dev.n_edges
        st = srv.stats()
        assert st["failed"] == 0 and st["cancelled"] == 2


def test_server_abandoned_tickets_are_freed_on_close(nl):
    from neighborlist_rs.serving import Server

    reqs = small_requests(nl, n=24, seed=32)
    srv = Server(hbm_budget_bytes=4 << 30, workers=2, max_batch=64)
    srv.pause(True)
    queued = [srv.submit(c, p, rc) for c, p, rc in reqs[:12]]
    srv.pause(False)
    finished = [srv.submit(c, p, rc, device_result=k % 2 == 0)
                for k, (c, p, rc) in enumerate(reqs[12:])]
    assert queued and finished
    srv.close()  # nothing was collected: queued ones cancelled, results freed
    with pytest.raises(RuntimeError, match="server is closed"):
        srv.stats()
    # a fresh server on the same device works
    with Server(hbm_budget_bytes=4 << 30, workers=1) as srv2:
        c, p, rc = reqs[0]
        assert_same(srv2.wait(srv2.submit(c, p, rc), timeout=60.0),
                    (lambda r: (r["edge_index"], r["shift"]))(nl.build_neighborlists(c, p, rc)),
                    "fresh server")


def test_server_batch_staging_failure_fails_only_that_request(nl, oracle):
    from neighborlist_rs import workloads as W
    from neighborlist_rs.serving import Server

    reqs = small_requests(nl, n=12, seed=33)
    rng = np.random.default_rng(34)
    rows = W.density_cell(6000, 0.1, rng, None, ortho=True)
    big = (nl.PyCell(rows.T.tolist()), rng.random((6000, 3)) @ rows, 6.0)  # single-system path
    with Server(hbm_budget_bytes=8 << 30, workers=1, max_batch=64) as srv:
        srv.pause(True)
        tickets = [srv.submit(c, p, rc) for c, p, rc in reqs]
        tb = srv.submit(*big)
        tb2 = srv.submit(*big)
        srv._debug_fail(tickets[5])
        srv._debug_fail(tb2)
        srv.pause(False)
        for i, ((c, p, rc), t) in enumerate(zip(reqs, tickets)):
            if i == 5:
                with pytest.raises(RuntimeError, match="staging failed"):
                    srv.wait(t, timeout=60.0)
                continue
            got = srv.wait(t, timeout=60.0)
            alone = nl.build_neighborlists(c, p, rc)
            assert_same(got, (alone["edge_index"], alone["shift"]), f"request {i}")
        c, p, rc = big
        ref = oracle.search_single(p, rows.T, PBC3, rc, nthreads=16)
        assert_same(srv.wait(tb, timeout=60.0), ref, "large request")
        with pytest.raises(RuntimeError, match="staging failed"):
            srv.wait(tb2, timeout=60.0)
        st = srv.stats()
    # 11 small requests and the first large one completed; two failed
    assert st["failed"] == 2 and st["completed"] == len(reqs)
