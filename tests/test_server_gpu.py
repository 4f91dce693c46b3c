"""Served request loop (continuous batching): every served result equals the
same request built alone (and the oracle), whatever else shares its batch;
HBM-budget admission, device-resident results, rejection and error paths."""

import threading

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
    import neighborlist_rs.serving  # noqa: F401

    return neighborlist_rs


@pytest.fixture(scope="module")
def stream():
    from neighborlist_rs import workloads

    return workloads.request_stream(64, seed=11, max_atoms=6000)


def same(got, ref, what):
    """assert_same for two result dicts (or a dict and an oracle tuple)."""
    if isinstance(ref, dict):
        ref = (ref["edge_index"], ref["shift"])
    assert_same(got, ref, what)


def cell_of(nl, rows, pbc=(True, True, True)):
    return None if rows is None else nl.PyCell(np.asarray(rows).T.tolist(), list(pbc))


def test_mixed_stream_equals_alone_and_oracle(nl, oracle, stream):
    from neighborlist_rs.serving import Server

    reqs = [(cell_of(nl, s.cell_rows), s.positions, s.cutoff, s.cell_rows) for s in stream]
    # Extra shapes: empty, one atom with self-images, mixed periodicity
    # (brute-force minimum image), a tiny box with many images.
    rng = np.random.default_rng(3)
    reqs.append((cell_of(nl, np.eye(3) * 10.0), np.zeros((0, 3)), 5.0, np.eye(3) * 10.0))
    reqs.append((cell_of(nl, np.eye(3) * 2.0), np.zeros((1, 3)), 5.0, np.eye(3) * 2.0))
    mixed = np.eye(3) * 20.0
    reqs.append((cell_of(nl, mixed, (True, False, True)), rng.random((300, 3)) * 20.0, 4.0,
                 mixed))
    tiny = np.array([[3.0, 0.0, 0.0], [0.7, 3.2, 0.0], [0.4, 0.5, 2.9]])
    reqs.append((cell_of(nl, tiny), rng.random((12, 3)) @ tiny, 7.5, tiny))
    with Server(hbm_budget_bytes=8 << 30, workers=2, max_batch=256) as srv:
        tickets = [srv.submit(c, p, rc) for c, p, rc, _ in reqs]
        served = [srv.wait(t, timeout=120.0) for t in tickets]
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["largest_batch"] > 1, "small requests were never batched"
    for i, ((c, p, rc, rows), got) in enumerate(zip(reqs, served)):
        alone = nl.build_neighborlists(c, np.ascontiguousarray(p, dtype=np.float64), rc)
        same(got, alone, f"request {i} (n={p.shape[0]}) served vs alone")
        if 0 < p.shape[0] <= 3000:
            pbc = None if c is None else [bool(x) for x in c._pbc]
            ref = oracle.search_single(p, None if rows is None else rows.T, pbc, rc, nthreads=8)
            assert_same(got, ref, f"request {i} served vs oracle")


def test_same_request_in_different_mixes(nl, stream):
    """One request served alone, in a batch of small systems and behind a
    large one gives the same arrays each time."""
    from neighborlist_rs.serving import Server

    probe = next(s for s in stream if 100 < s.positions.shape[0] <= 2048)
    pc = cell_of(nl, probe.cell_rows)
    outs = []
    with Server(hbm_budget_bytes=4 << 30, workers=1, max_batch=64) as srv:
        outs.append(srv.wait(srv.submit(pc, probe.positions, probe.cutoff)))
        ts = [srv.submit(cell_of(nl, s.cell_rows), s.positions, s.cutoff) for s in stream[:20]]
        tp = srv.submit(pc, probe.positions, probe.cutoff)
        for t in ts:
            srv.wait(t)
        outs.append(srv.wait(tp))
        big = max(stream, key=lambda s: s.positions.shape[0])
        tb = srv.submit(cell_of(nl, big.cell_rows), big.positions, big.cutoff)
        tp = srv.submit(pc, probe.positions, probe.cutoff)
        srv.wait(tb)
        outs.append(srv.wait(tp))
    for o in outs[1:]:
        same(o, outs[0], "probe request in another mix")


def test_budget_admission_and_rejection(nl, stream):
    from neighborlist_rs.serving import Server

    # A budget that holds only a few requests at a time: everything still
    # completes, in order, and nothing stays reserved afterwards.
    small = [s for s in stream if s.positions.shape[0] <= 2048][:24]
    with Server(hbm_budget_bytes=24 << 20, workers=2, max_batch=64) as srv:
        tickets = []
        for s in small:
            try:
                tickets.append((s, srv.submit(cell_of(nl, s.cell_rows), s.positions, s.cutoff)))
            except ValueError as e:
                assert "exceeds the server's HBM budget" in str(e)
        assert tickets
        for s, t in tickets:
            got = srv.wait(t, timeout=120.0)
            alone = nl.build_neighborlists(cell_of(nl, s.cell_rows), s.positions, s.cutoff)
            same(got, alone, "request under a small budget")
        st = srv.stats()
        assert st["reserved_bytes"] == 0 and st["queued"] == 0
        # A request larger than the whole budget is refused at submit.
        big = np.random.default_rng(0).random((200_000, 3)) * 120.0
        with pytest.raises(ValueError, match="exceeds the server's HBM budget"):
            srv.submit(cell_of(nl, np.eye(3) * 120.0), big, 8.0)


def test_device_results_and_release(nl, stream):
    import torch

    from neighborlist_rs.serving import DeviceResult, Server

    picks = [s for s in stream if s.positions.shape[0] <= 2048][:6]
    picks.append(max(stream, key=lambda s: s.positions.shape[0]))
    with Server(hbm_budget_bytes=4 << 30, workers=2) as srv:
        tickets = [srv.submit(cell_of(nl, s.cell_rows), s.positions, s.cutoff, device_result=True)
                   for s in picks]
        for s, t in zip(picks, tickets):
            r = srv.wait(t)
            assert isinstance(r, DeviceResult)
            d = r.to_torch()
            torch.cuda.synchronize()
            alone = nl.build_neighborlists(cell_of(nl, s.cell_rows), s.positions, s.cutoff)
            same({"edge_index": d["edge_index"].cpu().numpy(),
                  "shift": d["shift"].cpu().numpy()}, alone, "device-resident result")
            assert srv.stats()["reserved_bytes"] >= 28 * r.n_edges
            r.release()
        assert srv.stats()["reserved_bytes"] == 0


def test_concurrent_clients(nl, stream):
    from neighborlist_rs.serving import Server

    subset = stream[:32]
    expected = [nl.build_neighborlists(cell_of(nl, s.cell_rows), s.positions, s.cutoff)
                for s in subset]
    got = [None] * len(subset)
    errors = []
    with Server(hbm_budget_bytes=8 << 30, workers=3, max_batch=128) as srv:
        def client(k):
            try:
                for i in range(k, len(subset), 4):
                    s = subset[i]
                    got[i] = srv.wait(srv.submit(cell_of(nl, s.cell_rows), s.positions, s.cutoff))
            except Exception as e:  # reported below
                errors.append(e)

        threads = [threading.Thread(target=client, args=(k,)) for k in range(4)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    assert not errors, errors
    for i, (g, e) in enumerate(zip(got, expected)):
        same(g, e, f"client request {i}")


def test_server_validation(nl):
    from neighborlist_rs.serving import Server

    with Server(hbm_budget_bytes=1 << 30, workers=1) as srv:
        p = np.zeros((4, 3))
        with pytest.raises(ValueError, match="Cutoff must be positive and finite"):
            srv.submit(None, p, -1.0)
        with pytest.raises(ValueError, match="Cutoff must be positive and finite"):
            srv.submit(None, p, float("nan"))
        with pytest.raises(ValueError, match=r"Positions must be \(N, 3\)"):
            srv.submit(None, np.zeros((4, 2)), 5.0)
        with pytest.raises(ValueError, match="unknown ticket"):
            srv.wait(12345)
        t = srv.submit(None, p, 5.0)
        assert srv.wait(t)["edge_index"].shape[1] == 6
        with pytest.raises(ValueError, match="unknown ticket"):
            srv.wait(t)  # host results retire their ticket
    with pytest.raises(RuntimeError, match="server is closed"):
        srv.submit(None, p, 5.0)
    with pytest.raises(RuntimeError):
        Server(hbm_budget_bytes=0)


def test_mixed_host_and_device_results(nl, stream):
    """Host and device results in the same batches (the device ones share
    one pooled block) equal the requests built alone; released blocks
    return their reservation."""
    import torch

    from neighborlist_rs.serving import DeviceResult, Server

    picks = [s for s in stream if s.positions.shape[0] <= 2048][:16]
    with Server(hbm_budget_bytes=4 << 30, workers=1, max_batch=64) as srv:
        tickets = [srv.submit(cell_of(nl, s.cell_rows), s.positions, s.cutoff,
                              device_result=(i % 2 == 0)) for i, s in enumerate(picks)]
        got = [srv.wait(t) for t in tickets]
        assert srv.stats()["largest_batch"] > 1
        device_results = [r for r in got if isinstance(r, DeviceResult)]
        assert len(device_results) == len(got[0::2])
        for i, (s, r) in enumerate(zip(picks, got)):
            alone = nl.build_neighborlists(cell_of(nl, s.cell_rows), s.positions, s.cutoff)
            if i % 2 == 0:
                assert isinstance(r, DeviceResult)
                d = r.to_torch()
                torch.cuda.synchronize()
                r = {"edge_index": d["edge_index"].cpu().numpy(), "shift": d["shift"].cpu().numpy()}
            same(r, alone, f"mixed request {i}")
        for r in device_results:
            r.release()
        assert srv.stats()["reserved_bytes"] == 0
