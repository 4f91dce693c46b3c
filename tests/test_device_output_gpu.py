"""Zero-copy device results: build_neighborlists_torch returns tensors that
ARE the library's result blocks (written in place by the build, handed over,
returned to the library's pool when the tensors are freed), equal to the
oracle's lists; several results can be held at once; torch allocates
nothing for them."""

import ctypes
import gc

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


def as_np(r):
    return {"edge_index": r["edge_index"].cpu().numpy(), "shift": r["shift"].cpu().numpy()}


def test_owned_block_is_the_tensor_storage(nl):
    import torch

    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid(n_clusters=300, box=30.0, seed=7)
    cell = nl.PyCell(rows.T.tolist())
    d = torch.from_numpy(pos).cuda()
    h, pb = nl._cell_args(cell)
    r = nl._DevResult()
    stream = torch.cuda.current_stream().cuda_stream
    nl.set_stream(stream)
    try:
        assert nl._lib.nlb_build_device_owned(ctypes.c_void_p(d.data_ptr()), pos.shape[0], 6.0,
                                              h, pb, ctypes.byref(r)) == 0
    finally:
        nl.set_stream(None)
    m = int(r.n_edges)
    ei = torch.as_tensor(nl._DeviceBlock(r.edge_index, (2, m), "<i8", stream), device="cuda")
    sh = torch.as_tensor(nl._DeviceBlock(r.shift, (m, 3), "<i4", stream), device="cuda")
    assert ei.data_ptr() == r.edge_index and sh.data_ptr() == r.shift
    ref = nl.build_neighborlists(cell, pos, 6.0)
    assert_same(as_np({"edge_index": ei, "shift": sh}), (ref["edge_index"], ref["shift"]),
                "owned block")
    # Freeing a pointer twice, or one the library never handed out, is refused.
    assert nl._lib.nlb_device_free(ctypes.c_void_p(d.data_ptr()), None) == 1


def test_torch_results_zero_copy_and_oracle(nl, oracle):
    import torch

    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid()
    cell = nl.PyCell(rows.T.tolist())
    ref = oracle.search_single(pos, rows.T, PBC3, 6.0, nthreads=16)
    d = torch.from_numpy(pos).cuda()
    torch.cuda.synchronize()
    gc.collect()
    alloc0 = torch.cuda.memory_allocated()
    b0 = nl.device_blocks()
    held = []
    for k in range(5):  # direct, captured and replayed builds; results held at once
        r = nl.build_neighborlists_torch(cell, d, 6.0)
        held.append(r)
        assert r["edge_index"].is_cuda and r["edge_index"].dtype == torch.int64
        assert r["shift"].dtype == torch.int32 and r["shift"].shape == (ref[0].shape[1], 3)
    # torch allocated nothing for the result tensors
    assert torch.cuda.memory_allocated() == alloc0
    b1 = nl.device_blocks()
    assert b1["handed"] - b0["handed"] == 10
    assert b1["outstanding_bytes"] - b0["outstanding_bytes"] >= 5 * 28 * ref[0].shape[1]
    ptrs = {r["edge_index"].data_ptr() for r in held}
    assert len(ptrs) == 5, "every held result has its own block"
    torch.cuda.synchronize()
    for k, r in enumerate(held):
        assert_same(as_np(r), ref, f"held result {k}")
    del held, r
    gc.collect()
    b2 = nl.device_blocks()
    assert b2["returned"] - b1["returned"] == 10
    assert b2["outstanding_bytes"] == b0["outstanding_bytes"]
    # A build/consume/free loop reuses the pool's blocks.
    for k in range(4):
        r = nl.build_neighborlists_torch(cell, d, 6.0)
        assert int(r["edge_index"][0].sum()) == int(ref[0][0].sum())
        del r
    # Small and empty systems, and the multi-image / brute-force paths.
    tiny = np.array([[0.1, 0.2, 0.3], [1.0, 1.1, 0.9], [2.0, 0.1, 1.7]])
    for p, rows_t, rc in [(tiny, np.eye(3) * 3.0, 4.0), (tiny, None, 1.5),
                          (np.zeros((0, 3)), np.eye(3) * 5.0, 2.0)]:
        c = None if rows_t is None else nl.PyCell(rows_t.T.tolist())
        got = nl.build_neighborlists_torch(c, torch.from_numpy(p).cuda(), rc)
        want = oracle.search_single(p, None if rows_t is None else rows_t.T,
                                    None if rows_t is None else PBC3, rc)
        assert_same(as_np(got), want, f"small system rc {rc}")


def test_builds_on_two_streams_without_host_sync(nl, oracle):
    """A build on a caller's stream returns as soon as M is known; the next
    build on another stream reuses the workspace only after that work (the
    library orders it on the device).  Both lists, read after the fact, equal
    the oracle's; so do raw workspace results read on the producing stream
    right after the call."""
    import torch

    from neighborlist_rs import workloads as W

    pos_a, rows_a = W.cluster_liquid(n_clusters=1112, box=46.4, seed=3)
    pos_b, rows_b = W.cluster_liquid(n_clusters=600, box=38.0, seed=9)
    cell_a, cell_b = nl.PyCell(rows_a.T.tolist()), nl.PyCell(rows_b.T.tolist())
    sa, sb = torch.cuda.Stream(), torch.cuda.Stream()
    with torch.cuda.stream(sa):
        da = torch.from_numpy(pos_a).cuda()
    with torch.cuda.stream(sb):
        db = torch.from_numpy(pos_b).cuda()
    torch.cuda.synchronize()
    for _ in range(3):
        with torch.cuda.stream(sa):
            ra = nl.build_neighborlists_torch(cell_a, da, 6.0)
        with torch.cuda.stream(sb):
            rb = nl.build_neighborlists_torch(cell_b, db, 6.0)
        torch.cuda.synchronize()
        assert_same(as_np(ra), oracle.search_single(pos_a, rows_a.T, PBC3, 6.0, nthreads=8),
                    "stream A")
        assert_same(as_np(rb), oracle.search_single(pos_b, rows_b.T, PBC3, 6.0, nthreads=8),
                    "stream B")
    # Raw workspace results, copied out on the producing stream at once.
    nl.set_stream(sa.cuda_stream)
    try:
        m, ei_ptr, sh_ptr = nl.build_device_raw(cell_a, da.data_ptr(), pos_a.shape[0], 6.0)
        with torch.cuda.stream(sa):
            ei = torch.empty((2, m), dtype=torch.int64, device="cuda")
            sh = torch.empty((m, 3), dtype=torch.int32, device="cuda")
            assert nl._lib.nlb_copy_device(ctypes.c_void_p(ei.data_ptr()), ctypes.c_void_p(ei_ptr),
                                           16 * m, ctypes.c_void_p(sa.cuda_stream)) == 0
            assert nl._lib.nlb_copy_device(ctypes.c_void_p(sh.data_ptr()), ctypes.c_void_p(sh_ptr),
                                           12 * m, ctypes.c_void_p(sa.cuda_stream)) == 0
    finally:
        nl.set_stream(None)
    torch.cuda.synchronize()
    assert_same(as_np({"edge_index": ei, "shift": sh}),
                oracle.search_single(pos_a, rows_a.T, PBC3, 6.0, nthreads=8), "raw on stream A")
