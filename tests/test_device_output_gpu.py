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
