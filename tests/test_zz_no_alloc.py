"""nlb_build_noalloc: the build for callers that cannot allocate GPU memory.

It is called here through the C ABI with caller-owned device buffers (torch
tensors), and each result must equal, edge for edge, what the regular entry
point nlb_build returns for the same system.  Two different systems are built
in a row (a periodic cell-list system, then an isolated brute-force one, then
the first again), so stale contents of the shared scratch array would show.
This file is collected last on purpose, and it also passes on its own in a
fresh process.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import neighborlist_rs as nl

    lib = ctypes.CDLL(nl.LIB_PATH)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.nlb_build_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, dp,
                                      ctypes.POINTER(ctypes.c_uint8), ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_int64,
                                      ctypes.POINTER(ctypes.c_int64), ctypes.c_void_p]
    lib.nlb_last_error.restype = ctypes.c_char_p
    return torch, nl, lib


def noalloc_build(env, pos, rows, rc, max_edges):
    torch, nl, lib = env
    d_pos = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
    ei = torch.full((2, max_edges), -7, dtype=torch.int64, device="cuda")
    sh = torch.full((max_edges, 3), -7, dtype=torch.int32, device="cuda")
    m = ctypes.c_int64(-1)
    if rows is None:
        h = None
        pbc = None
    else:
        h9 = np.ascontiguousarray(rows.T.reshape(9))
        h = h9.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        pb = (ctypes.c_uint8 * 3)(1, 1, 1)
        pbc = pb
    stream = torch.cuda.current_stream().cuda_stream
    rc_code = lib.nlb_build_noalloc(d_pos.data_ptr(), pos.shape[0], rc, h, pbc, ei.data_ptr(),
                                    sh.data_ptr(), max_edges, ctypes.byref(m), stream)
    return rc_code, int(m.value), ei, sh


def regular_build(nl, pos, rows, rc):
    cell = None if rows is None else nl.PyCell(rows.T.tolist())
    return nl.build_neighborlists(cell, pos, rc)


def test_noalloc_matches_regular_entry_point(env):
    torch, nl, lib = env
    from neighborlist_rs import workloads as W

    pos_a, rows_a = W.cluster_liquid(n_clusters=139, box=23.2, seed=31)   # cell list
    pos_b = W.isolated_cube(n=700, side=19.0, seed=32)                     # brute force
    cap = 200_000
    for pos, rows, rc in [(pos_a, rows_a, 6.0), (pos_b, None, 5.0), (pos_a, rows_a, 6.0)]:
        code, m, ei, sh = noalloc_build(env, pos, rows, rc, cap)
        assert code == 0, lib.nlb_last_error().decode()
        ref = regular_build(nl, pos, rows, rc)
        assert m == ref["edge_index"].shape[1] > 0
        got_ei = torch.stack([ei[0, :m], ei[1, :m]]).cpu().numpy()
        assert np.array_equal(got_ei, ref["edge_index"])
        assert np.array_equal(sh[:m].cpu().numpy(), ref["shift"])
        # nothing written past the M valid columns
        assert bool((ei[:, m:] == -7).all()) and bool((sh[m:] == -7).all())


def test_noalloc_rejects_oversize(env):
    torch, nl, lib = env
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid(n_clusters=139, box=23.2, seed=31)
    code, m, ei, sh = noalloc_build(env, pos, rows, 6.0, 1000)
    assert code == 1 and m > 1000
    assert "output capacity" in lib.nlb_last_error().decode()
    assert bool((ei == -7).all())
    big = np.random.default_rng(0).random((20000, 3)) * 60.0
    code, m, _, _ = noalloc_build(env, big, None, 5.0, 10)
    assert code == 1 and "fixed capacity" in lib.nlb_last_error().decode()
