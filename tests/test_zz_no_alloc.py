"""nlb_build_noalloc: the build for callers that cannot allocate GPU memory.

It is called here through the C ABI with caller-owned device buffers (torch
tensors), and each result must equal, edge for edge, what the regular entry
point nlb_build returns for the same system.  Two different systems are built
in a row (a periodic cell-list system, then an isolated brute-force one, then
the first again), so stale contents of the shared scratch array would show.
The entry point is also checked against the CPU oracle directly, for its
size checks (refused before any launch), and for the property that defines
it: a series of calls leaves the device's free memory unchanged.
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


def test_noalloc_matches_oracle(env, oracle):
    """The entry point against the CPU oracle directly: a periodic cell-list
    system, an isolated brute-force one and a triclinic cell-list one, each
    twice in a row."""
    torch, nl, lib = env
    from neighborlist_rs import workloads as W

    pos_a, rows_a = W.cluster_liquid(n_clusters=139, box=23.2, seed=41)
    pos_b = W.isolated_cube(n=900, side=20.0, seed=42)
    pos_c, rows_c = W.triclinic_uniform(n=4000, seed=43, lengths=(30.0, 36.0))
    cases = [(pos_a, rows_a, 6.0), (pos_b, None, 5.0), (pos_c, rows_c, 5.0)]
    for pos, rows, rc in cases + cases:
        code, m, ei, sh = noalloc_build(env, pos, rows, rc, 300_000)
        assert code == 0, lib.nlb_last_error().decode()
        h = None if rows is None else rows.T
        pbc = None if rows is None else [True] * 3
        want_ei, want_sh = oracle.search_single(pos, h, pbc, rc, nthreads=4)
        assert m == want_ei.shape[1] > 0
        got_ei = torch.stack([ei[0, :m], ei[1, :m]]).cpu().numpy()
        assert np.array_equal(got_ei, want_ei)
        assert np.array_equal(sh[:m].cpu().numpy(), want_sh)


def test_noalloc_rejects_grids_beyond_capacity_before_launching(env):
    """A tiny cutoff in a huge cell asks for far more bins than the fixed
    scratch holds (and more than 2^21 along an axis): the call is refused
    with NLB_ERR_VALUE before any kernel touches the scratch array."""
    torch, nl, lib = env
    pos = np.random.default_rng(5).random((1200, 3)) * 1.0e9
    rows = np.diag([1.0e9, 1.0e9, 1.0e9])
    code, m, ei, _ = noalloc_build(env, pos, rows, 1e-3, 10)
    assert code == 1, lib.nlb_last_error().decode()
    assert "bins" in lib.nlb_last_error().decode()
    assert bool((ei == -7).all())
    # a grid of a few hundred thousand bins: within the per-axis limit, above
    # the scratch capacity
    pos = np.random.default_rng(6).random((1200, 3)) * 200.0
    code, m, _, _ = noalloc_build(env, pos, np.diag([200.0] * 3), 2.5, 10)
    assert code == 1 and "fixed capacity" in lib.nlb_last_error().decode()


def test_noalloc_allocates_no_device_memory(env):
    """The defining property: once the caller's buffers exist, a series of
    calls leaves the device's free memory unchanged (no cudaMalloc, no
    growing workspace)."""
    torch, nl, lib = env
    from neighborlist_rs import workloads as W

    pos, rows = W.cluster_liquid(n_clusters=139, box=23.2, seed=44)
    d_pos = torch.from_numpy(np.ascontiguousarray(pos)).cuda()
    cap = 200_000
    ei = torch.empty((2, cap), dtype=torch.int64, device="cuda")
    sh = torch.empty((cap, 3), dtype=torch.int32, device="cuda")
    h9 = np.ascontiguousarray(rows.T.reshape(9))
    h = h9.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    pbc = (ctypes.c_uint8 * 3)(1, 1, 1)
    m = ctypes.c_int64(-1)
    stream = torch.cuda.current_stream().cuda_stream

    def call():
        code = lib.nlb_build_noalloc(d_pos.data_ptr(), pos.shape[0], 6.0, h, pbc,
                                     ei.data_ptr(), sh.data_ptr(), cap, ctypes.byref(m), stream)
        assert code == 0, lib.nlb_last_error().decode()

    call()  # the first call on the device looks up the scratch address
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(20):
        call()
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert m.value > 0
