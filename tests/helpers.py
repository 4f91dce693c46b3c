"""Shared helpers for the parity tests."""

import numpy as np


def assert_same(got: dict, ref, what=""):
    """Bit-exact comparison of a product result dict with an oracle tuple
    (edge_index int64 (2,M), shift int32 (M,3)): same edges, same order."""
    ei, sh = ref
    g_ei, g_sh = got["edge_index"], got["shift"]
    assert g_ei.dtype == np.int64 and g_sh.dtype == np.int32, what
    assert g_ei.shape == ei.shape, f"{what}: edge_index shape {g_ei.shape} != {ei.shape}"
    assert g_sh.shape == sh.shape, f"{what}: shift shape {g_sh.shape} != {sh.shape}"
    if not np.array_equal(g_ei, ei) or not np.array_equal(g_sh, sh):
        bad = np.nonzero((g_ei != ei).any(axis=0) | (g_sh != sh).any(axis=1))[0]
        k = int(bad[0])
        raise AssertionError(
            f"{what}: {len(bad)} of {ei.shape[1]} edges differ; first at {k}: "
            f"got ({g_ei[0, k]}, {g_ei[1, k]}, {g_sh[k].tolist()}) "
            f"want ({ei[0, k]}, {ei[1, k]}, {sh[k].tolist()})")


def edge_set(ei, sh):
    return set(zip(ei[0].tolist(), ei[1].tolist(), map(tuple, sh.tolist())))
