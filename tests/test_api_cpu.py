"""Host-side behaviour of the drop-in module that needs no GPU: the C-ABI
library loads and exports every declared symbol, and the Python surface
raises the reference's errors (src/python_api.rs, tests/test_validation.py,
tests/test_api_extensions.py) before any device work."""

import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def nl():
    import neighborlist_rs

    return neighborlist_rs


def declared_functions():
    with open(os.path.join(ROOT, "include", "neighborlist_b200.h")) as f:
        text = f.read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nlb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(nl):
    lib = ctypes.CDLL(nl.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 16
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_version(nl):
    assert "sm_100a" in nl.version()


def test_cutoff_validation(nl):
    pos = np.random.rand(10, 3)
    for bad in (-1.0, 0.0, float("nan"), float("inf")):
        with pytest.raises(ValueError, match="Cutoff must be positive and finite"):
            nl.build_neighborlists(None, pos, bad)
    with pytest.raises(ValueError, match="Cutoff must be positive and finite"):
        nl.build_neighborlists_batch(pos, np.zeros(10, np.int32), None, -2.0)
    with pytest.raises(ValueError, match="All cutoffs must be positive and finite"):
        nl.build_neighborlists_multi(None, pos, [1.0, -2.0, 3.0])
    with pytest.raises(ValueError, match="All cutoffs must be positive and finite"):
        nl.build_neighborlists_batch_multi(pos, np.zeros(10, np.int32), None, [1.0, float("nan")])


def test_position_shape_validation(nl):
    with pytest.raises(ValueError, match=r"Positions must be \(N, 3\)"):
        nl.build_neighborlists(None, np.random.rand(10, 4), 5.0)
    with pytest.raises(ValueError, match=r"Positions must be \(N, 3\)"):
        nl.build_neighborlists_batch(np.random.rand(10, 2), np.zeros(10, np.int32), None, 5.0)
    with pytest.raises(ValueError, match=r"Positions must be \(N, 3\)"):
        nl.build_neighborlists_batch_multi(np.random.rand(10, 2), np.zeros(10, np.int32), None,
                                           [5.0])
    with pytest.raises(TypeError):
        nl.build_neighborlists(None, [[0.0, 0.0, 0.0]], 5.0)


def test_batch_validation(nl):
    pos = np.random.rand(10, 3)
    b = np.array([0, 0, 1, 1, 0, 0, 1, 1, 2, 2], np.int32)
    with pytest.raises(ValueError, match=r"Batch IDs must be monotonic \(non-decreasing\)"):
        nl.build_neighborlists_batch(pos, b, None, 5.0)
    with pytest.raises(ValueError, match="positions and batch must have the same length"):
        nl.build_neighborlists_batch(pos, np.zeros(9, np.int32), None, 5.0)
    with pytest.raises(ValueError, match="Expected at least 2 cells, but got 1"):
        nl.build_neighborlists_batch(np.random.rand(4, 3), np.array([0, 0, 1, 1], np.int32),
                                     cells=np.zeros((1, 3, 3)), cutoff=1.0)
    with pytest.raises(ValueError, match="Length of labels must match length of cutoffs"):
        nl.build_neighborlists_batch_multi(pos, np.zeros(10, np.int32), cutoffs=[1.0, 2.0],
                                           labels=["one"])


def test_empty_inputs_need_no_device(nl):
    pos = np.zeros((0, 3))
    r = nl.build_neighborlists(None, pos, 1.0)
    assert r["edge_index"].shape == (2, 0) and r["shift"].shape == (0, 3)
    assert r["edge_index"].dtype == np.int64 and r["shift"].dtype == np.int32
    m = nl.build_neighborlists_multi(None, pos, [1.0, 2.0])
    assert len(m) == 2 and m[0]["edge_index"].shape == (2, 0)
    assert nl.build_neighborlists_multi(None, np.random.rand(5, 3), []) == {}
    b = nl.build_neighborlists_batch(pos, np.zeros(0, np.int32), cutoff=1.0)
    assert b["edge_index"].shape == (2, 0)
    assert nl.build_neighborlists_batch_multi(np.random.rand(5, 3), np.zeros(5, np.int32),
                                              cutoffs=[]) == {}
    assert nl.build_neighborlists_batch_multi(pos, np.zeros(0, np.int32), cutoffs=[1.0]) == {}


def test_pycell(nl):
    c = nl.PyCell([[10.0, 0, 0], [0, 10.0, 0], [0, 0, 10.0]])
    assert c.wrap([15.0, -2.0, 8.0]) == pytest.approx([5.0, 8.0, 8.0])
    c2 = nl.PyCell([[10.0, 0, 0], [0, 10.0, 0], [0, 0, 10.0]], [True, False, False])
    assert c2.wrap([15.0, 15.0, 15.0]) == pytest.approx([5.0, 15.0, 15.0])
    with pytest.raises(ValueError, match="Cell matrix is not invertible"):
        nl.PyCell([[0, 0, 0], [0, 0, 0], [0, 0, 0]])
    with pytest.raises(ValueError, match="Cell matrix must be 3x3"):
        nl.PyCell([[1.0, 0.0], [0.0, 1.0]])
    r = repr(nl.PyCell([[10, 0, 0], [0, 10, 0], [0, 0, 10]], pbc=[True, False, True]))
    assert r == "PyCell(h=[[10, 0, 0], [0, 10, 0], [0, 0, 10]], pbc=[true, false, true])"


class FakeAtoms:
    """The three methods the reference calls on an ASE Atoms object."""

    def __init__(self, positions, cell, pbc):
        self._p = np.asarray(positions, np.float64)
        self._c = np.asarray(cell, np.float64)
        self._pbc = np.asarray(pbc, bool)

    def get_positions(self):
        return self._p.copy()

    def get_cell(self):
        return self._c

    def get_pbc(self):
        return self._pbc


def test_pycell_from_ase_transposes(nl):
    rows = np.array([[3.0, 0.0, 0.0], [1.0, 3.0, 0.0], [0.5, 0.2, 3.0]])
    c = nl.PyCell.from_ase(FakeAtoms(np.zeros((1, 3)), rows, [True, True, False]))
    assert np.array_equal(c._h9.reshape(3, 3), rows.T)
    assert "pbc=[true, true, false]" in repr(c)


def test_thresholds(nl):
    bf, par, st = (nl.get_brute_force_threshold(), nl.get_parallel_threshold(),
                   nl.get_stack_threshold())
    assert (bf, par, st) == (1000, 300, 1000)
    nl.set_brute_force_threshold(1234)
    nl.set_parallel_threshold(567)
    nl.set_stack_threshold(890)
    assert (nl.get_brute_force_threshold(), nl.get_parallel_threshold(),
            nl.get_stack_threshold()) == (1234, 567, 890)
    nl.set_stack_threshold(5000)
    assert nl.get_stack_threshold() == 1024  # clamped like src/config.rs:36-39
    with pytest.raises(OverflowError):
        nl.set_brute_force_threshold(-1)
    nl.set_brute_force_threshold(bf)
    nl.set_parallel_threshold(par)
    nl.set_stack_threshold(st)


def test_threads_and_logging(nl):
    assert nl.get_num_threads() > 0
    nl.set_num_threads(nl.get_num_threads() + 1)
    assert nl.get_num_threads() > 0
    nl.init_logging("debug")
    nl.init_logging(None)


def test_batch_launch_shapes_and_pinning(nl):
    """The batched kernels' launch-shape table and the pin / reset calls are
    host-side: every shape is a valid launch, pinning checks its range."""
    n = nl.set_batch_shape(None)
    assert n >= 2
    seen = set()
    for i in range(n):
        s = nl.batch_shape_info(i)
        assert s["small_threads"] in (64, 128, 256, 512)
        assert s["large_threads"] in (256, 512)
        assert s["chunk"] in (128, 256, 512) and s["large_atoms"] >= 256
        seen.add(tuple(s.values()))
    assert len(seen) == n, "duplicate shapes"
    assert nl.batch_shape_info(0) == {"small_threads": 256, "large_threads": 512, "chunk": 256,
                                      "large_atoms": 512}
    try:
        assert nl.set_batch_shape(n - 1) == n
    finally:
        nl.set_batch_shape(None)
    for bad in (n, -2):
        with pytest.raises(ValueError):
            nl.set_batch_shape(bad)
        with pytest.raises(ValueError):
            nl.batch_shape_info(bad)
    nl.batch_tuner_reset()
    assert nl.batch_tuner_state() == []


def test_pinned_stats_counters(nl):
    st = nl.pinned_stats()
    assert set(st) == {"host_alloc_calls", "host_alloc_us", "host_alloc_bytes", "host_free_calls",
                       "host_free_us", "cache_hits", "cached_bytes"}
    assert all(isinstance(v, int) and v >= 0 for v in st.values())


@pytest.mark.parametrize("offsets", [False, True])
def test_batch_validation_with_and_without_offsets(nl, offsets):
    """The batched calls raise the reference's errors before any device work
    (src/python_api.rs:315-423, src/batch.rs:18-46), with or without the
    per-system offset table."""
    pos = np.zeros((4, 3))
    with pytest.raises(ValueError, match="positions and batch must have the same length"):
        nl.build_neighborlists_batch(pos, np.zeros(3, np.int32), cutoff=5.0,
                                     return_offsets=offsets)
    with pytest.raises(ValueError, match="Batch IDs must be monotonic"):
        nl.build_neighborlists_batch(pos, np.array([0, 1, 0, 1], np.int32), cutoff=5.0,
                                     return_offsets=offsets)
    with pytest.raises(ValueError, match="Expected at least 2 cells, but got 1"):
        nl.build_neighborlists_batch(pos, np.array([0, 0, 1, 1], np.int32),
                                     cells=np.zeros((1, 3, 3)), cutoff=5.0,
                                     return_offsets=offsets)
    with pytest.raises(ValueError, match="All cutoffs must be positive and finite"):
        nl.build_neighborlists_batch_multi(pos, np.zeros(4, np.int32), cutoffs=[5.0, -1.0],
                                           return_offsets=offsets)
    r = nl.build_neighborlists_batch(np.zeros((0, 3)), np.zeros(0, np.int32), cutoff=5.0,
                                     return_offsets=offsets)
    assert r["edge_index"].shape == (2, 0)
    assert ("system_offsets" in r) == offsets


def test_device_block_release_survives_module_teardown(nl, monkeypatch):
    """A zero-copy device result whose last view dies after the module's
    globals are gone (interpreter shutdown) still calls the library's free
    function held by its class, and never raises."""
    calls = []

    class FakeFree:
        def __call__(self, ptr, stream):
            calls.append((ptr, stream))
            return 0

    monkeypatch.setattr(nl._DeviceBlock, "_free", FakeFree())
    monkeypatch.setattr(nl, "_lib", None)
    b = nl._DeviceBlock(0x1000, (2, 3), "<i8", 7)
    assert b.__cuda_array_interface__["shape"] == (2, 3)
    del b
    assert calls == [(0x1000, 7)]

    class Raising:
        def __call__(self, ptr, stream):
            raise RuntimeError("no CUDA context")

    monkeypatch.setattr(nl._DeviceBlock, "_free", Raising())
    b = nl._DeviceBlock(0x2000, (1,), "<i4", 0)
    del b  # swallowed, as at interpreter shutdown
