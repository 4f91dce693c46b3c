"""neighborlist_rs -- B200 drop-in for the Python module of solccp/neighborlist-rs.

Same functions, signatures, defaults, dict layout, dtypes and ValueError
messages as the reference's PyO3 module (src/python_api.rs:15-626,
neighborlist_rs.pyi); the search itself runs in the CUDA library
``_lib/libnlb200.so`` (C ABI: include/neighborlist_b200.h).  There is no CPU
fallback: importing this module fails if the library is missing, and every
build call fails if no CUDA device is available.

Results are numpy arrays that view pinned host memory owned by the library;
the memory is returned to the library when the arrays are garbage-collected.
"""

from __future__ import annotations

import ctypes
import math
import os

import numpy as np

__all__ = [
    "PyCell", "build_neighborlists", "build_from_ase", "build_neighborlists_multi",
    "build_multi_from_ase", "build_neighborlists_batch", "build_neighborlists_batch_multi",
    "get_num_threads", "set_num_threads", "init_logging", "get_brute_force_threshold",
    "set_brute_force_threshold", "get_parallel_threshold", "set_parallel_threshold",
    "get_stack_threshold", "set_stack_threshold",
]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libnlb200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"neighborlist_rs: CUDA library not found at {LIB_PATH}; build it with "
        "`python neighborlist-rs_b200/build.py` (nvcc, sm_100a)")


class _Result(ctypes.Structure):
    _fields_ = [("n_edges", ctypes.c_int64),
                ("edge_index", ctypes.c_void_p),
                ("shift", ctypes.c_void_p)]


_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)

_lib = ctypes.CDLL(LIB_PATH)
_lib.nlb_last_error.restype = ctypes.c_char_p
_lib.nlb_version.restype = ctypes.c_char_p
_lib.nlb_build.argtypes = [_dp, ctypes.c_int64, ctypes.c_double, _dp, _u8p, ctypes.c_int,
                           ctypes.POINTER(_Result)]
_lib.nlb_build_multi.argtypes = [_dp, ctypes.c_int64, _dp, ctypes.c_int32, _dp, _u8p,
                                 ctypes.c_int, ctypes.POINTER(_Result)]
_lib.nlb_build_batch.argtypes = [_dp, ctypes.c_int64, _i32p, ctypes.c_int64, ctypes.c_double,
                                 _dp, _u8p, _u8p, ctypes.c_int64, ctypes.c_int,
                                 ctypes.POINTER(_Result)]
_lib.nlb_build_batch_multi.argtypes = [_dp, ctypes.c_int64, _i32p, ctypes.c_int64, _dp,
                                       ctypes.c_int32, _dp, _u8p, _u8p, ctypes.c_int64,
                                       ctypes.c_int, ctypes.POINTER(_Result)]
_i64p = ctypes.POINTER(ctypes.c_int64)
_lib.nlb_build_batch_ex.argtypes = [_dp, ctypes.c_int64, _i32p, ctypes.c_int64, _dp,
                                    ctypes.c_int32, _dp, _u8p, _u8p, ctypes.c_int64,
                                    ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Result), _i64p]
_lib.nlb_result_free.argtypes = [ctypes.POINTER(_Result)]
_lib.nlb_host_free.argtypes = [ctypes.c_void_p]
_lib.nlb_cell_check.argtypes = [_dp]
_lib.nlb_cell_wrap.argtypes = [_dp, _u8p, _dp, _dp]
for _name in ("brute_force", "parallel", "stack"):
    getattr(_lib, f"nlb_get_{_name}_threshold").restype = ctypes.c_size_t
    getattr(_lib, f"nlb_set_{_name}_threshold").argtypes = [ctypes.c_size_t]

_NLB_ERR_VALUE = 1
_LOG_LEVEL = None


def _check(code: int) -> None:
    if code == 0:
        return
    msg = _lib.nlb_last_error().decode()
    if code == _NLB_ERR_VALUE:
        raise ValueError(msg)
    raise RuntimeError(f"neighborlist_rs (CUDA): {msg}")


class _HostBlock:
    """Owner of one library-allocated host block, exposed to numpy through
    the array interface (the array's base); the block is returned to the
    library when the last view is gone.  (A ctypes array type per length
    would cost ~20 us per result and grow ctypes' type cache.)"""

    __slots__ = ("__array_interface__", "_ptr")

    def __init__(self, ptr, count, typestr):
        self._ptr = ptr
        self.__array_interface__ = {"data": (ptr, False), "shape": (count,),
                                    "typestr": typestr, "version": 3}

    def __del__(self):
        try:
            _lib.nlb_host_free(ctypes.c_void_p(self._ptr))
        except Exception:  # interpreter shutdown
            pass


def _arr(ptr, count, dtype):
    """numpy view of `count` library-owned elements; freed with the array."""
    if count == 0:
        _lib.nlb_host_free(ptr)
        return np.zeros(0, dtype=dtype)
    return np.asarray(_HostBlock(ptr, count, np.dtype(dtype).str))


def _to_dict(r: _Result) -> dict:
    m = int(r.n_edges)
    ei = _arr(r.edge_index, 2 * m, np.int64).reshape(2, m)
    sh = _arr(r.shift, 3 * m, np.int32).reshape(m, 3)
    return {"edge_index": ei, "shift": sh}


def _empty() -> dict:
    return {"edge_index": np.zeros((2, 0), np.int64), "shift": np.zeros((0, 3), np.int32)}


def _positions(positions) -> np.ndarray:
    # PyReadonlyArray2<f64> (src/python_api.rs:116-137): a 2-D float64 array,
    # copied when not C-contiguous.
    if not isinstance(positions, np.ndarray) or positions.ndim != 2 or positions.dtype != np.float64:
        raise TypeError("positions must be a 2-D numpy array of float64")
    if positions.shape[1] != 3:
        raise ValueError("Positions must be (N, 3)")
    return np.ascontiguousarray(positions)


def _batch_ids(batch) -> np.ndarray:
    if not isinstance(batch, np.ndarray) or batch.ndim != 1 or batch.dtype != np.int32:
        raise TypeError("batch must be a 1-D numpy array of int32")
    return np.ascontiguousarray(batch)


def _check_cutoff(cutoff) -> float:
    c = float(cutoff)
    if not math.isfinite(c) or c <= 0.0:
        raise ValueError("Cutoff must be positive and finite")
    return c


def _cutoff_list(cutoffs) -> list:
    if isinstance(cutoffs, (str, bytes)):
        raise TypeError("cutoffs must be a sequence of floats")
    return [float(c) for c in cutoffs]


def _rust_float(x: float) -> str:
    """Rust's Display for f64 (shortest round-trip digits, never an exponent)."""
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    return np.format_float_positional(x, trim="-")


class PyCell:
    """Simulation cell (src/python_api.rs:15-99).

    ``h`` is a 3x3 nested list whose COLUMNS are the lattice vectors (the
    reference feeds it to ``Matrix3::new`` row by row); ``pbc`` defaults to
    all periodic.  ``from_ase`` transposes an ASE cell (rows = vectors).
    """

    __slots__ = ("_h9", "_pbc", "_args")

    def __init__(self, h, pbc=None):
        rows = [list(r) for r in h] if not isinstance(h, (str, bytes)) else []
        if len(rows) != 3 or any(len(r) != 3 for r in rows):
            raise ValueError("Cell matrix must be 3x3")
        self._h9 = np.ascontiguousarray(np.array(rows, dtype=np.float64).reshape(9))
        if pbc is None:
            pbc = (True, True, True)
        p = [bool(x) for x in pbc]
        if len(p) != 3:
            raise ValueError("pbc must have 3 entries")
        self._pbc = np.ascontiguousarray(np.array(p, dtype=np.uint8))
        # ctypes pointers made once (each data_as costs ~2 us per call)
        self._args = (self._h9.ctypes.data_as(_dp), self._pbc.ctypes.data_as(_u8p))
        _check(_lib.nlb_cell_check(self._args[0]))

    def wrap(self, pos):
        p = np.ascontiguousarray(np.array([float(x) for x in pos], dtype=np.float64))
        if p.shape != (3,):
            raise ValueError("pos must have 3 entries")
        out = np.zeros(3, np.float64)
        _check(_lib.nlb_cell_wrap(self._args[0], self._args[1],
                                  p.ctypes.data_as(_dp), out.ctypes.data_as(_dp)))
        return [float(v) for v in out]

    def __repr__(self):
        h = [_rust_float(float(v)) for v in self._h9]
        pb = ["true" if v else "false" for v in self._pbc]
        return (f"PyCell(h=[[{h[0]}, {h[1]}, {h[2]}], [{h[3]}, {h[4]}, {h[5]}], "
                f"[{h[6]}, {h[7]}, {h[8]}]], pbc=[{pb[0]}, {pb[1]}, {pb[2]}])")

    @staticmethod
    def from_ase(atoms) -> "PyCell":
        c = np.asarray(atoms.get_cell().__array__(), dtype=np.float64)
        if c.shape != (3, 3):
            raise ValueError("Cell must be 3x3")
        pbc = [bool(x) for x in atoms.get_pbc()]
        return PyCell(c.T.tolist(), pbc)


def _cell_args(cell):
    if cell is None:
        return None, None
    if not isinstance(cell, PyCell):
        raise TypeError("cell must be a PyCell or None")
    return cell._args


def build_neighborlists(cell, positions, cutoff, parallel=True):
    """src/python_api.rs:139-186.  Half list (i < j, or i == j with a non-zero
    image); returns {"edge_index": int64 (2, M), "shift": int32 (M, 3)}."""
    c = _check_cutoff(cutoff)
    pos = _positions(positions)
    n = pos.shape[0]
    if n == 0:
        return _empty()
    h, pb = _cell_args(cell)
    r = _Result()
    _check(_lib.nlb_build(pos.ctypes.data_as(_dp), n, c, h, pb, int(bool(parallel)),
                          ctypes.byref(r)))
    return _to_dict(r)


def _ase_inputs(atoms):
    # src/python_api.rs:188-209
    positions = atoms.get_positions()
    pbc = [bool(x) for x in atoms.get_pbc()]
    cell = PyCell.from_ase(atoms) if any(pbc) else None
    return positions, cell


def build_from_ase(atoms, cutoff):
    """src/python_api.rs:211-220."""
    positions, cell = _ase_inputs(atoms)
    return build_neighborlists(cell, positions, cutoff, True)


def _multi_dict(results, labels):
    out = {}
    for k, r in enumerate(results):
        out[labels[k] if labels is not None else k] = r
    return out


def build_neighborlists_multi(cell, positions, cutoffs, labels=None, disjoint=False):
    """src/python_api.rs:235-309.  One traversal for all cutoffs; returns a
    dict keyed by cutoff index (or label)."""
    pos = _positions(positions)
    cs = _cutoff_list(cutoffs)
    if not cs:
        return {}
    if any(not math.isfinite(c) or c <= 0.0 for c in cs):
        raise ValueError("All cutoffs must be positive and finite")
    if labels is not None:
        labels = [str(x) for x in labels]
        if len(labels) != len(cs):
            raise ValueError("Length of labels must match length of cutoffs")
    n = pos.shape[0]
    if n == 0:
        return _multi_dict([_empty() for _ in cs], labels)
    h, pb = _cell_args(cell)
    k = len(cs)
    carr = np.ascontiguousarray(np.array(cs, dtype=np.float64))
    outs = (_Result * k)()
    _check(_lib.nlb_build_multi(pos.ctypes.data_as(_dp), n, carr.ctypes.data_as(_dp), k, h, pb,
                                int(bool(disjoint)), outs))
    return _multi_dict([_to_dict(outs[q]) for q in range(k)], labels)


def build_multi_from_ase(atoms, cutoffs, labels=None, disjoint=False):
    """src/python_api.rs:222-233."""
    positions, cell = _ase_inputs(atoms)
    return build_neighborlists_multi(cell, positions, cutoffs, labels, disjoint)


def _batch_cells(cells, batch, need_count=False):
    """The (B,3,3) cells -> C arrays (src/python_api.rs:353-407): a zero
    matrix means isolated (auto-box); any other cell is transposed from ASE
    rows and gets pbc (T, T, T) (pbcs None: the library's default).  Every
    given cell is passed on; the library splits the systems and reports
    "Batch IDs must be monotonic (non-decreasing)" and "Expected at least {n}
    cells, but got {m}".  The system count is computed here only when the
    caller needs it (it is then also where a non-monotonic batch is
    reported)."""
    n_sys = -1
    if need_count:
        b1, b0 = batch[1:], batch[:-1]
        if (b1 < b0).any():
            raise ValueError("Batch IDs must be monotonic (non-decreasing)")
        n_sys = 1 + int(np.count_nonzero(b1 != b0))
    if cells is None:
        return n_sys, None, None, None, 0
    if not isinstance(cells, np.ndarray) or cells.ndim != 3 or cells.dtype != np.float64:
        raise TypeError("cells must be a 3-D numpy array of float64")
    if cells.shape[1:] != (3, 3):
        raise ValueError("cells must have shape (B, 3, 3)")
    nc = cells.shape[0]
    h9 = np.empty((nc, 9), np.float64)
    has = np.empty(nc, np.uint8)
    _lib.nlb_batch_cells(np.ascontiguousarray(cells).ctypes.data_as(_dp), nc,
                         h9.ctypes.data_as(_dp), has.ctypes.data_as(_u8p))
    return n_sys, h9, None, has, nc


_lib.nlb_batch_cells.argtypes = [_dp, ctypes.c_int64, _dp, _u8p]
_lib.nlb_batch_cells.restype = None


def build_neighborlists_batch(positions, batch, cells=None, cutoff=5.0, parallel=True, *,
                              return_offsets=False):
    """src/python_api.rs:315-423.  Systems split wherever the batch id
    changes; indices are global; systems concatenated in order.

    ``return_offsets=True`` (an addition) also returns ``system_offsets``,
    int64 (n_systems + 1,): system i's edges are [off[i], off[i + 1])."""
    c = _check_cutoff(cutoff)
    pos = _positions(positions)
    b = _batch_ids(batch)
    n = pos.shape[0]
    if b.shape[0] != n:
        raise ValueError("positions and batch must have the same length")
    if n == 0:
        res = _empty()
        if return_offsets:
            res["system_offsets"] = np.zeros(1, np.int64)
        return res
    n_sys, h9, pbcs, has, nc = _batch_cells(cells, b, need_count=return_offsets)
    r = _Result()
    cells_args = (h9.ctypes.data_as(_dp) if h9 is not None else None,
                  pbcs.ctypes.data_as(_u8p) if pbcs is not None else None,
                  has.ctypes.data_as(_u8p) if has is not None else None, nc)
    if not return_offsets:
        _check(_lib.nlb_build_batch(pos.ctypes.data_as(_dp), n, b.ctypes.data_as(_i32p), n, c,
                                    *cells_args, int(bool(parallel)), ctypes.byref(r)))
        return _to_dict(r)
    carr = np.array([c], dtype=np.float64)
    offs = np.zeros(n_sys + 1, np.int64)
    _check(_lib.nlb_build_batch_ex(pos.ctypes.data_as(_dp), n, b.ctypes.data_as(_i32p), n,
                                   carr.ctypes.data_as(_dp), 1, *cells_args, 0, 0,
                                   ctypes.byref(r), offs.ctypes.data_as(_i64p)))
    res = _to_dict(r)
    res["system_offsets"] = offs
    return res


def build_neighborlists_batch_multi(positions, batch, cells=None, cutoffs=(5.0,), labels=None,
                                    disjoint=False, *, return_offsets=False):
    """src/python_api.rs:425-546.  ``return_offsets=True`` (an addition) adds
    ``system_offsets`` to each list, as in build_neighborlists_batch."""
    pos = _positions(positions)
    b = _batch_ids(batch)
    n = pos.shape[0]
    if b.shape[0] != n:
        raise ValueError("positions and batch must have the same length")
    cs = _cutoff_list(cutoffs)
    if n == 0 or not cs:
        return {}
    if any(not math.isfinite(c) or c <= 0.0 for c in cs):
        raise ValueError("All cutoffs must be positive and finite")
    if labels is not None:
        labels = [str(x) for x in labels]
        if len(labels) != len(cs):
            raise ValueError("Length of labels must match length of cutoffs")
    n_sys, h9, pbcs, has, nc = _batch_cells(cells, b, need_count=return_offsets)
    k = len(cs)
    carr = np.ascontiguousarray(np.array(cs, dtype=np.float64))
    outs = (_Result * k)()
    cells_args = (h9.ctypes.data_as(_dp) if h9 is not None else None,
                  pbcs.ctypes.data_as(_u8p) if pbcs is not None else None,
                  has.ctypes.data_as(_u8p) if has is not None else None, nc)
    if not return_offsets:
        _check(_lib.nlb_build_batch_multi(
            pos.ctypes.data_as(_dp), n, b.ctypes.data_as(_i32p), n, carr.ctypes.data_as(_dp), k,
            *cells_args, int(bool(disjoint)), outs))
        return _multi_dict([_to_dict(outs[q]) for q in range(k)], labels)
    offs = np.zeros((k, n_sys + 1), np.int64)
    _check(_lib.nlb_build_batch_ex(
        pos.ctypes.data_as(_dp), n, b.ctypes.data_as(_i32p), n, carr.ctypes.data_as(_dp), k,
        *cells_args, int(bool(disjoint)), 1, outs, offs.ctypes.data_as(_i64p)))
    lists = []
    for q in range(k):
        d = _to_dict(outs[q])
        d["system_offsets"] = offs[q]
        lists.append(d)
    return _multi_dict(lists, labels)


# ---------------------------------------------------------------- configuration

def get_num_threads() -> int:
    """The reference reports its rayon pool size; the device path has no host
    thread pool, so this reports the host's logical CPU count (rayon's default)."""
    return os.cpu_count() or 1


def set_num_threads(n) -> None:
    """Accepted for API parity (src/python_api.rs:553-561); no effect on the GPU path."""
    int(n)


def init_logging(level=None) -> None:
    """src/python_api.rs:593-605.  Records the level; the library reports
    per-phase timings through bench.py / ncu rather than tracing spans."""
    global _LOG_LEVEL
    _LOG_LEVEL = level if level is not None else "info"


def _usize(val) -> int:
    v = int(val)
    if v < 0:
        raise OverflowError("can't convert negative int to unsigned")
    return v


def get_brute_force_threshold() -> int:
    return int(_lib.nlb_get_brute_force_threshold())


def set_brute_force_threshold(val) -> None:
    _lib.nlb_set_brute_force_threshold(_usize(val))


def get_parallel_threshold() -> int:
    return int(_lib.nlb_get_parallel_threshold())


def set_parallel_threshold(val) -> None:
    _lib.nlb_set_parallel_threshold(_usize(val))


def get_stack_threshold() -> int:
    return int(_lib.nlb_get_stack_threshold())


def set_stack_threshold(val) -> None:
    _lib.nlb_set_stack_threshold(_usize(val))


def version() -> str:
    return _lib.nlb_version().decode()


# ---------------------------------------------------------------- device-resident path

class _DevResult(ctypes.Structure):
    _fields_ = [("n_edges", ctypes.c_int64),
                ("edge_index", ctypes.c_void_p),
                ("shift", ctypes.c_void_p)]


_lib.nlb_build_device.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, _dp, _u8p,
                                  ctypes.POINTER(_DevResult)]
_lib.nlb_set_stream.argtypes = [ctypes.c_void_p]
_lib.nlb_kernel_launches.restype = ctypes.c_int64
_lib.nlb_profile.argtypes = [ctypes.c_int]
_lib.nlb_profile_read.argtypes = [_dp]
_lib.nlb_profile_read.restype = ctypes.c_int64
_lib.nlb_profile_host.argtypes = [_dp]
_lib.nlb_profile_host.restype = ctypes.c_int64
_lib.nlb_batch_shape.argtypes = [ctypes.c_int32]
_lib.nlb_batch_shape.restype = ctypes.c_int32
_lib.nlb_batch_shape_info.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_int32)]
_lib.nlb_batch_shape_info.restype = ctypes.c_int32
_lib.nlb_batch_tuner_state.argtypes = [ctypes.POINTER(ctypes.c_int64), ctypes.c_int32]
_lib.nlb_batch_tuner_state.restype = ctypes.c_int32
_lib.nlb_batch_tuner_reset.argtypes = []
_lib.nlb_batch_tuner_reset.restype = None


_lib.nlb_pinned_stats.argtypes = [ctypes.POINTER(ctypes.c_int64)]
_lib.nlb_pinned_stats.restype = None
_PINNED_STATS = ("host_alloc_calls", "host_alloc_us", "host_alloc_bytes", "host_free_calls",
                 "host_free_us", "cache_hits", "cached_bytes")


def pinned_stats() -> dict:
    """Counters of the pinned host pool behind every host result."""
    buf = (ctypes.c_int64 * len(_PINNED_STATS))()
    _lib.nlb_pinned_stats(buf)
    return dict(zip(_PINNED_STATS, (int(x) for x in buf)))


_lib.nlb_single_pipeline.argtypes = [ctypes.c_int32]
_lib.nlb_single_pipeline.restype = ctypes.c_int32
_lib.nlb_last_single_pipeline.restype = ctypes.c_int32


def last_single_pipeline() -> int:
    """Pipeline of this thread's last single-cutoff cell-list build: 0 = one
    launch, 1 = three launches, -1 = none yet."""
    return int(_lib.nlb_last_single_pipeline())


def set_single_pipeline(mode: int | None) -> int:
    """Single-system pipeline: 0 (or None) = automatic (one launch for count,
    offsets and emit on sparse grids), 1 = always the three-launch pair-task
    pipeline.  Identical results either way; returns the previous mode."""
    r = int(_lib.nlb_single_pipeline(0 if mode is None else int(mode)))
    if r < 0:
        raise ValueError(f"no single-system pipeline mode {mode}")
    return r


def set_batch_shape(shape: int | None) -> int:
    """Pin launch shape `shape` of the batched kernels (None: tune per kind of
    batch, the default).  Returns the number of shapes."""
    r = int(_lib.nlb_batch_shape(-1 if shape is None else int(shape)))
    if r < 0:
        raise ValueError(f"no batch launch shape {shape}")
    return r


def batch_shape_info(shape: int) -> dict:
    """{small_threads, large_threads, chunk, large_atoms} of launch shape `shape`."""
    out = (ctypes.c_int32 * 4)()
    if _lib.nlb_batch_shape_info(int(shape), out) != 0:
        raise ValueError(f"no batch launch shape {shape}")
    return dict(zip(("small_threads", "large_threads", "chunk", "large_atoms"), list(out)))


def batch_tuner_state() -> list:
    """One dict per kind of batch seen: its key, the chosen shape (-1: not
    decided yet) and the number of candidate shapes it was timed in."""
    n = int(_lib.nlb_batch_tuner_state(None, 0))
    buf = np.zeros(8 * max(n, 1), np.int64)
    n = min(n, int(_lib.nlb_batch_tuner_state(buf.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), n)))
    keys = ("device", "cutoffs", "systems_log2", "max_atoms_log2", "mean_atoms_log2",
            "cutoff_bucket", "shape", "candidates")
    return [dict(zip(keys, (int(v) for v in buf[8 * i:8 * i + 8]))) for i in range(n)]


def batch_tuner_reset() -> None:
    """Forget every tuned kind of batch (the next calls tune again)."""
    _lib.nlb_batch_tuner_reset()


def set_stream(stream_handle: int | None) -> None:
    """Launch the calling thread's subsequent builds on this cudaStream_t
    (e.g. ``torch.cuda.current_stream().cuda_stream``); None = library stream."""
    _lib.nlb_set_stream(ctypes.c_void_p(stream_handle) if stream_handle else None)


def kernel_launches() -> int:
    return int(_lib.nlb_kernel_launches())


def profile(enable: bool) -> None:
    _lib.nlb_profile(int(bool(enable)))


def profile_host_read():
    """(calls, {upload, device, results, total} host ms of profiled batched builds)."""
    ms = np.zeros(4, np.float64)
    calls = int(_lib.nlb_profile_host(ms.ctypes.data_as(_dp)))
    return calls, dict(zip(("upload", "device", "results", "total"), ms.tolist()))


def profile_read():
    """(calls, {build, count, scan, emit} ms accumulated with CUDA events)."""
    ms = np.zeros(4, np.float64)
    calls = int(_lib.nlb_profile_read(ms.ctypes.data_as(_dp)))
    return calls, dict(zip(("build", "count", "scan", "emit"), ms.tolist()))


def build_device_raw(cell, positions_ptr: int, n_atoms: int, cutoff: float):
    """Device-resident build: positions_ptr is a device pointer to n x 3
    float64.  Returns (n_edges, edge_index_ptr, shift_ptr): device pointers
    into the calling thread's workspace, valid until its next build."""
    c = _check_cutoff(cutoff)
    h, pb = _cell_args(cell)
    r = _DevResult()
    _check(_lib.nlb_build_device(ctypes.c_void_p(positions_ptr), int(n_atoms), c, h, pb,
                                 ctypes.byref(r)))
    return int(r.n_edges), r.edge_index, r.shift


_lib.nlb_build_device_owned.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, _dp,
                                       _u8p, ctypes.POINTER(_DevResult)]
_lib.nlb_device_free.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
_lib.nlb_device_blocks.argtypes = [ctypes.POINTER(ctypes.c_int64)]


class _DeviceBlock:
    """Owner of one device block handed over by nlb_build_device_owned,
    exposed through the CUDA array interface (version 3) so that torch (and
    CuPy, Numba, ...) view it without a copy; the block goes back to the
    library's pool (nlb_device_free, ordered on the producing stream) when
    the last view is gone."""

    __slots__ = ("ptr", "stream", "__cuda_array_interface__", "__weakref__")
    # (held by the class: module globals may already be gone when the last
    # view dies at interpreter shutdown)
    _free = _lib.nlb_device_free

    def __init__(self, ptr: int, shape, typestr: str, stream: int):
        self.ptr = ptr
        self.stream = stream
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": typestr,
                                         "data": (ptr, False), "version": 3, "strides": None,
                                         "stream": None}

    def __del__(self):
        if self.ptr:
            try:
                self._free(self.ptr, self.stream)
            except Exception:  # interpreter shutdown
                pass
            self.ptr = 0


def device_blocks() -> dict:
    """Counters of the zero-copy device result blocks: handed out, returned,
    and bytes still outstanding."""
    buf = (ctypes.c_int64 * 3)()
    _lib.nlb_device_blocks(buf)
    return {"handed": int(buf[0]), "returned": int(buf[1]), "outstanding_bytes": int(buf[2])}


def build_neighborlists_torch(cell, positions, cutoff, directed=False, vectors=False,
                              distances=False):
    """GPU-resident variant of build_neighborlists for torch pipelines:
    ``positions`` is a CUDA float64 tensor (N, 3); returns
    {"edge_index": int64 (2, M), "shift": int32 (M, 3)} as CUDA tensors on the
    same device, produced on the current torch stream.  The tensors are the
    library's result blocks themselves (zero-copy: the build writes them in
    place and hands them over; they return to the library's pool when the
    tensors are freed, ordered on the stream that was current for the build,
    so a consumer on another stream keeps them alive until its work there is
    done, as with torch's own record_stream rule).  directed / vectors /
    distances as in build_neighborlists_ex (adds "vectors" float64 (M, 3) and
    "distances" float64 (M,); those results are copied out of the library's
    workspace)."""
    if directed or vectors or distances:
        return _torch_ex(cell, positions, cutoff, directed, vectors, distances)
    import torch

    if not (isinstance(positions, torch.Tensor) and positions.is_cuda
            and positions.dtype == torch.float64 and positions.dim() == 2):
        raise TypeError("positions must be a CUDA float64 tensor of shape (N, 3)")
    if positions.shape[1] != 3:
        raise ValueError("Positions must be (N, 3)")
    pos = positions.contiguous()
    dev = pos.device
    n = pos.shape[0]
    if n == 0:
        _check_cutoff(cutoff)
        return {"edge_index": torch.zeros((2, 0), dtype=torch.int64, device=dev),
                "shift": torch.zeros((0, 3), dtype=torch.int32, device=dev)}
    c = _check_cutoff(cutoff)
    h, pb = _cell_args(cell)
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        set_stream(stream.cuda_stream)
        try:
            r = _DevResult()
            _check(_lib.nlb_build_device_owned(ctypes.c_void_p(pos.data_ptr()), n, c, h, pb,
                                               ctypes.byref(r)))
        finally:
            set_stream(None)
        m = int(r.n_edges)
        if m == 0:
            return {"edge_index": torch.zeros((2, 0), dtype=torch.int64, device=dev),
                    "shift": torch.zeros((0, 3), dtype=torch.int32, device=dev)}
        ei = torch.as_tensor(_DeviceBlock(r.edge_index, (2, m), "<i8", stream.cuda_stream),
                             device=dev)
        sh = torch.as_tensor(_DeviceBlock(r.shift, (m, 3), "<i4", stream.cuda_stream),
                             device=dev)
    return {"edge_index": ei, "shift": sh}


_lib.nlb_copy_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                 ctypes.c_void_p]


# ---------------------------------------------------------------- output options

class _ResultEx(ctypes.Structure):
    _fields_ = [("n_edges", ctypes.c_int64),
                ("edge_index", ctypes.c_void_p),
                ("shift", ctypes.c_void_p),
                ("vectors", ctypes.c_void_p),
                ("distances", ctypes.c_void_p)]


_NLB_DIRECTED, _NLB_VECTORS, _NLB_DISTANCES = 1, 2, 4
_lib.nlb_build_ex.argtypes = [_dp, ctypes.c_int64, ctypes.c_double, _dp, _u8p, ctypes.c_int,
                              ctypes.POINTER(_ResultEx)]
_lib.nlb_build_device_ex.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, _dp,
                                     _u8p, ctypes.c_int, ctypes.POINTER(_ResultEx)]
_lib.nlb_result_ex_free.argtypes = [ctypes.POINTER(_ResultEx)]


def _ex_flags(directed, vectors, distances) -> int:
    return ((_NLB_DIRECTED if directed else 0) | (_NLB_VECTORS if vectors else 0)
            | (_NLB_DISTANCES if distances else 0))


def build_neighborlists_ex(cell, positions, cutoff, directed=False, vectors=False,
                           distances=False):
    """build_neighborlists with the output options of the reference's
    specification (spec.md:100-108, RUST_API.md:89-90), computed on the GPU:

    * directed: the half list followed by every edge reversed, (j, i, -S)
      ("double the edges and negate the shifts");
    * vectors: "vectors" float64 (M, 3), d = (r_j - r_i) + H S (H columns =
      lattice vectors; r_j - r_i without a cell); reversed edges get -d;
    * distances: "distances" float64 (M,), |d| (correctly rounded sqrt).
    """
    c = _check_cutoff(cutoff)
    pos = _positions(positions)
    n = pos.shape[0]
    h, pb = _cell_args(cell)
    r = _ResultEx()
    _check(_lib.nlb_build_ex(pos.ctypes.data_as(_dp), n, c, h, pb,
                             _ex_flags(directed, vectors, distances), ctypes.byref(r)))
    m = int(r.n_edges)
    out = {"edge_index": _arr(r.edge_index, 2 * m, np.int64).reshape(2, m),
           "shift": _arr(r.shift, 3 * m, np.int32).reshape(m, 3)}
    if vectors:
        out["vectors"] = _arr(r.vectors, 3 * m, np.float64).reshape(m, 3)
    if distances:
        out["distances"] = _arr(r.distances, m, np.float64)
    return out


def _cudart_copy(dst, src, nbytes, stream):
    _check(_lib.nlb_copy_device(ctypes.c_void_p(dst), ctypes.c_void_p(src), nbytes,
                                ctypes.c_void_p(stream)))


def _torch_ex(cell, positions, cutoff, directed, vectors, distances):
    import torch

    if not (isinstance(positions, torch.Tensor) and positions.is_cuda
            and positions.dtype == torch.float64 and positions.dim() == 2):
        raise TypeError("positions must be a CUDA float64 tensor of shape (N, 3)")
    if positions.shape[1] != 3:
        raise ValueError("Positions must be (N, 3)")
    c = _check_cutoff(cutoff)
    pos = positions.contiguous()
    dev = pos.device
    n = pos.shape[0]
    h, pb = _cell_args(cell)
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev)
        set_stream(stream.cuda_stream)
        try:
            r = _ResultEx()
            _check(_lib.nlb_build_device_ex(ctypes.c_void_p(pos.data_ptr() if n else 0), n, c, h,
                                            pb, _ex_flags(directed, vectors, distances),
                                            ctypes.byref(r)))
            m = int(r.n_edges)
            out = {"edge_index": torch.empty((2, m), dtype=torch.int64, device=dev),
                   "shift": torch.empty((m, 3), dtype=torch.int32, device=dev)}
            if vectors:
                out["vectors"] = torch.empty((m, 3), dtype=torch.float64, device=dev)
            if distances:
                out["distances"] = torch.empty((m,), dtype=torch.float64, device=dev)
            if m:
                s = stream.cuda_stream
                _cudart_copy(out["edge_index"].data_ptr(), r.edge_index, 16 * m, s)
                _cudart_copy(out["shift"].data_ptr(), r.shift, 12 * m, s)
                if vectors:
                    _cudart_copy(out["vectors"].data_ptr(), r.vectors, 24 * m, s)
                if distances:
                    _cudart_copy(out["distances"].data_ptr(), r.distances, 8 * m, s)
        finally:
            set_stream(None)
    return out
