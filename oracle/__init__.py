"""CPU oracle for the neighbour-list path -- TEST INFRASTRUCTURE ONLY.

ctypes wrapper around ``oracle/_build/libnl_oracle.so`` (built from
``oracle/nl_oracle.cpp`` by ``oracle/Makefile``).  The C++ file restates the
search path of solccp/neighborlist-rs (src/cell.rs, src/search.rs,
src/single.rs, src/batch.rs); see its header for the line-by-line map.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs
import this module.  The product library (``neighborlist_rs``) never does.

Conventions follow the reference's Rust layer (src/api.rs):
  * ``h`` is a 3x3 matrix whose COLUMNS are the lattice vectors
    (``Matrix3::new`` takes row-major arguments, src/api.rs:93-98);
  * results are ``(edge_index int64 (2, M), shift int32 (M, 3))``.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))


def _has_avx2() -> bool:
    try:
        with open("/proc/cpuinfo") as f:
            return " avx2" in f.read()
    except OSError:
        return False


_LIB_PATH = os.path.join(_HERE, "_build", "libnl_oracle.so" if _has_avx2()
                         else "libnl_oracle_generic.so")


class _Edges(ctypes.Structure):
    _fields_ = [
        ("n_edges", ctypes.c_int64),
        ("edge_i", ctypes.POINTER(ctypes.c_int64)),
        ("edge_j", ctypes.POINTER(ctypes.c_int64)),
        ("shift", ctypes.POINTER(ctypes.c_int32)),
    ]


def build() -> str:
    """Compile the oracle library if it is missing or stale."""
    src = os.path.join(_HERE, "nl_oracle.cpp")
    if (not os.path.exists(_LIB_PATH)) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        u8p = ctypes.POINTER(ctypes.c_uint8)
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_set_thresholds.argtypes = [ctypes.c_int64, ctypes.c_int64]
        L.orc_edges_free.argtypes = [ctypes.POINTER(_Edges)]
        L.orc_cell_inverse.argtypes = [dp, dp]
        L.orc_perp_widths.argtypes = [dp, dp]
        L.orc_wrap.argtypes = [dp, u8p, dp, dp]
        L.orc_mic.argtypes = [dp, u8p, dp, dp, ctypes.POINTER(ctypes.c_int32), dp]
        L.orc_zorder.argtypes = [dp]
        L.orc_zorder.restype = ctypes.c_uint64
        L.orc_cell_list.argtypes = [dp, ctypes.c_int64, dp, ctypes.c_double,
                                    ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
        L.orc_search_single.argtypes = [dp, ctypes.c_int64, dp, u8p, ctypes.c_double,
                                        ctypes.c_int, ctypes.POINTER(_Edges)]
        L.orc_search_single_multi.argtypes = [dp, ctypes.c_int64, dp, u8p, dp, ctypes.c_int32,
                                              ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Edges)]
        L.orc_search_batch.argtypes = [dp, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32),
                                       ctypes.c_int64, dp, u8p, u8p, ctypes.c_int64, dp,
                                       ctypes.c_int32, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(_Edges)]
        i64p = ctypes.POINTER(ctypes.c_int64)
        L.orc_edge_extras.argtypes = [dp, dp, i64p, i64p, ctypes.POINTER(ctypes.c_int32),
                                      ctypes.c_int64, ctypes.c_int, i64p,
                                      ctypes.POINTER(ctypes.c_int32), dp, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _u8p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)) if a is not None else None


def _take(e: _Edges):
    m = int(e.n_edges)
    ei = np.ctypeslib.as_array(e.edge_i, shape=(max(m, 1),))[:m].copy()
    ej = np.ctypeslib.as_array(e.edge_j, shape=(max(m, 1),))[:m].copy()
    sh = np.ctypeslib.as_array(e.shift, shape=(max(3 * m, 1),))[: 3 * m].copy()
    lib().orc_edges_free(ctypes.byref(e))
    return np.stack([ei, ej]).astype(np.int64).reshape(2, m), sh.reshape(m, 3).astype(np.int32)


def _err():
    return RuntimeError(lib().orc_last_error().decode())


def _pos(positions):
    p = np.ascontiguousarray(np.asarray(positions, dtype=np.float64))
    if p.size == 0:
        p = p.reshape(0, 3)
    return p


def _cell(h, pbc):
    if h is None:
        return None, None
    h9 = np.ascontiguousarray(np.asarray(h, dtype=np.float64).reshape(9))
    pb = np.ascontiguousarray(np.asarray(pbc if pbc is not None else [True] * 3, dtype=np.uint8))
    return h9, pb


def set_thresholds(brute_force: int = 1000, parallel: int = 300) -> None:
    lib().orc_set_thresholds(int(brute_force), int(parallel))


def search_single(positions, h=None, pbc=None, cutoff=5.0, nthreads=1):
    """src/single.rs:8-90.  h=None selects the auto-box (isolated) cell."""
    p = _pos(positions)
    h9, pb = _cell(h, pbc)
    e = _Edges()
    if lib().orc_search_single(_dp(p), p.shape[0], _dp(h9), _u8p(pb), float(cutoff),
                               int(nthreads), ctypes.byref(e)):
        raise _err()
    return _take(e)


def search_single_multi(positions, h=None, pbc=None, cutoffs=(5.0,), disjoint=False,
                        nthreads=1):
    """src/single.rs:92-164.  Returns a list of (edge_index, shift) in input cutoff order."""
    p = _pos(positions)
    h9, pb = _cell(h, pbc)
    cs = np.ascontiguousarray(np.asarray(cutoffs, dtype=np.float64).reshape(-1))
    k = cs.shape[0]
    outs = (_Edges * max(k, 1))()
    if lib().orc_search_single_multi(_dp(p), p.shape[0], _dp(h9), _u8p(pb), _dp(cs), k,
                                     int(bool(disjoint)), int(nthreads), outs):
        raise _err()
    if p.shape[0] == 0 or k == 0:
        return [(np.zeros((2, 0), np.int64), np.zeros((0, 3), np.int32)) for _ in range(k)]
    return [_take(outs[q]) for q in range(k)]


def search_batch(positions, batch, cells=None, cutoffs=(5.0,), disjoint=False, nthreads=1):
    """src/batch.rs:10-290.

    ``cells`` is None (every system auto-boxed) or a list with one entry per
    system: None (auto-box) or ``(h, pbc)`` with h's columns the lattice vectors.
    Returns a list over cutoffs of (edge_index, shift).
    """
    p = _pos(positions)
    b = np.ascontiguousarray(np.asarray(batch, dtype=np.int32).reshape(-1))
    cs = np.ascontiguousarray(np.asarray(cutoffs, dtype=np.float64).reshape(-1))
    k = cs.shape[0]
    if cells is None:
        c9 = pb = has = None
        nc = 0
    else:
        nc = len(cells)
        c9 = np.zeros((max(nc, 1), 9), np.float64)
        pb = np.zeros((max(nc, 1), 3), np.uint8)
        has = np.zeros(max(nc, 1), np.uint8)
        for s, c in enumerate(cells):
            if c is not None:
                c9[s] = np.asarray(c[0], np.float64).reshape(9)
                pb[s] = np.asarray(c[1], np.uint8)
                has[s] = 1
    outs = (_Edges * max(k, 1))()
    if lib().orc_search_batch(_dp(p), p.shape[0], b.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                              b.shape[0], _dp(c9), _u8p(pb), _u8p(has), nc, _dp(cs), k,
                              int(bool(disjoint)), int(nthreads), outs):
        raise _err()
    return [_take(outs[q]) for q in range(k)]


def cell_inverse(h):
    h9 = np.ascontiguousarray(np.asarray(h, np.float64).reshape(9))
    out = np.zeros(9)
    if lib().orc_cell_inverse(_dp(h9), _dp(out)):
        raise RuntimeError("Cell matrix is not invertible")
    return out.reshape(3, 3)


def perpendicular_widths(h):
    h9 = np.ascontiguousarray(np.asarray(h, np.float64).reshape(9))
    out = np.zeros(3)
    if lib().orc_perp_widths(_dp(h9), _dp(out)):
        raise RuntimeError("Cell matrix is not invertible")
    return out


def wrap(h, pbc, pos):
    h9 = np.ascontiguousarray(np.asarray(h, np.float64).reshape(9))
    pb = np.ascontiguousarray(np.asarray(pbc, np.uint8))
    p = np.ascontiguousarray(np.asarray(pos, np.float64))
    out = np.zeros(3)
    if lib().orc_wrap(_dp(h9), _u8p(pb), _dp(p), _dp(out)):
        raise RuntimeError("Cell matrix is not invertible")
    return out


def minimum_image(h, pbc, ri, rj):
    h9 = np.ascontiguousarray(np.asarray(h, np.float64).reshape(9))
    pb = np.ascontiguousarray(np.asarray(pbc, np.uint8))
    a = np.ascontiguousarray(np.asarray(ri, np.float64))
    b = np.ascontiguousarray(np.asarray(rj, np.float64))
    s = np.zeros(3, np.int32)
    d = np.zeros(3)
    if lib().orc_mic(_dp(h9), _u8p(pb), _dp(a), _dp(b),
                     s.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _dp(d)):
        raise RuntimeError("Cell matrix is not invertible")
    return s, d


def zorder(frac):
    f = np.ascontiguousarray(np.asarray(frac, np.float64))
    return int(lib().orc_zorder(_dp(f)))


def cell_list(positions, h, cutoff):
    """Cell-list structure (src/search.rs:92-264): (num_bins, n_search, particles, atom_bin)."""
    p = _pos(positions)
    h9 = np.ascontiguousarray(np.asarray(h, np.float64).reshape(9))
    nb = np.zeros(3, np.int64)
    ns = np.zeros(3, np.int32)
    parts = np.zeros(max(p.shape[0], 1), np.int64)
    abin = np.zeros(max(p.shape[0], 1), np.int64)
    if lib().orc_cell_list(_dp(p), p.shape[0], _dp(h9), float(cutoff),
                           nb.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                           ns.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                           parts.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                           abin.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))):
        raise RuntimeError("Cell matrix is not invertible")
    return nb, ns, parts[: p.shape[0]], abin[: p.shape[0]]


def edge_extras(positions, h, edges, directed=False):
    """spec.md:100-108 / RUST_API.md:89-90 output options on a half list
    (edge_index (2, M), shift (M, 3)): returns (edge_index (2, Mo), shift
    (Mo, 3), vectors (Mo, 3), distances (Mo,)), Mo = 2M if directed.
    h=None: the system has no cell (vectors are r_j - r_i)."""
    p = _pos(positions)
    ei, sh = edges
    m = ei.shape[1]
    mo = 2 * m if directed else m
    src = np.ascontiguousarray(ei[0], dtype=np.int64)
    dst = np.ascontiguousarray(ei[1], dtype=np.int64)
    s = np.ascontiguousarray(sh, dtype=np.int32).reshape(-1)
    h9 = None if h is None else np.ascontiguousarray(np.asarray(h, dtype=np.float64).reshape(9))
    ei_out = np.zeros(max(2 * mo, 1), np.int64)
    sh_out = np.zeros(max(3 * mo, 1), np.int32)
    vec = np.zeros(max(3 * mo, 1), np.float64)
    dist = np.zeros(max(mo, 1), np.float64)
    i64p = ctypes.POINTER(ctypes.c_int64)
    i32p = ctypes.POINTER(ctypes.c_int32)
    lib().orc_edge_extras(_dp(p), _dp(h9), src.ctypes.data_as(i64p), dst.ctypes.data_as(i64p),
                          s.ctypes.data_as(i32p), m, int(bool(directed)),
                          ei_out.ctypes.data_as(i64p), sh_out.ctypes.data_as(i32p), _dp(vec),
                          _dp(dist))
    return (ei_out[: 2 * mo].reshape(2, mo), sh_out[: 3 * mo].reshape(mo, 3),
            vec[: 3 * mo].reshape(mo, 3), dist[:mo])


def verlet_filter(positions, h, edges, cutoff):
    """The filter step of the skin-list manager (no counterpart in the
    reference, whose spec.md:41-48 and 209-222 only describe it): the stored
    half list (i, j, S), built at cutoff + skin from the positions of the last
    rebuild, is kept in stored order where |(r_j - r_i) + H.S|^2 < cutoff^2
    with the current positions.  The displacement is edge_extras'
    expression; the squared norm is (d0^2 + d1^2) + d2^2, each operation a
    separately rounded FP64 multiply or add (numpy never fuses them).
    h=None: a system without a cell (d = r_j - r_i)."""
    ei, sh = edges
    if ei.shape[1] == 0:
        return ei.copy(), sh.copy()
    _, _, vec, _ = edge_extras(positions, h, edges)
    n2 = (vec[:, 0] * vec[:, 0] + vec[:, 1] * vec[:, 1]) + vec[:, 2] * vec[:, 2]
    keep = n2 < float(cutoff) * float(cutoff)
    return np.ascontiguousarray(ei[:, keep]), np.ascontiguousarray(sh[keep])
