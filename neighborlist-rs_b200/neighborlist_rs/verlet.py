"""Verlet (skin) neighbour lists for molecular dynamics.

``VerletList(cutoff, skin)`` keeps the exact half list at cutoff + skin of a
reference configuration on the GPU and, on every ``update``, returns the
pairs within ``cutoff`` of the current positions by filtering that list; it
rebuilds when an atom moved more than skin / 2 since the last rebuild, or
when the atom count, cell or periodicity changed.  This is the dynamic
manager the reference's specification describes (spec.md:41-48, 209-222;
``DynamicNeighborManager.update / needs_rebuild / get``).  The returned pairs
are the ones ``build_neighborlists(cell, positions, cutoff)`` finds (edges
within rounding of the cutoff aside), in the stored list's order.

    vl = VerletList(cutoff=5.0, skin=1.0)
    for step in range(n_steps):
        res = vl.update(cell, positions)   # numpy in -> numpy out
        ...                                # or CUDA float64 tensor in -> tensors out
"""

from __future__ import annotations

import ctypes

from . import (_DeviceBlock, _DevResult, _Result, _cell_args, _check, _check_cutoff, _dp, _lib,
               _positions, _to_dict, _u8p)

_lib.nlb_verlet_create.argtypes = [ctypes.c_double, ctypes.c_double]
_lib.nlb_verlet_create.restype = ctypes.c_void_p
_lib.nlb_verlet_update.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int64, _dp, _u8p,
                                   ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_Result)]
_lib.nlb_verlet_update_device.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _dp,
                                          _u8p, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(_DevResult)]
_lib.nlb_verlet_update_device_owned.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                                _dp, _u8p, ctypes.POINTER(ctypes.c_int),
                                                ctypes.POINTER(_DevResult)]
_lib.nlb_verlet_needs_rebuild.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, _dp,
                                          _u8p, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_double)]
_lib.nlb_verlet_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
_lib.nlb_verlet_destroy.argtypes = [ctypes.c_void_p]


def _is_cuda_tensor(x) -> bool:
    try:
        import torch
    except ImportError:
        return False
    return isinstance(x, torch.Tensor) and x.is_cuda


class VerletList:
    """Skin-list manager on the current CUDA device (see the module doc)."""

    def __init__(self, cutoff: float, skin: float):
        c = _check_cutoff(cutoff)
        h = _lib.nlb_verlet_create(c, float(skin))
        if not h:
            raise ValueError(_lib.nlb_last_error().decode())
        self._h = h
        self.cutoff = c
        self.skin = float(skin)
        self.rebuilt = False     # whether the last update rebuilt the list
        self.max_displacement = 0.0

    def _handle(self):
        if not self._h:
            raise RuntimeError("VerletList is closed")
        return self._h

    def update(self, cell, positions):
        """Pairs within the cutoff for these positions: numpy (N, 3) float64
        in -> build_neighborlists dict; CUDA float64 tensor in -> the same
        dict of CUDA tensors, produced on the current torch stream: the
        library's result blocks themselves (written in place, handed over,
        returned to the pool when the tensors are freed), as in
        build_neighborlists_torch."""
        h, pb = _cell_args(cell)
        flag = ctypes.c_int(0)
        if _is_cuda_tensor(positions):
            import torch

            from . import set_stream

            if positions.dtype != torch.float64 or positions.dim() != 2:
                raise TypeError("positions must be a CUDA float64 tensor of shape (N, 3)")
            if positions.shape[1] != 3:
                raise ValueError("Positions must be (N, 3)")
            pos = positions.contiguous()
            dev = pos.device
            with torch.cuda.device(dev):
                stream = torch.cuda.current_stream(dev)
                set_stream(stream.cuda_stream)
                try:
                    r = _DevResult()
                    _check(_lib.nlb_verlet_update_device_owned(
                        self._handle(), ctypes.c_void_p(pos.data_ptr()), pos.shape[0], h, pb,
                        ctypes.byref(flag), ctypes.byref(r)))
                finally:
                    set_stream(None)
                m = int(r.n_edges)
                if m == 0:
                    ei = torch.zeros((2, 0), dtype=torch.int64, device=dev)
                    sh = torch.zeros((0, 3), dtype=torch.int32, device=dev)
                else:
                    ei = torch.as_tensor(_DeviceBlock(r.edge_index, (2, m), "<i8",
                                                      stream.cuda_stream), device=dev)
                    sh = torch.as_tensor(_DeviceBlock(r.shift, (m, 3), "<i4",
                                                      stream.cuda_stream), device=dev)
            self.rebuilt = bool(flag.value)
            return {"edge_index": ei, "shift": sh}
        pos = _positions(positions)
        r = _Result()
        _check(_lib.nlb_verlet_update(self._handle(), pos.ctypes.data_as(_dp), pos.shape[0], h, pb,
                                      ctypes.byref(flag), ctypes.byref(r)))
        self.rebuilt = bool(flag.value)
        return _to_dict(r)

    def needs_rebuild(self, cell, positions) -> bool:
        """Whether the next update with these positions rebuilds; sets
        ``max_displacement`` (inf when the system changed or there is no
        list yet)."""
        h, pb = _cell_args(cell)
        needs = ctypes.c_int(1)
        disp = ctypes.c_double(0.0)
        if _is_cuda_tensor(positions):
            pos = positions.contiguous()
            ptr, n, on_dev = ctypes.c_void_p(pos.data_ptr()), pos.shape[0], 1
        else:
            pos = _positions(positions)
            ptr, n, on_dev = ctypes.c_void_p(pos.ctypes.data), pos.shape[0], 0
        _check(_lib.nlb_verlet_needs_rebuild(self._handle(), ptr, n, h, pb, on_dev,
                                             ctypes.byref(needs), ctypes.byref(disp)))
        self.max_displacement = disp.value
        return bool(needs.value)

    def stats(self) -> dict:
        buf = (ctypes.c_int64 * 4)()
        _lib.nlb_verlet_stats(self._handle(), buf)
        return dict(zip(("updates", "rebuilds", "stored_edges", "last_edges"),
                        (int(x) for x in buf)))

    def close(self) -> None:
        if self._h:
            _lib.nlb_verlet_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


__all__ = ["VerletList"]
