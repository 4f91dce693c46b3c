"""Served request loop: continuous batching of neighbour-list requests.

``Server`` wraps the library's request server (``nlb_server_*`` in
include/neighborlist_b200.h).  Requests are structures of any size, each
with its own cell and cutoff; worker threads batch the queued small ones
into single launches of the batched kernels and run large ones through the
single-system pipeline, admitting work against an HBM budget.  Every result
is the one ``build_neighborlists(cell, positions, cutoff)`` gives for the
same request.

    with Server(hbm_budget_bytes=40 << 30, workers=2) as srv:
        tickets = [srv.submit(cell, pos, 6.0) for cell, pos in structures]
        results = [srv.wait(t) for t in tickets]
"""

from __future__ import annotations

import ctypes
import threading

from . import (_Result, _cell_args, _check, _check_cutoff, _dp, _lib, _positions, _to_dict,
               _u8p)

_lib.nlb_server_create.argtypes = [ctypes.c_int, ctypes.c_int64, ctypes.c_int, ctypes.c_int]
_lib.nlb_server_create.restype = ctypes.c_void_p
_lib.nlb_server_submit.argtypes = [ctypes.c_void_p, _dp, ctypes.c_int64, _dp, _u8p,
                                   ctypes.c_double, ctypes.c_int]
_lib.nlb_server_submit.restype = ctypes.c_int64
_lib.nlb_server_wait.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double,
                                 ctypes.POINTER(_Result), ctypes.POINTER(ctypes.c_double)]
_lib.nlb_server_release.argtypes = [ctypes.c_void_p, ctypes.c_int64]
_lib.nlb_server_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]
_lib.nlb_server_pause.argtypes = [ctypes.c_void_p, ctypes.c_int]
_lib.nlb_server_cancel.argtypes = [ctypes.c_void_p, ctypes.c_int64]
_lib.nlb_server_debug_fail.argtypes = [ctypes.c_void_p, ctypes.c_int64]
_lib.nlb_server_destroy.argtypes = [ctypes.c_void_p]

_NLB_NOT_READY = 4
_STATS = ("submitted", "completed", "failed", "batches", "reserved_bytes", "queued",
          "largest_batch", "budget_bytes", "us_stage", "us_count_wait", "us_deliver",
          "us_emit_wait", "us_large", "cancelled", "us_queue_wait", "max_queued")


class DeviceResult:
    """A device-resident served result: ``edge_index`` ([src | dst], 2*M
    int64) and ``shift`` (3*M int32) are device pointers owned by the server
    until ``release()`` (their bytes stay reserved in its HBM budget)."""

    def __init__(self, server: "Server", ticket: int, r: _Result):
        self._server = server
        self.ticket = ticket
        self.n_edges = int(r.n_edges)
        self.edge_index = int(r.edge_index or 0)
        self.shift = int(r.shift or 0)

    def to_torch(self, device=None):
        """Copies into new CUDA tensors {"edge_index": (2, M), "shift": (M, 3)}."""
        import torch

        from . import _cudart_copy

        dev = torch.device("cuda", self._server.device) if device is None else device
        m = self.n_edges
        ei = torch.empty((2, m), dtype=torch.int64, device=dev)
        sh = torch.empty((m, 3), dtype=torch.int32, device=dev)
        if m:
            stream = torch.cuda.current_stream(dev).cuda_stream
            _cudart_copy(ei.data_ptr(), self.edge_index, 16 * m, stream)
            _cudart_copy(sh.data_ptr(), self.shift, 12 * m, stream)
        return {"edge_index": ei, "shift": sh}

    def release(self) -> None:
        if self.ticket:
            srv = self._server
            _check(_lib.nlb_server_release(srv._handle(), self.ticket))
            with srv._lock:
                srv._device_tickets.discard(self.ticket)
            self.ticket = 0


class Server:
    """Continuous-batching neighbour-list server on one CUDA device.

    hbm_budget_bytes: bound on the estimated device footprint of admitted
    requests; workers: host worker threads (each with its own stream);
    max_batch: most requests per batched launch."""

    def __init__(self, hbm_budget_bytes: int = 40 << 30, workers: int = 2,
                 max_batch: int = 4096, device: int = 0):
        self.device = int(device)
        h = _lib.nlb_server_create(self.device, int(hbm_budget_bytes), int(workers),
                                   int(max_batch))
        if not h:
            raise RuntimeError(
                f"neighborlist_rs (CUDA): {_lib.nlb_last_error().decode()}")
        self._h = h
        self._lock = threading.Lock()
        self._device_tickets: set[int] = set()

    def _handle(self):
        if not self._h:
            raise RuntimeError("server is closed")
        return self._h

    def submit(self, cell, positions, cutoff, device_result: bool = False) -> int:
        """Queues one structure; returns its ticket.  Validation and errors are
        those of build_neighborlists."""
        c = _check_cutoff(cutoff)
        pos = _positions(positions)
        h, pb = _cell_args(cell)
        t = int(_lib.nlb_server_submit(self._handle(), pos.ctypes.data_as(_dp), pos.shape[0], h,
                                       pb, c, int(bool(device_result))))
        if t < 0:
            _check(-t)
        if device_result:
            with self._lock:
                self._device_tickets.add(t)
        return t

    def wait_timed(self, ticket: int, timeout: float | None = None):
        """Returns (result, latency_ms from submit to completion).  The result
        is the build_neighborlists dict, or a DeviceResult for device_result
        requests.  Raises TimeoutError if not done within ``timeout`` s."""
        r = _Result()
        lat = ctypes.c_double(0.0)
        code = _lib.nlb_server_wait(self._handle(), int(ticket),
                                    -1.0 if timeout is None else float(timeout), ctypes.byref(r),
                                    ctypes.byref(lat))
        if code == _NLB_NOT_READY:
            raise TimeoutError(f"request {ticket} not done after {timeout} s")
        if code != 0:
            with self._lock:
                self._device_tickets.discard(int(ticket))
        _check(code)
        with self._lock:
            on_device = int(ticket) in self._device_tickets
        if on_device:
            return DeviceResult(self, int(ticket), r), lat.value
        return _to_dict(r), lat.value

    def wait(self, ticket: int, timeout: float | None = None):
        return self.wait_timed(ticket, timeout)[0]

    def pause(self, paused: bool = True) -> None:
        """Stops (or resumes) the workers taking new work; queued requests
        wait, running work finishes."""
        _check(_lib.nlb_server_pause(self._handle(), int(bool(paused))))

    def cancel(self, ticket: int) -> None:
        """Withdraws a queued request (it never runs) or frees a finished
        one's result; the ticket is retired.  Raises ValueError for a running
        request or an unknown ticket."""
        _check(_lib.nlb_server_cancel(self._handle(), int(ticket)))
        with self._lock:
            self._device_tickets.discard(int(ticket))

    def _debug_fail(self, ticket: int) -> None:
        """Failure-detection hook for tests: the staging of any batch holding
        this queued request fails; only this request reports the error."""
        _check(_lib.nlb_server_debug_fail(self._handle(), int(ticket)))

    def stats(self) -> dict:
        buf = (ctypes.c_int64 * len(_STATS))()
        _lib.nlb_server_stats(self._handle(), buf)
        return dict(zip(_STATS, (int(x) for x in buf)))

    def close(self) -> None:
        with self._lock:
            if self._h:
                _lib.nlb_server_destroy(self._h)
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
