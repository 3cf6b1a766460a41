"""Asynchronous :gradepro requests with continuous batching (pkde_submit / pkde_wait).

    srv = Server(device_id=0, lanes=2)
    t = srv.submit(grid, data, n_bootstraps=32, n_steps=100, seed=1)
    res = srv.wait(t)          # dict: density, selected_step, queue_ms, run_ms, ...

Requests queue in the library; each lane (worker thread + stream + device buffers)
takes the queued requests as one wave when it is free, so requests that arrive while
other work is on the GPU start as soon as a lane and memory are free, and their work
overlaps on the device.  Results equal those of a one-request call.
"""
import ctypes
import threading

import numpy as np

from ._lib import (PkdeGradeproParams, ArgumentError, CudaLibraryError, check, context, load, make_grid_struct,
                   make_params, ptr)

PKDE_OK, PKDE_EINVAL, PKDE_ETIMEDOUT = 0, 1, 5


class PkdeRequest(ctypes.Structure):
    _fields_ = [("params", PkdeGradeproParams), ("data", ctypes.c_void_p), ("n", ctypes.c_int64),
                ("boot_idx", ctypes.c_void_p), ("seed", ctypes.c_uint64), ("density_out", ctypes.c_void_p),
                ("selected_out", ctypes.c_void_p)]


class PkdeResult(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("batch_size", ctypes.c_int32), ("queue_ms", ctypes.c_double),
                ("run_ms", ctypes.c_double), ("total_ms", ctypes.c_double), ("message", ctypes.c_char * 256)]


def _bind(lib):
    if getattr(lib, "_pkde_serve_bound", False):
        return lib
    lib.pkde_serve_config.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64]
    lib.pkde_submit.argtypes = [ctypes.c_void_p, ctypes.POINTER(PkdeRequest), ctypes.POINTER(ctypes.c_uint64)]
    lib.pkde_wait.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(PkdeResult)]
    lib._pkde_serve_bound = True
    return lib


class Server:
    """Serving front end of one device's context."""

    def __init__(self, device_id=0, lanes=2, lane_memory_bytes=0):
        self.lib = _bind(load())
        self.ctx = context(device_id)
        rc = self.lib.pkde_serve_config(self.ctx, int(lanes), int(lane_memory_bytes))
        if rc == PKDE_EINVAL and b"before the first" in self.lib.pkde_last_error(self.ctx):
            pass  # already serving: keep the running configuration
        else:
            check(rc, self.ctx)
        self._keep = {}
        self._lock = threading.Lock()

    def submit(self, grid, data, n_bootstraps=100, n_steps=None, seed=0, bootstrap_idxs=None, **kwargs):
        """Queue one estimation of `data` (N x n) on `grid`; returns the ticket."""
        x = np.asarray(data, dtype=np.float64)
        if x.ndim == 1:
            x = x.reshape(1, -1)
        host = np.ascontiguousarray(x.T)
        G = int(np.prod(grid.dims))
        dens = np.empty(G)
        sel = np.empty(G, dtype=np.int32)
        idx = None if bootstrap_idxs is None else np.ascontiguousarray(bootstrap_idxs, dtype=np.int32)
        req = PkdeRequest()
        req.params = make_params(make_grid_struct(grid.lo, grid.hi, grid.h, grid.dims), n_bootstraps, n_steps,
                                 **kwargs)
        req.data = ptr(host)
        req.n = host.shape[0]
        req.boot_idx = ptr(idx)
        req.seed = int(seed) & (2**64 - 1)
        req.density_out = ptr(dens)
        req.selected_out = ptr(sel)
        t = ctypes.c_uint64()
        check(self.lib.pkde_submit(self.ctx, ctypes.byref(req), ctypes.byref(t)), self.ctx)
        with self._lock:
            self._keep[t.value] = (host, idx, dens, sel, tuple(reversed(grid.dims)))
        return t.value

    def wait(self, ticket, timeout_ms=-1):
        """The request's result (a dict), or None if it is not done within timeout_ms."""
        res = PkdeResult()
        rc = self.lib.pkde_wait(self.ctx, int(ticket), int(timeout_ms), ctypes.byref(res))
        if rc == PKDE_ETIMEDOUT:
            return None
        if rc != PKDE_OK:
            raise ArgumentError(self.lib.pkde_last_error(self.ctx).decode(errors="replace"))
        with self._lock:
            host, idx, dens, sel, shape = self._keep.pop(ticket)
        out = dict(status=res.status, batch_size=res.batch_size, queue_ms=res.queue_ms, run_ms=res.run_ms,
                   total_ms=res.total_ms, message=res.message.decode(errors="replace"))
        if res.status == PKDE_OK:
            out["density"] = dens.reshape(shape)
            out["selected_step"] = sel.reshape(shape)
        elif res.status == PKDE_EINVAL:
            out["error"] = ArgumentError(out["message"])
        else:
            out["error"] = CudaLibraryError(out["message"])
        return out
