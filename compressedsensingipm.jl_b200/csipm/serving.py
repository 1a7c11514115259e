"""Serving loop over the C ABI (csipm_server_*, include/csipm.h).

Many recoveries of uneven sizes are submitted as they arrive; the library's
slots (worker threads with one CUDA stream each) admit them in arrival order as
slots and device memory (each request's footprint, csipm_footprint) free up,
keep each admitted request's interior-point state resident on the device and
overlap their kernels.  The reference solves one recovery per call
(src/CompressedSensingIPM.jl:31-36); this layer has no counterpart there.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native
from ._native import check


def lib():
    from . import lib as _lib
    return _lib()


def footprint(size, precision="fp64", n_missing=0) -> int:
    """Device bytes one request of this size holds while it runs (upper bound)."""
    size = tuple(int(s) for s in size)
    arr = (ctypes.c_int * 3)(*(list(size) + [1] * (3 - len(size))))
    out = ctypes.c_size_t()
    prec = {"fp64": 0, "mixed": 1}[precision] if isinstance(precision, str) else int(precision)
    check(lib().csipm_footprint(len(size), arr, prec, int(n_missing), ctypes.byref(out)))
    return int(out.value)


@dataclass
class ServeResult:
    tag: int
    status: int
    stats: dict
    queue_ms: float
    latency_ms: float
    footprint: int
    beta: np.ndarray = field(repr=False, default=None)
    message: str = ""               # the failure's message when status != 0
    group: int = 1                  # requests solved together with this one, itself included


class Server:
    """csipm_server: `slots` concurrent solves within `hbm_budget` device bytes
    (0: 80% of the free memory); cuda_graphs: each request's iterations as one
    graph launch; batch > 1: each slot solves up to `batch` requests of one
    batch class together (csipm_solve_batch, FP64); batch_max_n > 0: requests
    of more samples are solved alone."""

    def __init__(self, slots=8, hbm_budget=0, device=-1, cuda_graphs=False, batch=1, batch_max_n=0):
        o = _native.ServerOptions(int(slots), int(hbm_budget), int(device), int(bool(cuda_graphs)), int(batch),
                                  int(batch_max_n))
        h = ctypes.c_void_p()
        check(lib().csipm_server_create(ctypes.byref(o), ctypes.byref(h)))
        self.handle = h
        self._live = {}
        self._next = 0

    def submit(self, size, z0, lam, missing=None, tag=None, **opts) -> int:
        """Queue one recovery.  z0: host float64 array of prod(size) values
        (column-major), zero at the missing samples; missing: 0-based linear
        indices.  opts as for FFTNLPModel (precision, tol, ipm_cg_rtol, ...)."""
        from . import _options
        size = tuple(int(s) for s in size)
        z0 = np.ascontiguousarray(np.asarray(z0, dtype=np.float64).reshape(-1, order="F"))
        n = int(np.prod(size))
        if z0.size != n:
            raise ValueError("z0 must hold prod(size) values")
        miss = np.ascontiguousarray(np.asarray([] if missing is None else missing, dtype=np.int64))
        beta = np.empty(n, dtype=np.float64)
        if tag is None:
            tag = self._next
        self._next = max(self._next, int(tag) + 1)
        r = _native.Request()
        r.problem.dim = len(size)
        for d in range(3):
            r.problem.size[d] = size[d] if d < len(size) else 1
        r.problem.lam = float(lam)
        r.problem.z0 = z0.ctypes.data
        r.problem.host_missing = miss.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)) if miss.size else None
        r.problem.n_missing = int(miss.size)
        opts.setdefault("rdft", True)
        r.options = _options(stream=0, **opts)
        r.beta_out = beta.ctypes.data
        r.tag = int(tag)
        if tag in self._live:
            raise ValueError(f"tag {tag} is still in flight")
        self._live[int(tag)] = (z0, miss, beta, r)
        check(lib().csipm_server_submit(self.handle, ctypes.byref(r)))
        return int(tag)

    def poll(self, max_results=64, timeout_ms=-1) -> list[ServeResult]:
        buf = (_native.Result * max_results)()
        n = ctypes.c_int()
        check(lib().csipm_server_poll(self.handle, buf, max_results, ctypes.byref(n), int(timeout_ms)))
        out = []
        for k in range(n.value):
            r = buf[k]
            z0, miss, beta, _ = self._live.pop(int(r.tag))
            out.append(ServeResult(int(r.tag), int(r.status), r.stats.as_dict(), float(r.queue_ms),
                                   float(r.latency_ms), int(r.footprint), beta,
                                   r.message.decode(errors="replace"), int(r.group)))
        return out

    def drain(self) -> list[ServeResult]:
        """Poll until every submitted request has returned."""
        out = []
        while self._live:
            out.extend(self.poll(timeout_ms=-1))
        return out

    def close(self):
        if getattr(self, "handle", None):
            lib().csipm_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
