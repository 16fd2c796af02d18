"""Heterogeneous batches of searches (the C ABI's sc_dd_pool).

A SearchPool runs a list of SearchRequest objects -- each with its own input, shape,
frequency resolution, drift range, threshold and storage precision -- in sub-batches
that fit a device scratch budget; kernels run once per sub-batch for up to 64 searches,
launch shapes are autotuned on first sight and repeated sub-batches replay a captured
CUDA graph.
"""
import ctypes
from dataclasses import dataclass
from typing import List, Optional

from . import _capi
from ._capi import check, lib
from .dedoppler import Dedopplerer, _stream_handle


@dataclass
class SearchRequest:
    input: object            # CUDA float32 tensor [rounded T][N] (unit channel stride)
    num_timesteps: int       # unrounded
    foff: float              # MHz
    tsamp: float             # s
    max_drift: float
    min_drift: float = 0.0
    snr_threshold: float = 10.0
    beam: int = -1
    coarse_channel: int = 0
    precision: str = "fp32"  # "fp32", "bf16" or "fp16"

    def to_c(self) -> _capi.ScDdRequest:
        t = self.input
        if not getattr(t, "is_cuda", False) or t.dim() != 2 or t.stride(1) != 1:
            raise TypeError("SearchRequest.input must be a 2-D CUDA tensor with unit channel stride")
        r = _capi.ScDdRequest()
        r.dev_input = t.data_ptr()
        r.row_stride = t.stride(0)
        r.num_timesteps = self.num_timesteps
        r.num_channels = t.shape[1]
        r.foff_mhz = self.foff
        r.tsamp_s = self.tsamp
        r.max_drift = self.max_drift
        r.min_drift = self.min_drift
        r.snr_threshold = self.snr_threshold
        r.beam = self.beam
        r.coarse_channel = self.coarse_channel
        r.precision = {"fp32": _capi.SC_DD_PRECISION_FP32, "bf16": _capi.SC_DD_PRECISION_BF16,
                       "fp16": _capi.SC_DD_PRECISION_FP16}[self.precision]
        return r


class SearchPool:
    def __init__(self, scratch_budget_bytes: int = 8 << 30, autotune: bool = True, cuda_graphs: bool = True):
        self._h = ctypes.c_void_p()
        check(lib().sc_dd_pool_create(scratch_budget_bytes, ctypes.byref(self._h)), pool=True)
        self._graphs = bool(cuda_graphs)
        self.configure(autotune)

    def configure(self, autotune: bool):
        """Turns the timing of new launch classes on or off (tuned classes stay tuned)."""
        check(lib().sc_dd_pool_configure(self._h, int(autotune), int(self._graphs)), pool=True)

    def close(self):
        if self._h:
            lib().sc_dd_pool_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def scratch_bytes(req: SearchRequest) -> int:
        r = req.to_c()
        return int(lib().sc_dd_request_scratch_bytes(ctypes.byref(r)))

    def search_raw(self, requests: List[SearchRequest], stream=None, capacity: int = 1 << 16):
        """One HitList of ScDdHit per request."""
        n = len(requests)
        if n == 0:
            return []
        reqs = (_capi.ScDdRequest * n)(*[r.to_c() for r in requests])
        counts = (ctypes.c_int * n)()
        cap = capacity
        while True:
            buf = self._hits if getattr(self, "_hits", None) is not None and len(self._hits) >= cap else None
            if buf is None:
                buf = self._hits = (_capi.ScDdHit * max(cap, 1))()
            rc = lib().sc_dd_pool_search(self._h, reqs, n, buf, cap, counts, _stream_handle(stream))
            if rc == _capi.SC_DD_ETRUNC:
                cap = sum(counts)
                continue
            check(rc, pool=True)
            return Dedopplerer._split_hits(buf, list(counts))

    def stats(self) -> _capi.ScDdPoolStats:
        s = _capi.ScDdPoolStats()
        check(lib().sc_dd_pool_stats_get(self._h, ctypes.byref(s)), pool=True)
        return s
