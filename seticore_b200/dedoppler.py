"""Python host interface mirroring seticore's dedoppler API.

Names, arguments and results follow the reference:
  * FilterbankBuffer      -- filterbank_buffer.h:11-48 (row-major [time][channel] float32)
  * FilterbankMetadata    -- filterbank_metadata.h:17-62 (the fields the search reads)
  * DedopplerHit          -- dedoppler_hit.h:11-66, dedoppler_hit.cpp:11-73
  * Dedopplerer           -- dedoppler.h:15-79 (search, addIncoherentPower, memoryUsage)

Device memory is held in torch CUDA tensors and work is queued on torch's current CUDA
stream; all arithmetic runs in the CUDA library through the C ABI.  There is no CPU
path: a search on a tensor that is not on a CUDA device raises.
"""
import ctypes
import math
from collections.abc import Sequence
from dataclasses import dataclass, field
from typing import List, Optional

from . import _capi
from ._capi import NO_BEAM, check, lib


def roundUpToPowerOfTwo(n: int) -> int:  # util.cpp:16-22
    r = 1
    while r < n:
        r *= 2
    return r


@dataclass
class FilterbankMetadata:
    """The metadata fields a search uses (filterbank_metadata.h:17-62)."""
    fch1: float = 0.0
    foff: float = 0.0  # MHz
    tsamp: float = 0.0  # s
    coarse_channel_size: int = 0
    num_timesteps: int = 0
    num_channels: int = 0
    num_coarse_channels: int = 0
    has_dc_spike: bool = False
    source_name: str = ""
    source_names: List[str] = field(default_factory=list)
    ras: List[float] = field(default_factory=list)   # hours, per coherent beam
    decs: List[float] = field(default_factory=list)  # degrees, per coherent beam
    tstart: float = 0.0  # MJD
    src_raj: float = 0.0  # hours
    src_dej: float = 0.0  # degrees
    telescope_id: int = 0

    def isCoherentBeam(self, beam: int) -> bool:  # filterbank_metadata.cpp:116-118
        return 0 <= beam < len(self.source_names)

    def getBeamSourceName(self, beam: int) -> str:  # filterbank_metadata.cpp:95-100
        return self.source_names[beam] if self.isCoherentBeam(beam) else self.source_name

    def getBeamRA(self, beam: int) -> float:  # filterbank_metadata.cpp:102-107
        return self.ras[beam] if self.isCoherentBeam(beam) else self.src_raj

    def getBeamDec(self, beam: int) -> float:  # filterbank_metadata.cpp:109-114
        return self.decs[beam] if self.isCoherentBeam(beam) else self.src_dej

    def getSubsetMetadata(self, beam: int, band: int, num_bands: int) -> "FilterbankMetadata":
        """The metadata of one band of one beam (filterbank_metadata.cpp:22-50)."""
        import dataclasses
        n = self.num_channels // num_bands
        assert n > 0
        return dataclasses.replace(
            self, source_name=self.getBeamSourceName(beam), source_names=list(self.source_names),
            ras=list(self.ras), decs=list(self.decs), num_channels=n,
            num_coarse_channels=self.num_coarse_channels // num_bands, fch1=self.fch1 + self.foff * n * band,
            src_raj=self.getBeamRA(beam), src_dej=self.getBeamDec(beam))


@dataclass
class DedopplerHit:
    """dedoppler_hit.h:11-66."""
    frequency: float
    index: int
    drift_steps: int
    drift_rate: float
    snr: float
    coarse_channel: int
    beam: int
    num_timesteps: int
    power: float
    incoherent_power: float = 0.0

    @classmethod
    def make(cls, metadata: FilterbankMetadata, index, drift_steps, drift_rate, snr, beam,
             coarse_channel, num_timesteps, power):
        """The reference constructor (dedoppler_hit.cpp:11-23)."""
        global_index = coarse_channel * metadata.coarse_channel_size + index
        return cls(frequency=metadata.fch1 + global_index * metadata.foff, index=index,
                   drift_steps=drift_steps, drift_rate=drift_rate, snr=snr,
                   coarse_channel=coarse_channel,
                   beam=beam if metadata.isCoherentBeam(beam) else NO_BEAM,
                   num_timesteps=num_timesteps, power=power)

    def toString(self) -> str:  # dedoppler_hit.cpp:25-30
        bins = "bin" if self.drift_steps in (1, -1) else "bins"
        return (f"coarse channel = {self.coarse_channel}, index = {self.index}, "
                f"snr = {self.snr:.5f}, drift rate = {self.drift_rate:.5f} "
                f"({self.drift_steps} {bins})")

    def lowIndex(self) -> int:
        return min(self.index, self.index + self.drift_steps)

    def highIndex(self) -> int:
        return max(self.index, self.index + self.drift_steps)

    def expectedIndex(self, timesteps: int) -> int:  # dedoppler_hit.cpp:40-44
        per = float(self.drift_steps) / float(self.num_timesteps - 1)
        return self.index + int(_round_half_away(timesteps * per))

    def score(self) -> float:  # dedoppler_hit.cpp:48-55
        if self.incoherent_power > 0:
            return self.power / self.incoherent_power
        return -1.0 / (1.0 + self.snr)

    def __lt__(self, other):  # dedoppler_hit.cpp:58-66
        if self.coarse_channel != other.coarse_channel:
            return self.coarse_channel < other.coarse_channel
        if self.lowIndex() != other.lowIndex():
            return self.lowIndex() < other.lowIndex()
        return self.highIndex() < other.highIndex()


def _round_half_away(x: float) -> float:
    return math.floor(x + 0.5) if x >= 0 else -math.floor(-x + 0.5)


def driftStepsLessThan(a: DedopplerHit, b: DedopplerHit) -> bool:  # dedoppler_hit.cpp:70-72
    return a.drift_steps < b.drift_steps


class FilterbankBuffer:
    """Row-major [time][channel] float32 power on a CUDA device (filterbank_buffer.h).

    FilterbankBuffer(T, N) allocates; FilterbankBuffer(T, N, data=tensor) is a view on an
    existing CUDA tensor (a 2-D view with unit channel stride, e.g. one coarse channel
    of a wider band: rows may be longer than N)."""

    def __init__(self, num_timesteps: int, num_channels: int, data=None, device=None):
        import torch
        self.num_timesteps = num_timesteps
        self.num_channels = num_channels
        if data is None:
            self.data = torch.zeros((num_timesteps, num_channels), dtype=torch.float32,
                                    device=device or "cuda")
            self.managed = True
        else:
            if data.dim() != 2 or data.shape[0] < num_timesteps or data.shape[1] < num_channels:
                raise ValueError("FilterbankBuffer view has the wrong shape")
            self.data = data
            self.managed = False

    @property
    def row_stride(self) -> int:
        return int(self.data.stride(0))

    def zero(self):
        self.data.zero_()

    def set(self, time: int, channel: int, value: float):
        self.data[time, channel] = value

    def get(self, time: int, channel: int) -> float:
        return float(self.data[time, channel])


def makeNoisyBuffer(num_timesteps: int, num_channels: int, device=None) -> FilterbankBuffer:
    """filterbank_buffer.cu:71-78: row 0 holds 0.1 * chan / N, everything else zero."""
    import torch
    buf = FilterbankBuffer(num_timesteps, num_channels, device=device)
    buf.data[0] = 0.1 * torch.arange(num_channels, dtype=torch.float64, device=buf.data.device).float() / num_channels
    return buf


def _device_input(input, num_rows: int, num_channels: int):
    import torch
    t = input.data if isinstance(input, FilterbankBuffer) else input
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError("dedoppler input must be a CUDA tensor or a FilterbankBuffer on a CUDA device")
    if t.dtype != torch.float32 or t.dim() != 2 or t.stride(1) != 1:
        raise TypeError("dedoppler input must be a 2-D float32 tensor with unit channel stride")
    if t.shape[0] != num_rows or t.shape[1] != num_channels:
        raise ValueError(f"input shape {tuple(t.shape)} != ({num_rows}, {num_channels}) "
                         "(dedoppler.cu:191-192 requires rounded timesteps x channels)")
    return t


class HitList(Sequence):
    """The hit records (ScDdHit) of one search from the raw calls.  The records are held in
    one private copy; a record object is made only when the list is indexed or iterated, so
    a call that returns thousands of hits does not build thousands of Python objects."""

    __slots__ = ("_records",)

    def __init__(self, records):
        self._records = records

    def __len__(self):
        return len(self._records)

    def __getitem__(self, i):
        return self._records[i]

    def __iter__(self):
        return iter(self._records)

    def __eq__(self, other):
        if isinstance(other, (list, tuple, HitList)):
            return len(self) == len(other) and all(a is b or _same_hit(a, b) for a, b in zip(self, other))
        return NotImplemented

    def __repr__(self):
        return f"HitList({len(self)} hits)"


def _same_hit(a, b) -> bool:
    return all(getattr(a, f) == getattr(b, f) for f, _ in _capi.ScDdHit._fields_)


def _stream_handle(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def prepare_coarse_channels(buffers, num_timesteps: int, has_dc_spike: bool, stream=None) -> None:
    """The device half of loading coarse channels (h5_reader.cpp:190-209), one launch for a
    [count][rounded T][N] CUDA tensor (or one [rounded T][N] tensor): zeroes the rows past
    num_timesteps and, with has_dc_spike, replaces the middle column of each loaded row by
    the mean of its neighbours (sc_dd_prepare_coarse_channels)."""
    t = buffers if buffers.dim() == 3 else buffers.unsqueeze(0)
    if not t.is_cuda or t.dtype.itemsize != 4 or t.stride(2) != 1:
        raise TypeError("prepare_coarse_channels needs a float32 CUDA tensor with unit channel stride")
    check(lib().sc_dd_prepare_coarse_channels(ctypes.c_void_p(t.data_ptr()), t.shape[0], t.stride(0), t.stride(1),
                                              num_timesteps, t.shape[1], t.shape[2], int(has_dc_spike),
                                              _stream_handle(stream)))


def gather_hit_slices(input, num_timesteps: int, num_channels: int, bounds, stream=None):
    """Rows [0, num_timesteps) and columns [begin, end) of a CUDA tensor for each (begin,
    end) in bounds, gathered by one kernel launch (sc_dd_gather_columns) and copied to the
    host once.  Returns a list of float32 numpy arrays."""
    import numpy as np
    import torch
    n = len(bounds)
    if n == 0:
        return []
    widths = [max(0, e - b) for b, e in bounds]
    offs = np.zeros(n + 1, dtype=np.int64)
    np.cumsum([num_timesteps * w for w in widths], out=offs[1:])
    dev = input.device
    ranges = torch.tensor([v for b, e in bounds for v in (b, max(b, e))], dtype=torch.int32, device=dev)
    offsets = torch.from_numpy(offs[:-1].copy()).to(dev)
    out = torch.empty(max(1, int(offs[-1])), dtype=torch.float32, device=dev)
    check(lib().sc_dd_gather_columns(ctypes.c_void_p(input.data_ptr()), input.stride(0), num_timesteps, num_channels,
                                     ctypes.c_void_p(ranges.data_ptr()), ctypes.c_void_p(offsets.data_ptr()), n,
                                     ctypes.c_void_p(out.data_ptr()), _stream_handle(stream)))
    if stream is not None:
        stream.synchronize()
    host = out.cpu().numpy()
    return [host[offs[k]:offs[k + 1]].reshape(num_timesteps, widths[k]) for k in range(n)]


class Dedopplerer:
    """The dedoppler search engine (dedoppler.h:15-79) on one CUDA device."""

    def __init__(self, num_timesteps: int, num_channels: int, foff: float, tsamp: float,
                 has_dc_spike: bool = False):
        self.num_timesteps = num_timesteps
        self.num_channels = num_channels
        self.foff = foff
        self.tsamp = tsamp
        self.has_dc_spike = has_dc_spike
        self.print_hits = False
        self._h = ctypes.c_void_p()
        check(lib().sc_dd_create(num_timesteps, num_channels, foff, tsamp, int(has_dc_spike),
                                 ctypes.byref(self._h)))
        self.rounded_num_timesteps = lib().sc_dd_rounded_timesteps(self._h)
        self.drift_timesteps = self.rounded_num_timesteps - 1
        self.drift_rate_resolution = 1e6 * foff / (self.drift_timesteps * tsamp)

    def close(self):
        if self._h:
            lib().sc_dd_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, precision: str) -> None:
        """'fp32' (the reference's form), 'bf16' or 'fp16' (normalised 16-bit storage with
        exact FP32 recomputation near the threshold; identical hit lists)."""
        code = {"fp32": _capi.SC_DD_PRECISION_FP32, "bf16": _capi.SC_DD_PRECISION_BF16,
                "fp16": _capi.SC_DD_PRECISION_FP16}[precision]
        check(lib().sc_dd_set_precision(self._h, code))
        self.precision = precision

    def memoryUsage(self) -> int:
        return int(lib().sc_dd_memory_usage(self._h))

    def _hit_buffer(self, cap: int):
        """A reusable host array of at least `cap` hit records (allocating and zeroing a fresh
        one per call costs milliseconds at 2^16 records)."""
        buf = getattr(self, "_hits", None)
        if buf is None or len(buf) < cap:
            buf = (_capi.ScDdHit * max(cap, 1))()
            self._hits = buf
        return buf

    @staticmethod
    def _copy_hits(buf, start: int, count: int) -> "HitList":
        """Records [start, start + count) of the reusable buffer, copied out (the buffer is
        overwritten by the next call)."""
        return Dedopplerer._split_hits(buf, [count], start)[0]

    @staticmethod
    def _split_hits(buf, counts, start: int = 0) -> list:
        """One HitList per count over consecutive records of the reusable buffer from `start`:
        a single copy of all of them, then views into it."""
        size = ctypes.sizeof(_capi.ScDdHit)
        total = sum(counts)
        block = (_capi.ScDdHit * max(total, 1))()
        if total:
            ctypes.memmove(block, ctypes.addressof(buf) + start * size, total * size)
        out, k = [], 0
        for c in counts:
            out.append(HitList((_capi.ScDdHit * c).from_buffer(block, k * size)))
            k += c
        return out

    def search_raw(self, input, beam: int, coarse_channel: int, max_drift: float,
                   min_drift: float, snr_threshold: float, stream=None, capacity: int = 4096):
        """Runs the search and returns the C ABI hit records (a HitList of ScDdHit)."""
        t = _device_input(input, self.rounded_num_timesteps, self.num_channels)
        cap = capacity
        while True:
            buf = self._hit_buffer(cap)
            n = ctypes.c_int(0)
            rc = lib().sc_dd_search(self._h, ctypes.c_void_p(t.data_ptr()), t.stride(0), beam,
                                    coarse_channel, max_drift, min_drift, snr_threshold, buf, cap,
                                    ctypes.byref(n), _stream_handle(stream))
            if rc == _capi.SC_DD_ETRUNC:
                cap = n.value
                continue
            check(rc)
            return self._copy_hits(buf, 0, n.value)

    def search_batch_raw(self, inputs, beams, coarse_channels, max_drift: float, min_drift: float,
                         snr_threshold: float, stream=None, capacity: int = 1 << 16):
        """Many searches of this engine's shape in one call (sc_dd_search_batch).  Returns one
        HitList of ScDdHit per input."""
        ts = [_device_input(x, self.rounded_num_timesteps, self.num_channels) for x in inputs]
        n = len(ts)
        if n == 0:
            return []
        ptrs = (ctypes.c_void_p * n)(*[t.data_ptr() for t in ts])
        strides = (ctypes.c_longlong * n)(*[t.stride(0) for t in ts])
        b = (ctypes.c_int * n)(*beams)
        c = (ctypes.c_int * n)(*coarse_channels)
        counts = (ctypes.c_int * n)()
        cap = capacity
        while True:
            buf = self._hit_buffer(cap)
            rc = lib().sc_dd_search_batch(self._h, n, ptrs, strides, b, c, max_drift, min_drift, snr_threshold,
                                          buf, cap, counts, _stream_handle(stream))
            if rc == _capi.SC_DD_ETRUNC:
                cap = sum(counts)
                continue
            check(rc)
            return self._split_hits(buf, list(counts))

    def search_batch(self, inputs, metadata: Optional[FilterbankMetadata], beams, coarse_channels,
                     max_drift: float, min_drift: float, snr_threshold: float, stream=None) -> list:
        """Batched Dedopplerer::search: one list of DedopplerHit per input."""
        meta = metadata or FilterbankMetadata(foff=self.foff, tsamp=self.tsamp,
                                              coarse_channel_size=self.num_channels)
        res = self.search_batch_raw(inputs, beams, coarse_channels, max_drift, min_drift, snr_threshold, stream)
        out = [[DedopplerHit.make(meta, h.index, h.drift_steps, h.drift_rate, h.snr, b, c, self.num_timesteps,
                                  h.power) for h in hits]
               for hits, b, c in zip(res, beams, coarse_channels)]
        if self.print_hits:
            for hits in out:
                for hit in hits:
                    print("hit: " + hit.toString())
        return out

    def search(self, input, metadata: Optional[FilterbankMetadata], beam: int, coarse_channel: int,
               max_drift: float, min_drift: float, snr_threshold: float,
               output: Optional[list] = None, stream=None) -> list:
        """Dedopplerer::search (dedoppler.cu:186-320); appends to `output` and returns it."""
        if output is None:
            output = []
        meta = metadata or FilterbankMetadata(foff=self.foff, tsamp=self.tsamp,
                                              coarse_channel_size=self.num_channels)
        for h in self.search_raw(input, beam, coarse_channel, max_drift, min_drift, snr_threshold, stream):
            hit = DedopplerHit.make(meta, h.index, h.drift_steps, h.drift_rate, h.snr, beam,
                                    coarse_channel, self.num_timesteps, h.power)
            if self.print_hits:
                print("hit: " + hit.toString())
            output.append(hit)
        return output

    def addIncoherentPower(self, input, hits: list, stream=None) -> None:
        """Dedopplerer::addIncoherentPower (dedoppler.cu:139-176): sorts `hits` by
        drift_steps (as the reference does) and fills incoherent_power."""
        t = _device_input(input, self.rounded_num_timesteps, self.num_channels)
        hits.sort(key=lambda h: h.drift_steps)
        if not hits:
            return
        arr = (_capi.ScDdHit * len(hits))()
        for i, h in enumerate(hits):
            arr[i].index = h.index
            arr[i].drift_steps = h.drift_steps
        check(lib().sc_dd_add_incoherent_power(self._h, ctypes.c_void_p(t.data_ptr()), t.stride(0), arr,
                                               len(hits), _stream_handle(stream)))
        for i, h in enumerate(hits):
            h.incoherent_power = arr[i].incoherent_power

    add_incoherent_power = addIncoherentPower

    def last_stats(self) -> _capi.ScDdStats:
        s = _capi.ScDdStats()
        check(lib().sc_dd_last_stats(self._h, ctypes.byref(s)))
        return s

    def channel_array(self, which: str):
        """Copy of the last search's per-channel 'top' path sums or 'colsum' column sums."""
        import torch
        out = torch.empty(self.num_channels, dtype=torch.float32, device="cuda")
        check(lib().sc_dd_copy_channel_array(self._h, {"top": 0, "colsum": 1, "top16": 2}[which],
                                             ctypes.c_void_p(out.data_ptr()), _stream_handle(None)))
        return out
