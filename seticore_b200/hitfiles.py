"""Hit output files: the .dat text table and the .hits Cap'n Proto stream.

  * DatFileWriter      -- dat_file_writer.cpp:14-73 (header lines, one tab-separated row per hit)
  * HitFileWriter      -- hit_file_writer.cpp:18-97 (one Hit message per hit, written to
                          <name>.tmp and renamed on close; each carries the hit's Signal and a
                          Filterbank slice of the input, 40 extra columns either side)
  * makeHitRecorder    -- hit_recorder.cpp:10-23 (chooses by file suffix)
  * read_hits          -- what hitls.cpp reads: the Hit messages of a .hits file

The Cap'n Proto encoding is written here from the published wire format (no capnp library
is needed): an unpacked message is a segment table (segment count - 1, then each segment's
size in words, padded to 8 bytes) followed by the segments; a struct pointer holds
(offset << 2 | 0, data words, pointer words), a list pointer (offset << 2 | 1, element size
code, element count).  The struct layouts follow hit.capnp's field order under capnp's
slot allocation and agree with the generated accessors (hit.capnp.h):

  Signal     data 6 words:  frequency f64 @w0, index i32 @s2, driftSteps i32 @s3,
                            driftRate f64 @w2, snr f32 @s6, coarseChannel i32 @s7,
                            beam i32 @s8, numTimesteps i32 @s9, power f32 @s10,
                            incoherentPower f32 @s11
  Filterbank data 9 words, 2 pointers:  fch1, foff, tstart, tsamp, ra, dec f64 @w0..w5,
                            telescopeId i32 @s12, numTimesteps @s13, numChannels @s14,
                            coarseChannel @s15, startChannel @s16, beam @s17;
                            sourceName text @p0, data List(Float32) @p1
  Hit        pointers 2:    signal @p0, filterbank @p1

(w = 64-bit word, s = 32-bit slot).  Objects are laid out in the order a MallocMessageBuilder
allocates them in HitFileWriter::recordHit -- root pointer, Hit, Signal, Filterbank, source
name, data -- in one segment, so the bytes match the reference writer's for messages that fit
its first segment (1024 words).  The filterbank slice is gathered on the GPU
(sc_dd_gather_columns) when the input is a device tensor.
"""
import os
import struct
from typing import List, Optional

import numpy as np

EXTRA_COLUMNS = 40  # hit_file_writer.cpp:16

# Struct sizes (data words, pointer words) of the current schema.
LAYOUT = {"Signal": (6, 0), "Filterbank": (9, 2), "Hit": (0, 2)}

# (field, kind, byte offset in the data section) -- kind: d f64, i i32, f f32
SIGNAL_FIELDS = [("frequency", "d", 0), ("index", "i", 8), ("driftSteps", "i", 12), ("driftRate", "d", 16),
                 ("snr", "f", 24), ("coarseChannel", "i", 28), ("beam", "i", 32), ("numTimesteps", "i", 36),
                 ("power", "f", 40), ("incoherentPower", "f", 44)]
FILTERBANK_FIELDS = [("fch1", "d", 0), ("foff", "d", 8), ("tstart", "d", 16), ("tsamp", "d", 24), ("ra", "d", 32),
                     ("dec", "d", 40), ("telescopeId", "i", 48), ("numTimesteps", "i", 52),
                     ("numChannels", "i", 56), ("coarseChannel", "i", 60), ("startChannel", "i", 64),
                     ("beam", "i", 68)]
_FMT = {"d": "<d", "i": "<i", "f": "<f"}


# ---------------------------------------------------------------- encoder

def _struct_ptr(offset: int, data_words: int, ptr_words: int) -> int:
    return ((offset & 0x3FFFFFFF) << 2) | (data_words << 32) | (ptr_words << 48)


def _list_ptr(offset: int, size_code: int, count: int) -> int:
    return 1 | ((offset & 0x3FFFFFFF) << 2) | (size_code << 32) | (count << 35)


class _Segment:
    def __init__(self):
        self.words = bytearray()

    def alloc(self, n_words: int) -> int:
        at = len(self.words) // 8
        self.words += b"\0" * (8 * n_words)
        return at

    def put_ptr(self, at_word: int, value: int):
        struct.pack_into("<Q", self.words, 8 * at_word, value)

    def point_struct(self, ptr_word: int, target: int, dw: int, pw: int):
        self.put_ptr(ptr_word, _struct_ptr(target - ptr_word - 1, dw, pw))

    def point_list(self, ptr_word: int, target: int, size_code: int, count: int):
        self.put_ptr(ptr_word, _list_ptr(target - ptr_word - 1, size_code, count))


def _fill(seg: _Segment, at_word: int, data_words: int, fields, values: dict):
    base = 8 * at_word
    for name, kind, off in fields:
        if off + struct.calcsize(_FMT[kind]) > 8 * data_words:
            continue  # not in this layout
        v = values.get(name, 0)
        struct.pack_into(_FMT[kind], seg.words, base + off, float(v) if kind in "df" else int(v))


def _put_signal(seg: _Segment, ptr_word: int, signal: dict, layout):
    sdw, spw = layout["Signal"]
    s = seg.alloc(sdw + spw)
    seg.point_struct(ptr_word, s, sdw, spw)
    _fill(seg, s, sdw, SIGNAL_FIELDS, signal)


def _put_filterbank(seg: _Segment, ptr_word: int, filterbank: dict, layout):
    fdw, fpw = layout["Filterbank"]
    f = seg.alloc(fdw + fpw)
    seg.point_struct(ptr_word, f, fdw, fpw)
    name = filterbank.get("sourceName", "").encode() + b"\0"
    t = seg.alloc((len(name) + 7) // 8)
    seg.point_list(f + fdw + 0, t, 2, len(name))
    seg.words[8 * t: 8 * t + len(name)] = name
    _fill(seg, f, fdw, FILTERBANK_FIELDS, filterbank)
    data = np.ascontiguousarray(filterbank.get("data", np.zeros(0, np.float32)), dtype="<f4").ravel()
    d = seg.alloc((data.size + 1) // 2)
    seg.point_list(f + fdw + 1, d, 4, data.size)
    seg.words[8 * d: 8 * d + 4 * data.size] = data.tobytes()


def _frame(seg: _Segment) -> bytes:
    return struct.pack("<II", 0, len(seg.words) // 8) + bytes(seg.words)


def encode_hit(signal: Optional[dict], filterbank: Optional[dict], layout=LAYOUT) -> bytes:
    """One Hit message (unpacked stream framing).  `filterbank["data"]` is a float32 array
    of numTimesteps x numChannels values (row-major) and `filterbank["sourceName"]` a str.
    Allocation order of HitFileWriter::recordHit: Hit, Signal, Filterbank, name, data."""
    seg = _Segment()
    root = seg.alloc(1)
    hdw, hpw = layout["Hit"]
    hit = seg.alloc(hdw + hpw)
    seg.point_struct(root, hit, hdw, hpw)
    if signal is not None:
        _put_signal(seg, hit + hdw + 0, signal, layout)
    if filterbank is not None:
        _put_filterbank(seg, hit + hdw + 1, filterbank, layout)
    return _frame(seg)


def encode_event(hits, layout=LAYOUT) -> bytes:
    """One Event message (hit.capnp: Event { hits @0 :List(Hit) }) for a list of
    (signal or None, filterbank) pairs.  Allocation order of EventFileWriter::write
    (event_file_writer.cpp:36-70): Event, the composite list of Hits, then per hit its
    Filterbank (name, data) followed by its Signal."""
    seg = _Segment()
    root = seg.alloc(1)
    event = seg.alloc(1)  # Event: 0 data words, 1 pointer
    seg.point_struct(root, event, 0, 1)
    hdw, hpw = layout["Hit"]
    n = len(hits)
    tag = seg.alloc(1 + n * (hdw + hpw))
    seg.point_list(event, tag, 7, n * (hdw + hpw))
    seg.put_ptr(tag, _struct_ptr(n, hdw, hpw))  # composite-list tag: element count and size
    for i, (signal, filterbank) in enumerate(hits):
        h = tag + 1 + i * (hdw + hpw)
        _put_filterbank(seg, h + hdw + 1, filterbank, layout)
        if signal is not None:
            _put_signal(seg, h + hdw + 0, signal, layout)
    return _frame(seg)


# ---------------------------------------------------------------- decoder

def _read_struct(seg: bytes, ptr_word: int):
    v = struct.unpack_from("<Q", seg, 8 * ptr_word)[0]
    if v == 0:
        return None
    if v & 3 != 0:
        raise ValueError("expected a struct pointer")
    off = (v >> 2) & 0x3FFFFFFF
    if off & 0x20000000:
        off -= 0x40000000
    return ptr_word + 1 + off, (v >> 32) & 0xFFFF, (v >> 48) & 0xFFFF


def _read_list(seg: bytes, ptr_word: int):
    v = struct.unpack_from("<Q", seg, 8 * ptr_word)[0]
    if v == 0:
        return None
    if v & 3 != 1:
        raise ValueError("expected a list pointer")
    off = (v >> 2) & 0x3FFFFFFF
    if off & 0x20000000:
        off -= 0x40000000
    return ptr_word + 1 + off, (v >> 32) & 7, v >> 35


def _get(seg, at, dw, fields):
    out = {}
    for name, kind, off in fields:
        size = struct.calcsize(_FMT[kind])
        out[name] = struct.unpack_from(_FMT[kind], seg, 8 * at + off)[0] if off + size <= 8 * dw else 0
    return out


def decode_hit(seg: bytes, ptr_word: int = 0) -> dict:
    """The Signal and Filterbank of a Hit whose struct pointer is at ptr_word (0: the root
    of a single-segment Hit message).  Fields missing from an older, smaller layout read as
    zero, as capnp's schema evolution defines."""
    r = _read_struct(seg, ptr_word)
    hit, hdw, hpw = r
    return _decode_hit_at(seg, hit, hdw, hpw)


def _decode_hit_at(seg: bytes, hit: int, hdw: int, hpw: int) -> dict:
    out = {"signal": None, "filterbank": None}
    if hpw > 0:
        s = _read_struct(seg, hit + hdw + 0)
        if s:
            out["signal"] = _get(seg, s[0], s[1], SIGNAL_FIELDS)
            out["signal"]["_layout"] = (s[1], s[2])
    if hpw > 1:
        f = _read_struct(seg, hit + hdw + 1)
        if f:
            at, dw, pw = f
            fb = _get(seg, at, dw, FILTERBANK_FIELDS)
            fb["_layout"] = (dw, pw)
            t = _read_list(seg, at + dw + 0) if pw > 0 else None
            fb["sourceName"] = bytes(seg[8 * t[0]: 8 * t[0] + t[2] - 1]).decode() if t else ""
            d = _read_list(seg, at + dw + 1) if pw > 1 else None
            fb["data"] = (np.frombuffer(seg, dtype="<f4", count=d[2], offset=8 * d[0]).copy()
                          if d else np.zeros(0, np.float32))
            out["filterbank"] = fb
    return out


def decode_event(seg: bytes) -> List[dict]:
    """The Hits of one single-segment Event message."""
    ev = _read_struct(seg, 0)
    lst = _read_list(seg, ev[0] + ev[1])
    if lst is None:
        return []
    at, size_code, _ = lst
    if size_code != 7:
        raise ValueError("Event.hits is not a composite list")
    tag = struct.unpack_from("<Q", seg, 8 * at)[0]
    n, dw, pw = (tag >> 2) & 0x3FFFFFFF, (tag >> 32) & 0xFFFF, (tag >> 48) & 0xFFFF
    return [_decode_hit_at(seg, at + 1 + i * (dw + pw), dw, pw) for i in range(n)]


def split_messages(blob: bytes):
    """Yields (raw message bytes, first segment) for each message of a stream."""
    off = 0
    while off < len(blob):
        nseg = struct.unpack_from("<I", blob, off)[0] + 1
        sizes = struct.unpack_from("<%dI" % nseg, blob, off + 4)
        head = (4 + 4 * nseg + 7) // 8 * 8
        if nseg != 1:
            raise ValueError("multi-segment messages are not supported by this reader")
        end = off + head + 8 * sum(sizes)
        yield blob[off:end], blob[off + head: end]
        off = end


def read_hits(filename: str) -> List[dict]:
    """Every Hit message of a .hits file (hitls.cpp:33-51 reads the same fields)."""
    with open(filename, "rb") as fh:
        blob = fh.read()
    return [decode_hit(seg) for _, seg in split_messages(blob)]


# ---------------------------------------------------------------- writers

def _slice_bounds(hit, coarse_channel_size: int):
    """[begin, end) of the stored columns: hit_file_writer.cpp:82-86 (end keeps the
    reference's `- 1`)."""
    begin = max(hit.lowIndex() - EXTRA_COLUMNS, 0)
    end = min(hit.highIndex() + EXTRA_COLUMNS, coarse_channel_size) - 1
    return begin, end


def gather_ranges(input, metadata, bounds) -> List[np.ndarray]:
    """The [num_timesteps][end - begin] slice of `input` for each (begin, end).  A CUDA
    tensor input is gathered by one kernel launch (sc_dd_gather_columns) and copied back
    once; a host array is sliced directly."""
    T = int(metadata.num_timesteps)
    N = int(metadata.coarse_channel_size)
    if hasattr(input, "is_cuda") and input.is_cuda:
        from .dedoppler import gather_hit_slices
        return gather_hit_slices(input, T, N, bounds)
    x = np.asarray(input, dtype=np.float32).reshape(-1, N)
    return [np.ascontiguousarray(x[:T, b:e]) for b, e in bounds]


def gather_slices(hits, input, metadata) -> List[np.ndarray]:
    """The slice a .hits file stores with each hit (gather_ranges of _slice_bounds)."""
    return gather_ranges(input, metadata, [_slice_bounds(h, int(metadata.coarse_channel_size)) for h in hits])


class HitRecorder:
    """hit_recorder.h: recordHit(hit, input); recordHits batches the slice gather."""

    def recordHit(self, hit, input) -> None:
        self.recordHits([hit], input)

    def recordHits(self, hits, input) -> None:
        raise NotImplementedError

    def close(self) -> None:
        pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class DatFileWriter(HitRecorder):
    """dat_file_writer.cpp:14-73."""

    def __init__(self, filename: str, metadata, max_drift: float):
        self.metadata = metadata
        self.hit_count = 0
        self.file = open(filename, "w")
        m = metadata
        f = self.file
        f.write("# -------------------------- o --------------------------\n")
        f.write("# File ID: " + filename.split("/")[-1] + " \n")
        f.write("# -------------------------- o --------------------------\n")
        f.write("# Source:" + m.source_name + "\n")
        f.write(f"# MJD: {m.tstart:18.12f}\tRA: {m.src_raj:.6f}\tDEC: {m.src_dej:.6f}\n")
        f.write(f"# DELTAT: {m.tsamp:10.6f}\tDELTAF(Hz): {m.foff * 1000000.0:10.6f}\t"
                f"max_drift_rate: {max_drift:10.6f}\tobs_length: {m.num_timesteps * m.tsamp:10.6f}\n")
        f.write("# --------------------------\n"
                "# Top_Hit_# \tDrift_Rate \tSNR \tUncorrected_Frequency \tCorrected_Frequency \tIndex \t"
                "freq_start \tfreq_end \tSEFD \tSEFD_freq \tCoarse_Channel_Number \tFull_number_of_hits \t\n"
                "# --------------------------\n")
        f.flush()

    def recordHits(self, hits, input=None) -> None:
        m = self.metadata
        for hit in hits:
            self.hit_count += 1
            global_index = hit.coarse_channel * m.coarse_channel_size + hit.index
            frequency = m.fch1 + global_index * m.foff
            self.file.write(f"{self.hit_count}\t{hit.drift_rate:10.6f}\t{hit.snr:10.6f}\t{frequency:14.6f}\t"
                            f"{frequency:14.6f}\t{hit.index}\t{frequency:14.6f}\t{frequency:14.6f}\t")
            self.file.write(f"0.0\t0.000000\t{hit.coarse_channel}\t1\t\n")
        self.file.flush()

    def close(self) -> None:
        if not self.file.closed:
            self.file.close()


def signal_fields(hit) -> dict:
    """buildSignal (hit_file_writer.cpp:49-60)."""
    return {"frequency": hit.frequency, "index": hit.index, "driftSteps": hit.drift_steps,
            "driftRate": hit.drift_rate, "snr": hit.snr, "coarseChannel": hit.coarse_channel, "beam": hit.beam,
            "numTimesteps": hit.num_timesteps, "power": hit.power, "incoherentPower": hit.incoherent_power}


def filterbank_fields(metadata, beam: int, coarse_channel: int, begin: int, end: int, data) -> dict:
    """buildFilterbank (hit_file_writer.cpp:62-97) for the columns [begin, end)."""
    m = metadata
    coarse_offset = coarse_channel * m.coarse_channel_size
    return {"sourceName": m.getBeamSourceName(beam), "ra": m.getBeamRA(beam), "dec": m.getBeamDec(beam),
            "telescopeId": m.telescope_id, "foff": m.foff, "tsamp": m.tsamp, "tstart": m.tstart,
            "numTimesteps": m.num_timesteps, "coarseChannel": coarse_channel, "beam": beam,
            "numChannels": end - begin, "fch1": m.fch1 + (coarse_offset + begin) * m.foff,
            "startChannel": begin, "data": data}


class HitFileWriter(HitRecorder):
    """hit_file_writer.cpp:18-47: appends one Hit message per hit to <filename>.tmp and
    renames it to <filename> on close."""

    def __init__(self, filename: str, metadata):
        self.metadata = metadata
        self.final_filename = filename
        self.tmp_filename = filename + ".tmp"
        fd = os.open(self.tmp_filename, os.O_WRONLY | os.O_CREAT, 0o664)
        self.file = os.fdopen(fd, "wb")

    def recordHits(self, hits, input) -> None:
        hits = list(hits)
        if not hits:
            return
        slices = gather_slices(hits, input, self.metadata)
        for hit, data in zip(hits, slices):
            b, e = _slice_bounds(hit, int(self.metadata.coarse_channel_size))
            self.file.write(encode_hit(signal_fields(hit),
                                       filterbank_fields(self.metadata, hit.beam, hit.coarse_channel, b, e, data)))

    def close(self) -> None:
        if not self.file.closed:
            self.file.close()
            os.replace(self.tmp_filename, self.final_filename)


def makeHitRecorder(filename: str, metadata, max_drift: float) -> HitRecorder:
    """hit_recorder.cpp:10-23."""
    if filename.endswith(".dat"):
        return DatFileWriter(filename, metadata, max_drift)
    if filename.endswith(".hits"):
        return HitFileWriter(filename, metadata)
    raise ValueError(f"could not recognize the file type of {filename}")
