"""End to end: a filterbank file to a hit file (run_dedoppler.cpp:30-53).

  * FilterbankFileReader / loadFilterbankFile -- filterbank_file_reader.cpp:11-28
  * FilReader            -- fil_reader.cpp:16-139 (sigproc header); its loadCoarseChannel,
                            a stub in the reference (fil_reader.cpp:151-154), reads the
                            coarse channel's columns of every row here
  * ArrayFilterbankFile  -- an in-memory file: the "non-file object that satisfies the
                            FilterbankFile interface" run_dedoppler.cpp:24-28 suggests
  * runDedoppler         -- run_dedoppler.cpp:30-53, pipelined over coarse channels

HDF5 (.h5) input needs libhdf5 and its filter plugins, which this package does not link;
loadFilterbankFile raises for it.

runDedoppler keeps three stages in flight: a host thread reads coarse channels j+2 into a
pinned buffer, a copy stream moves channels j+1 to the device, and the search runs on
channels j (a batch of `batch` coarse channels per call).  Padding rows and the DC-spike
fix are applied on the device (sc_dd_prepare_coarse_channels), which the reference does on
the host inside loadCoarseChannel (h5_reader.cpp:190-209).
"""
import os
import struct
import threading
from concurrent.futures import ThreadPoolExecutor
from typing import Optional

import numpy as np

from .dedoppler import (NO_BEAM, Dedopplerer, FilterbankMetadata, prepare_coarse_channels,
                        roundUpToPowerOfTwo)
from .hitfiles import makeHitRecorder

NO_TELESCOPE_ID = -1  # util.h:14
GREEN_BANK = 6        # util.h:16
ATA = 9               # util.h:17


def convertFromSigprocRaOrDec(sigproc: float) -> float:
    """HHMMSS.S (or DDMMSS.S) to hours (degrees) with a fraction (fil_reader.cpp:16-25)."""
    negative = sigproc < 0
    a = abs(sigproc)
    whole = int(np.floor(a / 10000.0))
    remnant = a - whole * 10000.0
    minutes = int(np.floor(remnant / 100.0))
    seconds = remnant - minutes * 100.0
    ans = whole + minutes / 60.0 + seconds / 3600.0
    return -ans if negative else ans


class FilterbankFileReader(FilterbankMetadata):
    """Metadata plus loadCoarseChannel (filterbank_file_reader.h)."""

    filename: str = ""

    def loadCoarseChannel(self, i: int, out: np.ndarray) -> None:
        """Copies rows [0, num_timesteps) of coarse channel i into out[:num_timesteps]."""
        raise NotImplementedError(f"cannot loadCoarseChannel from a base FilterbankFileReader: {self.filename}")

    def _infer_green_bank(self, nfpc: int) -> bool:  # filterbank_metadata.cpp:53-63
        if self.num_timesteps in (16, 32, 15) and self.num_channels % nfpc == 0:
            if self.coarse_channel_size == 0:
                self.coarse_channel_size = nfpc
            self.has_dc_spike = True
            return True
        return False

    def inferMetadata(self) -> None:
        """coarse_channel_size, has_dc_spike and num_coarse_channels from the other fields
        (filterbank_metadata.cpp:71-93)."""
        if self._infer_green_bank(1048576) or self._infer_green_bank(1033216) or self._infer_green_bank(999424):
            assert self.telescope_id in (NO_TELESCOPE_ID, GREEN_BANK)
        elif self.num_channels == 50331648:
            assert self.telescope_id in (NO_TELESCOPE_ID, ATA)
            if self.coarse_channel_size == 0:
                self.coarse_channel_size = 262144
            self.has_dc_spike = False
        elif self.coarse_channel_size > 0:
            self.has_dc_spike = self.telescope_id == GREEN_BANK
        else:
            raise ValueError(f"unable to infer coarse channel size for data with dimensions: "
                             f"{self.num_timesteps} x {self.num_channels}. please set the nfpc header.")
        self.num_coarse_channels = self.num_channels // self.coarse_channel_size


class ArrayFilterbankFile(FilterbankFileReader):
    """A filterbank held in a [num_timesteps][num_channels] float32 array (host memory or a
    numpy memmap) with the given metadata fields."""

    def __init__(self, data: np.ndarray, infer: bool = True, **metadata):
        super().__init__(**metadata)
        self.data = data
        self.num_timesteps, self.num_channels = int(data.shape[0]), int(data.shape[1])
        if infer:
            self.inferMetadata()
        else:
            self.num_coarse_channels = self.num_channels // self.coarse_channel_size

    def loadCoarseChannel(self, i: int, out: np.ndarray) -> None:
        n = self.coarse_channel_size
        out[: self.num_timesteps] = self.data[:, i * n:(i + 1) * n]


_INT_ATTRS = {"telescope_id", "machine_id", "data_type", "barycentric", "pulsarcentric", "nbits", "nsamples",
              "nchans", "nifs", "nbeams", "ibeam"}
_DOUBLE_ATTRS = {"az_start", "za_start", "tstart", "tsamp", "fch1", "foff", "refdm", "period", "src_raj", "src_dej"}
_STRING_ATTRS = {"rawdatafile", "source_name"}


class FilReader(FilterbankFileReader):
    """A sigproc filterbank (.fil) file of 32-bit floats (fil_reader.cpp:27-139)."""

    def __init__(self, filename: str):
        super().__init__()
        self.filename = filename
        with open(filename, "rb") as f:
            def read_string():
                n = struct.unpack("<I", f.read(4))[0]
                if n >= 256:
                    raise ValueError(f"{filename}: header string of {n} bytes")
                return f.read(n).decode("latin-1")

            if read_string() != "HEADER_START":
                raise ValueError(f"The file {filename} did not start with HEADER_START. Is it really a .fil file?")
            while True:
                name = read_string()
                if name == "HEADER_END":
                    break
                if name in _INT_ATTRS:
                    v = struct.unpack("<i", f.read(4))[0]
                    if name == "telescope_id":
                        self.telescope_id = v
                    elif name == "nbits" and v != 32:
                        raise ValueError(f"{filename}: only 32-bit float data is handled (nbits = {v})")
                    elif name == "nsamples":
                        self.num_timesteps = v
                    elif name == "nchans":
                        self.num_channels = v
                elif name in _DOUBLE_ATTRS:
                    v = struct.unpack("<d", f.read(8))[0]
                    if name in ("src_raj", "src_dej"):
                        v = convertFromSigprocRaOrDec(v)
                    if name in ("tstart", "tsamp", "fch1", "foff", "src_raj", "src_dej"):
                        setattr(self, name, v)
                elif name in _STRING_ATTRS:
                    v = read_string()
                    if name == "source_name":
                        self.source_name = v
                else:
                    raise ValueError(f"unhandled attr name: {name}")
            self.data_start = f.tell()
            f.seek(0, os.SEEK_END)
            nbytes = f.tell() - self.data_start
        if nbytes % 4:
            raise ValueError(f"indivisible amount of data is {nbytes} bytes")
        nfloats = nbytes // 4
        if nfloats % self.num_channels:
            raise ValueError(f"we have {nfloats} which does not divide into {self.num_channels} frequencies")
        inferred = nfloats // self.num_channels
        if self.num_timesteps == 0:
            self.num_timesteps = inferred
        elif self.num_timesteps != inferred:
            raise ValueError(f"header num timesteps is {self.num_timesteps} but inferred num timesteps is {inferred}")
        self.inferMetadata()
        self.data = np.memmap(filename, dtype="<f4", mode="r", offset=self.data_start,
                              shape=(self.num_timesteps, self.num_channels))

    def loadCoarseChannel(self, i: int, out: np.ndarray) -> None:
        n = self.coarse_channel_size
        out[: self.num_timesteps] = self.data[:, i * n:(i + 1) * n]


def write_fil(filename: str, data: np.ndarray, metadata: FilterbankMetadata) -> None:
    """Writes a sigproc .fil file of float32 [num_timesteps][num_channels] (the header fields
    FilReader reads; src_raj / src_dej are written in HHMMSS.S form)."""

    def to_sigproc(x):
        neg = x < 0
        a = abs(x)
        h = int(a)
        m = int((a - h) * 60)
        s = (a - h - m / 60.0) * 3600.0
        v = h * 10000.0 + m * 100.0 + s
        return -v if neg else v

    def s(x):
        b = x.encode("latin-1")
        return struct.pack("<I", len(b)) + b

    data = np.ascontiguousarray(data, dtype="<f4")
    h = s("HEADER_START")
    h += s("telescope_id") + struct.pack("<i", metadata.telescope_id)
    h += s("source_name") + s(metadata.source_name)
    for name, v in [("tstart", metadata.tstart), ("tsamp", metadata.tsamp), ("fch1", metadata.fch1),
                    ("foff", metadata.foff), ("src_raj", to_sigproc(metadata.src_raj)),
                    ("src_dej", to_sigproc(metadata.src_dej))]:
        h += s(name) + struct.pack("<d", v)
    h += s("nbits") + struct.pack("<i", 32) + s("nchans") + struct.pack("<i", data.shape[1])
    h += s("nifs") + struct.pack("<i", 1) + s("HEADER_END")
    with open(filename, "wb") as f:
        f.write(h)
        f.write(data.tobytes())


def loadFilterbankFile(filename: str) -> FilterbankFileReader:
    """filterbank_file_reader.cpp:17-28."""
    if filename.endswith(".h5"):
        raise RuntimeError(f"{filename}: HDF5 filterbank files need libhdf5, which this package does not link")
    if filename.endswith(".fil"):
        return FilReader(filename)
    raise ValueError(f"could not recognize the file type of {filename}")


def runDedoppler(input, output_filename: str, max_drift: float, min_drift: float, snr_threshold: float,
                 batch: int = 8, print_hits: bool = True, recorder=None) -> list:
    """Searches every coarse channel of `input` (a file name or a FilterbankFileReader) and
    records the hits in output_filename (.dat or .hits).  Returns the hits in the order
    they were recorded: coarse channel by coarse channel, each in search order."""
    import torch
    f = loadFilterbankFile(input) if isinstance(input, str) else input
    own_recorder = recorder is None
    if own_recorder:
        recorder = makeHitRecorder(output_filename, f, max_drift)
    T, N = int(f.num_timesteps), int(f.coarse_channel_size)
    Tr = roundUpToPowerOfTwo(T)
    dd = Dedopplerer(T, N, f.foff, f.tsamp, f.has_dc_spike)
    dd.print_hits = print_hits
    n_coarse = int(f.num_coarse_channels)
    B = max(1, min(batch, n_coarse, 64))
    chunks = [(j, min(B, n_coarse - j)) for j in range(0, n_coarse, B)]
    pinned = [torch.empty((B, T, N), dtype=torch.float32, pin_memory=True) for _ in range(2)]
    dev = [torch.empty((B, Tr, N), dtype=torch.float32, device="cuda") for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    compute = torch.cuda.current_stream()
    h2d_done = [torch.cuda.Event() for _ in range(2)]
    h2d_issued = [False, False]
    all_hits = []

    def load(ci):
        b = ci % 2
        if h2d_issued[b]:
            h2d_done[b].synchronize()  # the previous copy out of this pinned buffer has finished
        j, m = chunks[ci]
        host = pinned[b].numpy()
        for k in range(m):
            f.loadCoarseChannel(j + k, host[k])

    def issue_h2d(ci):
        b = ci % 2
        j, m = chunks[ci]
        with torch.cuda.stream(copy_stream):
            dev[b][:m, :T].copy_(pinned[b][:m], non_blocking=True)
            h2d_done[b].record(copy_stream)
        h2d_issued[b] = True

    try:
        with ThreadPoolExecutor(max_workers=1) as pool:
            load(0)
            issue_h2d(0)
            nxt = pool.submit(load, 1) if len(chunks) > 1 else None
            for ci, (j, m) in enumerate(chunks):
                b = ci % 2
                if ci + 1 < len(chunks):
                    nxt.result()
                    issue_h2d(ci + 1)  # overlaps this chunk's search
                    nxt = pool.submit(load, ci + 2) if ci + 2 < len(chunks) else None
                compute.wait_event(h2d_done[b])
                prepare_coarse_channels(dev[b][:m], T, f.has_dc_spike, stream=compute)
                inputs = [dev[b][k] for k in range(m)]
                res = dd.search_batch(inputs, f, [NO_BEAM] * m, list(range(j, j + m)), max_drift, min_drift,
                                      snr_threshold, stream=compute)
                for k in range(m):
                    recorder.recordHits(res[k], dev[b][k])
                    all_hits.extend(res[k])
    finally:
        dd.close()
        if own_recorder:
            recorder.close()
    return all_hits
