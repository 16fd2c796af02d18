"""Cadence event search (find_events.cpp:54-226): hits that appear in every "on"
observation of an ABACAD cadence, drifting consistently, and in no "off" observation.

  * findHit              -- find_events.cpp:26-45, including its behaviour of returning the
                            first hit at or after low_index even when it lies past
                            high_index
  * removeZeroDriftHits  -- find_events.cpp:47-53
  * match_events         -- the candidate loop of findEvents (find_events.cpp:154-224) on
                            per-file hit lists of one coarse channel, host logic
  * EventFileWriter      -- event_file_writer.cpp:17-70 (Event messages, .events files)
  * findEvents           -- find_events.cpp:64-226 with the searches on the GPU: file 0
                            alone first (a coarse channel without hits there is skipped, as
                            in the reference), then the other "on" files in one batched call
                            at snr_on and the "off" files in one at snr_off
"""
import bisect
import os
from typing import List, Optional, Sequence

from .dedoppler import NO_BEAM, DedopplerHit, Dedopplerer, _round_half_away, roundUpToPowerOfTwo
from .hitfiles import EXTRA_COLUMNS, encode_event, filterbank_fields, gather_ranges, signal_fields


def findHit(keys: Sequence[int], hits_by_key: dict, low_index: int, high_index: int):
    """(count, hit): count is 0, 1 or 2 (two or more); hit only when count is 1.  keys is
    the sorted list of hit start indices of one file."""
    i = bisect.bisect_left(keys, low_index)
    if i == len(keys):
        return 0, None
    answer = (1, hits_by_key[keys[i]])
    if i + 1 == len(keys) or keys[i + 1] > high_index:
        return answer
    return 2, None


def removeZeroDriftHits(hits: list) -> list:
    return [h for h in hits if h.drift_steps != 0]


def match_events(hit_lists: List[list], tstarts: Sequence[float], tsamp: float, coarse_channel_size: int):
    """The events of one coarse channel: a list of candidates, each a list parallel to the
    files holding the matched hit (None for the "off" files)."""
    maps = []
    for hits in hit_lists:
        m = {}
        for h in hits:
            m[h.index] = h  # a later hit with the same index replaces an earlier one, as std::map[] does
        maps.append((sorted(m), m))
    events = []
    t0 = tstarts[0]
    for key in maps[0][0]:
        initial = maps[0][1][key]
        ok = True
        low, high = 2 ** 31 - 1, -1
        for i in range(0, len(maps), 2):
            timesteps = int(_round_half_away((tstarts[i] - t0) / tsamp))
            expected = initial.expectedIndex(timesteps)
            count, hit = findHit(maps[i][0], maps[i][1], expected - 10, expected + 10)
            if count != 1:
                ok = False
                break
            low = min(low, hit.lowIndex())
            high = max(high, hit.highIndex())
        if not ok:
            continue
        assert low < coarse_channel_size and high >= 0
        candidate, good = [], True
        for i in range(len(maps)):
            ideal = 1 if i % 2 == 0 else 0
            # find_events.cpp:205 passes high_index - wiggle as the upper end; kept.
            count, hit = findHit(maps[i][0], maps[i][1], low - 50, high - 50)
            if count != ideal:
                good = False
                break
            candidate.append(hit)
        if good:
            events.append(candidate)
    return events


class EventFileWriter:
    """event_file_writer.cpp:17-70: one Event message per candidate, written to
    <filename>.tmp and renamed on close."""

    def __init__(self, filename: str, metadatas: list):
        self.metadatas = metadatas
        self.final_filename = filename
        self.tmp_filename = filename + ".tmp"
        self.file = os.fdopen(os.open(self.tmp_filename, os.O_WRONLY | os.O_CREAT, 0o664), "wb")

    def write(self, hits: list, buffers: list) -> None:
        """hits: parallel to the files (None where a file has no hit); buffers: each file's
        coarse-channel input (device tensors or host arrays)."""
        assert len(hits) == len(self.metadatas) == len(buffers) and hits[0] is not None
        low = min(h.lowIndex() for h in hits if h is not None)
        high = max(h.highIndex() for h in hits if h is not None)
        beam, cc = hits[0].beam, hits[0].coarse_channel
        pairs = []
        for i, (h, m) in enumerate(zip(hits, self.metadatas)):
            # buildFilterbank gets the event's low and high index for every file
            # (hit_file_writer.cpp:82-86 bounds, "- 1" included)
            b = max(low - EXTRA_COLUMNS, 0)
            e = min(high + EXTRA_COLUMNS, int(m.coarse_channel_size)) - 1
            data = gather_ranges(buffers[i], m, [(b, e)])[0]
            pairs.append((signal_fields(h) if h is not None else None,
                          filterbank_fields(m, beam, cc, b, e, data)))
        self.file.write(encode_event(pairs))

    def close(self) -> None:
        if not self.file.closed:
            self.file.close()
            os.replace(self.tmp_filename, self.final_filename)

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def check_cadence(files) -> None:
    """The metadata checks of findEvents (find_events.cpp:95-122)."""
    f0 = files[0]
    for i, f in enumerate(files):
        assert f.num_timesteps == f0.num_timesteps and f.coarse_channel_size == f0.coarse_channel_size
        assert f.num_coarse_channels == f0.num_coarse_channels and f.has_dc_spike == f0.has_dc_spike
        assert abs(f.foff - f0.foff) <= 1e-6 * max(1.0, abs(f0.foff)) or f.foff == f0.foff
        assert abs(f.tsamp - f0.tsamp) <= 1e-6 * max(1.0, abs(f0.tsamp))
        if i % 2 == 0:
            if f.source_name != f0.source_name:
                raise ValueError(f"file {f.filename} has source {f.source_name} when we expected source "
                                 f"{f0.source_name}")
        elif f.source_name == f0.source_name and f0.source_name != "VOYAGER-1":
            raise ValueError(f"file {f.filename} has source {f.source_name} but it is supposed to be an 'off'")


def findEvents(inputs: list, output_filename: str, max_drift: float, snr_on: float, snr_off: float,
               verbose: bool = True) -> list:
    """Returns the events found (lists of hits parallel to the files) and writes them to
    output_filename.  inputs: file names or FilterbankFileReader objects."""
    import torch
    from .run_dedoppler import loadFilterbankFile
    files = [loadFilterbankFile(x) if isinstance(x, str) else x for x in inputs]
    check_cadence(files)
    f0 = files[0]
    T, N = int(f0.num_timesteps), int(f0.coarse_channel_size)
    Tr = roundUpToPowerOfTwo(T)
    dd = Dedopplerer(T, N, f0.foff, f0.tsamp, f0.has_dc_spike)
    from .dedoppler import prepare_coarse_channels
    host = torch.empty((len(files), T, N), dtype=torch.float32, pin_memory=True)
    dev = torch.empty((len(files), Tr, N), dtype=torch.float32, device="cuda")
    ons = [i for i in range(2, len(files), 2)]
    offs = [i for i in range(1, len(files), 2)]
    all_events = []
    writer = EventFileWriter(output_filename, files)
    try:
        for cc in range(int(f0.num_coarse_channels)):
            def load(idx):
                for i in idx:
                    files[i].loadCoarseChannel(cc, host[i].numpy())
                for i in idx:
                    dev[i, :T].copy_(host[i], non_blocking=True)
                    prepare_coarse_channels(dev[i], T, files[i].has_dc_spike)

            load([0])
            first = dd.search(dev[0], files[0], NO_BEAM, cc, max_drift, 0.0, snr_on)
            hit_lists = [removeZeroDriftHits(first)] + [[] for _ in files[1:]]
            if not hit_lists[0]:
                continue
            load(ons + offs)
            for group, snr, is_on in ((ons, snr_on, True), (offs, snr_off, False)):
                if not group:
                    continue
                res = dd.search_batch_raw([dev[i] for i in group], [NO_BEAM] * len(group), [cc] * len(group),
                                          max_drift, 0.0, snr)
                for i, raw in zip(group, res):
                    hits = [DedopplerHit.make(files[i], h.index, h.drift_steps, h.drift_rate, h.snr, NO_BEAM, cc,
                                              T, h.power) for h in raw]
                    hit_lists[i] = removeZeroDriftHits(hits) if is_on else hits
            events = match_events(hit_lists, [f.tstart for f in files], f0.tsamp, N)
            for ev in events:
                if verbose:
                    print("found event starting at " + ev[0].toString())
                writer.write(ev, [dev[i] for i in range(len(files))])
            if verbose:
                print(f"{len(events)} event{'' if len(events) == 1 else 's'} found in coarse channel "
                      f"{cc}/{f0.num_coarse_channels}")
            all_events.extend(events)
    finally:
        writer.close()
        dd.close()
    return all_events
