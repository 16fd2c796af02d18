"""The callers either side of the search on the GPU: coarse-channel preparation (padding
rows, DC spike), the hit-slice gather, runDedoppler over a multi-coarse-channel file with
.dat and .hits output, and the in-place multibeam band search."""
import numpy as np
import pytest

from tests.conftest import has_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch


def _prepared_host(rows, Tr, dc_spike):
    """What H5Reader::loadCoarseChannel leaves in the buffer (h5_reader.cpp:190-209)."""
    T, N = rows.shape
    out = np.zeros((Tr, N), np.float32)
    out[:T] = rows
    if dc_spike:
        mid = N // 2
        out[:T, mid] = (out[:T, mid - 1] + out[:T, mid + 1]) / np.float32(2.0)
    return out


def test_prepare_coarse_channels(torch_cuda):
    torch = torch_cuda
    from seticore_b200.dedoppler import prepare_coarse_channels
    rng = np.random.default_rng(5)
    for T, Tr, N, dc in [(13, 16, 1001, True), (16, 16, 4096, True), (5, 8, 3000, False), (31, 32, 65536, True)]:
        raw = rng.random((3, Tr, N), dtype=np.float32) * 1e9
        dev = torch.from_numpy(raw).cuda()
        prepare_coarse_channels(dev, T, dc)
        got = dev.cpu().numpy()
        for k in range(3):
            want = _prepared_host(raw[k, :T], Tr, dc)
            assert np.array_equal(got[k].view(np.uint32), want.view(np.uint32)), (T, N, k)


def test_gather_columns(torch_cuda):
    torch = torch_cuda
    from seticore_b200.dedoppler import gather_hit_slices
    rng = np.random.default_rng(6)
    x = rng.random((16, 5000), dtype=np.float32)
    big = np.zeros((16, 7000), np.float32)
    big[:, :5000] = x
    dev = torch.from_numpy(big).cuda()[:, :5000]  # row stride 7000
    bounds = [(0, 81), (4919, 4999), (100, 100), (2500, 2600), (0, 4999)]
    got = gather_hit_slices(dev, 13, 5000, bounds)
    for (b, e), g in zip(bounds, got):
        np.testing.assert_array_equal(g, x[:13, b:e])


def _coarse_file(n_coarse, T, N, seed):
    from seticore_b200.run_dedoppler import ArrayFilterbankFile
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    parts = []
    for k in range(n_coarse):
        spec = SearchSpec(T, N, seed=seed + k, n_tones=5, snr_threshold=8.0)
        parts.append(make_filterbank_numpy(spec)[:T])
    data = np.concatenate(parts, axis=1)
    return ArrayFilterbankFile(data, coarse_channel_size=N, telescope_id=6, fch1=8421.0, foff=spec.foff_mhz,
                               tsamp=spec.tsamp, source_name="synthetic", tstart=60000.5)


def _direct_hits(torch, f, max_drift, snr):
    from seticore_b200 import Dedopplerer
    from seticore_b200.dedoppler import roundUpToPowerOfTwo
    T, N = f.num_timesteps, f.coarse_channel_size
    Tr = roundUpToPowerOfTwo(T)
    dd = Dedopplerer(T, N, f.foff, f.tsamp, f.has_dc_spike)
    hits, prepared = [], []
    for c in range(f.num_coarse_channels):
        host = np.zeros((T, N), np.float32)
        f.loadCoarseChannel(c, host)
        p = _prepared_host(host, Tr, f.has_dc_spike)
        prepared.append(p)
        hits.extend(dd.search(torch.from_numpy(p).cuda(), f, -1, c, max_drift, 0.0, snr))
    dd.close()
    return hits, prepared


def _key(h):
    return (h.coarse_channel, h.index, h.drift_steps, np.float32(h.power), np.float32(h.snr), h.beam)


def test_run_dedoppler_dat_and_hits(torch_cuda, tmp_path):
    from seticore_b200.hitfiles import read_hits
    from seticore_b200.run_dedoppler import runDedoppler
    f = _coarse_file(6, 13, 32768, seed=900)
    assert f.has_dc_spike and f.num_coarse_channels == 6
    want, prepared = _direct_hits(torch_cuda, f, 2.0, 8.0)
    assert len(want) >= 6
    got_dat = runDedoppler(f, str(tmp_path / "o.dat"), 2.0, 0.0, 8.0, batch=4, print_hits=False)
    got_hits = runDedoppler(f, str(tmp_path / "o.hits"), 2.0, 0.0, 8.0, batch=4, print_hits=False)
    assert [_key(h) for h in got_dat] == [_key(h) for h in want]
    assert [_key(h) for h in got_hits] == [_key(h) for h in want]
    rows = [ln for ln in open(tmp_path / "o.dat").read().split("\n") if ln and not ln.startswith("#")]
    assert len(rows) == len(want)
    recs = read_hits(str(tmp_path / "o.hits"))
    assert len(recs) == len(want)
    for h, r in zip(want, recs):
        s, fb = r["signal"], r["filterbank"]
        assert (s["index"], s["driftSteps"], s["coarseChannel"]) == (h.index, h.drift_steps, h.coarse_channel)
        b = fb["startChannel"]
        np.testing.assert_array_equal(fb["data"].reshape(13, -1),
                                      prepared[h.coarse_channel][:13, b:b + fb["numChannels"]])


def test_run_dedoppler_from_fil_file(torch_cuda, tmp_path):
    from seticore_b200.run_dedoppler import FilReader, runDedoppler, write_fil
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    spec = SearchSpec(16, 1 << 20, seed=950, n_tones=6, snr_threshold=10.0)
    x = make_filterbank_numpy(spec)
    fn = str(tmp_path / "g.fil")
    from seticore_b200 import FilterbankMetadata
    write_fil(fn, x, FilterbankMetadata(fch1=8421.0, foff=spec.foff_mhz, tsamp=spec.tsamp, telescope_id=6,
                                        source_name="synthetic", tstart=60000.5))
    f = FilReader(fn)
    assert f.coarse_channel_size == 1 << 20 and f.has_dc_spike
    want, _ = _direct_hits(torch_cuda, f, 4.0, 10.0)
    got = runDedoppler(fn, str(tmp_path / "g.dat"), 4.0, 0.0, 10.0, print_hits=False)
    assert len(got) >= 4 and [_key(h) for h in got] == [_key(h) for h in want]


def test_multibeam_band_search_in_place(torch_cuda):
    torch = torch_cuda
    from seticore_b200 import Dedopplerer, FilterbankMetadata
    from seticore_b200.multibeam import MultibeamBuffer, search_band
    from seticore_b200.synthetic import SearchSpec, make_filterbank_torch
    nb, T, fft, cpb = 4, 16, 32768, 3  # beams 0-2 coherent, beam 3 incoherent
    mb = MultibeamBuffer(nb, T, fft * cpb)
    for b in range(nb):
        for lc in range(cpb):
            spec = SearchSpec(T, fft, seed=1000 + 10 * b + lc, n_tones=4 if b < 3 else 0, snr_threshold=8.0)
            mb.data[b, :, lc * fft:(lc + 1) * fft] = make_filterbank_torch(spec)
    meta = FilterbankMetadata(fch1=1400.0, foff=spec.foff_mhz, tsamp=spec.tsamp, coarse_channel_size=fft,
                              num_timesteps=T, num_channels=fft * cpb * 2, num_coarse_channels=2 * cpb,
                              source_names=["b0", "b1", "b2"], ras=[1.0, 2.0, 3.0], decs=[4.0, 5.0, 6.0])
    dd = Dedopplerer(T, fft, spec.foff_mhz, spec.tsamp)
    band = 1
    got = search_band(dd, mb, meta, band, cpb, 3.0, 8.0)
    # The reference's way: copy each region to its own buffer, search, then add incoherent power.
    per_cc = {}
    for b in range(3):
        for lc in range(cpb):
            cc = band * cpb + lc
            region = mb.data[b, :, lc * fft:(lc + 1) * fft].contiguous()
            dd.search(region, meta, b, cc, 3.0, 0.0, 8.0, output=per_cc.setdefault(cc, []))
    for lc in range(cpb):
        dd.addIncoherentPower(mb.data[3, :, lc * fft:(lc + 1) * fft].contiguous(), per_cc[band * cpb + lc])
    want = [h for cc in sorted(per_cc) for h in per_cc[cc]]
    dd.close()
    assert len(want) >= 6
    assert [_key(h) + (np.float32(h.incoherent_power),) for h in got] == \
        [_key(h) + (np.float32(h.incoherent_power),) for h in want]
    assert {h.beam for h in got} == {0, 1, 2}
    assert all(h.incoherent_power > 0 for h in got)


def _tone(x, c0, steps_per_row, amp):
    for t in range(x.shape[0]):
        c = c0 + int(round(t * steps_per_row))
        if 0 <= c < x.shape[1]:
            x[t, c] += amp


def test_find_events_on_a_synthetic_cadence(torch_cuda, tmp_path):
    """ABACAD: a drifting tone in the three "on" files only is one event; a drifting tone in
    all six files (at lower channels) is not."""
    from seticore_b200.events import findEvents
    from seticore_b200.hitfiles import decode_event, split_messages
    from seticore_b200.run_dedoppler import ArrayFilterbankFile
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    N, T = 65536, 16
    files = []
    rate = 8.0 / 15.0  # channels per timestep
    for i in range(6):
        spec = SearchSpec(T, N, seed=3000 + i, n_tones=0)
        x = make_filterbank_numpy(spec)[:T]
        sigma = np.std(np.sort(x.sum(axis=0, dtype=np.float64))[int(np.ceil(0.05 * N)):int(0.95 * N) + 1])
        tstart = i * 300.0
        t_off = tstart / spec.tsamp
        _tone(x, 10000 + int(round(rate * t_off)), rate, 40 * sigma / T)  # in every file
        if i % 2 == 0:
            _tone(x, 40000 + int(round(rate * t_off)), rate, 40 * sigma / T)
        files.append(ArrayFilterbankFile(x, coarse_channel_size=N, telescope_id=6, foff=spec.foff_mhz,
                                         tsamp=spec.tsamp, tstart=tstart, fch1=8000.0,
                                         source_name="TGT" if i % 2 == 0 else f"OFF{i}"))
    out = str(tmp_path / "c.events")
    events = findEvents(files, out, 2.0, 20.0, 20.0, verbose=False)  # above the noise hits (SNR ~10-11)
    assert len(events) == 1
    ev = events[0]
    assert [h is None for h in ev] == [False, True, False, True, False, True]
    assert abs(ev[0].index - 40000) <= 2
    msgs = [decode_event(seg) for _, seg in split_messages(open(out, "rb").read())]
    assert len(msgs) == 1 and len(msgs[0]) == 6
    assert [m["signal"] is None for m in msgs[0]] == [False, True, False, True, False, True]
    assert [m["filterbank"]["sourceName"] for m in msgs[0]] == ["TGT", "OFF1", "TGT", "OFF3", "TGT", "OFF5"]
    assert all(m["filterbank"]["data"].size == T * m["filterbank"]["numChannels"] for m in msgs[0])
