"""The search, and the callers either side of it, against the reference's own GPU build.

oracle/_ref/libref_gpu.so is the reference's Dedopplerer (dedoppler.cu, taylor.cu, ...)
compiled for sm_100a.  Each test runs the same seeded input through it and through this
package and asks for the parity bar of tests/test_gpu_parity.py: identical (index,
drift_steps) lists, power bit-equal, SNR within 1e-4 relative, and a hit on one side only
accepted as a listed threshold tie (at most one per search).
"""
import numpy as np
import pytest

from tests.conftest import has_gpu
from tests.test_gpu_parity import compare_hits

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch


@pytest.fixture(scope="module")
def ref_gpu():
    from oracle.oracle import RefGpu, available
    if not available("reference_gpu"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    return RefGpu()


def ref_search(ref, x, T, spec_foff_mhz, tsamp, max_drift, min_drift, snr, beam=-1, coarse=0):
    ctx = ref.context(T, x.shape[1], spec_foff_mhz, tsamp)
    ctx.load(x)
    hits = ctx.search(beam, coarse, max_drift, min_drift, snr)
    ctx.close()
    return hits


def as_dicts(hits):
    return [dict(index=h.index, drift_steps=h.drift_steps, snr=h.snr, power=h.power, drift_rate=h.drift_rate)
            for h in hits]


def test_node_coarse_channels_match_reference_gpu(torch_cuda, ref_gpu):
    """Four coarse channels of the benchmark node (its own seeds), searched as one batch."""
    torch = torch_cuda
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import config_node, make_filterbank_numpy
    specs = config_node(4, base_seed=2000)
    xs = [make_filterbank_numpy(s) for s in specs]
    s0 = specs[0]
    dd = Dedopplerer(16, s0.num_channels, s0.foff_mhz, s0.tsamp)
    got = dd.search_batch_raw([torch.from_numpy(x).cuda() for x in xs], [-1] * 4, list(range(4)),
                              s0.max_drift, s0.min_drift, s0.snr_threshold)
    thr = dd.last_stats().threshold
    dd.close()
    total = 0
    for k, (s, x) in enumerate(zip(specs, xs)):
        want = ref_search(ref_gpu, x, 16, s.foff_mhz, s.tsamp, s.max_drift, s.min_drift, s.snr_threshold, coarse=k)
        ties = compare_hits(as_dicts(got[k]), want, thr, thr, f"node coarse {k}")
        assert len(ties) <= 1, ties
        total += len(want)
    assert total >= 16  # 4 tones + 2 spikes per coarse channel


@pytest.mark.parametrize("precision", ["bf16", "fp16"])
def test_16bit_forms_match_reference_gpu(torch_cuda, ref_gpu, precision):
    """The 16-bit forms -- whose 16- and 32-row trees add FP16 pairs of two drift blocks --
    against the reference's own GPU search: one node coarse channel (16 rows) and one 32-row
    search of the uneven model."""
    torch = torch_cuda
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import SearchSpec, config_node, make_filterbank_numpy
    cases = [config_node(1, base_seed=2100)[0],
             SearchSpec(32, 1 << 18, tsamp=18.253611 / 2, max_drift=3.0, seed=2101, n_tones=5, snr_threshold=10.0)]
    for s in cases:
        x = make_filterbank_numpy(s)
        dd = Dedopplerer(s.num_timesteps, s.num_channels, s.foff_mhz, s.tsamp)
        dd.set_precision(precision)
        got = dd.search_raw(torch.from_numpy(x).cuda(), -1, 0, s.max_drift, s.min_drift, s.snr_threshold)
        thr = dd.last_stats().threshold
        dd.close()
        want = ref_search(ref_gpu, x, s.num_timesteps, s.foff_mhz, s.tsamp, s.max_drift, s.min_drift, s.snr_threshold)
        ties = compare_hits(as_dicts(got), want, thr, thr, f"{precision} T{s.num_timesteps}")
        assert len(ties) <= 1, ties
        assert len(want) >= 3


def test_uneven_shapes_through_the_pool_match_reference_gpu(torch_cuda, ref_gpu):
    """64, 128 and 256 timesteps at 2^20 channels (the level path), mixed in one pool call."""
    torch = torch_cuda
    from seticore_b200 import SearchPool, SearchRequest
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    shapes = [(64, 3.0, 61), (128, 6.0, 62), (256, 10.0, 63)]
    specs = [SearchSpec(T, 1 << 20, tsamp=18.253611 * 16 / T, max_drift=md, seed=seed, n_tones=5,
                        tone_drift=min(md, 4.0), tone_snr=(12.0, 80.0), snr_threshold=10.0)
             for T, md, seed in shapes]
    xs = [make_filterbank_numpy(s) for s in specs]
    reqs = [SearchRequest(torch.from_numpy(x).cuda(), s.num_timesteps, s.foff_mhz, s.tsamp, s.max_drift, 0.0,
                          s.snr_threshold, beam=-1, coarse_channel=k)
            for k, (s, x) in enumerate(zip(specs, xs))]
    pool = SearchPool(scratch_budget_bytes=8 << 30)
    got = pool.search_raw(reqs)
    got2 = pool.search_raw(reqs)  # the second call replays the captured graphs
    pool.close()
    for k, (s, x) in enumerate(zip(specs, xs)):
        want = ref_search(ref_gpu, x, s.num_timesteps, s.foff_mhz, s.tsamp, s.max_drift, 0.0, s.snr_threshold,
                          coarse=k)
        g = [dict(index=h.index, drift_steps=h.drift_steps, snr=h.snr, power=h.power) for h in got[k]]
        compare_hits(g, want, 0.0, 0.0, f"pool T{s.num_timesteps}")  # threshold 0: no tie accepted
        assert len(want) >= 3, (s.num_timesteps, len(want))
        assert [(h.index, h.drift_steps, h.power) for h in got2[k]] == [(h.index, h.drift_steps, h.power)
                                                                         for h in got[k]]


def test_add_incoherent_power_matches_reference_gpu(torch_cuda, ref_gpu):
    """Dedopplerer::addIncoherentPower (dedoppler.cu:139-176): the reference's own tree over the
    incoherent beam, read at each hit's path, against path_values_kernel."""
    torch = torch_cuda
    from seticore_b200 import Dedopplerer, FilterbankMetadata
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    for T, N, seed in [(16, 1 << 17, 71), (64, 40000, 72)]:
        spec = SearchSpec(T, N, tsamp=18.253611 * 16 / T, max_drift=2.0, seed=seed, n_tones=10, tone_drift=2.0,
                          snr_threshold=8.0)
        x = make_filterbank_numpy(spec)
        inc = make_filterbank_numpy(SearchSpec(T, N, tsamp=spec.tsamp, seed=seed + 100, n_tones=3))
        dd = Dedopplerer(T, N, spec.foff_mhz, spec.tsamp)
        hits = dd.search(torch.from_numpy(x).cuda(), FilterbankMetadata(coarse_channel_size=N), -1, 0, 2.0, 0.0, 8.0)
        assert len(hits) >= 5
        dd.addIncoherentPower(torch.from_numpy(inc).cuda(), hits)
        dd.close()
        ctx = ref_gpu.context(T, N, spec.foff_mhz, spec.tsamp)
        ctx.load(inc)
        want = ctx.add_incoherent([dict(index=h.index, drift_steps=h.drift_steps, drift_rate=h.drift_rate,
                                        snr=h.snr, power=h.power) for h in hits])
        ctx.close()
        # both sort by drift_steps (dedoppler.cu:144); compare as (index, drift) -> value
        g = {(h.index, h.drift_steps): np.float32(h.incoherent_power) for h in hits}
        w = {(h["index"], h["drift_steps"]): np.float32(h["incoherent_power"]) for h in want}
        assert g == w, (T, g, w)
        assert [h.drift_steps for h in hits] == sorted(h.drift_steps for h in hits)


def test_quantised_power_matches_reference_gpu(torch_cuda, ref_gpu):
    """8-bit quantised power (what 8-bit filterbanks give): column sums with many exact ties,
    the case where the order of the reference's float variance sum matters most."""
    torch = torch_cuda
    from seticore_b200 import Dedopplerer
    rng = np.random.default_rng(91)
    for N, scale in [(1 << 18, 20.0), (1 << 20, 4.0)]:
        x = np.minimum(np.rint(rng.exponential(scale, size=(16, N))), 255).astype(np.float32)
        for c, v in ((1000, 60.0), (90000, 45.0), (200000, 40.0)):
            for t in range(16):
                x[t, c + t // 3] += v * scale / 20.0
        dd = Dedopplerer(16, N, 2.7939677e-6, 18.253611)
        got = dd.search_raw(torch.from_numpy(x).cuda(), -1, 0, 2.0, 0.0, 10.0)
        thr = dd.last_stats().threshold
        dd.close()
        want = ref_search(ref_gpu, x, 16, 2.7939677e-6, 18.253611, 2.0, 0.0, 10.0)
        ties = compare_hits(as_dicts(got), want, thr, thr, f"quantised N{N}")
        assert len(ties) <= 1, ties
        assert len(want) >= 3


def test_run_dedoppler_matches_reference_gpu(torch_cuda, ref_gpu, tmp_path):
    """runDedoppler (run_dedoppler.cpp:30-53) over a six-coarse-channel file against the
    reference's search of each prepared coarse channel (rows padded, DC spike replaced as
    h5_reader.cpp:190-209 does)."""
    from seticore_b200.run_dedoppler import runDedoppler
    from tests.test_gpu_driver import _coarse_file, _prepared_host
    f = _coarse_file(6, 13, 32768, seed=900)
    got = runDedoppler(f, str(tmp_path / "o.dat"), 2.0, 0.0, 8.0, batch=4, print_hits=False)
    n = 0
    for c in range(f.num_coarse_channels):
        host = np.zeros((f.num_timesteps, f.coarse_channel_size), np.float32)
        f.loadCoarseChannel(c, host)
        p = _prepared_host(host, 16, f.has_dc_spike)
        want = ref_search(ref_gpu, p, f.num_timesteps, f.foff, f.tsamp, 2.0, 0.0, 8.0, coarse=c)
        mine = [dict(index=h.index, drift_steps=h.drift_steps, snr=h.snr, power=h.power)
                for h in got if h.coarse_channel == c]
        compare_hits(mine, want, 0.0, 0.0, f"runDedoppler coarse {c}")  # threshold 0: no tie accepted
        n += len(want)
    assert n >= 6


def test_multibeam_band_matches_reference_gpu(torch_cuda, ref_gpu):
    """The in-place band search (search_band) against the reference's way: each region copied
    out and searched by the reference, then its addIncoherentPower over the incoherent beam."""
    torch = torch_cuda
    from seticore_b200 import Dedopplerer, FilterbankMetadata
    from seticore_b200.multibeam import MultibeamBuffer, search_band
    from seticore_b200.synthetic import SearchSpec, make_filterbank_torch
    nb, T, fft, cpb = 4, 16, 32768, 3  # beams 0-2 coherent, beam 3 incoherent
    mb = MultibeamBuffer(nb, T, fft * cpb)
    for b in range(nb):
        for lc in range(cpb):
            spec = SearchSpec(T, fft, seed=1100 + 10 * b + lc, n_tones=4 if b < 3 else 0, snr_threshold=8.0)
            mb.data[b, :, lc * fft:(lc + 1) * fft] = make_filterbank_torch(spec)
    meta = FilterbankMetadata(fch1=1400.0, foff=spec.foff_mhz, tsamp=spec.tsamp, coarse_channel_size=fft,
                              num_timesteps=T, num_channels=fft * cpb * 2, num_coarse_channels=2 * cpb,
                              source_names=["b0", "b1", "b2"], ras=[1.0, 2.0, 3.0], decs=[4.0, 5.0, 6.0])
    dd = Dedopplerer(T, fft, spec.foff_mhz, spec.tsamp)
    band = 1
    got = search_band(dd, mb, meta, band, cpb, 3.0, 8.0)
    dd.close()
    host = mb.data.cpu().numpy()
    want = []
    for lc in range(cpb):
        cc = band * cpb + lc
        hits = []
        for b in range(3):
            # the reference context's metadata lists no beams, so its hits carry NO_BEAM: keep b
            hits += [dict(h, beam=b) for h in ref_search(ref_gpu, host[b, :, lc * fft:(lc + 1) * fft], T,
                                                          spec.foff_mhz, spec.tsamp, 3.0, 0.0, 8.0, beam=b, coarse=cc)]
        ctx = ref_gpu.context(T, fft, spec.foff_mhz, spec.tsamp)
        ctx.load(np.ascontiguousarray(host[3, :, lc * fft:(lc + 1) * fft]))
        inc = ctx.add_incoherent(hits)
        ctx.close()
        incp = {(h["index"], h["drift_steps"]): np.float32(h["incoherent_power"]) for h in inc}
        want += [(cc, h["beam"], h["index"], h["drift_steps"], np.float32(h["power"]),
                  incp[(h["index"], h["drift_steps"])]) for h in hits]
    mine = [(h.coarse_channel, h.beam, h.index, h.drift_steps, np.float32(h.power), np.float32(h.incoherent_power))
            for h in got]
    assert sorted(mine) == sorted(want)
    assert len(want) >= 6


def _cadence(T, N, num_coarse, seed):
    """Six ABACAD files of num_coarse coarse channels with drifting tones placed so that some
    become events and some do not (in every file; zero drift; a matching hit in an "off")."""
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    # channels per timestep: a whole number of drift steps over the rounded rows, slow enough
    # with padding rows that expectedIndex (drift over num_timesteps - 1) stays in the wiggle
    rate = 8.0 / 15.0 if T == 16 else 0.25
    files = []
    for i in range(6):
        parts = []
        for cc in range(num_coarse):
            spec = SearchSpec(T, N, seed=seed + 10 * i + cc, n_tones=0)
            parts.append(make_filterbank_numpy(spec)[:T])
        x = np.concatenate(parts, axis=1)
        sigma = np.std(np.sort(parts[0].sum(axis=0, dtype=np.float64))[int(np.ceil(0.05 * N)):int(0.95 * N) + 1])
        tstart = i * 300.0
        t_off = tstart / spec.tsamp
        on = i % 2 == 0

        def tone(cc, c0, r, snr):
            for t in range(T):
                c = c0 + int(round(r * t_off)) + int(round(t * r))
                if 0 <= c < N:
                    x[t, cc * N + c] += snr * sigma / T

        tone(0, N // 8, rate, 40)                   # in every file: no event
        if on:
            tone(0, 5 * N // 8, rate, 40)           # ons only: an event
            tone(0, 3 * N // 8, rate, 40)           # ons, and an off below: no event
        if i == 3:
            tone(0, 3 * N // 8, rate, 18)
        if num_coarse > 1 and on:
            tone(1, N // 4, 0.0, 60)                # zero drift: removed
            tone(1, 3 * N // 4, -rate, 35)          # negative drift: an event
        files.append(dict(rows=x, source_name="TGT" if on else f"OFF{i}", tstart=tstart, coarse_size=N,
                          num_coarse=num_coarse, fch1=8000.0, foff=spec.foff_mhz, tsamp=spec.tsamp,
                          has_dc_spike=True))
    return files


@pytest.mark.parametrize("T,num_coarse", [(16, 2), (12, 1)])
def test_find_events_match_reference_gpu(torch_cuda, ref_gpu, tmp_path, T, num_coarse):
    """Cadence search (find_events.cpp:65-226) against the reference's own findEvents built
    with its Dedopplerer: the same events, each file's hit with the same index and drift,
    power bit-equal and SNR within 1e-4 relative (None in the same files)."""
    from seticore_b200.events import findEvents
    from seticore_b200.run_dedoppler import ArrayFilterbankFile
    N = 1 << 15
    files = _cadence(T, N, num_coarse, 7000 + T)
    max_drift, snr_on, snr_off = 2.0, 20.0, 14.0
    want = ref_gpu.find_events(files, max_drift, snr_on, snr_off)
    readers = [ArrayFilterbankFile(f["rows"], coarse_channel_size=N, telescope_id=6, foff=f["foff"],
                                   tsamp=f["tsamp"], tstart=f["tstart"], fch1=f["fch1"],
                                   source_name=f["source_name"]) for f in files]
    assert all(r.has_dc_spike for r in readers)
    got = findEvents(readers, str(tmp_path / "c.events"), max_drift, snr_on, snr_off, verbose=False)
    assert len(want) >= 1, want
    assert len(got) == len(want), (got, want)
    for ev_got, ev_want in zip(got, want):
        assert [h is None for h in ev_got] == [h is None for h in ev_want]
        for g, w in zip(ev_got, ev_want):
            if w is None:
                continue
            assert (g.index, g.drift_steps) == (w["index"], w["drift_steps"])
            assert np.float32(g.power) == np.float32(w["power"])
            assert abs(g.snr - w["snr"]) <= 1e-4 * abs(w["snr"])
