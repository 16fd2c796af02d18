"""GPU parity: the sm_100a search against the oracle and the reference's own GPU build.

Bar (per hit list): identical (index, drift_steps) lists, SNR within 1e-4 relative, top
path sums and column sums bit-identical to the oracle (integer-exact adds in the same
tree order).  A hit present on one side only is accepted only as a threshold tie: its
power lies within 1e-4 relative of the threshold (the thresholds differ by the
reference's float-accumulated variance, see dd_stats.cu); such ties are listed in the
assertion message.
"""
import os
import subprocess

import numpy as np
import pytest

from tests.conftest import has_gpu

pytestmark = pytest.mark.gpu

SNR_RTOL = 1e-4
TIE_RTOL = 1e-4


@pytest.fixture(scope="module")
def torch_cuda():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch


def run_gpu(torch, x, foff_mhz, tsamp, max_drift, min_drift, snr, T=None, beam=-1, coarse=0):
    from seticore_b200 import Dedopplerer
    Tr, N = x.shape
    dd = Dedopplerer(T or Tr, N, foff_mhz, tsamp)
    xt = torch.from_numpy(x).cuda()
    hits = dd.search_raw(xt, beam, coarse, max_drift, min_drift, snr)
    stats = dd.last_stats()
    top = dd.channel_array("top").cpu().numpy()
    colsum = dd.channel_array("colsum").cpu().numpy()
    dd.close()
    return ([dict(index=h.index, drift_steps=h.drift_steps, snr=h.snr, power=h.power, drift_rate=h.drift_rate)
             for h in hits], stats, top, colsum)


def compare_hits(got, want, thr_got, thr_want, label=""):
    """Asserts hit-list parity; returns the list of threshold ties."""
    g = {h["index"]: h for h in got}
    w = {h["index"]: h for h in want}
    ties = []
    for idx in sorted(set(g) ^ set(w)):
        h = g.get(idx) or w.get(idx)
        thr = float(thr_want)
        if abs(float(h["power"]) - thr) <= TIE_RTOL * abs(thr):
            ties.append(idx)
        else:
            raise AssertionError(f"{label}: hit at index {idx} only on one side "
                                 f"(gpu={idx in g}, ref={idx in w}): {h}; thresholds {thr_got} vs {thr_want}")
    for idx in sorted(set(g) & set(w)):
        a, b = g[idx], w[idx]
        assert a["drift_steps"] == b["drift_steps"], (label, idx, a, b)
        assert np.float32(a["power"]) == np.float32(b["power"]), (label, idx, a, b)
        assert abs(a["snr"] - b["snr"]) <= SNR_RTOL * abs(b["snr"]), (label, idx, a, b)
    return ties


CASES = [
    # T, N, foff_hz, tsamp, max_drift, n_tones, seed
    (2, 5000, 2.7939677, 18.253611, 1.0, 4, 1),
    (4, 6000, 2.7939677, 18.253611, 2.0, 5, 2),
    (8, 4099, -2.7939677, 18.253611, 2.0, 5, 3),
    (16, 8192, 2.7939677, 18.253611, 4.0, 6, 4),
    (16, 20000, -2.7939677, 18.253611, 4.0, 8, 5),
    (13, 5000, 2.7939677, 18.253611, 3.0, 5, 6),
    (16, 1001, 2.7939677, 18.253611, 0.3, 3, 7),
    (32, 4096, 2.7939677, 9.1268055, 2.0, 5, 8),
    (64, 3000, 2.7939677, 4.5634028, 1.0, 4, 9),
    (128, 2048, 2.7939677, 2.2817014, 1.0, 3, 10),
    (256, 4096, 3.814697265625, 0.268435456, 10.0, 4, 11),
    (16, 65536, 2.7939677, 18.253611, 8.0, 8, 12),
    # edges: fewer channels than a tile, drift ranges wider than the band, the smallest
    # band, and more than 256 rows (a 2-row level after the 16-row level)
    (16, 100, 2.7939677, 18.253611, 4.0, 1, 13),
    (8, 300, 2.7939677, 18.253611, 8.0, 2, 14),
    (2, 64, 2.7939677, 18.253611, 1.0, 1, 15),
    (512, 2048, 3.814697265625, 0.134217728, 4.0, 3, 16),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"T{c[0]}_N{c[1]}_md{c[4]}_s{c[6]}")
def test_search_matches_oracle(torch_cuda, port_oracle, case):
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    T, N, foff_hz, tsamp, md, ntones, seed = case
    spec = SearchSpec(T, N, foff_hz=foff_hz, tsamp=tsamp, max_drift=md, seed=seed, n_tones=ntones,
                      tone_drift=min(md, 4.0), snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    want, wstats, arrays = port_oracle.search(x, spec.foff_mhz, tsamp, md, 0.0, 8.0, arrays=True)
    got, gstats, top, colsum = run_gpu(torch_cuda, x, spec.foff_mhz, tsamp, md, 0.0, 8.0, T=T)
    np.testing.assert_array_equal(colsum, arrays["colsum"])
    np.testing.assert_array_equal(top, arrays["top"])
    assert gstats.window_size == wstats["window_size"]
    assert gstats.median == np.float32(wstats["median"])
    assert gstats.mean == np.float32(wstats["mean"])
    if gstats.order_exact:  # formed in the reference's nth_element order: bit for bit
        assert np.float32(gstats.std_dev) == np.float32(wstats["std_dev"])
        assert np.float32(gstats.threshold) == np.float32(wstats["threshold"])
    else:  # distinct column sums: the float variance emulated in channel order
        assert abs(gstats.std_dev - wstats["std_dev"]) <= 1e-4 * abs(wstats["std_dev"])
    ties = compare_hits(got, want, gstats.threshold, wstats["threshold"], label=str(case))
    assert len(ties) <= 1, ties


def test_known_answer(torch_cuda):
    """dedoppler_test.cpp:9-33 through the Python API."""
    from seticore_b200 import NO_BEAM, Dedopplerer, FilterbankMetadata, makeNoisyBuffer
    buf = makeNoisyBuffer(8, 1000)
    for t, c in enumerate([70, 70, 71, 71, 72, 72, 73, 73]):
        buf.set(t, c, 1.0)
    dd = Dedopplerer(8, 1000, 1.0, 1.0, False)
    hits = dd.search(buf, FilterbankMetadata(), NO_BEAM, 555, 0.01, 0.01, 200.0)
    assert len(hits) == 1
    assert hits[0].index == 70 and hits[0].drift_steps == 3
    assert hits[0].beam == NO_BEAM and hits[0].coarse_channel == 555


def test_golden_searches(torch_cuda):
    """The reference-generated golden hit lists (tests/golden/golden.json)."""
    import json
    from tests.golden.make_golden import search_spec
    from seticore_b200.synthetic import make_filterbank_numpy
    golden = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
    for entry in golden["search"]:
        spec = search_spec(entry["case"])
        x = make_filterbank_numpy(spec)
        got, gstats, _, _ = run_gpu(torch_cuda, x, spec.foff_mhz, spec.tsamp, spec.max_drift, spec.min_drift,
                                    spec.snr_threshold, T=spec.num_timesteps)
        compare_hits(got, entry["hits"], gstats.threshold, entry["stats"]["threshold"], entry["case"]["name"])


def test_full_size_single_coarse_channel(torch_cuda, port_oracle):
    """16 x 2^20, 8 tones, max_drift 4: bit-exact top sums and identical hits."""
    from seticore_b200.synthetic import config_single, make_filterbank_numpy
    spec = config_single()
    x = make_filterbank_numpy(spec)
    want, wstats, arrays = port_oracle.search(x, spec.foff_mhz, spec.tsamp, spec.max_drift, 0.0,
                                              spec.snr_threshold, arrays=True)
    got, gstats, top, colsum = run_gpu(torch_cuda, x, spec.foff_mhz, spec.tsamp, spec.max_drift, 0.0,
                                       spec.snr_threshold)
    np.testing.assert_array_equal(top, arrays["top"])
    np.testing.assert_array_equal(colsum, arrays["colsum"])
    compare_hits(got, want, gstats.threshold, wstats["threshold"], "full")
    assert len(got) >= 1


def test_matches_reference_gpu_build(torch_cuda):
    """The reference's own Dedopplerer (dedoppler.cu/taylor.cu built for sm_100a)."""
    from oracle.oracle import RefGpu, available
    if not available("reference_gpu"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    ref = RefGpu()
    for (T, N, md, seed) in [(16, 1 << 18, 4.0, 21), (8, 50000, 2.0, 22), (32, 30000, 2.0, 23), (64, 20000, 1.0, 24)]:
        spec = SearchSpec(T, N, max_drift=md, seed=seed, n_tones=6, tone_drift=min(md, 4.0),
                          tsamp=18.253611 * 16 / max(T, 16), snr_threshold=8.0)
        x = make_filterbank_numpy(spec)
        ctx = ref.context(T, N, spec.foff_mhz, spec.tsamp)
        ctx.load(x)
        want = ctx.search(-1, 3, md, 0.0, 8.0)
        ctx.close()
        got, gstats, _, _ = run_gpu(torch_cuda, x, spec.foff_mhz, spec.tsamp, md, 0.0, 8.0, T=T)
        thr = gstats.threshold
        ties = compare_hits(got, want, thr, thr, f"refgpu T{T}")
        assert len(ties) <= 1, ties
        assert len(want) >= 3


def test_incoherent_power(torch_cuda, port_oracle):
    from seticore_b200 import Dedopplerer, DedopplerHit, FilterbankMetadata
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    spec = SearchSpec(16, 20000, seed=31, n_tones=6, snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    inc = make_filterbank_numpy(SearchSpec(16, 20000, seed=32, n_tones=0))
    dd = Dedopplerer(16, 20000, spec.foff_mhz, spec.tsamp)
    hits = dd.search(torch_cuda.from_numpy(x).cuda(), FilterbankMetadata(coarse_channel_size=20000), -1, 0,
                     4.0, 0.0, 8.0)
    assert hits
    dd.addIncoherentPower(torch_cuda.from_numpy(inc).cuda(), hits)
    assert [h.drift_steps for h in hits] == sorted(h.drift_steps for h in hits)
    for h in hits:
        assert np.float32(h.incoherent_power) == np.float32(port_oracle.incoherent_power(inc, h.drift_steps, h.index))


def test_strided_view_equals_dense(torch_cuda):
    """Searching a [T][N] window of a wider [T][3N] buffer in place (the multibeam case)."""
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    torch = torch_cuda
    N = 10000
    wide = np.concatenate([make_filterbank_numpy(SearchSpec(16, N, seed=40 + i, n_tones=4)) for i in range(3)], axis=1)
    wt = torch.from_numpy(wide).cuda()
    dd = Dedopplerer(16, N, 2.7939677e-6, 18.253611)
    view_hits = dd.search_raw(wt[:, N:2 * N], -1, 1, 4.0, 0.0, 8.0)
    dense_hits = dd.search_raw(wt[:, N:2 * N].contiguous(), -1, 1, 4.0, 0.0, 8.0)
    assert [(h.index, h.drift_steps, h.power) for h in view_hits] == \
           [(h.index, h.drift_steps, h.power) for h in dense_hits]


def test_errors_are_status_codes(torch_cuda):
    from seticore_b200 import DedopplerError, Dedopplerer
    torch = torch_cuda
    dd = Dedopplerer(16, 1000, 2.7939677e-6, 18.253611)
    with pytest.raises(ValueError):
        dd.search_raw(torch.zeros((8, 1000), device="cuda"), -1, 0, 4.0, 0.0, 10.0)
    with pytest.raises(DedopplerError) as e:
        dd.search_raw(torch.zeros((16, 1000), device="cuda"), -1, 0, 0.0, 0.0, 10.0)
    assert e.value.code == 1
    with pytest.raises(TypeError):
        dd.search_raw(torch.zeros((16, 1000)), -1, 0, 4.0, 0.0, 10.0)
    with pytest.raises(DedopplerError):
        Dedopplerer(1, 1000, 1.0, 1.0)


def test_cpp_dropin_known_answer(torch_cuda):
    """tests/cpp/dedoppler_api_test.cpp: the reference's dedoppler test through the C++ header."""
    exe = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "seticore_b200", "_lib",
                       "dedoppler_api_test")
    if not os.path.exists(exe):
        pytest.fail("C++ test program not built (python -m seticore_b200.build)")
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr


def test_batch_equals_single_searches(torch_cuda):
    """sc_dd_search_batch over 70 inputs (two launches of up to 64) equals 70 single searches."""
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import SearchSpec, make_filterbank_torch
    torch = torch_cuda
    N = 1 << 15
    specs = [SearchSpec(16, N, seed=500 + i, n_tones=4, n_spikes=1, snr_threshold=8.0) for i in range(70)]
    data = torch.empty((70, 16, N), dtype=torch.float32, device="cuda")
    for i, s in enumerate(specs):
        make_filterbank_torch(s, out=data[i])
    dd = Dedopplerer(16, N, specs[0].foff_mhz, specs[0].tsamp)
    single = [dd.search_raw(data[i], -1, i, 4.0, 0.0, 8.0) for i in range(70)]
    batch = dd.search_batch_raw([data[i] for i in range(70)], [-1] * 70, list(range(70)), 4.0, 0.0, 8.0)
    assert len(batch) == 70
    for a, b in zip(single, batch):
        assert [(h.index, h.drift_steps, h.power, h.snr, h.coarse_channel) for h in a] == \
               [(h.index, h.drift_steps, h.power, h.snr, h.coarse_channel) for h in b]
    assert sum(len(x) for x in batch) > 70


@pytest.mark.parametrize("kind", ["integer", "half_zero"])
def test_order_statistics_with_heavy_ties(torch_cuda, port_oracle, kind):
    """Column sums with many equal values (integer-valued power).  The reference adds the
    squared deviations in float in the order std::nth_element leaves the array, and with this
    many exact ties that order decides which terms fall under half an ulp of the running sum
    (channel order is 4e-4 away here).  The GPU follows the same order: median, mean,
    deviation and SNR are bit-identical to the oracle's."""
    N = 1 << 18
    rng = np.random.default_rng(77)
    x = rng.integers(0, 3, size=(16, N)).astype(np.float32)
    if kind == "half_zero":
        x[:, rng.random(N) < 0.6] = 0.0
    for c, v in ((1000, 40.0), (90000, 30.0), (200000, 25.0)):  # a few drifting tones
        for t in range(16):
            x[t, c + t // 4] += v
    want, wstats = port_oracle.search(x, 2.7939677e-6, 18.253611, 2.0, 0.0, 10.0)
    got, gstats, _, _ = run_gpu(torch_cuda, x, 2.7939677e-6, 18.253611, 2.0, 0.0, 10.0, T=16)
    assert gstats.median == np.float32(wstats["median"])
    assert gstats.mean == np.float32(wstats["mean"])
    assert np.float32(gstats.std_dev) == np.float32(wstats["std_dev"]) and gstats.order_exact == 1
    assert [(h["index"], h["drift_steps"], np.float32(h["power"])) for h in got] == \
        [(h["index"], h["drift_steps"], np.float32(h["power"])) for h in want]
    for a, b in zip(got, want):
        assert np.float32(a["snr"]) == np.float32(b["snr"]), (kind, a, b)
    assert len(got) >= 3


def test_min_drift_filter(torch_cuda, port_oracle):
    """Hits whose |drift rate| is below min_drift are dropped (dedoppler.cu:310)."""
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    spec = SearchSpec(16, 20000, seed=41, n_tones=10, snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    for min_drift in (0.05, 0.5):
        want, wstats = port_oracle.search(x, spec.foff_mhz, spec.tsamp, 4.0, min_drift, 8.0)
        got, gstats, _, _ = run_gpu(torch_cuda, x, spec.foff_mhz, spec.tsamp, 4.0, min_drift, 8.0, T=16)
        compare_hits(got, want, gstats.threshold, wstats["threshold"], label=f"min_drift {min_drift}")
        assert all(abs(h["drift_rate"]) >= min_drift for h in got)


def test_constant_input_has_no_hits(torch_cuda):
    """Zero or constant power: every path sums to the median, nothing beats the threshold."""
    for value in (0.0, 3.5):
        x = np.full((16, 5000), value, dtype=np.float32)
        got, gstats, top, _ = run_gpu(torch_cuda, x, 2.7939677e-6, 18.253611, 4.0, 0.0, 10.0, T=16)
        assert got == []
        assert gstats.median == np.float32(16 * value)


@pytest.mark.parametrize("precision", ["fp32", "bf16"])
def test_staging_wait_give_up_is_reported(torch_cuda, port_oracle, precision):
    """The tree's bounded wait for its staged rows (an mbarrier poll with a try limit): with the
    limit set to 0 every staged item gives up at once -- nothing hangs or faults -- and the search
    reports SC_DD_EINTERNAL; with the default restored the same engine searches correctly.  BF16:
    the paired-FP16 tree, which stages its paired copy the same way."""
    from seticore_b200 import DedopplerError, Dedopplerer, _capi
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    spec = SearchSpec(16, 1 << 16, seed=51, n_tones=6, snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    xt = torch_cuda.from_numpy(x).cuda()
    dd = Dedopplerer(16, x.shape[1], spec.foff_mhz, spec.tsamp)
    if precision != "fp32":
        dd.set_precision(precision)
    L = _capi.lib()
    try:
        assert L.sc_dd_set_stage_wait_limit(0) == _capi.SC_DD_OK
        for _ in range(2):
            with pytest.raises(DedopplerError) as e:
                dd.search_raw(xt, -1, 0, spec.max_drift, 0.0, spec.snr_threshold)
            assert e.value.code == _capi.SC_DD_EINTERNAL
    finally:
        L.sc_dd_set_stage_wait_limit(-1)
    got = dd.search_raw(xt, -1, 0, spec.max_drift, 0.0, spec.snr_threshold)
    top = dd.channel_array("top").cpu().numpy()
    dd.close()
    want, _, arrays = port_oracle.search(x, spec.foff_mhz, spec.tsamp, spec.max_drift, 0.0, spec.snr_threshold,
                                         arrays=True)
    if precision == "fp32":
        np.testing.assert_array_equal(top, arrays["top"])
    assert [(h.index, h.drift_steps) for h in got] == [(h["index"], h["drift_steps"]) for h in want]


EDGE_CASES = [
    # T, N, max_drift (Hz/s at foff 2.79 Hz, tsamp 18.25 * 16 / T s): most strips sit near an
    # edge of the band, where the drift blocks reach past it
    (2, 1500, 40.0), (4, 2100, 30.0), (8, 2900, 25.0), (16, 3300, 20.0), (16, 1056, 12.0),
    (32, 4000, 10.0), (32, 1200, 6.0), (13, 2500, 18.0), (64, 5000, 8.0),
]


@pytest.mark.parametrize("case", EDGE_CASES, ids=lambda c: f"T{c[0]}_N{c[1]}_md{c[2]}")
def test_edge_strips_match_oracle(torch_cuda, port_oracle, case):
    """Edge strips (channels near the band's ends whose drift blocks reach past it): the
    generated tree with a range fold for the channels whose paths are all eligible, one path
    at a time for the partially eligible ones.  Top sums bit-identical to the oracle."""
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    T, N, md = case
    spec = SearchSpec(T, N, tsamp=18.253611 * 16 / max(T, 16), max_drift=md, seed=700 + T, n_tones=3,
                      tone_drift=4.0, snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    want, wstats, arrays = port_oracle.search(x, spec.foff_mhz, spec.tsamp, md, 0.0, 8.0, arrays=True)
    got, gstats, top, colsum = run_gpu(torch_cuda, x, spec.foff_mhz, spec.tsamp, md, 0.0, 8.0, T=T)
    assert wstats["window_size"] > 0 and spec.num_drift_blocks() >= 3
    np.testing.assert_array_equal(top, arrays["top"])
    ties = compare_hits(got, want, gstats.threshold, wstats["threshold"], label=str(case))
    assert len(ties) <= 1, ties
