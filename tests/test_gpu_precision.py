"""The precision form: 16-bit normalised storage with exact FP32 recomputation.

Bar: the BF16 and FP16 forms return exactly the FP32 form's hit list (index, drift,
power bit-for-bit, SNR); the approximate path sums they compute are compared with the
FP64 oracle (tree in double precision, same geometry) and the error is stated.
"""
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


def _hits(dd, xt, spec):
    return [(h.index, h.drift_steps, np.float32(h.power), np.float32(h.snr))
            for h in dd.search_raw(xt, -1, 0, spec.max_drift, spec.min_drift, spec.snr_threshold)]


CASES = [(16, 65536, 4.0, 1, 1), (16, 40000, 4.0, 2, 0), (8, 30000, 2.0, 3, 2), (13, 20000, 3.0, 4, 1),
         (4, 50000, 1.0, 5, 1), (2, 20000, 1.0, 6, 0), (16, 1 << 20, 4.0, 7, 2),
         (32, 65536, 4.0, 8, 1), (100, 32768, 2.0, 9, 0), (256, 131072, 2.0, 10, 1),
         # rows of a length that is not a whole number of 16-byte chunks: no bulk copy can take
         # them, so they are staged by per-thread loads
         (16, 30001, 4.0, 11, 1), (32, 12345, 3.0, 12, 0),
         # narrow bands: one block of channels, most strips at the band's edges
         (16, 1000, 2.0, 13, 0), (32, 700, 2.0, 14, 0)]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"T{c[0]}_N{c[1]}_s{c[3]}")
@pytest.mark.parametrize("precision", ["bf16", "fp16"])
def test_16bit_forms_return_the_fp32_hit_list(torch_cuda, case, precision):
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    T, N, md, seed, spikes = case
    spec = SearchSpec(T, N, max_drift=md, seed=900 + seed, n_tones=8, n_spikes=spikes, tone_drift=min(md, 4.0),
                      tsamp=18.253611 * 16 / max(T, 16), snr_threshold=8.0)
    xt = torch_cuda.from_numpy(make_filterbank_numpy(spec)).cuda()
    dd = Dedopplerer(T, N, spec.foff_mhz, spec.tsamp)
    want = _hits(dd, xt, spec)
    dd.set_precision(precision)
    got = _hits(dd, xt, spec)
    st = dd.last_stats()
    assert got == want
    assert len(want) >= 1
    assert 0 < st.recomputed_channels <= st.total_channels
    # a second call on the same engine (scratch reuse) gives the same answer
    assert _hits(dd, xt, spec) == want
    dd.close()


def _fp64_top(oracle, x, spec):
    """Per-channel maximum over eligible paths (the reference's rule), FP64 tree."""
    Tr, N = x.shape
    res = 1e6 * spec.foff_mhz / ((Tr - 1) * spec.tsamp)
    nmax = spec.max_drift / abs(res * (Tr - 1))
    top = np.zeros(N)
    c = np.arange(N)
    for db in range(int(np.floor(-nmax)), int(np.floor(nmax)) + 1):
        out = oracle.taylor_f64(x, db)
        e = (Tr - 1) * db
        for off in range(Tr):
            ok = (c + e >= 0) & (c + e + off < N)
            v = np.where(ok, out[off], -np.inf)
            top = np.maximum(top, np.nan_to_num(v, nan=-np.inf))
    return top


ERROR_CASES = {
    # the node's coarse-channel model (16 timesteps, GBT resolution), narrower for the oracle
    "node_16": dict(T=16, N=32768, foff_hz=2.7939677, tsamp=18.253611, max_drift=4.0),
    # the beamformed model (256 timesteps, 3.81 Hz, 0.268 s, 10 Hz/s)
    "beams_256": dict(T=256, N=8192, foff_hz=1e6 / 262144, tsamp=0.268435456, max_drift=10.0),
    # one of the uneven mix's shapes (64 timesteps, tsamp scaled to the same span)
    "uneven_64": dict(T=64, N=16384, foff_hz=2.7939677, tsamp=18.253611 * 16 / 64, max_drift=6.0),
}


@pytest.mark.parametrize("name", list(ERROR_CASES))
def test_path_sum_error_against_fp64_oracle(torch_cuda, port_oracle, name):
    """States the top-path-sum error of each form against the FP64 tree (printed as one JSON
    line per case), and bounds it: FP32 1e-6, FP16 1e-3 (2e-3 for 16 and 32 rows, whose tree
    adds in FP16: four or five levels of 2^-11), BF16 1e-2 relative (to the top sum), over the
    channels whose top is above the median top."""
    import json
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    c = ERROR_CASES[name]
    spec = SearchSpec(c["T"], c["N"], foff_hz=c["foff_hz"], tsamp=c["tsamp"], max_drift=c["max_drift"], seed=77,
                      n_tones=8, tone_drift=min(c["max_drift"], 4.0), snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    ref = _fp64_top(port_oracle, x, spec)
    xt = torch_cuda.from_numpy(x).cuda()
    dd = Dedopplerer(spec.num_timesteps, spec.num_channels, spec.foff_mhz, spec.tsamp)
    dd.search_raw(xt, -1, 0, spec.max_drift, 0.0, spec.snr_threshold)
    top32 = dd.channel_array("top").cpu().numpy().astype(np.float64)
    sel = ref > np.percentile(ref, 50)  # the approximate tops are floored at 0 in normalised units
    err = {"fp32": float(np.max(np.abs(top32[sel] - ref[sel]) / ref[sel]))}
    for prec, bound in (("fp16", 2e-3 if c["T"] <= 32 else 1e-3), ("bf16", 1e-2)):
        dd.set_precision(prec)
        dd.search_raw(xt, -1, 0, spec.max_drift, 0.0, spec.snr_threshold)
        st = dd.last_stats()
        approx = (dd.channel_array("top16").cpu().numpy().astype(np.float64) * st.norm_std
                  + spec.num_timesteps * st.norm_mean)
        err[prec] = float(np.max(np.abs(approx[sel] - ref[sel]) / ref[sel]))
        assert err[prec] < bound, (prec, err[prec])
    dd.close()
    print(json.dumps({"fp64_error_case": name, "shape": [spec.rounded_timesteps, spec.num_channels],
                      "drift_blocks": spec.num_drift_blocks(), "max_relative_top_error": err}))
    assert err["fp32"] < 1e-6


def _bound_patterns():
    rng = np.random.default_rng(77)
    out = []
    for T, N in ((16, 65536), (32, 32768), (64, 20000)):
        out.append((f"exponential_T{T}", rng.exponential(1.0, (T, N)).astype(np.float32)))
        out.append((f"heavy_tail_T{T}", (rng.exponential(1.0, (T, N)) ** 4).astype(np.float32)))
        x = rng.exponential(1.0, (T, N)).astype(np.float32)
        x[:, rng.integers(0, N, 40)] += 200.0  # bright columns and lines
        x[rng.integers(0, T, 30), rng.integers(0, N, 30)] += 1000.0
        out.append((f"spiky_T{T}", x))
        out.append((f"signed_T{T}", (rng.standard_normal((T, N)) * 5.0 - 1.0).astype(np.float32)))
        out.append((f"offset_T{T}", (1e4 + rng.exponential(1.0, (T, N))).astype(np.float32)))
    # one value so far above the rest that a 16-row FP16 sum could overflow: every channel
    # is listed and recomputed
    x = rng.exponential(1.0, (16, 65536)).astype(np.float32)
    x[7, 12345] = 3e7
    out.append(("overflow_T16", x))
    return out


@pytest.mark.parametrize("name,x", _bound_patterns(), ids=[p[0] for p in _bound_patterns()])
@pytest.mark.parametrize("precision", ["bf16", "fp16"])
@pytest.mark.parametrize("snr", [3.0, 10.0])
def test_flag_bound_covers_every_channel_at_the_threshold(torch_cuda, name, x, precision, snr):
    """The flag threshold is a rounding bound, not a fixed margin: at any SNR threshold, on
    noise, heavy tails, spikes, signed values and a large offset, every channel whose FP32
    top reaches the threshold is listed and recomputed (its top in the 16-bit form equals the
    FP32 top bit for bit), and the hit lists are identical."""
    from seticore_b200 import Dedopplerer
    T, N = x.shape
    xt = torch_cuda.from_numpy(x).cuda()
    dd = Dedopplerer(T, N, 2.7939677e-6, 18.253611 * 16 / T)
    h32 = [(h.index, h.drift_steps, np.float32(h.power)) for h in dd.search_raw(xt, -1, 0, 4.0, 0.0, snr)]
    top32 = dd.channel_array("top").cpu().numpy().copy()
    thr = np.float32(dd.last_stats().threshold)
    dd.set_precision(precision)
    h16 = [(h.index, h.drift_steps, np.float32(h.power)) for h in dd.search_raw(xt, -1, 0, 4.0, 0.0, snr)]
    top16 = dd.channel_array("top").cpu().numpy()
    st = dd.last_stats()
    dd.close()
    assert np.float32(st.threshold) == thr
    need = np.nonzero(top32 >= thr)[0]
    np.testing.assert_array_equal(top16[need].view(np.uint32), top32[need].view(np.uint32))
    assert h16 == h32
    assert st.recomputed_channels >= len(need)
    if name.startswith("overflow"):
        assert st.recomputed_channels == st.total_channels


def _round_bf16(y32):
    """float32 -> BF16 (round to nearest even), returned as float32 values."""
    b = y32.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32)


def _fp16_tree_top(y16, dmin, dmax):
    """Per-channel maximum, floored at 0, of the 16-row tree in FP16 arithmetic (every add
    rounded once to FP16, as __hadd2 does) over drift blocks dmin..dmax, leaves y16[t] read at
    c + db*t (0 outside the band)."""
    T, N = y16.shape
    top = np.zeros(N, dtype=np.float16)
    for db in range(dmin, dmax + 1):
        rows = []
        for t in range(T):
            r = np.zeros(N + 64, dtype=np.float16)
            lo, hi = max(0, -db * t), min(N, N - db * t)
            if hi > lo:
                r[lo:hi] = y16[t, lo + db * t:hi + db * t]
            rows.append(r)
        level = {(t, 0): rows[t] for t in range(T)}  # (block, offset) -> values at c
        L = 1
        while L < T:
            nxt = {}
            for b in range(T // (2 * L)):
                for o in range(2 * L):
                    a = level[(2 * b, o // 2)]
                    s = (o + 1) // 2
                    bb = np.zeros_like(a)
                    bb[:len(a) - s] = level[(2 * b + 1, o // 2)][s:]
                    nxt[(b, o)] = (a.astype(np.float64) + bb.astype(np.float64)).astype(np.float16)
            level = nxt
            L *= 2
        for o in range(T):
            top = np.maximum(top, level[(0, o)][:N])
    return top.astype(np.float32)


@pytest.mark.parametrize("T", [16, 32])
@pytest.mark.parametrize("precision", ["fp16", "bf16"])
def test_paired_fp16_tree_equals_the_fp16_recursion(torch_cuda, precision, T):
    """The 16- and 32-row trees of the 16-bit forms run two drift blocks per instruction in
    FP16 pairs.  Away from the band's edges its approximate tops equal, bit for bit, the tree's
    recursion evaluated in FP16 on the normalised copy (an odd drift-block count leaves the last
    pair half empty); and the hits equal the FP32 form's with the pairs on and off."""
    from seticore_b200 import Dedopplerer, _capi
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    L = _capi.lib()
    # a drift limit of exactly k drift blocks gives 2k + 1 of them (an odd count)
    tsamp = 18.253611 * 16 / T
    probe = SearchSpec(T, 8192, seed=4242, tsamp=tsamp)
    diag = (1e6 * probe.foff_mhz / ((T - 1) * probe.tsamp)) * (T - 1)
    k = next(k for k in range(3, 12) if (k * diag) / abs(diag) == k)
    spec = SearchSpec(T, 8192, max_drift=k * diag, seed=4242, n_tones=6, tone_drift=min(k * diag, 2.0),
                      snr_threshold=8.0, tsamp=tsamp)
    x = make_filterbank_numpy(spec)
    xt = torch_cuda.from_numpy(x).cuda()
    dd = Dedopplerer(T, 8192, spec.foff_mhz, spec.tsamp)
    want = _hits(dd, xt, spec)
    dd.set_precision(precision)
    got = _hits(dd, xt, spec)
    st = dd.last_stats()
    top16 = dd.channel_array("top16").cpu().numpy()
    assert got == want
    # the normalising pass's float arithmetic: (x - float(mean)) * float(1 / std), each step rounded
    y = (x.astype(np.float32) - np.float32(st.norm_mean)) * np.float32(1.0 / st.norm_std)
    if precision == "bf16":
        y = _round_bf16(y)
    y16 = y.astype(np.float16)
    res = 1e6 * spec.foff_mhz / ((T - 1) * spec.tsamp)
    nmax = spec.max_drift / abs(res * (T - 1))
    dmin, dmax = int(np.floor(-nmax)), int(np.floor(nmax))
    assert (dmax - dmin + 1) % 2 == 1  # an odd count: the last pair's second half is empty
    ref = _fp16_tree_top(y16, dmin, dmax)
    margin = (T - 1) * max(-dmin, dmax) + 2 * 1056
    mid = slice(margin, 8192 - margin)
    np.testing.assert_array_equal(top16[mid], ref[mid])
    try:
        assert L.sc_dd_set_paired_fp16(0) == _capi.SC_DD_OK
        assert _hits(dd, xt, spec) == want
        flat = dd.channel_array("top16").cpu().numpy()
        # the float-accumulating tree is within the FP16 tree's error of it
        assert np.max(np.abs(flat[mid] - ref[mid])) <= 5 * 2.0 ** -11 * np.max(np.abs(flat[mid])) * T
    finally:
        L.sc_dd_set_paired_fp16(1)
    dd.close()
