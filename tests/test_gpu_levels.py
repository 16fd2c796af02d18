"""Searches of 64 to 256 rounded timesteps: the 16-row first level and the last level run in
stripe passes (a range of channels and a few drift blocks per pass, sized so that the planes
between the levels stay in L2).  Whatever the pass size -- one 1056-channel stripe and one
drift block per pass, a few megabytes, whole rows -- the top path sums must equal the
oracle's bit for bit (the same adds in the same tree order as twoStageTaylorTree,
taylor.cu:298-327) and the hits must match.
"""
import numpy as np
import pytest

from tests.conftest import has_gpu
from tests.test_gpu_parity import compare_hits, run_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    return torch


@pytest.fixture(params=[256 << 10, 2 << 20, 0, -1], ids=["256KB", "2MB", "whole_rows", "default"])
def stripe_bytes(request):
    from seticore_b200 import _capi
    L = _capi.lib()
    assert L.sc_dd_set_level_stripe_bytes(request.param) == _capi.SC_DD_OK
    yield request.param
    L.sc_dd_set_level_stripe_bytes(-1)


CASES = [
    # T, N, foff_hz, tsamp, max_drift, n_tones, seed
    (64, 30000, 2.7939677, 4.5634028, 4.0, 5, 21),      # 14 drift blocks
    (128, 20000, -2.7939677, 2.2817014, 6.0, 4, 22),    # negative foff, 10 drift blocks
    (256, 12000, 3.814697265625, 0.268435456, 10.0, 4, 23),
    (256, 9000, 2.7939677, 1.1408507, 8.0, 3, 24),      # 8 drift blocks of 256 rows
    (64, 5000, 2.7939677, 4.5634028, 20.0, 3, 25),      # drifts wider than the band
    (100, 7000, 2.7939677, 2.2817014, 3.0, 3, 26),      # 100 timesteps, 28 zero rows
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"T{c[0]}_N{c[1]}_md{c[4]}")
def test_stripe_passes_match_oracle(torch_cuda, port_oracle, stripe_bytes, case):
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    T, N, foff_hz, tsamp, md, ntones, seed = case
    spec = SearchSpec(T, N, foff_hz=foff_hz, tsamp=tsamp, max_drift=md, seed=seed, n_tones=ntones,
                      tone_drift=min(md, 4.0), snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    want, wstats, arrays = port_oracle.search(x, spec.foff_mhz, tsamp, md, 0.0, 8.0, arrays=True)
    got, gstats, top, colsum = run_gpu(torch_cuda, x, spec.foff_mhz, tsamp, md, 0.0, 8.0, T=T)
    np.testing.assert_array_equal(top, arrays["top"])
    np.testing.assert_array_equal(colsum, arrays["colsum"])
    ties = compare_hits(got, want, gstats.threshold, wstats["threshold"], label=str(case))
    assert len(ties) <= 1, ties


@pytest.mark.parametrize("form", ["bf16", "fp16"])
def test_stripe_passes_in_16_bit_storage(torch_cuda, port_oracle, form):
    """The precision form's 16-bit rows keep the four-channels-per-thread first level whatever
    the stripe setting (the emitting tree stages float rows only); its flagged channels are
    recomputed in FP32, so the hit list equals the oracle's."""
    from seticore_b200 import Dedopplerer, _capi
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    L = _capi.lib()
    spec = SearchSpec(128, 20000, tsamp=2.2817014, max_drift=6.0, seed=31, n_tones=5, tone_drift=4.0,
                      snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    want, wstats = port_oracle.search(x, spec.foff_mhz, spec.tsamp, 6.0, 0.0, 8.0)
    assert L.sc_dd_set_level_stripe_bytes(1 << 20) == _capi.SC_DD_OK
    try:
        dd = Dedopplerer(128, 20000, spec.foff_mhz, spec.tsamp)
        dd.set_precision(form)
        hits = dd.search_raw(torch_cuda.from_numpy(x).cuda(), -1, 0, 6.0, 0.0, 8.0)
        thr = dd.last_stats().threshold
        dd.close()
    finally:
        L.sc_dd_set_level_stripe_bytes(-1)
    got = [dict(index=h.index, drift_steps=h.drift_steps, snr=h.snr, power=h.power) for h in hits]
    ties = compare_hits(got, want, thr, wstats["threshold"], label=form)
    assert len(ties) <= 1, ties


@pytest.mark.parametrize("T", [64, 256])
def test_stripe_pass_wait_give_up_is_reported(torch_cuda, port_oracle, T):
    """The stripe passes' bounded waits (the pipelined tree's stage and refill mbarriers, the
    plain tree's staging mbarrier): with the poll limit at 0 every wait gives up at once --
    nothing hangs or faults -- and the search reports SC_DD_EINTERNAL; with the default
    restored the same engine searches correctly."""
    from seticore_b200 import DedopplerError, Dedopplerer, _capi
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    spec = SearchSpec(T, 12000, foff_hz=3.814697265625, tsamp=0.268435456 * 256 / T, max_drift=10.0, seed=41,
                      n_tones=4, snr_threshold=8.0)
    x = make_filterbank_numpy(spec)
    xt = torch_cuda.from_numpy(x).cuda()
    dd = Dedopplerer(T, x.shape[1], spec.foff_mhz, spec.tsamp)
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
    np.testing.assert_array_equal(top, arrays["top"])
    assert [(h.index, h.drift_steps) for h in got] == [(h["index"], h["drift_steps"]) for h in want]
