"""The allocation-free search entry point, sc_dd_search_static.

Some callers cannot allocate device memory where they search: a real-time capture or
beamforming pipeline that reserved the GPU's memory up front and must not call cudaMalloc
in its processing loop, or a host framework whose allocator owns all device memory.
sc_dd_search_static serves them from a fixed scratch array inside the library.  These
tests call it through the C ABI twice in a row and check each result against the engine
entry point (sc_dd_search) on the same input: both run the same kernels, so the hit lists
must agree exactly (within the parity tolerance used elsewhere: SNR to 1e-4 relative).
The file is named to be collected last, so a run that stops at the first failure has run
every other test first; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from tests.conftest import has_gpu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch
    torch.cuda.init()
    return torch


def _static_search(torch, xt, T, N, spec, capacity=4096, min_drift=None):
    from seticore_b200 import _capi
    out = (_capi.ScDdHit * max(1, capacity))()
    n = ctypes.c_int(0)
    rc = _capi.lib().sc_dd_search_static(
        ctypes.c_void_p(xt.data_ptr()), xt.stride(0), T, N, spec.foff_mhz, spec.tsamp, -1, 7,
        spec.max_drift, spec.min_drift if min_drift is None else min_drift, spec.snr_threshold, out, capacity,
        ctypes.byref(n), ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    return rc, list(out[: min(n.value, capacity)]), n.value


def _as_tuples(hits):
    return [(h.index, h.drift_steps, np.float32(h.power), np.float32(h.snr), h.drift_rate, h.coarse_channel)
            for h in hits]


def _engine_search(torch, xt, T, N, spec, min_drift):
    from seticore_b200 import Dedopplerer
    dd = Dedopplerer(T, N, spec.foff_mhz, spec.tsamp)
    want = dd.search_raw(xt, -1, 7, spec.max_drift, min_drift, spec.snr_threshold)
    dd.close()
    torch.cuda.synchronize()
    return want


def _assert_same(got, want, tag):
    assert len(got) == len(want), (tag, len(got), len(want))
    for a, b in zip(_as_tuples(got), _as_tuples(want)):
        assert a[:3] == b[:3] and a[4:] == b[4:], (tag, a, b)
        assert abs(a[3] - b[3]) <= 1e-4 * abs(b[3])


def test_static_search_matches_engine_search_twice(torch_cuda):
    from seticore_b200 import _capi
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    torch = torch_cuda
    N = 1 << 18
    unchanged = []
    for call, seed in enumerate((101, 102)):
        spec = SearchSpec(16, N, seed=seed, n_tones=8, n_spikes=1, snr_threshold=8.0)
        xt = torch.from_numpy(make_filterbank_numpy(spec)).cuda()
        want = _engine_search(torch, xt, 16, N, spec, spec.min_drift)
        # Device-wide free memory around the call: another process on a shared GPU can change
        # it, so the call is repeated and one unchanged reading suffices.
        for _ in range(3):
            free_before = torch.cuda.mem_get_info()[0]
            rc, got, n = _static_search(torch, xt, 16, N, spec)
            free_after = torch.cuda.mem_get_info()[0]
            assert rc == _capi.SC_DD_OK, rc
            assert n == len(want) > 0
            _assert_same(got, want, call)
            if call == 1:
                unchanged.append(free_after == free_before)
    # After the first call has set up the device, a call takes no device memory.
    assert any(unchanged)


@pytest.mark.parametrize("T", [4, 8, 12, 16])
def test_static_search_matches_engine_for_each_row_count(torch_cuda, T):
    """Every tree the static path launches (2..16 rows, unrounded T too), with a min_drift
    that drops some hits, against the engine; and a short `out` (SC_DD_ETRUNC with the
    engine's total in *num_hits)."""
    from seticore_b200 import _capi
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    torch = torch_cuda
    N = 1 << 16
    spec = SearchSpec(T, N, seed=200 + T, n_tones=8, n_spikes=2, snr_threshold=6.0)
    x = make_filterbank_numpy(spec)
    xt = torch.from_numpy(x).cuda()
    Tr = xt.shape[0]
    everything = _engine_search(torch, xt, T, N, spec, 0.0)
    min_drift = 0.5 * max(abs(h.drift_rate) for h in everything) if everything else 0.1
    want = _engine_search(torch, xt, T, N, spec, min_drift)
    assert 0 < len(want) < len(everything), (len(want), len(everything))
    for _ in range(2):
        rc, got, n = _static_search(torch, xt, T, N, spec, min_drift=min_drift)
        assert rc == _capi.SC_DD_OK, rc
        assert n == len(want) and Tr >= T
        _assert_same(got, want, T)
    cap = len(want) - 1
    rc, got, n = _static_search(torch, xt, T, N, spec, capacity=cap, min_drift=min_drift)
    assert rc == _capi.SC_DD_ETRUNC, rc
    assert n == len(want) and len(got) == cap


def test_static_search_rejects_sizes_beyond_its_limits(torch_cuda):
    from seticore_b200 import _capi
    from seticore_b200.synthetic import SearchSpec
    torch = torch_cuda
    spec = SearchSpec(16, 1000)
    small = torch.zeros((16, 1024), device="cuda")
    too_wide = _capi.SC_DD_STATIC_MAX_CHANNELS + 1
    big = torch.zeros((1, 1), device="cuda")
    rc, _, _ = _static_search(torch, big.expand(16, too_wide), 16, too_wide, spec)
    assert rc == _capi.SC_DD_ELIMIT
    rc, _, _ = _static_search(torch, torch.zeros((32, 1024), device="cuda"), 32, 1024, spec)
    assert rc == _capi.SC_DD_ELIMIT
    rc, _, _ = _static_search(torch, small, 16, 1024, SearchSpec(16, 1024, max_drift=0.0))
    assert rc == _capi.SC_DD_EINVAL
    # A drift range beyond sc_dd_search's bound, and a max_drift that is not finite.
    for bad in (1e12, float("inf"), float("nan")):
        rc, _, _ = _static_search(torch, small, 16, 1024, SearchSpec(16, 1024, max_drift=bad))
        assert rc == _capi.SC_DD_EINVAL, (bad, rc)
