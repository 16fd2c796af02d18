"""The noise statistics of a search against the oracle.

The reference forms median, mean and deviation on the host (dedoppler.cu:242-262): three
std::nth_element calls, a double sum and a float sum of squared deviations, both in the order
the nth_element calls leave the column sums.  The oracle runs exactly that code.  A search of
two rows [c; 0] has column sums c + 0 = c, so any column-sum pattern can be fed to the GPU
statistics.

Median and mean always equal the oracle's.  With exact statistics on (every search), or by
default for column sums whose order statistics sit on values held by 8 or more column sums
(integer-valued power), the GPU forms them in the reference's own nth_element order and
std_dev and threshold are bit-identical too (order_exact).  Otherwise the float variance is
emulated in channel order: std_dev within the 1e-4 parity bar (about 2e-5 to 4e-5 on these
patterns), except on column sums whose squared deviations span many orders of magnitude,
where the order decides which terms vanish under the running sum's half ulp (the
exp_heavy_tail pattern, 3.3e-4): there only the exact mode matches.
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


def _patterns():
    rng = np.random.default_rng(123)
    out = []
    for n in (64, 65, 100, 1001, 4099, 20000, 65536, 300001, 1 << 20):
        out.append((f"random_{n}", (rng.random(n) * 1e9).astype(np.float32)))
    n = 1 << 18
    out += [
        ("sorted", np.arange(n, dtype=np.float32)),
        ("reversed", np.arange(n, 0, -1, dtype=np.float32)),
        ("constant", np.full(n, 7.0, np.float32)),
        ("two_values", rng.integers(0, 2, n).astype(np.float32)),
        ("few_values", rng.integers(0, 5, n).astype(np.float32) * 3.0),
        ("organ_pipe", np.concatenate([np.arange(n // 2), np.arange(n // 2, 0, -1)]).astype(np.float32)),
        ("sawtooth", (np.arange(n) % 97).astype(np.float32)),
        ("quantised_sums", rng.integers(0, 256, (16, n)).sum(axis=0).astype(np.float32)),
        ("exp_heavy_tail", rng.exponential(1.0, n).astype(np.float32) ** 6),
        ("wide_range", (np.float32(2.0) ** rng.integers(-60, 60, n)).astype(np.float32)),
        ("negative_mixed", (rng.standard_normal(n) * 1e6).astype(np.float32)),
        ("with_zeros", np.where(rng.random(n) < 0.5, 0.0, rng.random(n) * 1e10).astype(np.float32)),
        ("large_odd", (rng.random((1 << 20) + 7) * 1e10).astype(np.float32)),
    ]
    return out


@pytest.fixture(params=["auto", "always"])
def exact_mode(request):
    from seticore_b200 import _capi
    L = _capi.lib()
    assert L.sc_dd_set_exact_statistics(1 if request.param == "always" else 0) == _capi.SC_DD_OK
    yield request.param
    L.sc_dd_set_exact_statistics(0)


def _has_ties(c):
    s = np.sort(c.astype(np.float64))
    n = len(c)
    picks = [s[int(np.ceil(0.05 * n))], s[n // 2], s[int(np.floor(0.95 * n))]]
    return max(int(np.count_nonzero(s == v)) for v in picks) >= 8


@pytest.mark.parametrize("name,c", _patterns(), ids=[p[0] for p in _patterns()])
def test_statistics_against_oracle(torch_cuda, port_oracle, exact_mode, name, c):
    from seticore_b200 import Dedopplerer
    N = c.shape[0]
    x = np.zeros((2, N), np.float32)
    x[0] = c
    dd = Dedopplerer(2, N, 2.7939677e-6, 18.253611)
    dd.search_raw(torch_cuda.from_numpy(x).cuda(), -1, 0, 1.0, 0.0, 10.0)
    g = dd.last_stats()
    colsum = dd.channel_array("colsum").cpu().numpy()
    dd.close()
    np.testing.assert_array_equal(colsum.view(np.uint32), (c + np.float32(0.0)).view(np.uint32))
    _, w = port_oracle.search(x, 2.7939677e-6, 18.253611, 1.0, 0.0, 10.0)
    want_exact = exact_mode == "always" or _has_ties(c)
    assert g.order_exact == (1 if want_exact else 0), (name, exact_mode)
    assert np.float32(g.median) == np.float32(w["median"]), (name, g.median, w["median"])
    assert np.float32(g.mean).view(np.uint32) == np.float32(w["mean"]).view(np.uint32), (name, g.mean, w["mean"])
    if want_exact:
        assert np.float32(g.std_dev).view(np.uint32) == np.float32(w["std_dev"]).view(np.uint32), \
            (name, g.std_dev, w["std_dev"])
        assert np.float32(g.threshold) == np.float32(w["threshold"]), (name, g.threshold, w["threshold"])
    else:
        tol = 5e-4 if name == "exp_heavy_tail" else 1e-4
        assert abs(g.std_dev - w["std_dev"]) <= tol * abs(w["std_dev"]), (name, g.std_dev, w["std_dev"])


def test_statistics_of_a_batch(torch_cuda, port_oracle):
    """64 searches in one launch (one CTA each) with integer-valued column sums (ties): every
    one bit-exact."""
    from seticore_b200 import Dedopplerer
    rng = np.random.default_rng(5)
    N = 1 << 16
    xs = []
    for k in range(64):
        x = np.zeros((2, N), np.float32)
        x[0] = rng.integers(0, 40 + k, N).astype(np.float32)
        xs.append(x)
    dd = Dedopplerer(2, N, 2.7939677e-6, 18.253611)
    for k, x in enumerate(xs):
        dd.search_raw(torch_cuda.from_numpy(x).cuda(), -1, 0, 1.0, 0.0, 10.0)
        g = dd.last_stats()
        _, w = port_oracle.search(x, 2.7939677e-6, 18.253611, 1.0, 0.0, 10.0)
        assert np.float32(g.std_dev) == np.float32(w["std_dev"]), k
    # the same inputs as one batch: the first search's statistics are reported
    dd.search_batch_raw([torch_cuda.from_numpy(x).cuda() for x in xs], [-1] * 64, list(range(64)), 1.0, 0.0, 10.0)
    g = dd.last_stats()
    _, w = port_oracle.search(xs[0], 2.7939677e-6, 18.253611, 1.0, 0.0, 10.0)
    assert np.float32(g.std_dev) == np.float32(w["std_dev"]) and g.order_exact == 1
    dd.close()
