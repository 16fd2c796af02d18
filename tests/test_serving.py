"""Serving loop: admission logic on the CPU; results alone vs in the mix on the GPU."""
import numpy as np
import pytest

from tests.conftest import has_gpu


def test_admission_takes_the_fitting_prefix():
    from seticore_b200.serving import admit
    assert admit([10, 20, 30], 100, 64) == 3
    assert admit([10, 20, 30], 35, 64) == 2
    assert admit([50, 10], 40, 64) == 0          # in order: a large head blocks (no reordering)
    assert admit([1] * 100, 1000, 64) == 64      # batch cap
    assert admit([], 100, 64) == 0
    # a sample cap bounds a batch's work, but the head request is always taken
    assert admit([1, 1, 1], 100, 64, [40, 40, 40], 100) == 2
    assert admit([1, 1], 100, 64, [500, 10], 100) == 1
    assert admit([1, 1], 100, 64, [10, 10], None) == 2


def test_batch_cap_grows_with_the_queue():
    from seticore_b200.serving import batch_cap
    assert batch_cap(None, 10**9, 3, True) is None
    assert batch_cap(100, 90, 3, True) == 100        # a short queue keeps the cap
    assert batch_cap(100, 900, 3, True) == 300       # a long one is shared out per worker
    assert batch_cap(100, 900, 3, False) == 100


@pytest.mark.gpu
def test_served_results_equal_results_alone():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import torch  # noqa: F401
    from seticore_b200 import Dedopplerer, SearchRequest, SearchServer
    from seticore_b200.synthetic import SearchSpec, make_filterbank_torch
    rng = np.random.default_rng(3)
    reqs = []
    for i in range(40):
        T = int(rng.choice([8, 16, 32]))
        N = int(rng.choice([16384, 65536]))
        spec = SearchSpec(T, N, tsamp=18.253611 * 16 / max(T, 16), max_drift=float(rng.uniform(1, 5)),
                          seed=7000 + i, n_tones=3, snr_threshold=8.0)
        reqs.append(SearchRequest(make_filterbank_torch(spec), T, spec.foff_mhz, spec.tsamp, spec.max_drift, 0.0,
                                  8.0, coarse_channel=i, precision="bf16" if i % 3 == 0 else "fp32"))
    alone = []
    for r in reqs:
        dd = Dedopplerer(r.num_timesteps, r.input.shape[1], r.foff, r.tsamp)
        dd.set_precision(r.precision)
        alone.append([(h.index, h.drift_steps, h.power) for h in
                      dd.search_raw(r.input, -1, r.coarse_channel, r.max_drift, 0.0, 8.0)])
        dd.close()
    budget = 3 * max(r.input.numel() * 4 for r in reqs) + (256 << 20)
    server = SearchServer(hbm_budget_bytes=budget, workers=2, max_batch=8)
    futs = [server.submit(r) for r in reqs]
    served = [f.result(timeout=300) for f in futs]
    too_big = server.submit(SearchRequest(torch.zeros((16, 1 << 24), device="cuda"), 16, 2.79e-6, 18.25, 4.0))
    with pytest.raises(MemoryError):
        too_big.result(timeout=10)
    stats = dict(server.stats)
    server.close()
    for (hits, lat), want in zip(served, alone):
        assert [(h.index, h.drift_steps, h.power) for h in hits] == want
        assert lat > 0
    assert stats["requests"] == len(reqs)
    assert stats["max_inflight_bytes"] <= budget
    assert stats["batches"] >= 2
