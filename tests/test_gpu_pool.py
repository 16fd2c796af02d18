"""Heterogeneous batches (sc_dd_pool): every request's hits equal the engine's hits for
that request alone, whatever else is in the batch, across the first call (autotuning),
the second (graph capture) and later calls (graph replay)."""
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


def _key(hits):
    return [(h.index, h.drift_steps, np.float32(h.power), np.float32(h.snr), h.coarse_channel) for h in hits]


def _mixed_requests(torch, n=24, seed=60):
    from seticore_b200 import SearchRequest
    from seticore_b200.synthetic import SearchSpec, make_filterbank_torch
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        T = int(rng.choice([4, 8, 13, 16, 32, 64]))
        N = int(rng.choice([4096, 10000, 32768, 65536]))
        md = float(rng.uniform(0.5, 6.0))
        prec = str(rng.choice(["fp32", "fp32", "bf16", "fp16"]))
        spec = SearchSpec(T, N, tsamp=18.253611 * 16 / max(T, 16), max_drift=md, seed=seed * 100 + i,
                          n_tones=int(rng.integers(1, 6)), tone_drift=min(md, 4.0), snr_threshold=8.0)
        x = make_filterbank_torch(spec)
        reqs.append(SearchRequest(x, T, spec.foff_mhz, spec.tsamp, md, 0.0, 8.0, beam=-1, coarse_channel=i,
                                  precision=prec))
    return reqs


def _alone(req):
    from seticore_b200 import Dedopplerer
    dd = Dedopplerer(req.num_timesteps, req.input.shape[1], req.foff, req.tsamp)
    dd.set_precision(req.precision)
    hits = dd.search_raw(req.input, req.beam, req.coarse_channel, req.max_drift, req.min_drift, req.snr_threshold)
    dd.close()
    return _key(hits)


def test_mixed_batch_equals_each_request_alone(torch_cuda):
    from seticore_b200 import SearchPool
    reqs = _mixed_requests(torch_cuda)
    alone = [_alone(r) for r in reqs]
    total = sum(SearchPool.scratch_bytes(r) for r in reqs)
    pool = SearchPool(scratch_budget_bytes=total // 5)  # a small budget: several admitted sub-batches
    for call in range(3):
        got = pool.search_raw(reqs)
        assert [_key(h) for h in got] == alone, f"call {call}"
    st = pool.stats()
    assert st.calls == 3 and st.sub_batches >= 3 * 5
    assert st.graph_captures >= 1 and st.graph_replays >= 1
    assert st.tuned_launches >= 1
    pool.close()


def test_request_order_does_not_change_results(torch_cuda):
    from seticore_b200 import SearchPool
    reqs = _mixed_requests(torch_cuda, n=12, seed=61)
    pool = SearchPool()
    a = [_key(h) for h in pool.search_raw(reqs)]
    b = [_key(h) for h in pool.search_raw(list(reversed(reqs)))]
    assert a == list(reversed(b))
    pool.close()
