"""The engine replays a repeated batch from a captured CUDA graph (second sight: capture,
later: replay).  A replay must behave exactly like a direct call: it reads the input buffer's
current contents, reports the tree's time, and is not reused when a setting that changes the
launches (exact statistics, the staging-wait limit, the storage form, the 16-bit tree's form)
or the scratch changes.
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


def _keys(hits):
    return [(h.index, h.drift_steps, np.float32(h.power), np.float32(h.snr)) for h in hits]


def test_replayed_batches_match_direct_calls(torch_cuda, port_oracle):
    torch = torch_cuda
    from seticore_b200 import Dedopplerer, _capi
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    L = _capi.lib()
    specs = [SearchSpec(16, 1 << 16, seed=80 + i, n_tones=5, snr_threshold=8.0) for i in range(3)]
    xs = [make_filterbank_numpy(s) for s in specs]
    s0 = specs[0]
    buf = [torch.from_numpy(x).cuda() for x in xs[:2]]
    dd = Dedopplerer(16, 1 << 16, s0.foff_mhz, s0.tsamp)
    runs = [dd.search_batch_raw(buf, [-1, -1], [0, 1], s0.max_drift, 0.0, 8.0) for _ in range(4)]
    st = dd.last_stats()
    assert st.tree_ms > 0.0  # timed on a replay too
    for r in runs[1:]:
        assert [_keys(h) for h in r] == [_keys(h) for h in runs[0]]
    for k in range(2):
        want, _ = port_oracle.search(xs[k], s0.foff_mhz, s0.tsamp, s0.max_drift, 0.0, 8.0)
        assert [h.index for h in runs[0][k]] == [h["index"] for h in want]
    # new contents in the same buffers: a replay reads them
    buf[0].copy_(torch.from_numpy(xs[2]).cuda())
    got = dd.search_batch_raw(buf, [-1, -1], [0, 1], s0.max_drift, 0.0, 8.0)
    want, _ = port_oracle.search(xs[2], s0.foff_mhz, s0.tsamp, s0.max_drift, 0.0, 8.0)
    assert [h.index for h in got[0]] == [h["index"] for h in want]
    assert _keys(got[1]) == _keys(runs[0][1])
    # a setting that changes the launches is not served by the old graph
    try:
        assert L.sc_dd_set_exact_statistics(1) == _capi.SC_DD_OK
        for _ in range(3):
            dd.search_batch_raw(buf, [-1, -1], [0, 1], s0.max_drift, 0.0, 8.0)
            assert dd.last_stats().order_exact == 1
    finally:
        L.sc_dd_set_exact_statistics(0)
    dd.search_batch_raw(buf, [-1, -1], [0, 1], s0.max_drift, 0.0, 8.0)
    assert dd.last_stats().order_exact == 0
    # the storage form is part of the key as well
    dd.set_precision("bf16")
    for _ in range(3):
        got16 = dd.search_batch_raw(buf, [-1, -1], [0, 1], s0.max_drift, 0.0, 8.0)
        assert dd.last_stats().precision == _capi.SC_DD_PRECISION_BF16
    assert [[(h.index, h.drift_steps) for h in r] for r in got16] == [[(h.index, h.drift_steps) for h in r] for r in got]
    # and so is the 16-bit tree's form (paired FP16 or float accumulation): a replay captured
    # with one form is not served to the other, and the hits stay the same
    try:
        assert L.sc_dd_set_paired_fp16(0) == _capi.SC_DD_OK
        for _ in range(3):
            flat = dd.search_batch_raw(buf, [-1, -1], [0, 1], s0.max_drift, 0.0, 8.0)
            assert [[(h.index, h.drift_steps) for h in r] for r in flat] == \
                [[(h.index, h.drift_steps) for h in r] for r in got]
    finally:
        L.sc_dd_set_paired_fp16(1)
    again = dd.search_batch_raw(buf, [-1, -1], [0, 1], s0.max_drift, 0.0, 8.0)
    assert [[(h.index, h.drift_steps) for h in r] for r in again] == [[(h.index, h.drift_steps) for h in r] for r in got]
    dd.close()


def test_replayed_level_batches_match_direct_calls(torch_cuda, port_oracle):
    """A batch of more than 32 rows deals its searches over the level side streams; captured
    and replayed, the fork and join events hold them all in the graph and the results stay
    those of a direct call (and of the oracle)."""
    torch = torch_cuda
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy
    specs = [SearchSpec(64, 1 << 14, tsamp=18.253611 / 4, max_drift=2.0, seed=90 + i, n_tones=4,
                        snr_threshold=8.0) for i in range(5)]
    xs = [make_filterbank_numpy(s) for s in specs]
    s0 = specs[0]
    buf = [torch.from_numpy(x).cuda() for x in xs]
    dd = Dedopplerer(64, 1 << 14, s0.foff_mhz, s0.tsamp)
    runs = [dd.search_batch_raw(buf, [-1] * 5, list(range(5)), s0.max_drift, 0.0, 8.0) for _ in range(4)]
    for r in runs[1:]:
        assert [_keys(h) for h in r] == [_keys(h) for h in runs[0]]
    for k in range(5):
        want, _ = port_oracle.search(xs[k], s0.foff_mhz, s0.tsamp, s0.max_drift, 0.0, 8.0)
        assert [(h.index, h.drift_steps) for h in runs[0][k]] == [(h["index"], h["drift_steps"]) for h in want]
    # new contents in one buffer: the replay reads them
    buf[2].copy_(torch.from_numpy(xs[4]).cuda())
    got = dd.search_batch_raw(buf, [-1] * 5, list(range(5)), s0.max_drift, 0.0, 8.0)
    assert _keys(got[2]) == _keys(runs[0][4])
    dd.close()
