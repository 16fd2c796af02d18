"""The reference's own GPU search (dedoppler.cu / taylor.cu built for sm_100a) against this
package's search: identical hit lists and a per-search time on the same device, for one
coarse channel of 16 x 2^20 (54 drift blocks) and one beam of 256 x 131072.  The timing of
each side includes its results on the host (the reference's search ends with a blocking
device->host copy and host-side statistics).  Prints one JSON line per case."""
import json
import time

import numpy as np
import pytest

from tests.conftest import has_gpu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", ["coarse_16x2^20", "beam_256x131072"])
def test_faster_than_reference_gpu_with_identical_hits(case):
    if not has_gpu():
        pytest.skip("no CUDA device")
    from oracle.oracle import RefGpu, available
    if not available("reference_gpu"):
        pytest.skip("oracle/_ref/libref_gpu.so not built")
    import torch
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import config_beams, config_single, make_filterbank_numpy
    spec = config_single() if case.startswith("coarse") else config_beams(1)[0]
    x = make_filterbank_numpy(spec)
    T, N = spec.num_timesteps, spec.num_channels
    md, snr = spec.max_drift, spec.snr_threshold
    ref = RefGpu()
    ctx = ref.context(T, N, spec.foff_mhz, spec.tsamp)
    ctx.load(x)
    want = ctx.search(-1, 0, md, 0.0, snr)
    ref_ms = ctx.time_search(md, 0.0, snr, 5)
    ctx.close()

    dd = Dedopplerer(T, N, spec.foff_mhz, spec.tsamp)
    dev = torch.from_numpy(x).cuda()
    for _ in range(3):
        got = dd.search_raw(dev, -1, 0, md, 0.0, snr)
    torch.cuda.synchronize()
    iters = 20
    t0 = time.perf_counter()
    for _ in range(iters):
        got = dd.search_raw(dev, -1, 0, md, 0.0, snr)
    ours_ms = (time.perf_counter() - t0) * 1e3 / iters
    dd.close()
    assert [(h.index, h.drift_steps) for h in got] == [(w["index"], w["drift_steps"]) for w in want]
    for h, w in zip(got, want):
        assert np.float32(h.power) == np.float32(w["power"])
    print(json.dumps({"case": case, "drift_blocks": spec.num_drift_blocks(), "hits": len(got),
                      "reference_gpu_ms_per_search": ref_ms, "ours_ms_per_search": ours_ms,
                      "speedup": ref_ms / ours_ms}))
    assert ours_ms < ref_ms
