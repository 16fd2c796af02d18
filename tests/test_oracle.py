"""Pins the CPU oracle (oracle/dedoppler_oracle.cpp) to the reference.

* The reference's own unit tests, restated: taylor_test.cu:8-51 (the tree for every
  T in 4..128 and drift block in [-2, 2] on input 1 + t + c) and dedoppler_test.cpp:9-33
  (one hit at index 70 drifting 3 bins).
* Golden vectors made by the reference's own taylorOneStepOneChannel
  (tests/golden/make_golden.py through oracle/_ref/libref_cpu.so).
* When libref_cpu.so is present, a direct comparison on fresh inputs.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from oracle.oracle import Oracle, available
from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _ramp(T, N):
    return (1.0 + np.arange(T, dtype=np.float32)[:, None] + np.arange(N, dtype=np.float32)[None, :]).astype(np.float32)


def _noise(T, N, seed):
    return (np.random.default_rng(seed).standard_exponential((T, N), dtype=np.float32) * 1e9).astype(np.float32)


@pytest.mark.parametrize("case", GOLDEN["tree"], ids=lambda c: f"T{c['T']}_{c['kind']}_db{c['db']}")
def test_tree_matches_reference_golden(port_oracle, case):
    T, N = case["T"], case["N"]
    x = _ramp(T, N) if case["kind"] == "ramp" else _noise(T, N, 100 + T)
    assert _digest(x) == case["input_sha256"]
    out = port_oracle.taylor(x, case["db"])
    z = np.where(np.isnan(out), np.float32(0), out).astype(np.float32)
    assert _digest(z) == case["valid_sha256"]


def _golden_input(case):
    from tests.golden.make_golden import search_spec
    spec = search_spec(case)
    return spec, make_filterbank_numpy(spec)


@pytest.mark.parametrize("entry", GOLDEN["search"], ids=lambda e: e["case"]["name"])
def test_search_matches_reference_golden(port_oracle, entry):
    spec, x = _golden_input(entry["case"])
    assert _digest(x) == entry["input_sha256"]
    hits, stats = port_oracle.search(x, spec.foff_mhz, spec.tsamp, spec.max_drift, spec.min_drift,
                                     spec.snr_threshold)
    assert [(h["index"], h["drift_steps"]) for h in hits] == [(h["index"], h["drift_steps"]) for h in entry["hits"]]
    for a, b in zip(hits, entry["hits"]):
        assert np.float32(a["snr"]) == np.float32(b["snr"])
        assert np.float32(a["power"]) == np.float32(b["power"])
    assert stats["window_size"] == entry["stats"]["window_size"]
    assert np.float32(stats["threshold"]) == np.float32(entry["stats"]["threshold"])


def test_reference_unit_test_taylor_basic_vs_all_T(port_oracle):
    """taylor_test.cu:8-51 restated: every valid path sum of the tree for 1 + t + c equals
    the closed form sum over the path, for T = 4..128 and drift blocks -2..2."""
    N = 1000
    for T in (4, 8, 16, 32, 64, 128):
        x = _ramp(T, N)
        for db in range(-2, 3):
            out = port_oracle.taylor(x, db)
            rng = np.random.default_rng(T * 10 + db + 2)
            for _ in range(40):
                off = int(rng.integers(0, T))
                c = int(rng.integers(0, N))
                last = (T - 1) * db + off + c
                if not (0 <= last < N):
                    assert np.isnan(out[off, c])
                    continue
                ps = port_oracle.path_sum(x, db, off, c)
                assert out[off, c] == np.float32(ps)


def test_reference_unit_test_dedoppler_known_answer(port_oracle):
    """dedoppler_test.cpp:9-33: makeNoisyBuffer(8, 1000) plus a line 70 -> 73."""
    T, N = 8, 1000
    x = np.zeros((T, N), np.float32)
    x[0] = (0.1 * np.arange(N, dtype=np.float64) / N).astype(np.float32)
    for t, c in enumerate([70, 70, 71, 71, 72, 72, 73, 73]):
        x[t, c] = 1.0
    hits, _ = port_oracle.search(x, 1.0, 1.0, 0.01, 0.01, 200.0)
    assert len(hits) == 1
    assert hits[0]["index"] == 70 and hits[0]["drift_steps"] == 3


@pytest.mark.skipif(not available("reference"), reason="libref_cpu.so not built (needs the reference tree)")
@pytest.mark.parametrize("T,N,db", [(16, 2000, -3), (16, 2000, 2), (32, 1500, -1), (64, 777, 1), (2, 500, -4)])
def test_port_equals_reference_driven_tree(port_oracle, T, N, db):
    ref = Oracle("reference")
    x = _noise(T, N, 7 + T + db)
    a = port_oracle.taylor(x, db)
    b = ref.taylor(x, db)
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b))
    np.testing.assert_array_equal(np.nan_to_num(a), np.nan_to_num(b))


def test_fp64_twin_close(port_oracle):
    x = _noise(16, 3000, 5)
    a = port_oracle.taylor(x, 1)
    b = port_oracle.taylor_f64(x, 1)
    ok = ~np.isnan(a)
    rel = np.abs(a[ok] - b[ok]) / np.abs(b[ok])
    assert rel.max() < 1e-6


def test_incoherent_power_uses_float_drift_block(port_oracle):
    x = _noise(16, 1000, 9)
    # drift_steps 15 maps to drift block 1, offset 0: the same path as block 0 offset 15
    a = port_oracle.incoherent_power(x, 15, 100)
    assert a == np.float32(port_oracle.path_sum(x, 1, 0, 100)) == np.float32(port_oracle.path_sum(x, 0, 15, 100))
    b = port_oracle.incoherent_power(x, -1, 500)
    assert b == np.float32(port_oracle.path_sum(x, -1, 14, 500))
