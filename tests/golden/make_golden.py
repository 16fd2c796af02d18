"""Generates tests/golden/golden.json from the reference's own code.

Run in a container where the reference tree exists (make -C oracle builds
oracle/_ref/libref_cpu.so from it): `python tests/golden/make_golden.py`.
Every tree step in libref_cpu.so is the reference's taylorOneStepOneChannel
(taylor.h:30-86); the per-channel top, statistics and window logic of that library is
the restatement in oracle/dedoppler_oracle.cpp.  The fixtures store, per case:
  * tree: sha256 of the float32 path sums of every valid path (invalid entries zeroed),
    for inputs 1 + t + c (the reference's taylor_test.cu:8-51 input) and seeded noise;
  * search: the hit list and statistics of seeded synthetic searches.
Inputs are regenerated from their seeds; their sha256 is stored to detect drift.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle.oracle import Oracle  # noqa: E402
from seticore_b200.synthetic import SearchSpec, make_filterbank_numpy  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def tree_valid_digest(out):
    z = np.where(np.isnan(out), np.float32(0), out).astype(np.float32)
    return digest(z)


def ramp_input(T, N):
    t = np.arange(T, dtype=np.float32)[:, None]
    c = np.arange(N, dtype=np.float32)[None, :]
    return (1.0 + t + c).astype(np.float32)


def noise_input(T, N, seed):
    return (np.random.default_rng(seed).standard_exponential((T, N), dtype=np.float32) * 1e9).astype(np.float32)


SEARCH_CASES = [
    dict(name="t16_n8192", T=16, N=8192, seed=11, n_tones=6, max_drift=4.0, snr=10.0, foff_hz=2.7939677),
    dict(name="t8_n4099_negfoff", T=8, N=4099, seed=12, n_tones=5, max_drift=2.0, snr=8.0, foff_hz=-2.7939677),
    dict(name="t4_n3000", T=4, N=3000, seed=13, n_tones=4, max_drift=1.0, snr=6.0, foff_hz=2.7939677),
    dict(name="t32_n4096", T=32, N=4096, seed=14, n_tones=5, max_drift=2.0, snr=10.0, foff_hz=2.7939677),
    dict(name="t13_n5000_padded", T=13, N=5000, seed=15, n_tones=5, max_drift=3.0, snr=9.0, foff_hz=2.7939677),
    dict(name="t64_n2048", T=64, N=2048, seed=16, n_tones=3, max_drift=0.5, snr=10.0, foff_hz=2.7939677),
]


def search_spec(case):
    return SearchSpec(case["T"], case["N"], foff_hz=case["foff_hz"], max_drift=case["max_drift"],
                      snr_threshold=case["snr"], seed=case["seed"], n_tones=case["n_tones"],
                      tone_drift=min(case["max_drift"], 4.0), tsamp=18.253611 * 16 / max(case["T"], 16))


def main():
    ref = Oracle("reference")
    out = {"generator": "tests/golden/make_golden.py", "tree": [], "search": []}
    for T in (4, 8, 16, 32, 64, 128):
        for kind in ("ramp", "noise"):
            N = 1000
            x = ramp_input(T, N) if kind == "ramp" else noise_input(T, N, 100 + T)
            for db in range(-2, 3):
                out["tree"].append(dict(T=T, N=N, kind=kind, db=db, input_sha256=digest(x),
                                        valid_sha256=tree_valid_digest(ref.taylor(x, db))))
    for case in SEARCH_CASES:
        spec = search_spec(case)
        x = make_filterbank_numpy(spec)
        hits, stats = ref.search(x, spec.foff_mhz, spec.tsamp, spec.max_drift, spec.min_drift,
                                 spec.snr_threshold)
        out["search"].append(dict(case=case, input_sha256=digest(x), hits=hits,
                                  stats={k: (float(v) if isinstance(v, float) else v) for k, v in stats.items()}))
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path, len(out["tree"]), "tree cases,", len(out["search"]), "searches")


if __name__ == "__main__":
    main()
