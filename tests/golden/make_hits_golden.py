"""Generates tests/golden/voyager_hits.npz from the reference's own .hits file.

Run where the reference tree exists (`REF=<tree> python tests/golden/make_hits_golden.py`;
REF defaults to oracle/Makefile's).  The
reference ships data/voyager.hits, written by its HitFileWriter (hit_file_writer.cpp) with
an earlier hit.capnp in which Signal had 4 data words and Filterbank 8 (the fields that
later versions appended read as zero).  The fixture keeps, per message, the sha256 of the
message's bytes, its struct sizes and its decoded fields, so a test can re-encode the
fields with seticore_b200.hitfiles and compare digests without the reference tree.
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from seticore_b200.hitfiles import decode_hit, split_messages  # noqa: E402

sys.path.insert(0, os.path.join(ROOT, "tests"))
from conftest import reference_root  # noqa: E402  ($REF, else oracle/Makefile's default)

SRC = os.path.join(reference_root(), "data", "voyager.hits")
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "voyager_hits.npz")


def main():
    blob = open(SRC, "rb").read()
    meta, arrays = [], {}
    for k, (raw, seg) in enumerate(split_messages(blob)):
        h = decode_hit(seg)
        fb = dict(h["filterbank"])
        arrays[f"data{k}"] = fb.pop("data")
        meta.append({"sha256": hashlib.sha256(raw).hexdigest(), "bytes": len(raw),
                     "signal": {a: b for a, b in h["signal"].items()}, "filterbank": fb})
    np.savez_compressed(OUT, meta=np.array(json.dumps(meta)), file_sha256=np.array(hashlib.sha256(blob).hexdigest()),
                        **arrays)
    print(f"wrote {OUT}: {len(meta)} messages")


if __name__ == "__main__":
    main()
