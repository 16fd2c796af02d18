"""The generated Taylor-tree strip code, executed on the CPU.

gen_taylor_stream.py writes the register-streaming strip functions that the tree kernels run
(seticore_b200/csrc/generated/taylor_stream_gen.cuh).  These tests translate each generated
function line by line into Python, run it on random float32 rows (numpy float32 adds round
to nearest like the device's float adds) and compare its result bit for bit with a direct
evaluation of the reference's recursion (taylor.h:30-86, drift block 0 inside the sheared
strip): node(L, b, o)[p] = node(L/2, 2b, o/2)[p] + node(L/2, 2b+1, o/2)[p + (o+1)/2].

The max-folding form must give, per channel, the maximum over its offsets floored at 0 (the
root offsets 2q and 2q+1 are folded through their shared left operand; leaves may be read again
instead of carried).  The emitting form must hand every root value to the sink.  The paired-FP16
form must give, for each of its two packed trees, the maximum of the FP16 recursion (every add
rounded to nearest FP16, as __hadd2 does).
"""
import os
import re
import sys

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "seticore_b200", "csrc")
sys.path.insert(0, CSRC)
import gen_taylor_stream as gen  # noqa: E402

sys.path.pop(0)


def _translate(code):
    """C++ strip function (the generator's restricted form) -> Python source of its body."""
    out, depth = [], 0
    for raw in code.splitlines():
        s = raw.strip()
        if (not s or s.startswith("template") or s.startswith("__device__") or s.startswith("const Row")
                or s.startswith("#pragma")):
            continue
        m = re.match(r"for \(int it = 0; it < (\d+); \+\+it\) \{$", s)
        if m:
            out.append("    " * depth + f"for it in range({m.group(1)}):")
            depth += 1
            continue
        if s == "}":
            depth = max(0, depth - 1)
            continue
        s = s.rstrip(";")
        s = re.sub(r"^float (\w+)\[(\d+)\]$", r"\1 = [None] * \2", s)
        s = re.sub(r"^const (?:float|int) ", "", s)
        s = re.sub(r"^float ", "", s)
        s = s.replace("0.0f", "F0")
        m = re.match(r"fold\(mrow, (.*), (\w+)\)$", s)
        if m:
            s = f"fold({m.group(1)}, {m.group(2)})"
        m = re.match(r"sink\.put\((\d+), (.*), (.*)\)$", s)
        if m:
            s = f"put({m.group(1)}, {m.group(2)}, {m.group(3)})"
        out.append("    " * depth + s)
    return "\n".join(out)


def _fmaxf(a, b):
    return a if a >= b else b


def _run(code, rows, S, emit=False):
    F0 = np.float32(0.0)
    top = [F0] * S
    vals = {}

    def fold(i, v):
        if v > top[i]:
            top[i] = v

    def put(i, c, v):
        vals[(i, c)] = v

    env = {"row": rows, "F0": F0, "fmaxf": _fmaxf, "fmax3": lambda a, b, c: max(a, b, c), "fold": fold,
           "put": put}
    exec(compile(_translate(code), "<generated>", "exec"), env)
    return vals if emit else top


def _reference(rows, R, lo, hi, S):
    memo = {}

    def node(L, b, o, p):
        key = (L, b, o, p)
        if key not in memo:
            if L == 1:
                memo[key] = rows[b][p]
            else:
                memo[key] = np.float32(node(L // 2, 2 * b, o // 2, p) + node(L // 2, 2 * b + 1, o // 2, p + (o + 1) // 2))
        return memo[key]

    return {(o - lo, p): node(R, 0, o, p) for o in range(lo, hi) for p in range(S)}


def _rows(R, S, seed):
    rng = np.random.default_rng(seed)
    # mixed signs and magnitudes, so that maxima, ties and the floor at 0 all occur
    return [(rng.standard_normal(S + R + 2) * rng.choice([1.0, 100.0])).astype(np.float32) for _ in range(R)]


def _configs():
    for cfg in gen.LOOP_CONFIGS:
        R, nparts, U, IT = cfg[:4]
        reload = cfg[4] if len(cfg) > 4 else 0
        step = R // nparts
        for k in range(nparts):
            yield R, k * step, (k + 1) * step, U, IT, reload


@pytest.mark.parametrize("R,lo,hi,U,IT,reload", list(_configs()),
                         ids=lambda v: str(v))
def test_max_form_equals_recursion(R, lo, hi, U, IT, reload):
    S = U * IT
    for seed in range(3):
        rows = _rows(R, S, 100 * R + 10 * lo + seed)
        got = _run(gen.gen_strip_loop(R, lo, hi, U, IT, reload=reload), rows, S)
        ref = _reference(rows, R, lo, hi, S)
        for p in range(S):
            want = max([np.float32(0.0)] + [ref[(o - lo, p)] for o in range(lo, hi)])
            assert got[p] == want, (R, lo, hi, reload, seed, p, got[p], want)
            assert np.float32(got[p]).tobytes() == np.float32(want).tobytes() or want == 0.0


@pytest.mark.parametrize("R,nparts,U,IT", gen.EMIT_CONFIGS)
def test_emit_form_writes_every_root_value(R, nparts, U, IT):
    S = U * IT
    step = R // nparts
    for k in range(nparts):
        lo, hi = k * step, (k + 1) * step
        rows = _rows(R, S, 7 + k)
        got = _run(gen.gen_strip_loop(R, lo, hi, U, IT, emit=True), rows, S, emit=True)
        ref = _reference(rows, R, lo, hi, S)
        assert set(got) == set(ref)
        for key, v in ref.items():
            assert np.float32(got[key]).tobytes() == v.tobytes(), (k, key)


def test_root_pairs_and_reload_are_used():
    """The 16-row long-strip form folds its roots in pairs and reads wide leaves again."""
    code = gen.gen_strip_loop(16, 0, 16, 11, 3, reload=12)
    assert code.count("fmaxf(") == 11 * 8  # eight pairs per channel, eleven channels per iteration
    assert "s1_15_0" not in code and "s1_11_0" in code  # leaf 15's window is reread, leaf 11's carried


def _run_direct(code, rows, CH):
    """Runs a generated taylor_direct_M function: ld(t, pos) = rows[t][pos]."""
    body = []
    for raw in code.splitlines():
        s = raw.strip()
        if not s or s.startswith("template") or s.startswith("__device__") or s == "}":
            continue
        s = s.rstrip(";")
        s = re.sub(r"^const float ", "", s)
        body.append(s)
    out, sunk = {}, {}

    def sink(o, *vals):
        for j, v in enumerate(vals):
            sunk[(o, j)] = v

    env = {"ld": lambda t, pos: rows[t][pos], "out": out, "sink": sink}
    exec(compile("\n".join(body), "<generated>", "exec"), env)
    if CH == 1:
        return {(o, 0): v for o, v in out.items()}
    return sunk


@pytest.mark.parametrize("M,CH", [(m, 1) for m in gen.DIRECT_SIZES] + list(gen.DIRECT_MULTI))
def test_direct_level_equals_recursion(M, CH):
    """The one-level subtrees of the level path: all M offsets at CH consecutive channels."""
    for seed in range(3):
        rows = _rows(M, CH + M, 300 + 10 * M + seed)
        got = _run_direct(gen.gen_direct(M, CH), rows, CH)
        ref = _reference(rows, M, 0, M, CH)
        assert set(got) == set(ref)
        for key, v in ref.items():
            assert np.float32(got[key]).tobytes() == v.tobytes(), (M, CH, seed, key)


def _h16(x):
    return np.float16(x)


def _hadd2(a, b):
    # the exact sum of two FP16 values fits a float64, so this rounds once, like __hadd2
    return np.array([_h16(np.float64(a[0]) + np.float64(b[0])), _h16(np.float64(a[1]) + np.float64(b[1]))],
                    dtype=np.float16)


def _hmax2(a, b):
    return np.array([max(a[0], b[0]), max(a[1], b[1])], dtype=np.float16)


def _run_h2(code, rows2, S):
    """Runs a generated paired-FP16 strip function: rows2[t][p] is the (2,) FP16 pair."""
    body, depth = [], 0
    for raw in code.splitlines():
        st = raw.strip()
        if (not st or st.startswith("template") or st.startswith("__device__") or st.startswith("const Row")
                or st.startswith("#pragma")):
            continue
        m = re.match(r"for \(int it = 0; it < (\d+); \+\+it\) \{$", st)
        if m:
            body.append("    " * depth + f"for it in range({m.group(1)}):")
            depth += 1
            continue
        if st == "}":
            depth = max(0, depth - 1)
            continue
        st = st.rstrip(";")
        st = re.sub(r"^__half2 (\w+)\[(\d+)\]$", r"\1 = [None] * \2", st)
        st = re.sub(r"^__half2 (\w+) = __float2half2_rn\(0.0f\)$", r"\1 = Z2", st)
        st = re.sub(r"^const (?:__half2|int) ", "", st)
        st = st.replace("__hadd2(", "hadd2(").replace("__hmax2(", "hmax2(")
        m = re.match(r"fold\(mrow, (.*), (\w+)\)$", st)
        if m:
            st = f"fold({m.group(1)}, {m.group(2)})"
        body.append("    " * depth + st)
    top = [[np.float16(0.0), np.float16(0.0)] for _ in range(S)]

    def fold(i, v):
        for h in range(2):
            if v[h] > top[i][h]:
                top[i][h] = v[h]

    env = {"row": rows2, "Z2": np.zeros(2, dtype=np.float16), "hadd2": _hadd2, "hmax2": _hmax2, "fold": fold}
    exec(compile("\n".join(body), "<generated>", "exec"), env)
    return top


def _reference_h16(rows, R, lo, hi, S):
    memo = {}

    def node(L, b, o, p):
        key = (L, b, o, p)
        if key not in memo:
            if L == 1:
                memo[key] = rows[b][p]
            else:
                memo[key] = _h16(np.float64(node(L // 2, 2 * b, o // 2, p)) +
                                 np.float64(node(L // 2, 2 * b + 1, o // 2, p + (o + 1) // 2)))
        return memo[key]

    return {(o - lo, p): node(R, 0, o, p) for o in range(lo, hi) for p in range(S)}


@pytest.mark.parametrize("R,nparts,U,IT,reload", gen.H2_CONFIGS)
def test_paired_fp16_form_equals_fp16_recursion(R, nparts, U, IT, reload):
    S = U * IT
    step = R // nparts
    for k in range(nparts):
        lo, hi = k * step, (k + 1) * step
        for seed in range(2):
            a = [r.astype(np.float16) for r in _rows(R, S, 500 + 10 * k + seed)]
            b = [r.astype(np.float16) for r in _rows(R, S, 900 + 10 * k + seed)]
            rows2 = [np.stack([a[t], b[t]], axis=1) for t in range(R)]
            got = _run_h2(gen.gen_strip_loop(R, lo, hi, U, IT, reload=reload, h2=True), rows2, S)
            for h, rows in enumerate((a, b)):
                ref = _reference_h16(rows, R, lo, hi, S)
                for p in range(S):
                    want = max([np.float16(0.0)] + [ref[(o - lo, p)] for o in range(lo, hi)])
                    assert got[p][h] == want, (R, lo, hi, reload, seed, h, p, got[p][h], want)
