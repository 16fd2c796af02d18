"""Generates the register-streaming Taylor-tree strip functions (taylor_stream_gen.cuh).

A lane owns a strip of S consecutive output channels of one drift block.  The input
rows sit in shared memory already sheared for that drift block, so inside the strip the
tree is the drift-block-0 recursion of the reference (taylor.h:30-86): the sum over a
block of L rows with in-block offset o starting at channel p is

    node(L, b, o)[p] = node(L/2, 2b, o/2)[p] + node(L/2, 2b+1, o/2)[p + (o+1)/2]

with node(1, t, 0)[p] = row t at channel p.  Streaming along p, every tree node value is
computed exactly once (one add) and kept in a register only while a later channel still
needs it, so the lane does the tree's minimal work -- R adds per level per channel -- and
reads each input value from shared memory once.  The in-block offsets [lo, hi) of the
root are a parameter: splitting the offsets over two warps halves the registers a lane
needs without duplicating any add (the two halves share no tree node above the leaves).

The emitted function is a loop over the strip, U channels per iteration: a prologue
fills every node's window for the first channel, the loop body is straight-line code for
U channels, and the values a later iteration still needs are carried in registers across
the back edge.  Looping (rather than unrolling the whole strip) keeps the code of one
offset half small enough for the instruction cache.  Each channel's outputs are folded into
a running maximum (starting at 0, so NaN and negative sums never count) that the caller's
fold merges into the CTA's per-channel maxima in shared memory: every channel, or only the
channels whose paths are all eligible where the band's edges exclude some.  The emitting form
(taylor_strip_emit) hands every root value to a sink instead: the first level of a tree of
more than 32 rows, whose output planes the next level reads.
"""
import os
import sys


def consumption(R, lo, hi):
    """Relative channel positions at which each (L, b, o) node value is consumed."""
    pos = {(R, 0, o): {0} for o in range(lo, hi)}
    L = R
    while L > 1:
        for (LL, b, o), P in list(pos.items()):
            if LL != L:
                continue
            h, s = o // 2, (o + 1) // 2
            pos.setdefault((L // 2, 2 * b, h), set()).update(P)
            pos.setdefault((L // 2, 2 * b + 1, h), set()).update(p + s for p in P)
        L //= 2
    return pos


def lead(R, lo, hi):
    """Largest channel offset a strip reads beyond its last output channel."""
    pos = consumption(R, lo, hi)
    return max(max(P) for (L, b, o), P in pos.items() if L == 1)


def gen_strip_loop(R, lo, hi, U, ITERS, emit=False, reload=0, h2=False):
    """Looped form: a prologue fills every node's window for step 0, then ITERS iterations
    of a U-step body; values still needed after an iteration are carried into the next
    (the loop-carried registers), and each iteration folds its U per-channel maxima into the
    warp's row of shared memory (mrow[0..U*ITERS)).

    reload > 0: leaves whose window spans `reload` positions or more are not carried; each
    use reads the row again (a shared-memory load per use instead of a register per window
    slot), which trades load bandwidth for registers and so for warps per SM.

    h2: every value is a pair of FP16 sums (__half2) of two independent trees with the same
    pairing -- two drift blocks, whose leaves the caller packs side by side -- added with
    __hadd2 and folded with __hmax2, so one instruction does the work of two float adds; the
    fold receives the pair."""
    T = "__half2" if h2 else "float"

    def add(x, y):
        return f"__hadd2({x}, {y})" if h2 else f"{x} + {y}"

    def mx(x, y):
        return f"__hmax2({x}, {y})" if h2 else f"fmaxf({x}, {y})"
    pos = consumption(R, lo, hi)
    nodes = {k: (min(P), max(P)) for k, P in pos.items() if k[0] != R}  # (mn, lead)
    reloaded = {k for k, (mn, ld) in nodes.items() if reload and k[0] == 1 and ld - mn >= reload}
    roots = [(R, 0, o) for o in range(lo, hi)]

    def nm(L, b, o):
        return f"{L}_{b}_{o}"

    def val(L, b, o, j):
        return f"v{nm(L, b, o)}_{j}".replace("-", "m")

    def st(L, b, o, k):
        return f"s{nm(L, b, o)}[{k}]"

    order = sorted(nodes.keys(), key=lambda k: k[0])  # leaves first, then bottom-up
    lines = []
    # state arrays
    for (L, b, o) in order:
        mn, ld = nodes[(L, b, o)]
        if ld - mn >= 1 and (L, b, o) not in reloaded:
            lines.append(f"  {T} s{nm(L, b, o)}[{ld - mn}];")
    # prologue: positions [mn, lead-1] of every node (bottom-up)
    def compute(L, b, o, j, src_pos_name):
        if L == 1:
            return f"row[{b}][{j}]"
        sh = (o + 1) // 2
        return add(src_pos_name(L // 2, 2 * b, o // 2, j), src_pos_name(L // 2, 2 * b + 1, o // 2, j + sh))

    def prologue_name(L, b, o, j):
        if (L, b, o) in reloaded:
            return f"row[{b}][{j}]"
        mn, ld = nodes[(L, b, o)]
        return st(L, b, o, j - mn)

    # Prologue in order of position then level, so children exist before parents.
    pro = []
    for (L, b, o) in order:
        if (L, b, o) in reloaded:
            continue
        mn, ld = nodes[(L, b, o)]
        for j in range(mn, ld):
            pro.append((j - ld, L, f"  {prologue_name(L, b, o, j)} = {compute(L, b, o, j, prologue_name)};"))
    pro.sort(key=lambda x: (x[0], x[1]))
    lines += [t for _, _, t in pro]
    lines.append(f"#pragma unroll 1")
    lines.append(f"  for (int it = 0; it < {ITERS}; ++it) {{")
    lines.append(f"    const int base = it * {U};")

    # body: value names for positions j in [mn, U-1+lead] relative to iteration start
    def body_name(L, b, o, j):
        if (L, b, o) in reloaded:
            return f"row[{b}][base + {j}]"
        mn, ld = nodes[(L, b, o)]
        if j < ld:
            return st(L, b, o, j - mn)
        return val(L, b, o, j)

    body = []
    for (L, b, o) in order:
        if (L, b, o) in reloaded:
            continue
        mn, ld = nodes[(L, b, o)]
        for j in range(ld, U + ld):
            if L == 1:
                expr = f"row[{b}][base + {j}]"
            else:
                expr = compute(L, b, o, j, body_name)
            body.append((j - ld, L, f"    const {T} {val(L, b, o, j)} = {expr};"))
    for s in range(U):
        outs = []
        for (_, _, o) in roots:
            sh = (o + 1) // 2
            outs.append(f"{body_name(R // 2, 0, o // 2, s)} + {body_name(R // 2, 1, o // 2, s + sh)}")
        if emit:
            for i, e in enumerate(outs):
                body.append((s, R, f"    sink.put({i}, base + {s}, {e});"))
            continue
        body.append((s, R, f"    __half2 m{s} = __float2half2_rn(0.0f);" if h2 else f"    float m{s} = 0.0f;"))
        # Offsets 2q and 2q + 1 share their left operand: their larger sum is
        # left + max(right at +q, right at +q + 1), exactly (rounding is monotonic, and a NaN
        # sum never counts on either side), so the pair costs one add and one max.
        outs = []
        his = {o for (_, _, o) in roots}
        for (_, _, o) in roots:
            q = o // 2
            if o % 2 == 0 and o + 1 in his:
                left = body_name(R // 2, 0, q, s)
                r0, r1 = body_name(R // 2, 1, q, s + q), body_name(R // 2, 1, q, s + q + 1)
                outs.append(add(left, mx(r0, r1)))
            elif o % 2 == 1 and o - 1 in his:
                continue
            else:
                sh = (o + 1) // 2
                outs.append(add(body_name(R // 2, 0, q, s), body_name(R // 2, 1, q, s + sh)))
        for i, e in enumerate(outs):
            body.append((s, R, f"    const {T} o{s}_{i} = {e};"))
        acc = f"m{s}"
        i = 0
        while i < len(outs):
            if i + 1 < len(outs):
                if h2:  # no three-input form for pairs
                    body.append((s, R + 1, f"    {acc} = __hmax2({acc}, __hmax2(o{s}_{i}, o{s}_{i + 1}));"))
                else:
                    body.append((s, R + 1, f"    {acc} = fmax3({acc}, o{s}_{i}, o{s}_{i + 1});"))
                i += 2
            else:
                body.append((s, R + 1, f"    {acc} = {mx(acc, f'o{s}_{i}')};"))
                i += 1
        body.append((s, R + 2, f"    fold(mrow, base + {s}, {acc});"))
    body.sort(key=lambda x: (x[0], x[1]))
    lines += [t for _, _, t in body]
    # carry: new state k holds position U + mn + k
    carry = []
    for (L, b, o) in order:
        if (L, b, o) in reloaded:
            continue
        mn, ld = nodes[(L, b, o)]
        for k in range(ld - mn):
            carry.append(f"    {st(L, b, o, k)} = {body_name(L, b, o, U + mn + k)};")
    lines += carry
    lines.append("  }")
    body_text = "\n".join(lines)
    if emit:
        return (f"template <typename Row, typename Sink>\n"
                f"__device__ __forceinline__ void taylor_strip_emit_{R}_{lo}_{hi}_{U}_{ITERS}(\n"
                f"    const Row (&row)[{R}], Sink& sink) {{\n{body_text}\n}}\n")
    return (f"template <typename Row, typename Fold>\n__device__ __forceinline__ void "
            f"{loop_name(R, lo, hi, U, ITERS, reload, h2)}(\n"
            f"    const Row (&row)[{R}], float* __restrict__ mrow, const Fold& fold) {{\n{body_text}\n}}\n")


def loop_name(R, lo, hi, U, ITERS, reload=0, h2=False):
    return (f"taylor_strip_loop{'_h2' if h2 else ''}_{R}_{lo}_{hi}_{U}_{ITERS}" +
            (f"_r{reload}" if reload else ""))


def gen_direct(M, CH=1):
    """All M root values of an M-row Taylor subtree at CH consecutive channels, as
    straight-line code: every (node, position) value the roots need is computed once from
    leaf loads ld(t, pos) (row t of the block at relative channel pos; the caller applies
    the shear), so neighbouring channels share their common nodes and leaves."""
    lines = []
    done = set()

    def nm(L, b, o, j):
        return f"n{L}_{b}_{o}_{j}"

    def emit(L, b, o, j):
        """Depth-first: a value is computed right before its first use, so leaves are
        loaded late and few values are live at once."""
        if (L, b, o, j) in done:
            return
        if L > 1:
            sh = (o + 1) // 2
            emit(L // 2, 2 * b, o // 2, j)
            emit(L // 2, 2 * b + 1, o // 2, j + sh)
            expr = f"{nm(L // 2, 2 * b, o // 2, j)} + {nm(L // 2, 2 * b + 1, o // 2, j + sh)}"
        else:
            expr = f"ld({b}, {j})"
        done.add((L, b, o, j))
        if L == M and CH == 1:
            lines.append(f"  out[{o}] = {expr};")
        else:
            lines.append(f"  const float {nm(L, b, o, j)} = {expr};")

    if CH > 1:
        # offset-major: the CH values of one offset are complete together and go to the sink
        # at once, so the outputs do not stay live until the end
        for o in range(M):
            for j in range(CH):
                emit(M, 0, o, j)
            args = ", ".join(nm(M, 0, o, j) for j in range(CH))
            lines.append(f"  sink({o}, {args});")
        body = "\n".join(lines)
        return (f"template <typename Ld, typename Sink>\n__device__ __forceinline__ void "
                f"taylor_direct_{M}x{CH}(const Ld& ld, const Sink& sink) {{\n{body}\n}}\n")
    for o in range(M):
        emit(M, 0, o, 0)
    body = "\n".join(lines)
    return (f"template <typename Ld>\n__device__ __forceinline__ void taylor_direct_{M}(const Ld& ld, "
            f"float (&out)[{M}]) {{\n{body}\n}}\n")


# (R, offset parts, U steps per iteration, iterations[, reload]) compiled into the library; a
# strip is S = U * ITERS channels (odd, so a warp's 32 strips start in 32 distinct banks);
# reload: leaves with windows of that many positions or more are read again at each use.
LOOP_CONFIGS = [(2, 1, 11, 3), (4, 1, 11, 3), (8, 1, 11, 3), (16, 1, 11, 3, 12), (16, 1, 11, 3, 8),
                # 32 rows in two parts of sixteen offsets
                (32, 2, 11, 3),
                # short strips (S = 11) for launches whose jobs each stage their own rows
                (2, 1, 11, 1), (4, 1, 11, 1), (8, 1, 11, 1), (16, 2, 11, 1)]


# (R, offset parts, U, iterations, reload) of the paired-FP16 form (two drift blocks per lane,
# the 16-bit forms' 16- and 32-row trees).
H2_CONFIGS = [(16, 1, 11, 3, 12), (16, 1, 11, 3, 10), (32, 2, 11, 3, 0)]


# (R, offset parts, U, iterations) of the emitting form: every root value goes to a sink
# (the level kernels' output planes, through a per-warp shared-memory buffer) instead of a
# running maximum.  Short strips (S = 11) keep a warp's buffer of one tile small.
EMIT_CONFIGS = [(16, 2, 11, 1), (16, 1, 11, 1)]
# Subtree sizes of the one-thread-per-channel level kernel (dd_levels.cu).
DIRECT_SIZES = [2, 4, 8, 16]
# (rows, consecutive channels per thread) of the level kernel's multi-channel form.
DIRECT_MULTI = [(16, 2), (16, 4)]


def main(out_path):
    parts = ["// GENERATED by gen_taylor_stream.py -- do not edit.\n#pragma once\n"]
    for R, nparts, U, IT, *rl in LOOP_CONFIGS:
        step = R // nparts
        for k in range(nparts):
            parts.append(gen_strip_loop(R, k * step, (k + 1) * step, U, IT, reload=rl[0] if rl else 0))
    for R, nparts, U, IT in EMIT_CONFIGS:
        step = R // nparts
        for k in range(nparts):
            parts.append(gen_strip_loop(R, k * step, (k + 1) * step, U, IT, emit=True))
    for R, nparts, U, IT, rl in H2_CONFIGS:
        step = R // nparts
        for k in range(nparts):
            parts.append(gen_strip_loop(R, k * step, (k + 1) * step, U, IT, reload=rl, h2=True))

    # Dispatcher: taylor_strip_loop<R, LO, HI, U, ITERS, RELOAD>(row, mrow, fold) for any element
    # accessor and fold (which merges a channel's maximum: all channels, or a range of them).
    parts.append("template <int R, int LO, int HI, int U, int ITERS, int RELOAD = 0, typename Row, typename Fold>\n"
                 "__device__ __forceinline__ void taylor_strip_loop(const Row (&row)[R], float* __restrict__ mrow, "
                 "const Fold& fold) {")
    for R, nparts, U, IT, *rl in LOOP_CONFIGS:
        step = R // nparts
        rel = rl[0] if rl else 0
        for k in range(nparts):
            lo, hi = k * step, (k + 1) * step
            parts.append(f"  if constexpr (R == {R} && LO == {lo} && HI == {hi} && U == {U} && ITERS == {IT} && "
                         f"RELOAD == {rel}) {loop_name(R, lo, hi, U, IT, rel)}(row, mrow, fold);")
    parts.append("}")
    parts.append("template <int R, int LO, int HI, int U, int ITERS, int RELOAD, typename Row, typename Fold>\n"
                 "__device__ __forceinline__ void taylor_strip_loop_h2(const Row (&row)[R], float* __restrict__ mrow, "
                 "const Fold& fold) {")
    for R, nparts, U, IT, rel in H2_CONFIGS:
        step = R // nparts
        for k in range(nparts):
            lo, hi = k * step, (k + 1) * step
            parts.append(f"  if constexpr (R == {R} && LO == {lo} && HI == {hi} && U == {U} && ITERS == {IT} && "
                         f"RELOAD == {rel}) {loop_name(R, lo, hi, U, IT, rel, True)}(row, mrow, fold);")
    parts.append("}")
    parts.append("template <int R, int LO, int HI, int U, int ITERS, typename Row, typename Sink>\n"
                 "__device__ __forceinline__ void taylor_strip_emit(const Row (&row)[R], Sink& sink) {")
    for R, nparts, U, IT in EMIT_CONFIGS:
        step = R // nparts
        for k in range(nparts):
            lo, hi = k * step, (k + 1) * step
            parts.append(f"  if constexpr (R == {R} && LO == {lo} && HI == {hi} && U == {U} && ITERS == {IT}) "
                         f"taylor_strip_emit_{R}_{lo}_{hi}_{U}_{IT}(row, sink);")
    parts.append("}")
    _write(out_path, "\n".join(parts))
    direct = ["// GENERATED by gen_taylor_stream.py -- do not edit.\n#pragma once\n"]
    for M in DIRECT_SIZES:
        direct.append(gen_direct(M))
    for M, CH in DIRECT_MULTI:
        direct.append(gen_direct(M, CH))
    _write(os.path.join(os.path.dirname(out_path), "taylor_direct_gen.cuh"), "\n".join(direct))


def _write(path, text):
    if os.path.exists(path) and open(path).read() == text:
        return
    with open(path, "w") as f:
        f.write(text)


if __name__ == "__main__":
    main(sys.argv[1])
