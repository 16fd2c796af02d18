"""Benchmark: dedoppler Gsamples/s and % of the HBM roofline on one wide-band node.

Workload ("node"): 64 coarse channels x 16 timesteps x 2^20 fine channels of float32
power (4.3 GB), the same noise/bandpass model per coarse channel with independent seeds,
4 drifting tones and 2 broadband spikes each; max_drift 4 Hz/s, snr_threshold 10.  One
step searches all 64 coarse channels.  Inputs live in HBM before the timed region; the
node is larger than L2, so consecutive coarse channels do not share cache.  Data are
synthetic (seticore_b200.synthetic).

`value` is the device-timed throughput (CUDA events, max over ranks); `e2e` is the same
metric through the public API with the inputs in pinned host memory, so the host->device
copy of every coarse channel is inside the timed region (copies overlap the previous
channel's search on a second stream).  Multi-GPU runs are independent replicas (weak
scaling): every rank searches its own node; nothing is exchanged.

A 1-GPU run also adds, as extra keys of the same line, the other workloads with a few timed
steps each: "beams" (64 x 256 x 131072, the level path), "uneven" (512 searches of mixed
shapes through the pool) and "serve" (Poisson arrivals of the uneven mix, p50/p99).  Each
also runs alone with --workload.

--impl reference times the reference's own CPU Taylor path (oracle/_ref/libref_cpu.so:
the reference's taylorOneStepOneChannel over all channels, all host threads) on a
bounded sample of the same workload.
"""
import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from seticore_b200.replicas import barrier, max_over_ranks  # noqa: E402

N_COARSE = 64
T = 16
N = 1 << 20
MAX_DRIFT, MIN_DRIFT, SNR = 4.0, 0.0, 10.0
METRIC = "dedoppler Gsamples/s (FP32, 64 coarse x 16 x 2^20 node)"
UNIT = "Gsamples/s"
# DRAM bytes per searched coarse channel in the tree kernel (dram__bytes_read.sum +
# dram__bytes_write.sum of one ncu capture of a launch over 4 coarse channels: 285.93 MB +
# 27.68 MB, with the command that made it in the tree kernel's profile summary); a launch
# covering k coarse channels moves k times this.
TREE_DRAM_BYTES = 78400384
# Warp instructions the tree kernel executes per coarse channel of the node (ncu
# smsp__inst_executed.sum of the same capture: 748.2 M for 4 coarse channels).
TREE_WARP_INSTR = 748.2e6 / 4
# Level path of the beams workload, DRAM bytes per beam of 256 x 131072 (2 drift blocks, one
# whole-row pass): the emitting first level 134.3 + 213.1 MB and the last level 269.5 + 3.9 MB
# (ncu, one launch each, summarised with the level kernels' profile).
BEAMS_DRAM_BYTES = 620.7e6
# Kernels of one FP32 batch of up to 64 searches of 2^20 channels and at most 32 rows (the
# launch list of one node step under ncu): clear, tree, range, three
# histogram passes, compaction, order-statistic finish, two variance kernels, window, drift
# recovery, and the exact statistics' launches, which exit at once when no search needs them
# (reset, init, 15 partition rounds of three launches, two finishers, moments).
LAUNCHES_PER_BATCH = 62


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        out, _ = self.proc.communicate(timeout=10)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak_hbm():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def bytes_read_per_drift_block(Tr, n, ndb):
    """The reference's schedule, per search: one stats read, one tree read per drift block and
    a (sum, drift, offset) write per channel: 4*Tr*N*(ndb+1) + 12*N.  The fused tree reads its
    input about once, so this is not a bound for it; it is reported only under this name."""
    return 4 * Tr * n * (ndb + 1) + 12 * n


def bytes_fused_fp32(Tr, n):
    """What the fused FP32 tree must move per search: the input read once and the per-channel
    top sums and column sums written, 4*Tr*N + 8*N."""
    return 4 * Tr * n + 8 * n


def bytes_paired_16bit(Tr, n):
    """What the 16-bit forms of a 16-row search must move, their tree adding FP16 pairs of two
    drift blocks: the float32 input read once by the normalising pass (plus three sampled rows
    for its scale), the paired copy (4 bytes per value) written and read once by the tree, and
    the per-channel tops and column sums: 4*Tr*N + 12*N + 4*Tr*N*2 + 8*N."""
    return 12 * Tr * n + 20 * n


def num_sms():
    import torch
    return torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count


def cpu_baseline(kind="reference", steps=1):
    """The reference CPU Taylor path on one coarse channel of the node (bounded sample)."""
    from oracle.oracle import Oracle, available
    from seticore_b200.synthetic import config_node, make_filterbank_numpy
    if kind == "reference" and not available("reference"):
        kind = "port"
    orc = Oracle(kind)
    threads = orc.max_threads()
    spec = config_node(1)[0]
    x = make_filterbank_numpy(spec)
    times = []
    for _ in range(steps):
        t0 = time.perf_counter()
        orc.search(x, spec.foff_mhz, spec.tsamp, MAX_DRIFT, MIN_DRIFT, SNR)
        times.append(time.perf_counter() - t0)
    sec = float(np.median(times))
    value = spec.samples() / sec / 1e9
    return {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "ms_per_step": sec * 1e3,
            "sample": f"1 coarse channel (16 x 2^20, {spec.num_drift_blocks()} drift blocks), "
                      f"{sec:.2f} s per search, median of {steps}"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    for _ in range(args.warmup):
        pass  # the CPU path has no warm-up state beyond the first call below
    cb = cpu_baseline("reference", steps=max(1, args.steps))
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": cb["ms_per_step"],
            "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "node: 64 coarse x 16 x 2^20 float32, max_drift 4 Hz/s, snr 10 "
                                   "(CPU sample: 1 coarse channel per step)"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _hit_keys(res):
    return [[(h.index, h.drift_steps, h.power) for h in hs] for hs in res]


def _uneven_requests(torch, n, precision="fp32", seed=4000):
    """The uneven mix on the device: T in {16..256}, N in {2^16..2^20}, max_drift U(1, 10)."""
    from seticore_b200 import SearchRequest
    from seticore_b200.synthetic import config_uneven, make_filterbank_torch
    specs = config_uneven(n, base_seed=seed)
    reqs = []
    for i, sp in enumerate(specs):
        x = make_filterbank_torch(sp)
        reqs.append(SearchRequest(x, sp.num_timesteps, sp.foff_mhz, sp.tsamp, sp.max_drift, sp.min_drift,
                                  sp.snr_threshold, beam=-1, coarse_channel=i, precision=precision))
    torch.cuda.synchronize()
    return specs, reqs


def _with_precision(reqs, prec):
    import dataclasses
    return [dataclasses.replace(r, precision=prec) for r in reqs]


def _time_pool(torch, pool, reqs, steps, warmup, stream):
    for _ in range(max(3, warmup)):
        pool.search_raw(reqs, stream=stream)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        res = pool.search_raw(reqs, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, res


def uneven_result(world, rank, local, n, steps, warmup, subsets=True):
    """Batched uneven searches through the pool (sc_dd_pool): autotuned on the first call,
    captured as CUDA graphs on the second, replayed afterwards; FP32 and BF16 storage (the
    whole mix, and the searches of 16 timesteps on their own)."""
    import torch
    from seticore_b200 import SearchPool
    specs, reqs = _uneven_requests(torch, n, seed=4000 + 1000 * rank)
    samples = sum(r.input.shape[0] * r.input.shape[1] for r in reqs)
    stream = torch.cuda.current_stream()
    pool = SearchPool(scratch_budget_bytes=16 << 30)
    barrier(world)
    clocks = Clocks(local)
    clocks.start()
    ms, res32 = _time_pool(torch, pool, reqs, steps, warmup, stream)
    clk = clocks.stop()
    ms = max_over_ranks(ms, world)
    st = pool.stats()
    calls = max(1, st.calls)
    out = {"metric": "dedoppler Gsamples/s (FP32, 512 uneven searches)", "value": world * samples / (ms / 1e3) / 1e9,
           "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"uneven: {n} searches, T in {{16,32,64,128,256}}, N in {{2^16,2^17,2^18,2^20}}, "
                                  "max_drift U(1,10) Hz/s, 0-6 tones SNR 12-80", "samples_per_step": samples,
                      "input_bytes": samples * 4, "l2": "inputs larger than L2; no flush"},
           "pool": {"sub_batches_per_call": st.sub_batches / calls, "graph_captures": st.graph_captures,
                    "graph_replays": st.graph_replays, "tuned_launches": st.tuned_launches},
           "clocks": clk, "hits_per_step": sum(len(h) for h in res32)}
    keys32 = _hit_keys(res32)
    # The searches of 16 timesteps alone, FP32 against BF16 / FP16 storage (identical hits required).
    t16 = [r for r in reqs if r.input.shape[0] <= 16]
    sub = {}
    if t16 and subsets:
        s16 = sum(r.input.shape[0] * r.input.shape[1] for r in t16)
        for prec in ["fp32", "bf16", "fp16"]:
            rq = _with_precision(t16, prec)
            p = SearchPool(scratch_budget_bytes=16 << 30)
            m, r = _time_pool(torch, p, rq, steps, warmup, stream)
            m = max_over_ranks(m, world)
            sub[prec] = {"value": world * s16 / (m / 1e3) / 1e9, "ms_per_step": m}
            if prec == "fp32":
                k32 = _hit_keys(r)
            else:
                sub[prec]["hits_identical_to_fp32"] = _hit_keys(r) == k32
            p.close()
        sub["searches"] = len(t16)
        sub["samples_per_step"] = s16
    out["t16_subset"] = sub
    # The whole mix with BF16 storage.
    rq = _with_precision(reqs, "bf16")
    p = SearchPool(scratch_budget_bytes=16 << 30)
    m, r = _time_pool(torch, p, rq, steps, warmup, stream)
    m = max_over_ranks(m, world)
    out["bf16_mix"] = {"value": world * samples / (m / 1e3) / 1e9, "ms_per_step": m,
                       "hits_identical_to_fp32": _hit_keys(r) == keys32}
    p.close()
    pool.close()
    del reqs, rq
    return out


def run_uneven(args, world, rank, local):
    out = uneven_result(world, rank, local, args.count or 512, args.steps, args.warmup)
    if rank == 0:
        print(json.dumps(out), flush=True)


# Serving shape: three workers (streams) and batches of at most 1e8 samples while the queue is
# short (the cap grows to a third of the queued samples when more waits).  On the uneven mix
# this measured capacity 57.5 Gsamples/s with p50 / p99 of 9.1 / 24.9 ms at 1.0x load; a fixed
# cap 48.0-55.7 with 6.9-7.4 / 15.6-16.7 ms; no cap and two workers 62.0 with 11.0 / 28.6 ms.
SERVE_WORKERS = 3
SERVE_BATCH_SAMPLES = 100_000_000


def serve_result(world, rank, local, n_inputs, serve_seconds):
    """Continuous batching (seticore_b200.serving): Poisson arrivals of searches drawn from
    the uneven mix, admitted by a 120 GB HBM budget, inputs resident on the device.
    Capacity is measured first with every request submitted at once; then arrivals are
    offered at 0.5, 0.8, 1.0 and 1.2 x capacity.  Latency is arrival to result (wall clock)."""
    import torch
    from seticore_b200 import SearchPool, SearchServer, run_load
    specs, reqs = _uneven_requests(torch, n_inputs, seed=5000 + 1000 * rank)
    stream = torch.cuda.current_stream()
    ref = SearchPool(scratch_budget_bytes=16 << 30)
    ref_keys = _hit_keys(ref.search_raw(reqs, stream=stream))
    ref.close()
    budget = 120 << 30
    out = {"metric": "serving p50/p99 latency and Gsamples/s (uneven mix)", "unit": "s", "n_gpus": world,
           "data": "synthetic", "higher_is_better": False,
           "config": {"workload": f"serve: {n_inputs} resident inputs from the uneven mix, Poisson arrivals, "
                                  "120 GB HBM budget, 3 workers, at most 64 requests and 1e8 samples per batch "
                                  "(or a third of the queued samples, if more)",
                      "budget_bytes": budget, "workers": SERVE_WORKERS, "max_batch_samples": SERVE_BATCH_SAMPLES},
           "forms": {}}
    for form in ["fp32", "bf16"]:
        base = reqs if form == "fp32" else _with_precision(reqs, "bf16")
        server = SearchServer(hbm_budget_bytes=budget, workers=SERVE_WORKERS, max_batch=64,
                              max_batch_samples=SERVE_BATCH_SAMPLES)
        # warm-up: every request alone (identical-hits check), then the capacity pattern once,
        # so that the launch classes the timed runs meet are tuned; then tuning is off
        got = [f.result() for f in [server.submit(r) for r in base]]
        identical = _hit_keys([g[0] for g in got]) == ref_keys
        n_cap = 2 * n_inputs
        for f in [server.submit(base[i % n_inputs]) for i in range(n_cap)]:
            f.result()
        server.set_autotune(False)
        # capacity: the median of three saturated runs, so that a one-off stall (a pool
        # growing its arena, a first launch) does not set the offered loads
        cap_runs = []
        for _ in range(3):
            t0 = time.perf_counter()
            futs = [server.submit(base[i % n_inputs]) for i in range(n_cap)]
            for f in futs:
                f.result()
            cap_runs.append(time.perf_counter() - t0)
        cap_s = float(np.median(cap_runs))
        cap_rps = n_cap / cap_s
        # each input's latency alone (submitted on an idle server): the service time that
        # the loaded latencies are divided by (the mix spans 16 x 2^16 to 256 x 2^20, so the
        # plain p99 / p50 mostly reflects request size, not queueing)
        alone = np.array([server.submit(base[i]).result()[1] for i in range(n_inputs)])
        samples = sum(base[i % n_inputs].input.shape[0] * base[i % n_inputs].input.shape[1] for i in range(n_cap))
        points = []
        for load in [0.5, 0.8, 1.0, 1.2]:
            rate = load * cap_rps
            n_req = int(min(16 * n_inputs, max(64, rate * serve_seconds)))
            _, lat, wall, smp = run_load(lambda i: base[i % n_inputs], n_req, rate, server, seed=int(load * 100))
            slow = lat / alone[np.arange(n_req) % n_inputs]
            points.append({"offered_load": load, "rate_per_s": rate, "requests": n_req,
                           "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                           "slowdown_p50": float(np.percentile(slow, 50)),
                           "slowdown_p99": float(np.percentile(slow, 99)),
                           "gsamples_per_s": smp / wall / 1e9})
        st = dict(server.stats)
        server.close()
        out["forms"][form] = {"capacity_requests_per_s": cap_rps, "capacity_gsamples_per_s": samples / cap_s / 1e9,
                              "capacity_runs_s": cap_runs,
                              "alone_p50_s": float(np.percentile(alone, 50)),
                              "alone_p99_s": float(np.percentile(alone, 99)),
                              "hits_identical_to_fp32": identical, "points": points, "server": st}
    del reqs
    return out


def run_serve(args, world, rank, local):
    out = serve_result(world, rank, local, args.count or 128, args.serve_seconds)
    if rank == 0:
        print(json.dumps(out), flush=True)


def beams_result(world, rank, local, n, steps, warmup):
    """Beamformed-style case: 64 beams x 256 timesteps x 131072 channels (foff 3.81 Hz,
    tsamp 0.268 s, max_drift 10 Hz/s), one batched call; more than 32 rows, so the
    level path runs."""
    import torch
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import config_beams, make_filterbank_torch
    specs = config_beams(n, base_seed=3000 + 1000 * rank)
    sp = specs[0]
    data = torch.empty((n, sp.rounded_timesteps, sp.num_channels), dtype=torch.float32, device="cuda")
    for i, s in enumerate(specs):
        make_filterbank_torch(s, out=data[i])
    torch.cuda.synchronize()
    dd = Dedopplerer(sp.num_timesteps, sp.num_channels, sp.foff_mhz, sp.tsamp)
    stream = torch.cuda.current_stream()
    inputs = [data[i] for i in range(n)]
    for _ in range(max(3, warmup)):
        res = dd.search_batch_raw(inputs, list(range(n)), [0] * n, sp.max_drift, 0.0, sp.snr_threshold, stream=stream)
    barrier(world)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        res = dd.search_batch_raw(inputs, list(range(n)), [0] * n, sp.max_drift, 0.0, sp.snr_threshold, stream=stream)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1) / steps, world)
    samples = n * sp.rounded_timesteps * sp.num_channels
    keys32 = _hit_keys(res)
    precision = {}
    for prec in ["bf16", "fp16"]:
        dd.set_precision(prec)
        for _ in range(max(3, warmup)):
            got = dd.search_batch_raw(inputs, list(range(n)), [0] * n, sp.max_drift, 0.0, sp.snr_threshold,
                                      stream=stream)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        for _ in range(steps):
            dd.search_batch_raw(inputs, list(range(n)), [0] * n, sp.max_drift, 0.0, sp.snr_threshold, stream=stream)
        p1.record(stream)
        torch.cuda.synchronize()
        st = dd.last_stats()
        p_ms = max_over_ranks(p0.elapsed_time(p1) / steps, world)
        precision[prec] = {"value": world * n * sp.rounded_timesteps * sp.num_channels / (p_ms / 1e3) / 1e9,
                           "ms_per_step": p_ms, "hits_identical_to_fp32": _hit_keys(got) == keys32,
                           "recomputed_channels_first_search": f"{st.recomputed_channels}/{st.total_channels}"}
    dd.set_precision("fp32")
    peak, peak_src = measured_peak_hbm()
    ndb = sp.num_drift_blocks()
    out = {"metric": "dedoppler Gsamples/s (FP32, 64 beams x 256 x 131072)", "value": world * samples / (ms / 1e3) / 1e9,
           "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warmup, "ms_per_step": ms,
           "higher_is_better": True, "scaling": "weak", "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"beams: {n} x 256 x 131072, foff 3.81 Hz, tsamp 0.268 s, max_drift 10 Hz/s",
                      "drift_blocks": sp.num_drift_blocks(), "input_bytes": samples * 4},
           "clocks": clk, "hits_per_step": sum(len(h) for h in res), "precision_forms": precision,
           "hbm": {"peak_gbs": peak, "peak_source": peak_src,
                   "dram_bytes_per_beam": BEAMS_DRAM_BYTES,
                   "dram_frac_of_step": n * BEAMS_DRAM_BYTES / (ms / 1e3) / 1e9 / peak,
                   "input_read_once_frac_of_step": 4 * samples / (ms / 1e3) / 1e9 / peak,
                   "bytes_if_read_per_drift_block_frac": n * bytes_read_per_drift_block(
                       sp.rounded_timesteps, sp.num_channels, ndb) / (ms / 1e3) / 1e9 / peak}}
    dd.close()
    del data, inputs
    return out


def run_beams(args, world, rank, local):
    out = beams_result(world, rank, local, args.count or 64, args.steps, args.warmup)
    if rank == 0:
        print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--fp32-only", action="store_true", help="skip the BF16/FP16 precision-form lines")
    ap.add_argument("--coarse", type=int, default=N_COARSE,
                    help="coarse channels per node (64; fewer only for small profiling captures)")
    ap.add_argument("--workload", default="node", choices=["node", "uneven", "serve", "beams"],
                    help="node (the headline line); uneven, serve and beams print their own lines")
    ap.add_argument("--count", type=int, default=0, help="searches of the uneven / serve / beams workloads")
    ap.add_argument("--serve-seconds", type=float, default=8.0, help="offered-load duration per serving point")
    ap.add_argument("--no-extra", action="store_true",
                    help="node line only (by default a 1-GPU run adds the beams, uneven and serve results)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.impl == "ours" and args.workload != "node":
        {"uneven": run_uneven, "serve": run_serve, "beams": run_beams}[args.workload](args, world, rank, local)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
        return

    import torch
    from seticore_b200 import Dedopplerer
    from seticore_b200.synthetic import config_node, make_filterbank_torch

    n_coarse = args.coarse
    specs = config_node(n_coarse, base_seed=2000 + 1000 * rank)
    data = torch.empty((n_coarse, T, N), dtype=torch.float32, device="cuda")
    for i, s in enumerate(specs):
        make_filterbank_torch(s, out=data[i])
    torch.cuda.synchronize()
    spec0 = specs[0]
    dd = Dedopplerer(T, N, spec0.foff_mhz, spec0.tsamp)
    stream = torch.cuda.current_stream()

    tree_ms = []
    hits_per_step = []
    inputs = [data[i] for i in range(n_coarse)]
    beams = [-1] * n_coarse
    coarse = list(range(n_coarse))

    def step(record=False):
        res = dd.search_batch_raw(inputs, beams, coarse, MAX_DRIFT, MIN_DRIFT, SNR, stream=stream)
        if record:
            tree_ms.append(dd.last_stats().tree_ms)
        hits_per_step.append(sum(len(h) for h in res))

    for _ in range(max(3, args.warmup)):
        step()
    barrier(world)
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(record=True)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, world)
    samples_per_step = n_coarse * T * N
    value = world * samples_per_step / (ms / 1e3) / 1e9

    # The precision forms on the same node: identical hit lists required.
    ref_hits = dd.search_batch_raw(inputs, beams, coarse, MAX_DRIFT, MIN_DRIFT, SNR, stream=stream)
    ref_key = [[(h.index, h.drift_steps, h.power) for h in hs] for hs in ref_hits]
    precision = {}
    for prec in ([] if args.fp32_only else ["bf16", "fp16"]):
        dd.set_precision(prec)
        for _ in range(max(3, args.warmup)):
            got = dd.search_batch_raw(inputs, beams, coarse, MAX_DRIFT, MIN_DRIFT, SNR, stream=stream)
        identical = [[(h.index, h.drift_steps, h.power) for h in hs] for hs in got] == ref_key
        barrier(world)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        ptree = []
        for _ in range(args.steps):
            dd.search_batch_raw(inputs, beams, coarse, MAX_DRIFT, MIN_DRIFT, SNR, stream=stream)
            ptree.append(dd.last_stats().tree_ms)
        p1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        st = dd.last_stats()
        p_ms = max_over_ranks(p0.elapsed_time(p1) / args.steps, world)
        alg16 = bytes_paired_16bit(T, N) * n_coarse
        peak16, _ = measured_peak_hbm()
        precision[prec] = {"value": world * samples_per_step / (p_ms / 1e3) / 1e9, "unit": UNIT, "ms_per_step": p_ms,
                           "hbm_frac_of_step": alg16 / (p_ms / 1e3) / 1e9 / peak16,
                           "bytes_per_step": alg16,
                           "bytes_per_step_note": "three sampled rows + one normalising read, the paired FP16 "
                                                  "copy written and read once by the tree, tops and column sums "
                                                  "(12*Tr*N + 20*N per search)",
                           "hits_identical_to_fp32": identical,
                           "recomputed_channels_first_search": f"{st.recomputed_channels}/{st.total_channels}",
                           "tree_ms": float(np.median(ptree)) if ptree else None,
                           "tree_note": "the 16-row tree launch (paired FP16: two drift blocks per __hadd2), "
                                        "CUDA events on the launching stream",
                           "speedup_vs_fp32": ms / p_ms}
    dd.set_precision("fp32")

    # End to end through the public API: host (pinned) -> device copies inside the timing,
    # in chunks of E2E_CHUNK coarse channels; the copy of chunk j+1 overlaps the search of j.
    e2e = None
    if not args.no_e2e:
        E2E_CHUNK = 8
        host = torch.empty((n_coarse, T, N), dtype=torch.float32, pin_memory=True)
        host.copy_(data)
        bufs = [torch.empty((E2E_CHUNK, T, N), dtype=torch.float32, device="cuda") for _ in range(2)]
        copy_stream = torch.cuda.Stream()
        done = [torch.cuda.Event() for _ in range(2)]
        freed = [torch.cuda.Event() for _ in range(2)]
        chunks = [(j, min(E2E_CHUNK, n_coarse - j)) for j in range(0, n_coarse, E2E_CHUNK)]

        def issue_copy(ci):
            j, m = chunks[ci]
            b = ci % 2
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(freed[b])
                bufs[b][:m].copy_(host[j:j + m], non_blocking=True)
                done[b].record(copy_stream)

        def e2e_step():
            nbytes = 0
            issue_copy(0)
            for ci, (j, m) in enumerate(chunks):
                b = ci % 2
                if ci + 1 < len(chunks):
                    issue_copy(ci + 1)
                stream.wait_event(done[b])
                dd.search_batch_raw([bufs[b][k] for k in range(m)], [-1] * m, list(range(j, j + m)),
                                    MAX_DRIFT, MIN_DRIFT, SNR, stream=stream)
                freed[b].record(stream)
                # the bytes the call copied device -> host (headers and candidates), as the
                # library counted them
                nbytes += dd.last_stats().d2h_bytes
            return nbytes

        for f in freed:
            f.record(stream)
        e2e_step()
        torch.cuda.synchronize()
        e2e_steps = max(1, min(args.steps, 3))
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d2h = 0
        for _ in range(e2e_steps):
            d2h = e2e_step()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        e_ms = max_over_ranks(e0.elapsed_time(e1) / e2e_steps, world)
        e2e = {"value": world * samples_per_step / (e_ms / 1e3) / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(host.numel() * 4), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e_ms}
        del host

    ndb = spec0.num_drift_blocks()
    per_launch = min(n_coarse, 64)
    # tree_ms times the one tree-kernel launch that covers the first (up to) 64 searches
    tree_launch_ms = float(np.mean(tree_ms))
    peak, peak_src = measured_peak_hbm()
    alg = bytes_fused_fp32(T, N) * per_launch
    achieved = alg / (tree_launch_ms / 1e3) / 1e9
    traffic = TREE_DRAM_BYTES * per_launch
    sms = num_sms()
    sm_mhz = clk.get("sm_mhz") or 1965.0
    # Instruction issue: 4 warp instructions per clock per SM at the sampled SM clock.
    issue_roof_ms = TREE_WARP_INSTR * per_launch / (sms * 4 * sm_mhz * 1e6) * 1e3
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_source": peak_src,
                "kernel": "tree_max_kernel<float,16,1,33> (8 warps, 2 CTAs per SM, leaves reread from 12)",
                "searches_per_launch": per_launch, "kernel_ms": tree_launch_ms,
                "algorithmic_bytes_per_launch": alg,
                "algorithmic_bytes_note": "input read once + top sums and column sums written, 4*Tr*N + 8*N "
                                          "per search",
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per coarse channel "
                                  "(one capture of a 4-channel launch) x searches per launch",
                "traffic_frac": traffic / (tree_launch_ms / 1e3) / 1e9 / peak,
                "binding_limit": "instruction issue",
                "issue_roof": {"warp_instructions_per_launch": TREE_WARP_INSTR * per_launch, "sms": sms,
                               "sm_mhz": sm_mhz, "roof_ms": issue_roof_ms, "frac": issue_roof_ms / tree_launch_ms,
                               "source": "ncu smsp__inst_executed.sum (one capture of a 4-channel launch)"},
                "bytes_if_read_per_drift_block": bytes_read_per_drift_block(T, N, ndb) * per_launch,
                "bytes_if_read_per_drift_block_note": "the reference's schedule (one input read per drift "
                                                      "block); not a bound for the fused kernel"}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"node: {n_coarse} coarse x 16 x 2^20 float32, 4 tones + 2 spikes per coarse "
                                   "channel, max_drift 4 Hz/s, snr 10", "drift_blocks": ndb,
                       "l2": "inputs (4.3 GB) larger than L2; no flush", "parallelism": f"replicas x{world}"},
            "clocks": clk, "roofline": roofline, "e2e": e2e,
            "precision_forms": precision,
            # per batch of up to 64 coarse channels (LAUNCHES_PER_BATCH)
            "gpu_launches": len(tree_ms) * LAUNCHES_PER_BATCH * ((n_coarse + 63) // 64),
            "hits_per_step": hits_per_step[-1]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline("reference", steps=3)
    dd.close()
    if world == 1 and not args.no_extra:
        # The other workloads, each bounded to a few seconds of timed work, as extra keys of this
        # line: the node's buffers are released first (the uneven mix holds 71 GB of inputs).
        inputs = data = bufs = host = None  # noqa: F841
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        extra_steps = max(1, min(args.steps, 3))
        for key, fn in (("beams", lambda: beams_result(world, rank, local, 64, max(1, min(args.steps, 5)), 3)),
                        ("uneven", lambda: uneven_result(world, rank, local, 512, extra_steps, 3, subsets=False)),
                        ("serve", lambda: serve_result(world, rank, local, 64, min(args.serve_seconds, 2.0)))):
            try:
                line[key] = fn()
            except Exception as exc:  # recorded, so that the headline line still prints
                line[key] = {"error": f"{type(exc).__name__}: {exc}"}
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
