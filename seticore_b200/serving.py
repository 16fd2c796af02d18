"""A serving loop for dedoppler searches: continuous batching under an HBM budget.

Requests arrive at any time (submit() returns a Future).  Each request carries its input
(already on the device or copied there at admission) and its search arguments.  Worker
threads -- one CUDA stream and one SearchPool each -- take every pending request that
fits the free HBM budget (input + search scratch) when they become free, run them as one
heterogeneous batch, release the memory and complete the futures.  With two or more
workers, a batch is admitted and launched while another is still on the GPU, so work
from requests that arrived at different times overlaps on the device.  A request larger
than the whole budget is rejected.

run_load() drives the server with Poisson arrivals and reports throughput and the p50 /
p99 latency (arrival to result).
"""
import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .pool import SearchPool, SearchRequest


def admit(pending_bytes, free_bytes: int, max_batch: int, pending_samples=None, max_samples=None) -> int:
    """How many of the pending requests (in arrival order) the next batch takes: the
    longest prefix whose bytes fit the free budget, at most max_batch, and -- when
    max_samples is given -- whose samples (timesteps x channels) stay within max_samples,
    though the first request is always taken if it fits the budget."""
    n = 0
    work = 0
    for i, b in enumerate(pending_bytes):
        if n >= max_batch or b > free_bytes:
            break
        if max_samples is not None and n > 0 and work + pending_samples[i] > max_samples:
            break
        free_bytes -= b
        if max_samples is not None:
            work += pending_samples[i]
        n += 1
    return n


def batch_cap(max_samples, queued_samples: int, workers: int, adaptive: bool):
    """The sample cap of the next batch: max_samples, or, when adaptive and more waits than
    the workers' share of it, an equal share of the queued samples per worker."""
    if max_samples is None or not adaptive:
        return max_samples
    return max(max_samples, queued_samples // max(1, workers))


@dataclass
class _Pending:
    req: SearchRequest
    bytes: int
    arrival: float
    samples: int = 0
    future: Future = field(default_factory=Future)


class SearchServer:
    def __init__(self, hbm_budget_bytes: int = 120 << 30, workers: int = 2, max_batch: int = 64,
                 input_bytes=None, max_batch_samples: Optional[int] = None, adaptive_cap: bool = True):
        import torch
        self.budget = int(hbm_budget_bytes)
        self.used = 0
        self.max_batch = max_batch
        self.max_batch_samples = max_batch_samples
        self.adaptive_cap = adaptive_cap
        self._input_bytes = input_bytes or (lambda r: r.input.numel() * r.input.element_size())
        self._q: deque = deque()
        self._cv = threading.Condition()
        self._stop = False
        self.stats = {"batches": 0, "requests": 0, "max_inflight_bytes": 0, "overlapped_batches": 0}
        self._running = 0
        self._threads = []
        self._pools = []
        self._autotune = True
        for i in range(workers):
            t = threading.Thread(target=self._work, args=(torch.cuda.Stream(),), daemon=True, name=f"dd-serve-{i}")
            t.start()
            self._threads.append(t)

    def submit(self, req: SearchRequest) -> Future:
        cost = self._input_bytes(req) + SearchPool.scratch_bytes(req)
        p = _Pending(req, cost, time.perf_counter(), int(req.input.shape[0]) * int(req.input.shape[1]))
        if cost > self.budget:
            p.future.set_exception(MemoryError(f"request needs {cost} bytes, budget is {self.budget}"))
            return p.future
        with self._cv:
            self._q.append(p)
            self._cv.notify()
        return p.future

    def close(self):
        with self._cv:
            self._stop = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()

    def set_autotune(self, enabled: bool):
        """Tuning times each new launch class on first sight, with synchronisations that stall
        a worker: a server warmed on its traffic turns it off, and classes not seen during the
        warm-up then take the default launch shape."""
        with self._cv:
            self._autotune = bool(enabled)
            for p in self._pools:
                p.configure(self._autotune)

    def _take(self) -> List[_Pending]:
        """Pending requests, in arrival order, that fit the free budget (at most max_batch
        requests and max_batch_samples samples).  When more work waits than the workers'
        share of the sample cap, the cap grows to an equal share of the queue per worker: a
        long queue is drained in large batches (throughput), a short one in small ones
        (latency)."""
        cap = batch_cap(self.max_batch_samples, sum(p.samples for p in self._q), len(self._threads),
                        self.adaptive_cap)
        n = admit([p.bytes for p in self._q], self.budget - self.used, self.max_batch,
                  [p.samples for p in self._q], cap)
        return [self._q.popleft() for _ in range(n)]

    def _work(self, stream):
        import torch
        # Arrival-time batches rarely repeat a composition, so captured graphs would seldom
        # replay; launch shapes are still tuned per shape class on first sight.
        pool = SearchPool(scratch_budget_bytes=max(1 << 30, self.budget // 8), cuda_graphs=False)
        with self._cv:
            pool.configure(self._autotune)
            self._pools.append(pool)
        while True:
            with self._cv:
                while not self._stop and not (self._q and self._q[0].bytes <= self.budget - self.used):
                    self._cv.wait(0.05)
                if self._stop and not self._q:
                    break
                batch = self._take()
                if not batch:
                    continue
                nbytes = sum(p.bytes for p in batch)
                self.used += nbytes
                if self._running > 0:
                    self.stats["overlapped_batches"] += 1
                self._running += 1
                self.stats["max_inflight_bytes"] = max(self.stats["max_inflight_bytes"], self.used)
            try:
                with torch.cuda.stream(stream):
                    res = pool.search_raw([p.req for p in batch], stream=stream)
                err = None
            except Exception as e:  # noqa: BLE001
                res, err = None, e
            done = time.perf_counter()
            with self._cv:
                self.used -= nbytes
                self._running -= 1
                self.stats["batches"] += 1
                self.stats["requests"] += len(batch)
                self._cv.notify_all()
            for i, p in enumerate(batch):
                if err is not None:
                    p.future.set_exception(err)
                else:
                    p.future.set_result((res[i], done - p.arrival))
        pool.close()


def run_load(make_request, n_requests: int, rate_per_s: float, server: SearchServer, seed: int = 0):
    """Poisson arrivals at rate_per_s; returns (results, latencies_s, wall_s, samples)."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_per_s, size=n_requests)
    futures, samples = [], 0
    t0 = time.perf_counter()
    t_next = t0
    for i in range(n_requests):
        t_next += gaps[i]
        now = time.perf_counter()
        if t_next > now:
            time.sleep(t_next - now)
        req = make_request(i)
        samples += req.input.shape[0] * req.input.shape[1]
        futures.append(server.submit(req))
    out = [f.result() for f in futures]
    wall = time.perf_counter() - t0
    lat = np.array([o[1] for o in out])
    return [o[0] for o in out], lat, wall, samples
