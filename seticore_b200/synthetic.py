"""Seeded synthetic filterbanks for tests and benchmarks.

There are no real observations on the machines this runs on, so every workload is
generated: power[t][c] = bandpass(c) * Exp(1) * 1e9, with bandpass(c) = 1 + 0.2 P(c/N)
for a seeded degree-4 polynomial P scaled to max |P| = 1 on [0, 1].  Linear drifting tones
add A = snr * sigma / T per row along chan(t) = c0 + round(rate * t * tsamp / foff_hz),
where sigma is the 5-95 % standard deviation of the noise's column sums (the statistic the
search normalises by).  Broadband spikes add A = snr * sigma / T to one channel in every
row.  Rows between the unrounded and rounded timestep counts stay zero, as a zero-padded
coarse channel does.

Parameters are drawn with numpy's PCG64 (seeded), so a spec always yields the same
signals; the noise comes from numpy (backend="numpy") or torch's generator on a CUDA
device (backend="torch", for gigabyte workloads).
"""
from dataclasses import dataclass, field
from typing import List, Tuple

import numpy as np

GBT_FOFF_HZ = 2.7939677
GBT_TSAMP = 18.253611


@dataclass
class Signal:
    kind: str  # "tone" or "spike"
    start_channel: int
    drift_rate: float  # Hz/s (0 for spikes)
    snr: float


@dataclass
class SearchSpec:
    num_timesteps: int
    num_channels: int
    foff_hz: float = GBT_FOFF_HZ
    tsamp: float = GBT_TSAMP
    max_drift: float = 4.0
    min_drift: float = 0.0
    snr_threshold: float = 10.0
    seed: int = 0
    n_tones: int = 8
    tone_snr: Tuple[float, float] = (15.0, 100.0)
    tone_drift: float = 4.0  # |rate| <= this, Hz/s
    n_spikes: int = 0
    spike_snr: float = 50.0
    signals: List[Signal] = field(default_factory=list)

    @property
    def rounded_timesteps(self) -> int:
        r = 1
        while r < self.num_timesteps:
            r *= 2
        return r

    @property
    def foff_mhz(self) -> float:
        return self.foff_hz * 1e-6

    def num_drift_blocks(self) -> int:
        tr = self.rounded_timesteps
        res = 1e6 * self.foff_mhz / ((tr - 1) * self.tsamp)
        nmax = self.max_drift / abs(res * (tr - 1))
        return int(np.floor(nmax)) - int(np.floor(-nmax)) + 1

    def samples(self) -> int:
        return self.rounded_timesteps * self.num_channels


def _bandpass(rng, n):
    coef = rng.normal(size=5)
    x = np.linspace(0.0, 1.0, 4097)
    p = np.polyval(coef, x)
    scale = np.max(np.abs(p))
    xc = np.arange(n, dtype=np.float64) / n
    return (1.0 + 0.2 * np.polyval(coef, xc) / scale).astype(np.float32)


def _sigma_numpy(power):
    cs = power.sum(axis=0, dtype=np.float64)
    n = cs.size
    s = np.sort(cs)
    first, last = int(np.ceil(0.05 * n)), int(np.floor(0.95 * n))
    return float(np.std(s[first:last + 1]))


def _plan_signals(spec: SearchSpec, rng):
    sigs = []
    n = spec.num_channels
    span = spec.tone_drift * spec.tsamp * spec.num_timesteps / spec.foff_hz
    margin = int(min(n // 4, span + 8))
    for _ in range(spec.n_tones):
        sigs.append(Signal("tone", int(rng.integers(margin, n - margin)),
                           float(rng.uniform(-spec.tone_drift, spec.tone_drift)),
                           float(rng.uniform(*spec.tone_snr))))
    for _ in range(spec.n_spikes):
        sigs.append(Signal("spike", int(rng.integers(0, n)), 0.0, spec.spike_snr))
    return sigs


def _inject(spec, power_set, sigma, sigs):
    """power_set(t, c, value) adds value at (t, c)."""
    T = spec.num_timesteps
    for s in sigs:
        amp = s.snr * sigma / T
        for t in range(T):
            if s.kind == "spike":
                c = s.start_channel
            else:
                c = s.start_channel + int(np.round(s.drift_rate * t * spec.tsamp / spec.foff_hz))
            if 0 <= c < spec.num_channels:
                power_set(t, c, amp)


def make_filterbank_numpy(spec: SearchSpec) -> np.ndarray:
    """[rounded T][N] float32 host array for `spec` (and fills spec.signals)."""
    rng = np.random.default_rng(spec.seed)
    bp = _bandpass(rng, spec.num_channels)
    sigs = _plan_signals(spec, rng)
    noise_rng = np.random.default_rng([spec.seed, 1])
    out = np.zeros((spec.rounded_timesteps, spec.num_channels), dtype=np.float32)
    out[: spec.num_timesteps] = noise_rng.standard_exponential(
        (spec.num_timesteps, spec.num_channels), dtype=np.float32) * np.float32(1e9) * bp
    sigma = _sigma_numpy(out[: spec.num_timesteps])

    def add(t, c, v):
        out[t, c] += np.float32(v)

    _inject(spec, add, sigma, sigs)
    spec.signals = sigs
    return out


def make_filterbank_torch(spec: SearchSpec, out=None, device="cuda"):
    """The same model generated on a CUDA device with torch's generator (fast for
    gigabyte workloads).  Writes into `out` ([rounded T][N] float32) if given."""
    import torch
    rng = np.random.default_rng(spec.seed)
    bp = torch.from_numpy(_bandpass(rng, spec.num_channels)).to(device)
    sigs = _plan_signals(spec, rng)
    if out is None:
        out = torch.zeros((spec.rounded_timesteps, spec.num_channels), dtype=torch.float32, device=device)
    else:
        out.zero_()
    g = torch.Generator(device=device)
    g.manual_seed(int(spec.seed) * 7919 + 17)
    body = out[: spec.num_timesteps]
    body.exponential_(1.0, generator=g)
    body.mul_(1e9).mul_(bp)
    cs = body.sum(dim=0, dtype=torch.float64)
    s, _ = torch.sort(cs)
    n = spec.num_channels
    first, last = int(np.ceil(0.05 * n)), int(np.floor(0.95 * n))
    sigma = float(s[first:last + 1].std(unbiased=False))
    ts, cs_, vs = [], [], []

    def add(t, c, v):
        ts.append(t)
        cs_.append(c)
        vs.append(v)

    _inject(spec, add, sigma, sigs)
    if ts:
        idx_t = torch.tensor(ts, device=device)
        idx_c = torch.tensor(cs_, device=device)
        out.index_put_((idx_t, idx_c), torch.tensor(vs, dtype=torch.float32, device=device), accumulate=True)
    spec.signals = sigs
    return out


# ---- the benchmark configurations (shapes and value distributions) ----

def config_single(seed=1000) -> SearchSpec:
    """Plain FP32 single coarse channel: 16 x 2^20, 8 tones SNR 15-100, +-4 Hz/s."""
    return SearchSpec(16, 1 << 20, seed=seed, n_tones=8, max_drift=4.0, snr_threshold=10.0)


def config_node(n_coarse=64, base_seed=2000) -> List[SearchSpec]:
    """One wide-band node: 64 coarse channels x 16 x 2^20, 4 tones + 2 spikes each."""
    return [SearchSpec(16, 1 << 20, seed=base_seed + i, n_tones=4, n_spikes=2, max_drift=4.0,
                       snr_threshold=10.0) for i in range(n_coarse)]


def config_beams(n_beams=64, base_seed=3000) -> List[SearchSpec]:
    """Beamformed-style: 64 beams x 256 x 131072, foff ~3.81 Hz, tsamp ~0.27 s, 10 Hz/s."""
    return [SearchSpec(256, 131072, foff_hz=1e6 / 262144, tsamp=0.268435456, max_drift=10.0,
                       seed=base_seed + i, n_tones=4, tone_drift=10.0, tone_snr=(15.0, 100.0))
            for i in range(n_beams)]


def config_uneven(n=512, base_seed=4000) -> List[SearchSpec]:
    """512 uneven searches: T in {16..256}, N in {2^16, 2^17, 2^18, 2^20}, max_drift U(1,10)."""
    rng = np.random.default_rng(base_seed)
    out = []
    for i in range(n):
        T = int(rng.choice([16, 32, 64, 128, 256]))
        N = int(rng.choice([65536, 131072, 262144, 1 << 20]))
        md = float(rng.uniform(1.0, 10.0))
        out.append(SearchSpec(T, N, tsamp=GBT_TSAMP * 16 / T, max_drift=md, seed=base_seed + 1 + i,
                              n_tones=int(rng.integers(0, 7)), tone_snr=(12.0, 80.0),
                              tone_drift=min(md, 4.0)))
    return out
