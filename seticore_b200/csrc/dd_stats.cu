// Column sums and the noise statistics of a search, on the GPU.
//
// The reference copies the column sums to the host and uses std::nth_element for the
// median and the 5% / 95% order statistics, then a mean and standard deviation over the
// sorted positions [ceil(0.05 N), floor(0.95 N)] (dedoppler.cu:322-342).  Here:
//   * colsum_kernel: sumColumns (dedoppler.cu:63-72), same sequential float order.
//   * select_pass (x4): MSB-first radix select of the three order statistics at once,
//     8 bits per pass; the last CTA of each pass picks the digits.  Exact.
//   * moments_kernel: the sum (FP64, as the reference's std::accumulate with a double
//     start) of the values between the two percentiles, with boundary ties counted
//     exactly; per-CTA partials are combined by the last CTA in a fixed order.  It forms
//     the mean with the reference's roundings (float sum, float division).
//   * var_chunk_kernel + var_emulate_kernel: the variance.  The reference accumulates
//     (f - m)^2 in FLOAT, one term at a time (dedoppler.cu:337-341).  Once the
//     accumulator is large, every term is rounded to the accumulator's ulp and terms
//     under half an ulp vanish, which biases the sum low (about 4e-4 relative at 2^20
//     channels, nearly independent of the order).  An exact FP64 variance would
//     therefore differ from the reference's by more than the SNR tolerance.  These two
//     kernels reproduce the float accumulation in parallel: an exact prefix sum gives
//     the accumulator A_i each term meets (in channel order), and the term contributes
//     rint(t_i / ulp(float(A_i))) * ulp(float(A_i)).  The result tracks a sequential
//     float sum to about 1e-5 relative; the remaining difference comes from the order
//     (the reference's order is whatever std::nth_element leaves).
#include <algorithm>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

constexpr int kSelectCtasPerSm = 16;

// Column sums of search blockIdx.y (dedoppler.cu:63-72: a float sum in row order); block 0
// also resets that search's select state.
__global__ void colsum_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& d = b.s[blockIdx.y];
  SelectState* st = d.sel;
  if (blockIdx.x == 0) {
    if (threadIdx.x < 3) {
      const int r = threadIdx.x == 0 ? d.first : (threadIdx.x == 1 ? d.mid : d.last);
      st->prefix[threadIdx.x] = 0;
      st->mask[threadIdx.x] = 0;
      st->rank[threadIdx.x] = (uint32_t)r;
      if (threadIdx.x == 0) st->ticket = 0;
    }
    for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&st->hist[0][0])[i] = 0;
  }
  const float* in = d.input;
  const long long row_stride = d.row_stride;
  const int N = d.N, Tr = d.Tr;
  const bool vec = ((reinterpret_cast<uintptr_t>(in) & 15) == 0) && ((row_stride & 3) == 0) && ((N & 3) == 0);
  if (vec) {
    const int c4 = blockIdx.x * blockDim.x + threadIdx.x;
    if (c4 * 4 >= N) return;
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
    for (int t = 0; t < Tr; ++t) {
      const float4 v = __ldg(reinterpret_cast<const float4*>(in + (long long)t * row_stride) + c4);
      acc.x += v.x;
      acc.y += v.y;
      acc.z += v.z;
      acc.w += v.w;
    }
    reinterpret_cast<float4*>(d.colsum)[c4] = acc;
  } else {
    const int c_end = min(N, (blockIdx.x + 1) * blockDim.x * 4);
    for (int c = blockIdx.x * blockDim.x * 4 + threadIdx.x; c < c_end; c += blockDim.x) {
      float acc = 0.0f;
      for (int t = 0; t < Tr; ++t) acc += __ldg(in + (long long)t * row_stride + c);
      d.colsum[c] = acc;
    }
  }
}

// Adds 1 to hist[d] for every lane whose predicate holds.  When every counted lane has
// the same digit (common for the leading digits: neighbouring channels have similar sums)
// one atomic adds them all; otherwise each lane adds to its warp's private histogram, so
// only lanes of one warp with equal digits contend.
__device__ __forceinline__ void warp_hist_add(unsigned* hist, uint32_t d, bool pred) {
  const unsigned active = __ballot_sync(0xffffffffu, pred);
  if (active == 0u) return;
  const int first = __ffs(active) - 1;
  const uint32_t d0 = __shfl_sync(0xffffffffu, d, first);
  const bool same = __all_sync(0xffffffffu, !pred || d == d0);
  if (same) {
    if ((int)(threadIdx.x & 31) == first) atomicAdd(&hist[d0], (unsigned)__popc(active));
  } else if (pred) {
    atomicAdd(&hist[d], 1u);
  }
}

// Picks, for each target, the digit whose cumulative count passes its rank: 256 threads
// scan the 256 bins in parallel.
__device__ void select_digits(SelectState* st, int shift) {
  __shared__ unsigned cnt[256];
  __shared__ unsigned incl[256];
  for (int j = 0; j < 3; ++j) {
    const int d = threadIdx.x;
    const uint32_t rank = st->rank[j];  // read before any thread can update it below
    if (d < 256) cnt[d] = __ldcg(&st->hist[j][d]);
    __syncthreads();
    if (d < 256) {
      unsigned v = cnt[d];
      // inclusive scan over 256 bins (8 warps x 32) via shared memory doubling
      incl[d] = v;
    }
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
      unsigned add = 0;
      if (d < 256 && d >= o) add = incl[d - o];
      __syncthreads();
      if (d < 256) incl[d] += add;
      __syncthreads();
    }
    if (d < 256) {
      const unsigned before = incl[d] - cnt[d];
      if (rank >= before && rank < incl[d]) {
        st->rank[j] = rank - before;
        st->prefix[j] |= (uint32_t)d << shift;
        st->mask[j] |= 255u << shift;
      }
    }
    __syncthreads();
  }
}

// One 8-bit radix-select pass for the three target ranks.
__global__ void __launch_bounds__(256) select_pass(const __grid_constant__ SearchBatch b, int shift) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ x = sd.colsum;
  const int N = sd.N;
  SelectState* st = sd.sel;
  __shared__ unsigned whist[8][3][256];  // one histogram per warp
  __shared__ bool last_block;
  for (int i = threadIdx.x; i < 8 * 3 * 256; i += blockDim.x) (&whist[0][0][0])[i] = 0;
  __syncthreads();
  unsigned (*hist)[256] = whist[threadIdx.x >> 5];
  const uint32_t p0 = st->prefix[0], p1 = st->prefix[1], p2 = st->prefix[2];
  const uint32_t m0 = st->mask[0], m1 = st->mask[1], m2 = st->mask[2];
  const int stride = gridDim.x * blockDim.x;
  const int n_round = ((N + stride - 1) / stride) * stride;  // every lane runs the same trip count
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += stride) {
    const bool in = i < N;
    const uint32_t k = in ? float_key(x[i]) : 0u;
    const uint32_t d = (k >> shift) & 255u;
    warp_hist_add(hist[0], d, in && (k & m0) == p0);
    warp_hist_add(hist[1], d, in && (k & m1) == p1);
    warp_hist_add(hist[2], d, in && (k & m2) == p2);
  }
  __syncthreads();
  const int nw = blockDim.x >> 5;
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) {
    unsigned v = 0;
    for (int w = 0; w < nw; ++w) v += (&whist[w][0][0])[i];
    if (v) atomicAdd(&st->hist[0][0] + i, v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last_block = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last_block) return;
  __threadfence();
  // The last CTA: choose each target's digit, then clear the histogram for the next pass.
  select_digits(st, shift);
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&st->hist[0][0])[i] = 0;
  if (threadIdx.x == 0) st->ticket = 0;
}

__global__ void moments_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ x = sd.colsum;
  const int N = sd.N;
  SelectState* st = sd.sel;
  const int first = sd.first, last = sd.last;
  MomentPartial* partials = sd.partials;
  SearchHeader* hdr = sd.hdr;
  __shared__ MomentPartial red[32];
  __shared__ bool last_block;
  const float v_first = key_float(st->prefix[0]);
  const float v_mid = key_float(st->prefix[1]);
  const float v_last = key_float(st->prefix[2]);
  MomentPartial acc = {0.0, 0.0, 0ull, 0ull, 0ull, 0ull};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const float f = x[i];
    if (f > v_first && f < v_last) {
      acc.s1 += (double)f;
    }
    acc.lt_first += (f < v_first);
    acc.eq_first += (f == v_first);
    acc.lt_last += (f < v_last);
    acc.eq_last += (f == v_last);
  }
  // Warp then block reduction in a fixed order.
  for (int o = 16; o > 0; o >>= 1) {
    acc.s1 += __shfl_down_sync(0xffffffffu, acc.s1, o);
    acc.lt_first += __shfl_down_sync(0xffffffffu, acc.lt_first, o);
    acc.eq_first += __shfl_down_sync(0xffffffffu, acc.eq_first, o);
    acc.lt_last += __shfl_down_sync(0xffffffffu, acc.lt_last, o);
    acc.eq_last += __shfl_down_sync(0xffffffffu, acc.eq_last, o);
  }
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[warp] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    MomentPartial b = red[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      b.s1 += red[w].s1;
      b.lt_first += red[w].lt_first;
      b.eq_first += red[w].eq_first;
      b.lt_last += red[w].lt_last;
      b.eq_last += red[w].eq_last;
    }
    partials[blockIdx.x] = b;
    __threadfence();
    last_block = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last_block) return;
  __threadfence();
  // Fixed-order reduction of the per-CTA partials: thread i folds partials i, i+256, ...,
  // then the block reduces in warp/lane order (deterministic for a given grid).
  MomentPartial t = {0.0, 0.0, 0ull, 0ull, 0ull, 0ull};
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    t.s1 += __ldcg(&partials[b].s1);
    t.lt_first += __ldcg(&partials[b].lt_first);
    t.eq_first += __ldcg(&partials[b].eq_first);
    t.lt_last += __ldcg(&partials[b].lt_last);
    t.eq_last += __ldcg(&partials[b].eq_last);
  }
  for (int o = 16; o > 0; o >>= 1) {
    t.s1 += __shfl_down_sync(0xffffffffu, t.s1, o);
    t.lt_first += __shfl_down_sync(0xffffffffu, t.lt_first, o);
    t.eq_first += __shfl_down_sync(0xffffffffu, t.eq_first, o);
    t.lt_last += __shfl_down_sync(0xffffffffu, t.lt_last, o);
    t.eq_last += __shfl_down_sync(0xffffffffu, t.eq_last, o);
  }
  __syncthreads();
  if (lane == 0) red[warp] = t;
  __syncthreads();
  if (threadIdx.x != 0) return;
  t = red[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
    t.s1 += red[w].s1;
    t.lt_first += red[w].lt_first;
    t.eq_first += red[w].eq_first;
    t.lt_last += red[w].lt_last;
    t.eq_last += red[w].eq_last;
  }
  st->ticket = 0;
  const long long n = (long long)last - first + 1;
  double s1;
  if (v_first == v_last) {
    s1 = (double)n * v_first;
  } else {
    // Sorted positions holding v_first are [lt_first, lt_first + eq_first - 1], those
    // holding v_last are [lt_last, lt_last + eq_last - 1]; count the ones in [first, last].
    const long long lo_end = min((long long)t.lt_first + (long long)t.eq_first - 1, (long long)last);
    const long long n_lo = lo_end - first + 1;
    const long long n_hi = (long long)last - max((long long)t.lt_last, (long long)first) + 1;
    s1 = t.s1 + (double)n_lo * v_first + (double)n_hi * v_last;
  }
  const float sum_f = (float)s1;
  const float m = sum_f / (float)n;  // dedoppler.cu:335-336: float sum / count
  hdr->median = v_mid;
  hdr->mean = m;
  st->mean = m;
  st->n = n;
  if (v_first == v_last) {
    st->n_lo = n;
    st->n_hi = 0;
  } else {
    const long long lo_end = min((long long)t.lt_first + (long long)t.eq_first - 1, (long long)last);
    st->n_lo = lo_end - first + 1;
    st->n_hi = (long long)last - max((long long)t.lt_last, (long long)first) + 1;
  }
}


__device__ __forceinline__ double float_ulp_above(double a) {
  const float af = __double2float_rn(a);
  if (af <= 0.0f) return 1.401298464324817e-45;  // 2^-149: the first add is exact
  return (double)(__uint_as_float(__float_as_uint(af) + 1u) - af);
}

// The squared deviation the reference adds: (f - m) * (f - m) in float.
__device__ __forceinline__ float var_term(float f, float m) {
  const float d = f - m;
  return __fmul_rn(d, d);
}

__device__ __forceinline__ bool var_inside(float f, float lo, float hi) { return f > lo && f < hi; }

// Per-chunk exact sums of the terms of the channels strictly between the percentiles.
__global__ void var_chunk_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ x = sd.colsum;
  const int N = sd.N;
  const SelectState* st = sd.sel;
  const int chunk = (N + gridDim.x - 1) / gridDim.x;
  double* chunk_sum = sd.var;
  __shared__ double red[32];
  const float lo = key_float(st->prefix[0]), hi = key_float(st->prefix[2]);
  const float m = st->mean;
  const long long b0 = (long long)blockIdx.x * chunk;
  const long long b1 = min((long long)N, b0 + chunk);
  double acc = 0.0;
  for (long long i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
    const float f = x[i];
    if (var_inside(f, lo, hi)) acc += (double)var_term(f, m);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) b += red[w];
    chunk_sum[blockIdx.x] = b;
  }
}

// Exclusive block scan of one double per thread (blockDim.x <= 1024, multiple of 32).
__device__ double block_exclusive_scan(double v, double* warp_tot, double* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  double inc = v;
  for (int o = 1; o < 32; o <<= 1) {
    const double y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += y;
  }
  if (lane == 31) warp_tot[warp] = inc;
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    double w = (lane < nw) ? warp_tot[lane] : 0.0;
    double wi = w;
    for (int o = 1; o < 32; o <<= 1) {
      const double y = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += y;
    }
    if (lane < nw) warp_tot[lane] = wi - w;  // exclusive prefix of the warp totals
    if (lane == nw - 1) *total = wi;
  }
  __syncthreads();
  const double r = warp_tot[warp] + (inc - v);
  __syncthreads();
  return r;
}

// Emulates the float accumulation over every included term, in channel order, then the
// boundary copies; the last CTA forms the standard deviation and the threshold.
__global__ void var_emulate_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ x = sd.colsum;
  const int N = sd.N;
  SelectState* st = sd.sel;
  const int chunk = (N + gridDim.x - 1) / gridDim.x;
  const double* chunk_sum = sd.var;
  double* chunk_part = sd.var + kVarChunks;
  const double snr_threshold = sd.snr_threshold;
  SearchHeader* hdr = sd.hdr;
  __shared__ double warp_tot[32];
  __shared__ double tile_total;
  __shared__ double red[32];
  __shared__ bool last_block;
  const float lo = key_float(st->prefix[0]), hi = key_float(st->prefix[2]);
  const float m = st->mean;
  // Exact sum of the preceding chunks, reduced in parallel.
  double pre_part = 0.0;
  for (int b = threadIdx.x; b < (int)blockIdx.x; b += blockDim.x) pre_part += chunk_sum[b];
  for (int o = 16; o > 0; o >>= 1) pre_part += __shfl_down_sync(0xffffffffu, pre_part, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = pre_part;
  __syncthreads();
  double base = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) base += red[w];
  __syncthreads();
  const long long b0 = (long long)blockIdx.x * chunk;
  const long long b1 = min((long long)N, b0 + chunk);
  double contrib = 0.0;
  for (long long t0 = b0; t0 < b1; t0 += blockDim.x) {
    const long long i = t0 + threadIdx.x;
    double term = 0.0;
    if (i < b1) {
      const float f = x[i];
      if (var_inside(f, lo, hi)) term = (double)var_term(f, m);
    }
    const double pre = block_exclusive_scan(term, warp_tot, &tile_total);
    if (term != 0.0) {
      const double u = float_ulp_above(base + pre);
      contrib += rint(term / u) * u;
    }
    base += tile_total;
  }
  for (int o = 16; o > 0; o >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = contrib;
  __syncthreads();
  if (threadIdx.x == 0) {
    double c = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) c += red[w];
    chunk_part[blockIdx.x] = c;
    __threadfence();
    last_block = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last_block) return;
  __threadfence();
  double pa = 0.0, pe = 0.0;
  for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
    pa += __ldcg(chunk_part + b);
    pe += __ldcg(chunk_sum + b);
  }
  for (int o = 16; o > 0; o >>= 1) {
    pa += __shfl_down_sync(0xffffffffu, pa, o);
    pe += __shfl_down_sync(0xffffffffu, pe, o);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    red[threadIdx.x >> 5] = pa;
    warp_tot[threadIdx.x >> 5] = pe;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  double acc = 0.0, exact = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    acc += red[w];
    exact += warp_tot[w];
  }
  // The percentile values themselves (ties at the boundaries), added after the rest.
  const double tlo = (double)var_term(lo, m), thi = (double)var_term(hi, m);
  for (long long k = 0; k < st->n_lo + st->n_hi; ++k) {
    const double term = (k < st->n_lo) ? tlo : thi;
    if (term != 0.0) {
      const double u = float_ulp_above(exact);
      acc += rint(term / u) * u;
    }
    exact += term;
  }
  st->ticket = 0;
  const float accum_f = (float)acc;
  const float std_dev = sqrtf(accum_f / (float)st->n);  // dedoppler.cu:342
  hdr->std_dev = std_dev;
  hdr->threshold = (float)(snr_threshold * (double)std_dev + (double)hdr->median);  // dedoppler.cu:353
}

}  // namespace

cudaError_t column_sums_batch(const SearchBatch& b, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  dim3 cgrid((b.maxN + 4 * 256 - 1) / (4 * 256), b.count);
  colsum_kernel<<<cgrid, 256, 0, stream>>>(b);
  return cudaGetLastError();
}

cudaError_t search_stats_batch(const SearchBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  const int maxN = b.maxN;
  // About four CTAs per SM over the whole batch, at least 8 per search.
  int sblocks = (4 * num_sms + b.count - 1) / b.count;
  if (sblocks < 8) sblocks = 8;
  if (sblocks > 2 * num_sms) sblocks = 2 * num_sms;
  if (sblocks > (maxN + 255) / 256) sblocks = (maxN + 255) / 256;
  dim3 sgrid(sblocks, b.count);
  // The select passes are latency-bound (a load, three warp votes and shared atomics per
  // value): many more CTAs than the moment kernels, which need one partial per CTA.
  int selblocks = (kSelectCtasPerSm * num_sms + b.count - 1) / b.count;
  if (selblocks > (maxN + 255) / 256) selblocks = (maxN + 255) / 256;
  if (selblocks < 1) selblocks = 1;
  dim3 selgrid(selblocks, b.count);
  for (int shift = 24; shift >= 0; shift -= 8) select_pass<<<selgrid, 256, 0, stream>>>(b, shift);
  moments_kernel<<<sgrid, 256, 0, stream>>>(b);
  // The variance emulation walks each chunk in 256-term tiles, one block scan per tile: short
  // chunks (16384 channels) keep that serial walk short.
  int vchunks = std::max(sblocks, (maxN + 16383) / 16384);
  if (vchunks > kVarChunks) vchunks = kVarChunks;
  dim3 vgrid(vchunks, b.count);
  var_chunk_kernel<<<vgrid, 256, 0, stream>>>(b);
  var_emulate_kernel<<<vgrid, 256, 0, stream>>>(b);
  return cudaGetLastError();
}

}  // namespace scb
