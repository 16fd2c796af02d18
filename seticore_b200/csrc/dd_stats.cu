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
#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

__global__ void colsum_kernel(const float* __restrict__ in, long long row_stride, int Tr, int N,
                              float* __restrict__ colsum, SelectState* st, int r_first, int r_mid,
                              int r_last) {
  if (blockIdx.x == 0 && threadIdx.x < 3) {
    const int r[3] = {r_first, r_mid, r_last};
    st->prefix[threadIdx.x] = 0;
    st->mask[threadIdx.x] = 0;
    st->rank[threadIdx.x] = (uint32_t)r[threadIdx.x];
    if (threadIdx.x == 0) st->ticket = 0;
  }
  if (blockIdx.x == 0) {
    for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&st->hist[0][0])[i] = 0;
  }
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
    reinterpret_cast<float4*>(colsum)[c4] = acc;
  } else {
    for (int c = blockIdx.x * blockDim.x * 4 + threadIdx.x; c < min(N, (blockIdx.x + 1) * blockDim.x * 4);
         c += blockDim.x) {
      float acc = 0.0f;
      for (int t = 0; t < Tr; ++t) acc += __ldg(in + (long long)t * row_stride + c);
      colsum[c] = acc;
    }
  }
}

// One 8-bit radix-select pass for the three target ranks.
__global__ void select_pass(const float* __restrict__ x, int N, SelectState* st, int shift) {
  __shared__ unsigned hist[3][256];
  __shared__ bool last_block;
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&hist[0][0])[i] = 0;
  __syncthreads();
  const uint32_t p0 = st->prefix[0], p1 = st->prefix[1], p2 = st->prefix[2];
  const uint32_t m0 = st->mask[0], m1 = st->mask[1], m2 = st->mask[2];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const uint32_t k = float_key(x[i]);
    const uint32_t d = (k >> shift) & 255u;
    if ((k & m0) == p0) atomicAdd(&hist[0][d], 1u);
    if ((k & m1) == p1) atomicAdd(&hist[1][d], 1u);
    if ((k & m2) == p2) atomicAdd(&hist[2][d], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) {
    const unsigned v = (&hist[0][0])[i];
    if (v) atomicAdd(&st->hist[0][0] + i, v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last_block = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last_block) return;
  __threadfence();
  // The last CTA: choose each target's digit, then clear the histogram for the next pass.
  if (threadIdx.x < 3) {
    const int j = threadIdx.x;
    uint32_t rank = st->rank[j];
    unsigned cum = 0;
    int digit = 255;
    for (int d = 0; d < 256; ++d) {
      const unsigned h = __ldcg(&st->hist[j][d]);
      if (rank < cum + h) {
        digit = d;
        break;
      }
      cum += h;
    }
    st->rank[j] = rank - cum;
    st->prefix[j] |= (uint32_t)digit << shift;
    st->mask[j] |= 255u << shift;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 3 * 256; i += blockDim.x) (&st->hist[0][0])[i] = 0;
  if (threadIdx.x == 0) st->ticket = 0;
}

__global__ void moments_kernel(const float* __restrict__ x, int N, SelectState* st, int first,
                               int last, double snr_threshold, MomentPartial* partials,
                               SearchHeader* hdr) {
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
  if (!last_block || threadIdx.x != 0) return;
  __threadfence();
  MomentPartial t = {0.0, 0.0, 0ull, 0ull, 0ull, 0ull};
  for (int b = 0; b < (int)gridDim.x; ++b) {
    const MomentPartial q = partials[b];
    t.s1 += q.s1;
    t.lt_first += q.lt_first;
    t.eq_first += q.eq_first;
    t.lt_last += q.lt_last;
    t.eq_last += q.eq_last;
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
__global__ void var_chunk_kernel(const float* __restrict__ x, int N, const SelectState* st, int chunk,
                                 double* chunk_sum) {
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
__global__ void var_emulate_kernel(const float* __restrict__ x, int N, SelectState* st, int chunk,
                                   const double* chunk_sum, double* chunk_part, double snr_threshold,
                                   SearchHeader* hdr) {
  __shared__ double warp_tot[32];
  __shared__ double tile_total;
  __shared__ double red[32];
  __shared__ bool last_block;
  const float lo = key_float(st->prefix[0]), hi = key_float(st->prefix[2]);
  const float m = st->mean;
  double base = 0.0;
  for (int b = 0; b < (int)blockIdx.x; ++b) base += chunk_sum[b];
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
  if (!last_block || threadIdx.x != 0) return;
  __threadfence();
  double acc = 0.0, exact = 0.0;
  for (int b = 0; b < (int)gridDim.x; ++b) {
    acc += __ldcg(chunk_part + b);
    exact += __ldcg(chunk_sum + b);
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

cudaError_t search_stats(const float* input, long long row_stride, int Tr, int N, float* colsum,
                         SelectState* st, MomentPartial* partials, int n_partials, double* var_scratch,
                         double snr_threshold, SearchHeader* hdr, int num_sms, cudaStream_t stream) {
  const int first = (int)ceil(0.05 * N);
  const int last = (int)floor(0.95 * N);
  const int mid = N / 2;
  const int cblocks = (N + 4 * 256 - 1) / (4 * 256);
  colsum_kernel<<<cblocks, 256, 0, stream>>>(input, row_stride, Tr, N, colsum, st, first, mid, last);
  int sblocks = 2 * num_sms;
  const int max_needed = (N + 255) / 256;
  if (sblocks > max_needed) sblocks = max_needed;
  for (int shift = 24; shift >= 0; shift -= 8) select_pass<<<sblocks, 256, 0, stream>>>(colsum, N, st, shift);
  int mblocks = sblocks < n_partials ? sblocks : n_partials;
  moments_kernel<<<mblocks, 256, 0, stream>>>(colsum, N, st, first, last, snr_threshold, partials, hdr);
  int vchunks = 2 * num_sms;
  if (vchunks > kVarChunks) vchunks = kVarChunks;
  if (vchunks > (N + 255) / 256) vchunks = (N + 255) / 256;
  const int chunk = (N + vchunks - 1) / vchunks;
  vchunks = (N + chunk - 1) / chunk;
  var_chunk_kernel<<<vchunks, 256, 0, stream>>>(colsum, N, st, chunk, var_scratch);
  var_emulate_kernel<<<vchunks, 256, 0, stream>>>(colsum, N, st, chunk, var_scratch, var_scratch + kVarChunks,
                                                  snr_threshold, hdr);
  return cudaGetLastError();
}

}  // namespace scb
