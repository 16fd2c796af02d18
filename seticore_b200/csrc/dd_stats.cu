// Column sums and the noise statistics of a search, on the GPU.
//
// The reference copies the column sums to the host and uses std::nth_element for the
// median and the 5% / 95% order statistics, then a mean and standard deviation over the
// sorted positions [ceil(0.05 N), floor(0.95 N)] (dedoppler.cu:322-342).  Here:
//   * colsum_kernel: sumColumns (dedoppler.cu:63-72), same sequential float order.
//   * select_pass (x4): MSB-first radix select of the three order statistics at once,
//     8 bits per pass; the last CTA of each pass picks the digits.  Exact.
//   * moments_kernel: sum and sum of squares (FP64) of the values between the two
//     percentiles, with boundary ties counted exactly; per-CTA partials are combined
//     by the last CTA in a fixed order, so the result does not depend on scheduling.
//     It then forms mean, standard deviation and threshold with the reference's float
//     roundings (float mean from the rounded sum; float sqrt; float threshold).
// The reference accumulates the variance in float over an nth_element-permuted order;
// the FP64 sum here differs from it only by that float rounding (about 1e-5 relative
// at 2^20 channels).
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
      acc.s2 += (double)f * (double)f;
    }
    acc.lt_first += (f < v_first);
    acc.eq_first += (f == v_first);
    acc.lt_last += (f < v_last);
    acc.eq_last += (f == v_last);
  }
  // Warp then block reduction in a fixed order.
  for (int o = 16; o > 0; o >>= 1) {
    acc.s1 += __shfl_down_sync(0xffffffffu, acc.s1, o);
    acc.s2 += __shfl_down_sync(0xffffffffu, acc.s2, o);
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
      b.s2 += red[w].s2;
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
    t.s2 += q.s2;
    t.lt_first += q.lt_first;
    t.eq_first += q.eq_first;
    t.lt_last += q.lt_last;
    t.eq_last += q.eq_last;
  }
  st->ticket = 0;
  const long long n = (long long)last - first + 1;
  double s1, s2;
  if (v_first == v_last) {
    s1 = (double)n * v_first;
    s2 = (double)n * (double)v_first * (double)v_first;
  } else {
    // Sorted positions holding v_first are [lt_first, lt_first + eq_first - 1], those
    // holding v_last are [lt_last, lt_last + eq_last - 1]; count the ones in [first, last].
    const long long lo_end = min((long long)t.lt_first + (long long)t.eq_first - 1, (long long)last);
    const long long n_lo = lo_end - first + 1;
    const long long n_hi = (long long)last - max((long long)t.lt_last, (long long)first) + 1;
    s1 = t.s1 + (double)n_lo * v_first + (double)n_hi * v_last;
    s2 = t.s2 + (double)n_lo * (double)v_first * (double)v_first + (double)n_hi * (double)v_last * (double)v_last;
  }
  const float sum_f = (float)s1;
  const float m = sum_f / (float)n;  // dedoppler.cu:336: float sum / count
  const double md = (double)m;
  const double accum = s2 - 2.0 * md * s1 + (double)n * md * md;
  const float accum_f = (float)(accum > 0.0 ? accum : 0.0);
  const float std_dev = sqrtf(accum_f / (float)n);
  hdr->median = v_mid;
  hdr->mean = m;
  hdr->std_dev = std_dev;
  hdr->threshold = (float)(snr_threshold * (double)std_dev + (double)v_mid);  // dedoppler.cu:353
}

}  // namespace

cudaError_t search_stats(const float* input, long long row_stride, int Tr, int N, float* colsum,
                         SelectState* st, MomentPartial* partials, int n_partials,
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
  return cudaGetLastError();
}

}  // namespace scb
