// Column sums and the noise statistics of a search, on the GPU.
//
// The reference copies the column sums to the host and uses std::nth_element for the
// median and the 5% / 95% order statistics, then a mean and standard deviation over the
// sorted positions [ceil(0.05 N), floor(0.95 N)] (dedoppler.cu:242-262).  Here:
//   * colsum_kernel: sumColumns (dedoppler.cu:63-72), same sequential float order.
//   * range_kernel, hist_kernel (x3), compact_kernel, select_finish_kernel: the three order
//     statistics at once.  The key range [kmin, kmax] is cut into 4096 bins; the bin holding
//     each target rank becomes that target's range, and further passes cut it again until
//     the range is one key or holds at most 4096 values, which are then collected and
//     sorted in shared memory.  Exact, and typically two reads of the column sums after the
//     range: one histogram and the compaction.  The compaction also sums (FP64, as the
//     reference's std::accumulate with a double start) the values between the two
//     percentiles' ranges; the finaliser adds the boundary candidates and ties exactly and
//     forms the mean with the reference's roundings (float sum, float division).
//   * var_chunk_kernel + var_emulate_kernel: the variance (searches whose order statistics
//     sit on repeated values are redone exactly in the reference's order by dd_order.cu).  The reference accumulates
//     (f - m)^2 in FLOAT, one term at a time (dedoppler.cu:257-261).  Once the
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
#include <climits>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

constexpr int kSelThreads = 512;   // histogram and finaliser blocks

// Column sums of search blockIdx.y (dedoppler.cu:63-72: a float sum in row order); block 0
// also resets that search's select state.
__global__ void colsum_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& d = b.s[blockIdx.y];
  SelectState* st = d.sel;
  if (blockIdx.x == 0) reset_select(st, d.first, d.mid, d.last);
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
// Visits the column sums of one search, four at a time where the array allows, with every
// lane of a warp running the same trip count (for warp-wide votes inside fn).
template <typename Fn>
__device__ __forceinline__ void for_each_colsum(const float* __restrict__ x, int N, Fn fn) {
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  const int n4 = vec ? N / 4 : 0;
  const int r4 = (n4 + stride - 1) / stride * stride;
  for (int i = tid; i < r4; i += stride) {
    const bool in = i < n4;
    const float4 v = in ? __ldg(reinterpret_cast<const float4*>(x) + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    fn(v.x, in);
    fn(v.y, in);
    fn(v.z, in);
    fn(v.w, in);
  }
  const int rest = N - 4 * n4;
  const int rr = (rest + stride - 1) / stride * stride;
  for (int i = tid; i < rr; i += stride) {
    const bool in = i < rest;
    fn(in ? x[4 * n4 + i] : 0.0f, in);
  }
}

// The smallest and largest key of each search's column sums.
__global__ void __launch_bounds__(256) range_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  uint32_t kmn = 0xffffffffu, kmx = 0u;
  for_each_colsum(sd.colsum, sd.N, [&](float f, bool in) {
    if (in) {
      const uint32_t k = sel_key(f);
      kmn = min(kmn, k);
      kmx = max(kmx, k);
    }
  });
  kmn = __reduce_min_sync(0xffffffffu, kmn);
  kmx = __reduce_max_sync(0xffffffffu, kmx);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&sd.sel->kmin, kmn);
    atomicMax(&sd.sel->kmax, kmx);
  }
}

// Number of bits that hold v (0 for 0).
__device__ __forceinline__ uint32_t bit_width(uint32_t v) { return 32u - (uint32_t)__clz((int)v); }

// One histogram pass of the order statistics.  Pass 0 bins the whole key range of the search
// ([kmin, kmax], one histogram for the three targets); later passes bin, for each target
// still in mode 0, the range its previous pass chose.  The last CTA of the search picks each
// active target's bin and updates its range, rank and mode.  Exact: the ranges nest, and
// a range of width one is the target's key.
__global__ void __launch_bounds__(kSelThreads) hist_kernel(const __grid_constant__ SearchBatch b, int pass) {
  const SearchDesc& sd = b.s[blockIdx.y];
  SelectState* st = sd.sel;
  const int N = sd.N;
  extern __shared__ unsigned sh_hist[];  // [slots][kSelBins]
  __shared__ uint32_t s_lo[3], s_ws[3];
  __shared__ int s_slot[3];
  __shared__ int s_slots;
  __shared__ bool last_block;
  if (threadIdx.x == 0) {
    int slots = 0;
    for (int j = 0; j < 3; ++j) {
      s_slot[j] = -1;
      uint32_t lo, ws;
      bool active;
      if (pass == 0) {
        lo = st->kmin;
        ws = bit_width(st->kmax - st->kmin);  // the range [kmin, kmin + 2^ws) holds kmax
        active = N > 0;
      } else {
        lo = st->lo[j];
        ws = st->wshift[j];
        active = st->mode[j] == 0 && N > 0;
      }
      s_lo[j] = lo;
      s_ws[j] = ws;
      if (!active) continue;
      for (int i = 0; i < j; ++i)  // targets with the same range share a histogram
        if (s_slot[i] >= 0 && s_lo[i] == lo && s_ws[i] == ws) s_slot[j] = s_slot[i];
      if (s_slot[j] < 0) s_slot[j] = slots++;
    }
    s_slots = slots;
  }
  __syncthreads();
  const int slots = s_slots;
  if (slots == 0) return;  // every target is resolved or collected: nothing to bin
  for (int i = threadIdx.x; i < slots * kSelBins; i += blockDim.x) sh_hist[i] = 0;
  uint32_t lo[3], bs[3];
  unsigned long long width[3];
  int slot_of[3];
  int first_of_slot[3] = {-1, -1, -1};
  for (int j = 0; j < 3; ++j) {
    lo[j] = s_lo[j];
    width[j] = 1ull << s_ws[j];
    bs[j] = s_ws[j] > 12u ? s_ws[j] - 12u : 0u;  // 2^bs keys per bin: at most kSelBins bins
    slot_of[j] = s_slot[j];
    if (slot_of[j] >= 0 && first_of_slot[slot_of[j]] < 0) first_of_slot[slot_of[j]] = j;
  }
  // Per-slot range, in registers for the loop below (s is a constant there).
  uint32_t slo[3] = {0u, 0u, 0u}, sbs[3] = {0u, 0u, 0u};
  unsigned long long swidth[3] = {0ull, 0ull, 0ull};
  for (int s = 0; s < 3; ++s) {
    const int j = first_of_slot[s];
    if (j < 0) continue;
    slo[s] = lo[j];
    sbs[s] = bs[j];
    swidth[s] = width[j];  // 0 for unused slots: nothing is binned there
  }
  __syncthreads();
  for_each_colsum(sd.colsum, N, [&](float f, bool in) {
    if (!in) return;
    const uint32_t k = sel_key(f);
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const uint32_t d = k - slo[s];
      if (k >= slo[s] && (unsigned long long)d < swidth[s]) atomicAdd(&sh_hist[s * kSelBins + (d >> sbs[s])], 1u);
    }
  });
  __syncthreads();
  for (int i = threadIdx.x; i < slots * kSelBins; i += blockDim.x) {
    const unsigned v = sh_hist[i];
    if (v) atomicAdd(&st->hist[0][0] + i, v);
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last_block = (atomicAdd(&st->ticket, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last_block) return;
  __threadfence();
  // The last CTA: for each active target, the bin that holds its rank.  Thread t owns bins
  // [t * per, (t + 1) * per) of the slot; a block scan of the per-thread totals places them.
  constexpr int per = kSelBins / kSelThreads;
  __shared__ unsigned warp_sum[kSelThreads / 32];
  for (int j = 0; j < 3; ++j) {
    const int s = slot_of[j];
    if (s < 0) continue;
    const unsigned* h = st->hist[s];
    unsigned c[per];
    unsigned tot = 0;
#pragma unroll
    for (int q = 0; q < per; ++q) {
      c[q] = __ldcg(h + threadIdx.x * per + q);
      tot += c[q];
    }
    // exclusive scan of tot over the block
    unsigned inc = tot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) warp_sum[warp] = inc;
    __syncthreads();
    unsigned before = 0;
    for (int w = 0; w < warp; ++w) before += warp_sum[w];
    before += inc - tot;
    const uint32_t rank = st->rank[j];  // every thread reads it before the owner updates it
    __syncthreads();
    if (rank >= before && rank < before + tot) {
      unsigned acc = before;
      for (int q = 0; q < per; ++q) {
        if (rank < acc + c[q]) {
          const uint32_t bin = (uint32_t)(threadIdx.x * per + q);
          const uint32_t nlo = lo[j] + (bin << bs[j]);
          st->lo[j] = nlo;
          st->wshift[j] = bs[j];
          st->rank[j] = rank - acc;
          st->count[j] = c[q];
          const uint32_t mode = bs[j] == 0 ? 2u : (c[q] <= (unsigned)kSelCands ? 1u : 0u);
          st->mode[j] = mode;
          if (mode == 2) st->prefix[j] = nlo;
          break;
        }
        acc += c[q];
      }
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < slots * kSelBins; i += blockDim.x) (&st->hist[0][0])[i] = 0;
  if (threadIdx.x == 0) st->ticket = 0;
}

// Collects the values of each mode-1 target's range (at most kSelCands each) and sums, in
// FP64, the values strictly between the first and the last target's ranges: the part of the
// 5-95 % mean that needs no exact boundary.  One partial per CTA.
__global__ void __launch_bounds__(256) compact_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  SelectState* st = sd.sel;
  __shared__ double red[8];
  uint32_t lo[3], mode[3];
  unsigned long long width[3];
  for (int j = 0; j < 3; ++j) {
    lo[j] = st->lo[j];
    width[j] = 1ull << st->wshift[j];
    mode[j] = st->mode[j];
  }
  // The ranges of two targets are equal or disjoint (they refine the same bins).  Interior:
  // keys above the first target's range and below the last's.  After the first histogram a
  // range is at most 2^20 keys wide, so each test is one 32-bit unsigned compare of k - lo.
  const bool disjoint = lo[0] != lo[2];
  const uint32_t in_lo = lo[0] + (uint32_t)width[0];
  const uint32_t in_len = disjoint ? lo[2] - in_lo : 0u;
  uint32_t w[3];
  for (int j = 0; j < 3; ++j) w[j] = mode[j] == 1 ? (uint32_t)width[j] : 0u;  // 0: collects nothing
  const int lane = threadIdx.x & 31;
  double acc = 0.0;
  // Appends the values of lane-local mask bits to the lists: rare (a few thousand values per
  // search), so it runs only when some lane of the warp holds one.
  auto collect = [&](uint32_t k, bool t0, bool t1, bool t2) {
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const bool take = j == 0 ? t0 : (j == 1 ? t1 : t2);
      const unsigned m = __ballot_sync(0xffffffffu, take);
      if (m == 0) continue;
      const int leader = __ffs(m) - 1;
      unsigned base = 0;
      if (lane == leader) base = atomicAdd(&st->ncand[j], (unsigned)__popc(m));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (take) {
        const unsigned at = base + (unsigned)__popc(m & ((1u << lane) - 1u));
        if (at < (unsigned)kSelCands) st->cand[j][at] = k;
      }
    }
  };
  const float* __restrict__ x = sd.colsum;
  const int N = sd.N;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x;
  const int stride = gridDim.x * blockDim.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
  const int n4 = vec ? N / 4 : 0;
  const int r4 = (n4 + stride - 1) / stride * stride;
  for (int i = tid; i < r4; i += stride) {
    const bool in = i < n4;
    const float4 v = in ? __ldg(reinterpret_cast<const float4*>(x) + i) : make_float4(0.f, 0.f, 0.f, 0.f);
    const float f[4] = {v.x, v.y, v.z, v.w};
    uint32_t k[4];
    bool any = false;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      k[q] = sel_key(f[q]);
      if (in && k[q] - in_lo < in_len) acc += (double)f[q];
      any |= in && ((k[q] - lo[0] < w[0]) | (k[q] - lo[1] < w[1]) | (k[q] - lo[2] < w[2]));
    }
    if (__ballot_sync(0xffffffffu, any) == 0u) continue;  // the common case: no candidate in the warp
#pragma unroll
    for (int q = 0; q < 4; ++q)
      collect(k[q], in && k[q] - lo[0] < w[0], in && k[q] - lo[1] < w[1], in && k[q] - lo[2] < w[2]);
  }
  const int rest = N - 4 * n4;
  const int rr = (rest + stride - 1) / stride * stride;
  for (int i = tid; i < rr; i += stride) {
    const bool in = i < rest;
    const float f = in ? x[4 * n4 + i] : 0.0f;
    const uint32_t k = sel_key(f);
    if (in && k - in_lo < in_len) acc += (double)f;
    collect(k, in && k - lo[0] < w[0], in && k - lo[1] < w[1], in && k - lo[2] < w[2]);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if (lane == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    MomentPartial mp{};
    mp.s1 = t;
    sd.partials[blockIdx.x] = mp;
  }
}

// Sorts n (<= kSelCands) keys in shared memory, ascending (bitonic, padded with the largest
// key).
__device__ void sort_keys(uint32_t* k, int n) {
  int p = 1;
  while (p < n) p <<= 1;
  for (int i = n + threadIdx.x; i < p; i += blockDim.x) k[i] = 0xffffffffu;
  __syncthreads();
  for (int size = 2; size <= p; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int i = threadIdx.x; i < p / 2; i += blockDim.x) {
        const int lo = 2 * i - (i & (stride - 1));
        const int hi = lo + stride;
        const bool up = (lo & size) == 0;
        const uint32_t a = k[lo], c = k[hi];
        if ((a > c) == up) {
          k[lo] = c;
          k[hi] = a;
        }
      }
      __syncthreads();
    }
  }
}

// One CTA per search: the exact order statistics from the collected candidates, then the
// mean over the sorted positions [first, last] as the reference forms it (dedoppler.cu:255-256):
// a double sum of the floats, rounded to float, divided by the count in float.
__global__ void __launch_bounds__(kSelThreads) select_finish_kernel(const __grid_constant__ SearchBatch b,
                                                                    int n_partials) {
  const SearchDesc& sd = b.s[blockIdx.y];
  SelectState* st = sd.sel;
  SearchHeader* hdr = sd.hdr;
  __shared__ uint32_t keys[kSelCands];
  __shared__ uint32_t s_key[3];
  __shared__ long long s_lt[3], s_eq[3];
  __shared__ double red[kSelThreads / 32];
  if (sd.N <= 0) return;
  const int ranks[3] = {sd.first, sd.mid, sd.last};
  for (int j = 0; j < 3; ++j) {
    const uint32_t mode = st->mode[j];
    const uint32_t rank = st->rank[j];
    const long long below = (long long)ranks[j] - rank;  // values under the target's range
    if (mode == 2) {
      if (threadIdx.x == 0) {
        s_key[j] = st->prefix[j];
        s_lt[j] = below;
        s_eq[j] = st->count[j];
      }
      continue;
    }
    // mode 1: exactly count[j] candidates were collected
    const int n = (int)min(st->ncand[j], (unsigned)kSelCands);
    for (int i = threadIdx.x; i < n; i += blockDim.x) keys[i] = __ldcg(&st->cand[j][i]);
    __syncthreads();
    sort_keys(keys, n);
    // The rank is below the range's count, which is the number collected; the clamp only
    // keeps the read inside the array.
    const int r = n > 0 ? min((int)rank, n - 1) : 0;
    const uint32_t key = n > 0 ? keys[r] : st->lo[j];
    // first and last occurrence of the key among the candidates
    if (threadIdx.x == 0) {
      int a = r, z = r;
      while (a > 0 && keys[a - 1] == key) --a;
      while (z + 1 < n && keys[z + 1] == key) ++z;
      s_key[j] = key;
      s_lt[j] = below + a;
      s_eq[j] = z - a + 1;
      st->prefix[j] = key;
    }
    __syncthreads();
  }
  __syncthreads();
  const float v_first = key_float(s_key[0]);
  const float v_mid = key_float(s_key[1]);
  const float v_last = key_float(s_key[2]);
  // Values strictly between the two percentiles: the interior partials plus the candidates
  // of the boundary ranges (once when the first and last ranges are the same).
  double acc = 0.0;
  for (int i = threadIdx.x; i < n_partials; i += blockDim.x) acc += __ldcg(&sd.partials[i].s1);
  const bool same = st->lo[0] == st->lo[2];
  for (int j = 0; j < 3; j += 2) {
    if (st->mode[j] != 1 || (j == 2 && same)) continue;
    const int n = (int)min(st->ncand[j], (unsigned)kSelCands);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      const float f = key_float(__ldcg(&st->cand[j][i]));
      if (f > v_first && f < v_last) acc += (double)f;
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x != 0) return;
  double inner = 0.0;
  for (int w = 0; w < kSelThreads / 32; ++w) inner += red[w];
  const int first = sd.first, last = sd.last;
  const long long n = (long long)last - first + 1;
  double s1;
  long long n_lo, n_hi;
  if (v_first == v_last) {
    s1 = (double)n * v_first;
    n_lo = n;
    n_hi = 0;
  } else {
    // Sorted positions holding v_first are [lt_first, lt_first + eq_first - 1], those
    // holding v_last are [lt_last, lt_last + eq_last - 1]; count the ones in [first, last].
    const long long lo_end = min(s_lt[0] + s_eq[0] - 1, (long long)last);
    n_lo = lo_end - first + 1;
    n_hi = (long long)last - max(s_lt[2], (long long)first) + 1;
    s1 = inner + (double)n_lo * v_first + (double)n_hi * v_last;
  }
  const float sum_f = (float)s1;
  const float m = sum_f / (float)n;  // dedoppler.cu:255-256: float sum / count
  hdr->median = v_mid;
  hdr->mean = m;
  // How often the most repeated of the three order-statistic values occurs: column sums with
  // many equal values (integer-valued power) are where the order of the float variance sum
  // matters, and those searches take the exact statistics of dd_order.cu.
  hdr->ties = (int)min(max(s_eq[0], max(s_eq[1], s_eq[2])), (long long)INT_MAX);
  hdr->order_exact = 0;
  st->mean = m;
  st->n = n;
  st->n_lo = n_lo;
  st->n_hi = n_hi;
  // reset for the next search in this slot
  for (int j = 0; j < 3; ++j) st->ncand[j] = 0;
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

// Channels per variance chunk: a multiple of 8, so every chunk starts 32-byte aligned.
__device__ __forceinline__ int var_chunk_len(int N, int chunks) { return ((N + chunks - 1) / chunks + 7) & ~7; }

// Per-chunk exact sums of the terms of the channels strictly between the percentiles.
__global__ void var_chunk_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ x = sd.colsum;
  const int N = sd.N;
  const SelectState* st = sd.sel;
  const int chunk = var_chunk_len(N, gridDim.x);
  double* chunk_sum = sd.var;
  __shared__ double red[32];
  const float lo = key_float(st->prefix[0]), hi = key_float(st->prefix[2]);
  const float m = st->mean;
  const long long b0 = (long long)blockIdx.x * chunk;
  const long long b1 = min((long long)N, b0 + chunk);
  double acc = 0.0;
  // 16-byte loads over the chunk (chunks start 32-byte aligned), then the ragged end.
  const bool vec = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
  const long long n4 = vec ? (b1 - b0) / 4 : 0;
  for (long long i = threadIdx.x; i < n4; i += blockDim.x) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(x + b0) + i);
    if (var_inside(v.x, lo, hi)) acc += (double)var_term(v.x, m);
    if (var_inside(v.y, lo, hi)) acc += (double)var_term(v.y, m);
    if (var_inside(v.z, lo, hi)) acc += (double)var_term(v.z, m);
    if (var_inside(v.w, lo, hi)) acc += (double)var_term(v.w, m);
  }
  for (long long i = b0 + 4 * n4 + threadIdx.x; i < b1; i += blockDim.x) {
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
  const int chunk = var_chunk_len(N, gridDim.x);
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
  // Tiles of 8 consecutive channels per thread: one block scan per 8 * blockDim.x channels;
  // each thread then walks its 8 in channel order.  The ulp of a float is a power of two,
  // so term / ulp is the exact product with its reciprocal.
  constexpr int K = 8;
  const bool vec = (reinterpret_cast<uintptr_t>(x) & 15) == 0;
  for (long long t0 = b0; t0 < b1; t0 += (long long)blockDim.x * K) {
    const long long i0 = t0 + (long long)threadIdx.x * K;
    float v[K];
    if (vec && i0 + K <= b1) {
      const float4 p = __ldg(reinterpret_cast<const float4*>(x + i0));
      const float4 q = __ldg(reinterpret_cast<const float4*>(x + i0) + 1);
      v[0] = p.x; v[1] = p.y; v[2] = p.z; v[3] = p.w;
      v[4] = q.x; v[5] = q.y; v[6] = q.z; v[7] = q.w;
    } else {
#pragma unroll
      for (int k = 0; k < K; ++k) v[k] = (i0 + k < b1) ? x[i0 + k] : lo;  // lo: not inside
    }
    double term[K];
    double tsum = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      term[k] = var_inside(v[k], lo, hi) ? (double)var_term(v[k], m) : 0.0;
      tsum += term[k];
    }
    double a = base + block_exclusive_scan(tsum, warp_tot, &tile_total);
#pragma unroll
    for (int k = 0; k < K; ++k) {
      if (term[k] != 0.0) {
        const double u = float_ulp_above(a);
        contrib += rint(term[k] * __drcp_rn(u)) * u;
      }
      a += term[k];
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
  const float std_dev = sqrtf(accum_f / (float)st->n);  // dedoppler.cu:262
  hdr->std_dev = std_dev;
  hdr->threshold = (float)(snr_threshold * (double)std_dev + (double)hdr->median);  // dedoppler.cu:273
}

}  // namespace

cudaError_t column_sums_batch(const SearchBatch& b, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  dim3 cgrid((b.maxN + 4 * 256 - 1) / (4 * 256), b.count);
  colsum_kernel<<<cgrid, 256, 0, stream>>>(b);
  return cudaGetLastError();
}

cudaError_t search_stats_emulated(const SearchBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  const int maxN = b.maxN;
  // About four CTAs per SM over the whole batch, at least 8 per search.
  int sblocks = (4 * num_sms + b.count - 1) / b.count;
  if (sblocks < 8) sblocks = 8;
  if (sblocks > 2 * num_sms) sblocks = 2 * num_sms;
  if (sblocks > (maxN + 255) / 256) sblocks = (maxN + 255) / 256;
  dim3 sgrid(sblocks, b.count);
  // Order statistics: the key range, up to three histogram passes (the second and third exit
  // at once unless a target's bin still holds more than kSelCands values), the compaction
  // with the interior sum of the mean, and one CTA per search for the exact pick.
  range_kernel<<<sgrid, 256, 0, stream>>>(b);
  const int hist_smem = 3 * kSelBins * (int)sizeof(unsigned);
  cudaError_t e = cudaFuncSetAttribute(hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
  if (e != cudaSuccess) return e;
  int hblocks = (2 * num_sms + b.count - 1) / b.count;
  if (hblocks > (maxN + 4 * kSelThreads - 1) / (4 * kSelThreads)) hblocks = (maxN + 4 * kSelThreads - 1) / (4 * kSelThreads);
  if (hblocks < 1) hblocks = 1;
  for (int pass = 0; pass < 3; ++pass) hist_kernel<<<dim3(hblocks, b.count), kSelThreads, hist_smem, stream>>>(b, pass);
  compact_kernel<<<sgrid, 256, 0, stream>>>(b);
  select_finish_kernel<<<dim3(1, b.count), kSelThreads, 0, stream>>>(b, sblocks);
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
