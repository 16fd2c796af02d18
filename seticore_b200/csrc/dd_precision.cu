// The precision form: searches over normalised 16-bit spectra with exact hits.
//
//   1. norm_sample_kernel: per search, the FP64 mean and standard deviation of three of
//      the unrounded rows (first, middle, last): the scale of the 16-bit values.
//   2. normalize_kernel, one read of the original float32 power: y = (x - mean) / std in
//      FP64, rounded to BF16 or FP16 (padded rows stay 0), into a dense [Tr][N] 16-bit copy
//      -- half the bytes of the input -- and, in the same read, the float32 column sums the
//      statistics need and the minimum and maximum of the unrounded rows.
//   3. (dd_tree.cu, dd_levels.cu) the tree over y, accumulating in FP32 (or, for 16 rows,
//      in FP16 pairs: two drift blocks per instruction), gives approximate tops.  A path
//      sum of y equals (P - T*mean) / std for the path sum P of x, so the order of path sums
//      is kept up to the rounding.
//   4. flag_channels_kernel: lists every channel whose approximate top reaches the flag
//      threshold, the threshold mapped to y units less a bound on the rounding of the
//      16-bit values and of both float trees (flag_threshold).
//   5. recompute_direct_kernel (up to 16 rows: one thread per channel and drift block,
//      all offsets from the subtree's leaves) or recompute_kernel (one path per thread):
//      for each listed channel, every eligible path is summed from the original power in
//      the tree's own pairing (bit-identical to the plain form's tree) and the maximum,
//      floored at 0, becomes its top.  Every other channel keeps top 0:
//      its approximate top is below the flag threshold, so its exact top is below the
//      threshold and it can neither become a window candidate nor beat one
//      (dedoppler.cu:275-302 compares only with values above the threshold).  The hit list
//      is therefore the plain form's, whatever the threshold or the data.
// The statistics (median, standard deviation, threshold) always come from the float32
// column sums, exactly as in the plain form.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>
#include <cstring>
#include <type_traits>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

// Block-wide reduction of (sum, sum of squares, min, max) into the search's moments
// buffer: per-block partials, then the last block to arrive (a ticket) folds them.  Returns
// true in thread 0 of that last block, with the totals in *a, *q, *mn, *mx.
__device__ bool fold_moments(const PrecisionDesc& d, double s1, double s2, float mn, float mx, double* a, double* q,
                             double* omn, double* omx) {
  __shared__ double r1[32], r2[32], r3[32], r4[32];
  __shared__ bool last_block;
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
    mn = fminf(mn, __shfl_down_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_down_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) {
    r1[threadIdx.x >> 5] = s1;
    r2[threadIdx.x >> 5] = s2;
    r3[threadIdx.x >> 5] = mn;
    r4[threadIdx.x >> 5] = mx;
  }
  __syncthreads();
  double* part = d.moments;  // sums [0, K), squares [K, 2K), minima and maxima from 2K + 4
  if (threadIdx.x == 0) {
    double x1 = 0.0, x2 = 0.0, m = r3[0], M = r4[0];
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      x1 += r1[w];
      x2 += r2[w];
      m = fmin(m, r3[w]);
      M = fmax(M, r4[w]);
    }
    part[blockIdx.x] = x1;
    part[kVarChunks + blockIdx.x] = x2;
    part[2 * kVarChunks + 4 + 2 * blockIdx.x] = m;
    part[2 * kVarChunks + 5 + 2 * blockIdx.x] = M;
    __threadfence();
    last_block = (atomicAdd(d.ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last_block) return false;
  __threadfence();
  double x1 = 0.0, x2 = 0.0, m = __longlong_as_double(0x7ff0000000000000ll), M = -m;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
    x1 += __ldcg(part + k);
    x2 += __ldcg(part + kVarChunks + k);
    m = fmin(m, __ldcg(part + 2 * kVarChunks + 4 + 2 * k));
    M = fmax(M, __ldcg(part + 2 * kVarChunks + 5 + 2 * k));
  }
  for (int o = 16; o > 0; o >>= 1) {
    x1 += __shfl_down_sync(0xffffffffu, x1, o);
    x2 += __shfl_down_sync(0xffffffffu, x2, o);
    m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
    M = fmax(M, __shfl_down_sync(0xffffffffu, M, o));
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    r1[threadIdx.x >> 5] = x1;
    r2[threadIdx.x >> 5] = x2;
    r3[threadIdx.x >> 5] = m;
    r4[threadIdx.x >> 5] = M;
  }
  __syncthreads();
  if (threadIdx.x != 0) return false;
  x1 = 0.0;
  x2 = 0.0;
  m = r3[0];
  M = r4[0];
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    x1 += r1[w];
    x2 += r2[w];
    m = fmin(m, r3[w]);
    M = fmax(M, r4[w]);
  }
  *d.ticket = 0;
  *a = x1;
  *q = x2;
  *omn = m;
  *omx = M;
  return true;
}

// The normalisation's mean and standard deviation, in FP64, from a sample of the unrounded
// rows: the first, middle and last.  Exactness does not depend on them (the flag bound uses
// whatever they are); they only set the 16-bit values' scale.
__global__ void norm_sample_kernel(const __grid_constant__ PrecisionBatch b) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  const int rows[3] = {0, d.T / 2, d.T - 1};
  const int nrows = d.T >= 3 ? 3 : d.T;
  double s1 = 0.0, s2 = 0.0;
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  const bool vec = (d.N % 4 == 0) && (d.row_stride % 4 == 0) && ((reinterpret_cast<uintptr_t>(d.input) & 15) == 0);
  for (int r = 0; r < nrows; ++r) {
    const float* row = d.input + (long long)rows[r] * d.row_stride;
    if (vec) {
      for (long long c = tid; c < d.N / 4; c += nth) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(row) + c);
        const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < 4; ++i)
          if (e[i] == e[i]) {  // NaNs do not enter the scale
            s1 += (double)e[i];
            s2 += (double)e[i] * (double)e[i];
          }
      }
    } else {
      for (long long c = tid; c < d.N; c += nth) {
        const double x = __ldg(row + c);
        if (x == x) {
          s1 += x;
          s2 += x * x;
        }
      }
    }
  }
  double a, q, mn, mx;
  if (!fold_moments(d, s1, s2, 0.0f, 0.0f, &a, &q, &mn, &mx)) return;
  const double n = (double)nrows * d.N;
  const double mean = a / n;
  double var = q / n - mean * mean;
  if (!(var > 0.0) || !(mean == mean)) var = 1.0;  // constant sample: any positive scale keeps the order
  d.moments[2 * kVarChunks] = (mean == mean) ? mean : 0.0;
  d.moments[2 * kVarChunks + 1] = sqrt(var);
}

template <typename E>
__device__ __forceinline__ E from_float(float v);
template <>
__device__ __forceinline__ __nv_bfloat16 from_float<__nv_bfloat16>(float v) {
  return __float2bfloat16_rn(v);
}
template <>
__device__ __forceinline__ __half from_float<__half>(float v) {
  return __float2half_rn(v);
}

// The normalised value in float: (x - m) * inv with m = float(mean) and inv = float(1 / std),
// each step rounded to nearest (no contraction).  The subtraction of two floats is exact or
// off by 2^-24 of its result, so against (x - mean) / std the value carries a relative error
// under 2^-22 (three roundings) and an absolute one of at most 1.01 * 2^-24 * |mean| / std
// (the rounding of the mean): flag_threshold counts both.
__device__ __forceinline__ float normalized(float x, float m, float inv) { return __fmul_rn(__fsub_rn(x, m), inv); }

// One read of the original power: y = (x - mean) / std in float (normalized), rounded to BF16
// or FP16, into the dense [Tr][N] 16-bit copy (padded rows 0); in the same read the float32 column sums in
// row order (sumColumns, dedoppler.cu:63-72, bit-identical to colsum_kernel) and the minimum
// and maximum of the unrounded rows, which the flag bound needs.  A thread takes four
// columns (one with unaligned rows) down all Tr rows.
template <typename E>
__global__ void normalize_kernel(const __grid_constant__ PrecisionBatch b) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  const float mean = (float)d.moments[2 * kVarChunks];
  const float inv = (float)(1.0 / d.moments[2 * kVarChunks + 1]);
  E* out = static_cast<E*>(d.norm);
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nth = (long long)gridDim.x * blockDim.x;
  float mn = __int_as_float(0x7f800000), mx = -mn;  // NaNs are skipped (they flag themselves)
  const bool vec = (d.N % 4 == 0) && (d.row_stride % 4 == 0) && ((reinterpret_cast<uintptr_t>(d.input) & 15) == 0);
  if (vec) {
    for (long long c = tid; c < d.N / 4; c += nth) {
      float4 cs = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int t = 0; t < d.Tr; ++t) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(d.input + (long long)t * d.row_stride) + c);
        cs.x += v.x;
        cs.y += v.y;
        cs.z += v.z;
        cs.w += v.w;
        E y[4] = {from_float<E>(0.0f), from_float<E>(0.0f), from_float<E>(0.0f), from_float<E>(0.0f)};
        if (t < d.T) {
          y[0] = from_float<E>(normalized(v.x, mean, inv));
          y[1] = from_float<E>(normalized(v.y, mean, inv));
          y[2] = from_float<E>(normalized(v.z, mean, inv));
          y[3] = from_float<E>(normalized(v.w, mean, inv));
          mn = fminf(mn, fminf(fminf(v.x, v.y), fminf(v.z, v.w)));
          mx = fmaxf(mx, fmaxf(fmaxf(v.x, v.y), fmaxf(v.z, v.w)));
        }
        uint2 packed;
        memcpy(&packed, y, sizeof(packed));
        reinterpret_cast<uint2*>(out + (long long)t * d.N)[c] = packed;
      }
      if (d.colsum) reinterpret_cast<float4*>(d.colsum)[c] = cs;
    }
  } else {
    for (long long c = tid; c < d.N; c += nth) {
      float cs = 0.0f;
      for (int t = 0; t < d.Tr; ++t) {
        const float x = __ldg(d.input + (long long)t * d.row_stride + c);
        cs += x;
        float y = 0.0f;
        if (t < d.T) {
          y = normalized(x, mean, inv);
          mn = fminf(mn, x);
          mx = fmaxf(mx, x);
        }
        out[(long long)t * d.N + c] = from_float<E>(y);
      }
      if (d.colsum) d.colsum[c] = cs;
    }
  }
  double a, q, omn, omx;
  if (!fold_moments(d, 0.0, 0.0, mn, mx, &a, &q, &omn, &omx)) return;
  d.moments[2 * kVarChunks + 2] = omn;
  d.moments[2 * kVarChunks + 3] = omx;
}

// The normalised value y as the FP16 bits the paired tree adds: rounded to the storage form
// first (BF16 values are then exact in FP16 within its normal range, and at most 2^-25 off
// below it).
template <typename E>
__device__ __forceinline__ unsigned short pair_bits(float y) {
  if constexpr (std::is_same<E, __half>::value) {
    return __half_as_ushort(__float2half_rn(y));
  } else {
    return __half_as_ushort(__float2half_rn(__bfloat162float(__float2bfloat16_rn(y))));
  }
}

// The paired copy of a 16- or 32-row search (the paired-FP16 tree's input): the same single
// read as normalize_kernel -- y in float, rounded to the storage form, the float32 column sums
// in row order and the extremes -- but it writes, for row t and channel x in [-kPairPad, N),
// the word (y[t][x], y[t][x + t]) as two FP16 values (0 outside [0, N)): the leaves of drift
// blocks k and k + 1 side by side, since the tree reads row t of drift block k + 1 t channels
// further.  A block takes kPairCols channels at a time, four per thread (256 threads), and
// the rows sixteen at a time: their values, and those of the next kPairPad channels, go to
// shared memory, then every word of those rows is written whole (16-byte stores).
constexpr int kPairCols = 1024;
template <typename E, int TR>
__global__ void __launch_bounds__(256, 4) normalize_pair_kernel(const __grid_constant__ PrecisionBatch b) {
  static_assert(TR == 16 || TR == 32, "paired copies hold 16 or 32 rows");
  const PrecisionDesc& d = b.s[blockIdx.y];
  // sixteen rows of kPairCols + kPairPad values (2112 bytes: every 4-value group is 8-byte
  // aligned)
  __shared__ __align__(16) unsigned short ys[16][kPairCols + kPairPad];
  const float mean = (float)d.moments[2 * kVarChunks];
  const float inv = (float)(1.0 / d.moments[2 * kVarChunks + 1]);
  uint32_t* out = static_cast<uint32_t*>(d.norm);
  const long long np = ((long long)d.N + kPairPad + 3) / 4 * 4;  // pair_row_words(N)
  const int N = d.N, T = d.T;
  float mn = __int_as_float(0x7f800000), mx = -mn;  // NaNs are skipped (they flag themselves)
  const bool vec = (N % 4 == 0) && (d.row_stride % 4 == 0) && ((reinterpret_cast<uintptr_t>(d.input) & 15) == 0);
  for (long long c0 = (long long)blockIdx.x * kPairCols; c0 < N; c0 += (long long)gridDim.x * kPairCols) {
    const long long c = c0 + 4 * threadIdx.x;
    const bool full = vec && c + 3 < N;
    const int nin = c >= N ? 0 : (c + 3 < N ? 4 : (int)(N - c));
    float cs[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 1
    for (int g = 0; g < TR; g += 16) {
      // the next kPairPad channels' values of these rows (the second elements of the last
      // words): two per thread, issued before the block's own loads
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int v = threadIdx.x + 256 * h;
        const int u = v >> 5, i = v & 31;
        const long long x = c0 + kPairCols + i;
        unsigned short hv = 0;
        if (x < N && g + u < T)
          hv = pair_bits<E>(normalized(__ldg(d.input + (long long)(g + u) * d.row_stride + x), mean, inv));
        ys[u][kPairCols + i] = hv;
      }
      // four channels per thread down the sixteen rows, eight rows' loads in flight at a
      // time; channels past N are 0 and do not enter the sums or the extremes
#pragma unroll
      for (int g8 = 0; g8 < 16; g8 += 8) {
        float e[8][4];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const float* row = d.input + (long long)(g + g8 + u) * d.row_stride;
          if (full) {
            const float4 q = __ldg(reinterpret_cast<const float4*>(row + c));
            e[u][0] = q.x;
            e[u][1] = q.y;
            e[u][2] = q.z;
            e[u][3] = q.w;
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i) e[u][i] = i < nin ? __ldg(row + c + i) : 0.0f;
          }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const int t = g + g8 + u;
          unsigned long long packed = 0;
#pragma unroll
          for (int i = 0; i < 4; ++i) cs[i] += e[u][i];
          if (t < T) {
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              if (i < nin) {
                packed |= (unsigned long long)pair_bits<E>(normalized(e[u][i], mean, inv)) << (16 * i);
                mn = fminf(mn, e[u][i]);
                mx = fmaxf(mx, e[u][i]);
              }
            }
          }
          *reinterpret_cast<unsigned long long*>(&ys[g8 + u][4 * threadIdx.x]) = packed;
        }
      }
      __syncthreads();
      // words (y[t][j], y[t][j + t]): the second values are the four starting t further, taken
      // from two aligned 8-byte loads by a constant shift (the loop is unrolled over u; t's
      // low two bits are u's)
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int t = g + u;
        const int sh = t & ~3;  // g is a multiple of 16, so t & 3 == u & 3
        const unsigned long long lo = *reinterpret_cast<const unsigned long long*>(&ys[u][4 * threadIdx.x]);
        const unsigned long long ha = *reinterpret_cast<const unsigned long long*>(&ys[u][4 * threadIdx.x + sh]);
        const unsigned long long hb = *reinterpret_cast<const unsigned long long*>(&ys[u][4 * threadIdx.x + sh + 4]);
        const unsigned long long hi = (u & 3) ? (ha >> (16 * (u & 3))) | (hb << (64 - 16 * (u & 3))) : ha;
        const uint32_t l0 = (uint32_t)lo, l1 = (uint32_t)(lo >> 32), h0 = (uint32_t)hi, h1 = (uint32_t)(hi >> 32);
        const uint4 w = make_uint4(__byte_perm(l0, h0, 0x5410), __byte_perm(l0, h0, 0x7632),
                                   __byte_perm(l1, h1, 0x5410), __byte_perm(l1, h1, 0x7632));
        uint32_t* dst = out + (long long)t * np + kPairPad + c;
        if (nin == 4) {
          *reinterpret_cast<uint4*>(dst) = w;
        } else {
          const uint32_t ws[4] = {w.x, w.y, w.z, w.w};
          for (int i = 0; i < nin; ++i) dst[i] = ws[i];
        }
      }
      // the kPairPad words before channel 0: (0, y[t][x + t])
      if (c0 == 0 && threadIdx.x < 16) {
        const int u = threadIdx.x, t = g + u;
        for (int x = -kPairPad; x < 0; ++x)
          out[(long long)t * np + kPairPad + x] = x + t >= 0 ? (uint32_t)ys[u][x + t] << 16 : 0u;
      }
      __syncthreads();
    }
    if (d.colsum) {
      if (nin == 4) {
        reinterpret_cast<float4*>(d.colsum + c)[0] = make_float4(cs[0], cs[1], cs[2], cs[3]);
      } else {
        for (int i = 0; i < nin; ++i) d.colsum[c + i] = cs[i];
      }
    }
  }
  double a, q, omn, omx;
  if (!fold_moments(d, 0.0, 0.0, mn, mx, &a, &q, &omn, &omx)) return;
  d.moments[2 * kVarChunks + 2] = omn;
  d.moments[2 * kVarChunks + 3] = omx;
}

// The flag threshold in normalised path-sum units: every channel whose float32 top P_f
// (the plain form's, tree order) reaches the search's threshold `thr` has an approximate
// top S~ (the 16-bit tree's) of at least this value, so it is listed and recomputed.
//
// Rounding bounds, per path of the T unrounded rows (padded rows are 0 on both sides):
//  * y_i = (x_i - mean) / std, formed in float (normalized: relative error under 2^-22,
//    absolute 1.01 * 2^-24 * |mean| / std), then rounded to 16 bits:
//    |y~_i - y_i| <= u |y_i| + e_abs with u = 2^-8 + 2^-22 (BF16; 2^-11 + 2^-22 for FP16) and
//    e_abs = 1.01 * 2^-24 * |mean| / std, plus 2^-25 below FP16's normal range (its
//    subnormals and its flush to zero).
//  * float sums of n terms in the tree's pairwise order (depth L = log2 Tr): the error is
//    at most g * sum|terms| with g = 1.01 L 2^-24, for both P_f and S~.
//  * y_i >= -Ym with Ym = max(0, (mean - min x) / std), so sum|y_i| <= S_y + 2 T Ym along a
//    path whose exact normalised sum is S_y = (P - T mean) / std; likewise
//    sum|x_i| <= P + 2 T Xn with Xn = max(0, -min x).
// If P_f >= thr then P >= a_x := thr - g (|thr| + 2 T Xn) (1 + 2g), i.e. S_y >= a =
// (a_x - T mean) / std, and S~ >= S_y - c (|S_y| + 2 T Ym) - T e_abs with c = u + g (1 + u).
// The right side grows with S_y (c < 1), so its value at S_y = a bounds S~ from below.
//
// The paired-FP16 tree (pair16) adds in FP16 instead: each add is off by at most 2^-11 of
// its result or, below FP16's normal range, by 2^-25 absolute, so its sums are within
// h sum|terms| + Tr 2^-25 (1.01) with h = 1.01 L 2^-11; BF16 leaves are rounded to FP16 on the
// way (its 2^-25 below FP16's normal range then applies to both forms).  Then
// S~ >= S_y - c (|S_y| + 2 T Ym) - T e_abs (1 + h) - 1.01 Tr 2^-25 with c = u + h (1 + u).  No partial sum can overflow while Tr * ymax
// stays below 60000 (FP16's largest value is 65504); beyond it every channel is listed.
// A margin of 2^-20 relative guards the double arithmetic here; NaN inputs and NaN tops are
// always listed.
__device__ __forceinline__ float flag_threshold(const PrecisionDesc& d, int elem) {
  const double mean = d.moments[2 * kVarChunks], sd = d.moments[2 * kVarChunks + 1];
  const double xmin = d.moments[2 * kVarChunks + 2], xmax = d.moments[2 * kVarChunks + 3];
  const double thr = (double)d.hdr->threshold;
  const int L = 31 - __clz(d.Tr);
  const double g = 1.01 * L * 0x1p-24;
  const bool fp16 = (elem == kElemF16);
  const bool pair = d.pair16 != 0;
  const double h = pair ? 1.01 * L * 0x1p-11 : g;  // the 16-bit tree's own add bound
  const double u = (fp16 ? 0x1p-11 : 0x1p-8) + 0x1p-22;
  const double e_abs = ((fp16 || pair) ? 0x1p-25 : 0.0) + 1.01 * 0x1p-24 * fabs(mean) / sd;
  const double T = (double)d.T;
  const double xn = xmin < 0.0 ? -xmin : 0.0;
  const double ym = fmax(0.0, (mean - xmin) / sd);
  const double a_x = thr - g * (fabs(thr) + 2.0 * T * xn) * (1.0 + 2.0 * g);
  const double a = (a_x - T * mean) / sd;
  const double c = u + h * (1.0 + u);
  const double sub = pair ? 1.01 * (double)d.Tr * 0x1p-25 : 0.0;
  const double lo = a - c * (fabs(a) + 2.0 * T * ym) - T * e_abs * (1.0 + h) - sub;
  // Normalised values beyond the 16-bit range (a scale from an unrepresentative sample), or
  // paired-FP16 sums that could overflow, void the bounds: then every channel is listed.
  const double ymax = fmax(fabs(xmax - mean), fabs(xmin - mean)) / sd;
  const double ylim = pair ? 60000.0 / (double)d.Tr : (fp16 ? 60000.0 : 1e38);
  if (!(ymax < ylim)) return __int_as_float(0xff800000);  // -inf
  return (float)(lo - 0x1p-20 * (fabs(lo) + 1.0));
}

// Appends channel c to the flag list for every lane whose f holds (one atomic per warp).
__device__ __forceinline__ void flag_append(const PrecisionDesc& d, bool f, int c) {
  const unsigned m = __ballot_sync(0xffffffffu, f);
  if (m) {
    const int lane = threadIdx.x & 31;
    int base = 0;
    if (lane == 0) base = atomicAdd(d.flag_count, __popc(m));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (f) d.flag_list[base + __popc(m & ((1u << lane) - 1u))] = c;
  }
}

// Four channels per thread (16-byte loads) where the tops allow; the list's order does not
// matter (each listed channel is recomputed on its own).
__global__ void flag_channels_kernel(const __grid_constant__ PrecisionBatch b) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  const float thr_y = flag_threshold(d, b.elem);
  if (d.N % 4 == 0 && (reinterpret_cast<uintptr_t>(d.top16) & 15) == 0) {
    const int n4 = d.N / 4;
    for (int i0 = blockIdx.x * blockDim.x; i0 < n4; i0 += gridDim.x * blockDim.x) {
      const int i = i0 + threadIdx.x;
      const bool in = i < n4;
      const float4 v = in ? __ldg(reinterpret_cast<const float4*>(d.top16) + i) : make_float4(0.f, 0.f, 0.f, 0.f);
      flag_append(d, in && !(v.x < thr_y), 4 * i);  // NaN is flagged
      flag_append(d, in && !(v.y < thr_y), 4 * i + 1);
      flag_append(d, in && !(v.z < thr_y), 4 * i + 2);
      flag_append(d, in && !(v.w < thr_y), 4 * i + 3);
    }
    return;
  }
  for (int c0 = blockIdx.x * blockDim.x; c0 < d.N; c0 += gridDim.x * blockDim.x) {
    const int c = c0 + threadIdx.x;
    flag_append(d, c < d.N && !(d.top16[c] < thr_y), c);  // NaN is flagged
  }
}

#include "generated/taylor_direct_gen.cuh"

// Up to 16 rows: one thread per (listed channel, drift block) computes all Tr in-block
// offsets at once from the Tr-row subtree's leaves (taylor_direct_M, the tree's pairing);
// leaves outside [0, N) read as zero, which only ineligible paths touch.
template <int M>
__global__ void recompute_direct_kernel(const __grid_constant__ PrecisionBatch b) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  const long long n = *d.flag_count;
  const int ndb = d.dmax - d.dmin + 1;
  const int N = d.N;
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n * ndb;
       u += (long long)gridDim.x * blockDim.x) {
    const long long k = u / ndb;
    const int db = d.dmin + (int)(u - k * ndb);
    const int c = d.flag_list[k];
    const long long e = (long long)(M - 1) * db;
    float best = 0.0f;
    if (c + e >= 0) {  // otherwise no offset of this drift block is eligible (dedoppler.cu:40-46)
      auto ld = [&](int t, int pos) {
        const long long x = c + (long long)db * t + pos;
        return (x >= 0 && x < N) ? __ldg(d.input + t * d.row_stride + x) : 0.0f;
      };
      float out[M];
      if constexpr (M == 16) taylor_direct_16(ld, out);
      else if constexpr (M == 8) taylor_direct_8(ld, out);
      else if constexpr (M == 4) taylor_direct_4(ld, out);
      else taylor_direct_2(ld, out);
#pragma unroll
      for (int off = 0; off < M; ++off)
        if (c + e + off < N) best = fmaxf(best, out[off]);
    }
    if (best > 0.0f) atomicMax(reinterpret_cast<int*>(d.top) + c, __float_as_int(best));
  }
}

// Work unit = (listed channel, block of blockDim.x of its (drift block, offset) paths),
// one path per thread; the channel's maximum meets in global memory (atomicMax on the
// float bits: every candidate is >= 0).
__global__ void recompute_kernel(const __grid_constant__ PrecisionBatch b) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  const long long n = *d.flag_count;
  const int Tr = d.Tr, N = d.N;
  const int levels = 31 - __clz(Tr);  // Tr is a power of two
  const int paths = (d.dmax - d.dmin + 1) * Tr;
  const int nblk = (paths + blockDim.x - 1) / blockDim.x;
  for (long long u = blockIdx.x; u < n * nblk; u += gridDim.x) {
    const long long k = u / nblk;
    const int pth = (int)(u - k * nblk) * blockDim.x + threadIdx.x;
    const int c = d.flag_list[k];
    float best = 0.0f;
    if (pth < paths) {
      const int db = d.dmin + pth / Tr;
      const int off = pth - (pth / Tr) * Tr;
      const long long e = (long long)(Tr - 1) * db;
      if (c + e >= 0 && c + e + off < N) {  // findTopPathSums' early return (dedoppler.cu:40-46)
        const float* base = d.input + c;
        best = fmaxf(0.0f, path_sum_pow2(levels, off, [&](int t, int pos) {
          return __ldg(base + (long long)t * d.row_stride + (long long)db * t + pos);
        }));
      }
    }
    for (int o = 16; o > 0; o >>= 1) best = fmaxf(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best > 0.0f) atomicMax(reinterpret_cast<int*>(d.top) + c, __float_as_int(best));
  }
}

}  // namespace

cudaError_t normalize_batch(const PrecisionBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  // About 64 sampled values per thread (three rows), at most kVarChunks blocks per search.
  int blocks = (int)std::min<long long>(kVarChunks, std::max<long long>(8, (3ll * b.maxN + 16383) / 16384));
  norm_sample_kernel<<<dim3(blocks, b.count), 256, 0, stream>>>(b);
  // At most kVarChunks blocks per search (the partials of the minimum and maximum).
  int nb = (8 * num_sms + b.count - 1) / b.count;
  if (nb < 8) nb = 8;
  if (nb > kVarChunks) nb = kVarChunks;
  // The searches that take the paired-FP16 tree get the paired copy, the others the dense one.
  PrecisionBatch plain, paired;
  plain.count = paired.count = 0;
  plain.maxN = paired.maxN = b.maxN;
  plain.elem = paired.elem = b.elem;
  for (int k = 0; k < b.count; ++k) {
    PrecisionBatch& dst = b.s[k].pair16 ? paired : plain;
    dst.s[dst.count++] = b.s[k];
  }
  if (plain.count) {
    if (b.elem == kElemBF16) normalize_kernel<__nv_bfloat16><<<dim3(nb, plain.count), 256, 0, stream>>>(plain);
    else normalize_kernel<__half><<<dim3(nb, plain.count), 256, 0, stream>>>(plain);
  }
  // paired copies, one launch per row count
  for (int tr : {16, 32}) {
    PrecisionBatch q;
    q.count = 0;
    q.maxN = b.maxN;
    q.elem = b.elem;
    for (int k = 0; k < paired.count; ++k)
      if (paired.s[k].Tr == tr) q.s[q.count++] = paired.s[k];
    if (!q.count) continue;
    const dim3 grid(nb, q.count);
    if (b.elem == kElemBF16) {
      if (tr == 16) normalize_pair_kernel<__nv_bfloat16, 16><<<grid, 256, 0, stream>>>(q);
      else normalize_pair_kernel<__nv_bfloat16, 32><<<grid, 256, 0, stream>>>(q);
    } else {
      if (tr == 16) normalize_pair_kernel<__half, 16><<<grid, 256, 0, stream>>>(q);
      else normalize_pair_kernel<__half, 32><<<grid, 256, 0, stream>>>(q);
    }
  }
  return cudaGetLastError();
}

cudaError_t flag_channels_batch(const PrecisionBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  int blocks = std::max(1, (b.maxN / 4 + 255) / 256);
  const int cap = (16 * num_sms + b.count - 1) / b.count;
  if (blocks > cap) blocks = cap < 1 ? 1 : cap;
  flag_channels_kernel<<<dim3(blocks, b.count), 256, 0, stream>>>(b);
  return cudaGetLastError();
}

cudaError_t recompute_batch(const PrecisionBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  int blocks = (16 * num_sms + b.count - 1) / b.count;
  if (blocks < 1) blocks = 1;
  // Searches of one rounded timestep count share a launch: the direct form per row count up
  // to 16, the per-path form beyond.
  for (int R : {2, 4, 8, 16, 0}) {
    PrecisionBatch q;
    q.count = 0;
    q.maxN = 0;
    q.elem = b.elem;
    for (int k = 0; k < b.count; ++k)
      if (R ? b.s[k].Tr == R : b.s[k].Tr > 16) {
        q.s[q.count++] = b.s[k];
        q.maxN = std::max(q.maxN, b.s[k].N);
      }
    if (!q.count) continue;
    const dim3 grid(blocks, q.count);
    switch (R) {
      case 2: recompute_direct_kernel<2><<<grid, 128, 0, stream>>>(q); break;
      case 4: recompute_direct_kernel<4><<<grid, 128, 0, stream>>>(q); break;
      case 8: recompute_direct_kernel<8><<<grid, 128, 0, stream>>>(q); break;
      case 16: recompute_direct_kernel<16><<<grid, 128, 0, stream>>>(q); break;
      default: recompute_kernel<<<grid, 256, 0, stream>>>(q); break;
    }
  }
  return cudaGetLastError();
}

}  // namespace scb
