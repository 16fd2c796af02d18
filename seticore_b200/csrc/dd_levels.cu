// Searches with more than 16 rounded timesteps.
//
// The Taylor tree of Tr = M1*...*Mk*16 rows factors into levels.  After a level of M
// rows has summed every block of M consecutive rows with in-block offset o (drift D of
// the enclosing problem), what remains is, for each o, a tree over Tr/M "rows" (the
// block sums of offset o) with drift o + M*D whose in-block offset r maps to the final
// offset o*(Tr/M) + r (same recursion, taylor.h:48-54).  Numbering the sub-problems
// p*M + o keeps this linear: after the emit levels, problem k has drift
// k + (M1*...*Mk)*db and final offsets 16k + r, so the last level is one launch of the
// fused max kernel over all problems (dd_tree.cu, one staged window per problem).
//
// Default splits:
//  * Tr = 64, 128, 256, float rows: one 16-row level, the emitting form of the fused tree
//    (dd_tree.cu; each CTA stages a 16-row group once for the pass's drift blocks and writes
//    the 16 in-block offsets of a 352-channel strip through a shared buffer as whole bulk
//    rows), then the last level over the 16 sub-problems.  Both run in passes of drift
//    blocks and channels (stripes_search): the planes hold, per block row, only the channels
//    the last level reads in that row (each block row has its own channel origin).
//  * 16-bit rows and Tr > 256: direct16x4_kernel (four channels per thread from global
//    memory), then emit_kernel's 4- and 2-row levels while more than 16 rows remain.
// The pool's autotuner times these against the other splits per shape class.  The pairing
// of the adds is the tree's own at every level, so every path sum is bit-identical to the
// reference's twoStageTaylorTree (taylor.cu:298-327).
#include <algorithm>
#include <atomic>
#include <cstdlib>

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

#include "generated/taylor_direct_gen.cuh"


namespace {

__device__ __forceinline__ float as_float(float v) { return v; }
__device__ __forceinline__ float as_float(__nv_bfloat16 v) { return __bfloat162float(v); }
__device__ __forceinline__ float as_float(__half v) { return __half2float(v); }

template <typename E>
__device__ __forceinline__ float ld_or_zero(const E* row, long long c, int N) {
  return (c >= 0 && c < N) ? as_float(row[c]) : 0.0f;
}

// One level of M in {2, 4} rows for every problem.  blockIdx.y = p*(Tp/M) + q.
template <int M>
__global__ void emit_kernel(const float* __restrict__ src, long long src_stride, int Tp, int D0,
                            float* __restrict__ dst, long long dst_stride, int N) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int nb = Tp / M;
  const int p = blockIdx.y / nb;
  const int q = blockIdx.y - p * nb;
  const long long D = (long long)D0 + p;
  const float* r0 = src + ((long long)p * Tp + (long long)q * M) * src_stride;
  float out[M];
  if constexpr (M == 2) {
    const float x0 = ld_or_zero(r0, c, N);
    out[0] = x0 + ld_or_zero(r0 + src_stride, c + D, N);
    out[1] = x0 + ld_or_zero(r0 + src_stride, c + D + 1, N);
  } else {
    const float* r1 = r0 + src_stride;
    const float* r2 = r1 + src_stride;
    const float* r3 = r2 + src_stride;
    const float x0 = ld_or_zero(r0, c, N);
    const float a0 = x0 + ld_or_zero(r1, c + D, N);
    const float a1 = x0 + ld_or_zero(r1, c + D + 1, N);
    const long long y = c + 2 * D;
    const float b0y0 = ld_or_zero(r2, y, N) + ld_or_zero(r3, y + D, N);
    const float b0y1 = ld_or_zero(r2, y + 1, N) + ld_or_zero(r3, y + 1 + D, N);
    const float b1y1 = ld_or_zero(r2, y + 1, N) + ld_or_zero(r3, y + 1 + D + 1, N);
    const float b1y2 = ld_or_zero(r2, y + 2, N) + ld_or_zero(r3, y + 2 + D + 1, N);
    out[0] = a0 + b0y0;
    out[1] = a0 + b0y1;
    out[2] = a1 + b1y1;
    out[3] = a1 + b1y2;
  }
#pragma unroll
  for (int o = 0; o < M; ++o) dst[(((long long)p * M + o) * nb + q) * dst_stride + c] = out[o];
}

// One level of M in {8, 16} rows, one thread per channel: all M in-block offsets of the
// M-row subtree at channel c from its 136 (M = 16) or 36 (M = 8) leaves, in the tree's
// pairing (taylor_direct_M, generated).  Loads of neighbouring threads overlap, so most
// come from L1; the level reads its input from HBM once and writes the planes once.
// Problem p reads rows from src + p * src_problem_rows rows (0: every problem reads the same
// rows, as the first level does for a chunk of drift blocks) with drift D0 + p.
template <int M, typename E>
__global__ void __launch_bounds__(128, 6) direct_kernel(const E* __restrict__ src, long long src_stride,
                                                        long long src_problem_rows, int Tp, int D0,
                                                        float* __restrict__ dst, long long dst_stride, int N) {
  const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= N) return;
  const int nb = Tp / M;
  const int p = blockIdx.y / nb;
  const int q = blockIdx.y - p * nb;
  const long long D = (long long)D0 + p;
  const E* r0 = src + ((long long)p * src_problem_rows + (long long)q * M) * src_stride;
  float out[M];
  // Leaves lie in [c + min(0, (M-1)D), c + (M-1) + max(0, (M-1)D)]: inside the row for
  // most channels, which then load without bounds checks.
  static_assert(M == 8, "16 rows use direct16x4_kernel");
  const long long span = (long long)(M - 1) * D;
  const bool inside = c + (span < 0 ? span : 0) >= 0 && c + (M - 1) + (span > 0 ? span : 0) < N;
  if (inside) {
    auto ld = [&](int t, int pos) { return as_float(r0[t * src_stride + c + D * t + pos]); };
    taylor_direct_8(ld, out);
  } else {
    auto ld = [&](int t, int pos) { return ld_or_zero(r0 + t * src_stride, c + pos + D * t, N); };
    taylor_direct_8(ld, out);
  }
#pragma unroll
  for (int o = 0; o < M; ++o) dst[(((long long)p * M + o) * nb + q) * dst_stride + c] = out[o];
}

// The 16-row level with four consecutive channels per thread: neighbouring channels share
// leaves and nodes (46 leaf loads and 86 adds per channel instead of 136 and 152), and the
// four results of each offset leave as one 16-byte store.  Plane rows are padded to whole
// tiles (a multiple of 4 channels), so the last thread of a row stores inside its plane.
template <typename E>
__global__ void __launch_bounds__(128, 4) direct16x4_kernel(const E* __restrict__ src, long long src_stride,
                                                            long long src_problem_rows, int Tp, int D0,
                                                            float* __restrict__ dst, long long dst_stride, int N) {
  const long long c = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (c >= N) return;
  const int nb = Tp / 16;
  const int p = blockIdx.y / nb;
  const int q = blockIdx.y - p * nb;
  const long long D = (long long)D0 + p;
  const E* r0 = src + ((long long)p * src_problem_rows + (long long)q * 16) * src_stride;
  float* out = dst + ((long long)p * 16 * nb + q) * dst_stride + c;  // offset 0's plane
  const long long plane = (long long)nb * dst_stride;
  auto sink = [&](int o, float v0, float v1, float v2, float v3) {
    *reinterpret_cast<float4*>(out + o * plane) = make_float4(v0, v1, v2, v3);
  };
  const long long span = 15 * D;
  const bool inside = c + (span < 0 ? span : 0) >= 0 && c + 18 + (span > 0 ? span : 0) < N;
  if (inside) {
    auto ld = [&](int t, int pos) { return as_float(r0[t * src_stride + c + D * t + pos]); };
    taylor_direct_16x4(ld, sink);
  } else {
    auto ld = [&](int t, int pos) { return ld_or_zero(r0 + t * src_stride, c + pos + D * t, N); };
    taylor_direct_16x4(ld, sink);
  }
}

}  // namespace

namespace {

// The fused max level over the problems left after the emit levels: problem k of drift
// block db has drift k + dscale*db and rows src + k*final_rows*N (row stride N).
TreeGroup final_group(const float* src, long long Np, int N, int final_rows, int P, long long dscale, int db, int Tr,
                      float* top) {
  TreeGroup tp{};
  tp.rows = src;
  tp.row_stride = Np;
  tp.job_row_stride = (long long)final_rows * Np;
  tp.N = N;
  tp.d_first = (int)(dscale * db);
  tp.d_step = 1;
  tp.n_jobs = P;
  tp.db_first = db;
  tp.db_step = 0;
  tp.off_base = 0;
  tp.off_step = final_rows;
  tp.elig_T1 = Tr - 1;
  tp.top = top;
  return tp;
}

// The emitting 16-row tree for drift blocks db0 .. db0 + nj - 1 of the input's Tr rows
// (whole rows, the plane layout of the other level kernels): group q reads rows
// 16q .. 16q + 15 (one trapezoid for the nj drift blocks) and writes plane r*(Tr/16) + q of
// drift block j to out + j*job_stride.
cudaError_t emit16(const float* input, long long row_stride, int Tr, int N, long long Np, int db0, int nj,
                   float* out, long long job_stride, int num_sms, cudaStream_t stream, int* status) {
  const int nb = Tr / 16;
  TreeBatch eb;
  eb.count = nb;
  eb.n_items = 0;
  for (int q = 0; q < nb; ++q) {
    TreeGroup& g = eb.g[q];
    g = TreeGroup{};
    g.rows = input + (long long)16 * q * row_stride;
    g.row_stride = row_stride;
    g.job_row_stride = 0;
    g.N = N;
    g.d_first = db0;
    g.d_step = 1;
    g.n_jobs = nj;
    g.emit_out = out + (long long)q * Np;
    g.emit_job_stride = job_stride;
    g.emit_plane_stride = (long long)nb * Np;
    g.status = status;
  }
  return tree_emit_batch(eb, num_sms, stream);
}

constexpr int kEmitTile = 352;     // channels per work item of the emitting tree
constexpr int kStripeUnit = 5280;  // stripes start at multiples of every tree tile width (160, 352, 1056)

// Bytes of planes one stripe pass may write: set_level_stripe_bytes, else
// SETICORE_B200_LEVEL_L2_MB, else 0, which keeps whole rows (as many drift blocks per pass
// as the level buffers hold).  Passes narrower than the row mark their input reads
// evict-first and their planes evict-last in L2, but on 64 x 256 x 131072 beams budgets of
// 32 to 96 MB still measured 0.6-0.95x the whole-row passes: the last level's reads did not
// come from L2, and the narrow passes leave each launch too few items per CTA.
std::atomic<long long> g_stripe_bytes{-1};
size_t level_l2_bytes() {
  const long long set = g_stripe_bytes.load();
  if (set >= 0) return (size_t)set;
  static const size_t mb = [] {
    const char* e = getenv("SETICORE_B200_LEVEL_L2_MB");
    const long v = e ? strtol(e, nullptr, 10) : -1;
    return (v >= 0 && v <= 4096) ? (size_t)v : (size_t)0;
  }();
  return mb << 20;
}

// L2 hints in stripe passes (SETICORE_B200_LEVEL_HINTS=0 turns them off, for comparisons).
bool level_cache_hints() {
  static const bool on = [] {
    const char* e = getenv("SETICORE_B200_LEVEL_HINTS");
    return !(e && e[0] == '0');
  }();
  return on;
}

// Drift blocks per stripe pass at most (SETICORE_B200_LEVEL_MAXJ, for tuning; default 64).
int level_max_chunk() {
  static const int v = [] {
    const char* e = getenv("SETICORE_B200_LEVEL_MAXJ");
    const long x = e ? strtol(e, nullptr, 10) : 0;
    return (x >= 1 && x <= kMaxBatch) ? (int)x : kMaxBatch;
  }();
  return v;
}

// Row length of a stripe pass's planes: a stripe of L channels, nj drift blocks, a last
// level of fr rows.  Block row q of the planes starts at channel x_b - 704 + 16*d0*q (its
// own origin, so a row holds only the channels that the last level reads in that row):
// the stripe, the shears of the nj drift blocks' sixteen sub-problems over q <= fr - 1
// rows, the last tile's lead and the rounding of both tile widths.
long long stripe_row_length(long long L, int nj, int fr) {
  return (L + (16ll * nj - 1) * (fr - 1) + fr + 1062 + 3) / 4 * 4;
}

// One stripe pass of a one-level split (Tr = 16 * fr rows, fr <= 16): the emitting 16-row
// tree writes, for drift blocks d0 .. d0 + nj - 1, the planes that the last level reads for
// the output tiles of [x_b, x_e), then the last level folds them into top.  plane(r, q) of
// drift block j at channel c is G[j*Tr*Lp + r*fr*Lp + q*(Lp - 16*d0) + c], with
// G = buf + 704 - x_b (each block row has its own channel origin).  A pass's planes fit the
// L2 budget, so the last level reads them from L2 and the next pass rewrites the same lines.
cudaError_t stripe_pass(const float* input, long long row_stride, int Tr, int N, int d0, int nj,
                        long long x_b, long long x_e, long long Lp, float* buf, float* top, int nparts, int num_sms,
                        cudaStream_t stream, int* status) {
  const int fr = Tr / 16;
  const long long etile = kEmitTile;
  float* G = buf + 704 - x_b;
  const long long qstride = Lp - 16ll * d0;
  // The last level's tiles: 352 channels, 1056 for last levels of 4 rows or fewer
  // (tree_max_batch's choice for jobs with their own rows).
  const long long WF = fr <= 4 ? 1056 : kEmitTile;
  const long long x_tiles_end = (x_e + WF - 1) / WF * WF;
  TreeBatch eb;
  eb.count = fr;
  eb.n_items = 0;
  eb.cache_mode = level_cache_hints() && (x_b > 0 || x_e < N) ? 1 : 0;  // stripes narrower than the row
  for (int q = 0; q < fr; ++q) {
    TreeGroup& g = eb.g[q];
    g = TreeGroup{};
    g.rows = input + (long long)16 * q * row_stride;
    g.row_stride = row_stride;
    g.job_row_stride = 0;
    g.N = N;
    g.d_first = d0;
    g.d_step = 1;
    g.n_jobs = nj;
    g.emit_out = G + q * qstride;
    g.emit_job_stride = (long long)Tr * Lp;
    g.emit_plane_stride = (long long)fr * Lp;
    // Channels the last level reads in block row q: shears 16*(d0 + j) + k per row for
    // k < 16, j < nj; staged windows rounded out to 16-byte chunks.
    const long long lo = x_b + 16ll * d0 * q - 3;
    const long long hi = x_tiles_end + (16ll * (d0 + nj - 1) + 15) * q + fr + 7;
    const long long xb = std::max<long long>(0, lo >= 0 ? lo / etile * etile : 0);
    const long long xe = std::min<long long>(N, hi);
    // Every tile the level writes (and so every channel the last level reads) lies inside
    // block row q's part of the buffer, [origin, origin + Lp).
    const long long origin = x_b - 704 + 16ll * d0 * q;
    const long long wend = (xe + etile - 1) / etile * etile;
    if (xe > xb && (xb < origin || wend > origin + Lp)) return cudaErrorInvalidValue;
    g.x_begin = (int)xb;
    g.x_end = xe > xb ? (int)xe : -1;  // no tiles when the last level reads none of [0, N) here
    g.status = status;
  }
  cudaError_t err = tree_emit_batch(eb, num_sms, stream, 0, nparts);
  if (err != cudaSuccess) return err;
  TreeBatch tb;
  tb.count = nj;
  tb.n_items = 0;
  for (int j = 0; j < nj; ++j) {
    TreeGroup& tp = tb.g[j];
    tp = TreeGroup{};
    tp.rows = G + (long long)j * Tr * Lp;
    tp.row_stride = qstride;
    tp.job_row_stride = (long long)fr * Lp;
    tp.N = N;
    tp.d_first = 16 * (d0 + j);
    tp.d_step = 1;
    tp.n_jobs = 16;
    tp.db_first = d0 + j;
    tp.db_step = 0;
    tp.off_base = 0;
    tp.off_step = fr;
    tp.elig_T1 = Tr - 1;
    tp.top = top;
    tp.x_begin = (int)x_b;
    tp.x_end = (int)x_e;
    tp.status = status;
  }
  return tree_max_batch(tb, fr, num_sms, stream);
}

// The one-level split with the emitting first level, in stripe passes.  The planes of a
// pass (nj drift blocks x Tr rows x the stripe) fit the L2 budget where one is set, else
// the level buffers (`cap` floats).
cudaError_t stripes_search(const float* input, long long row_stride, int Tr, int N, int dmin, int dmax,
                           float* buf, long long cap, float* top, int nparts, int num_sms, cudaStream_t stream,
                           int* status) {
  const int fr = Tr / 16;
  const int ndb = dmax - dmin + 1;
  // The whole row as one stripe (x_b = 0 suits every tile width, so any tile multiple will do).
  const long long Nt = ((long long)N + 1055) / 1056 * 1056;
  const long long l2 = (long long)(level_l2_bytes() / sizeof(float));
  const long long budget = l2 > 0 ? std::min(l2, cap) : cap;
  // Drift blocks per pass (J) and stripe length (L).  Whole-row mode: the fewest passes,
  // ceil(ndb / J) x stripes, counting a narrow remainder stripe as a full pass (each pass
  // costs a launch's fill and drain), the larger J on a tie, and stripes of equal length.
  // With an L2 budget: the largest J whose stripes span at least four stripe units.
  int J = 0;
  long long L = 0, best_passes = -1;
  for (int j = std::min(ndb, std::min(kMaxBatch, level_max_chunk()));; j = (j + 1) / 2) {
    const long long avail = budget / ((long long)j * Tr) - stripe_row_length(0, j, fr);
    long long lj = 0, stripes = 0;
    if (avail >= Nt) {
      lj = Nt;
      stripes = 1;
    } else {
      const long long lmax = std::max<long long>(0, avail) / kStripeUnit * kStripeUnit;
      if (lmax >= kStripeUnit) {
        stripes = (N + lmax - 1) / lmax;
        lj = ((N + stripes - 1) / stripes + kStripeUnit - 1) / kStripeUnit * kStripeUnit;
      }
    }
    if (stripes > 0) {
      if (l2 > 0) {
        if (lj >= std::min<long long>(Nt, 4 * kStripeUnit) || j == 1) {
          J = j;
          L = lj;
          break;
        }
      } else {
        const long long passes = (long long)((ndb + j - 1) / j) * stripes;
        if (best_passes < 0 || passes < best_passes) {
          best_passes = passes;
          J = j;
          L = lj;
        }
      }
    }
    if (j == 1) break;
  }
  if (J == 0) {  // no stripe fits the budget: the smallest one, one drift block per pass
    J = 1;
    L = std::min<long long>(kStripeUnit, Nt);
  }
  if (L < Nt) L = std::min<long long>(std::max<long long>(L, kStripeUnit), Nt);
  long long Lp = stripe_row_length(L, J, fr);
  if ((long long)J * Tr * Lp > cap) {  // the smallest stripe is too long for the buffers: whole rows
    J = 1;
    L = Nt;
    Lp = stripe_row_length(L, J, fr);
    if ((long long)Tr * Lp > cap) return cudaErrorInvalidValue;  // level buffers too small
  }
  cudaError_t err;
  for (int d0 = dmin; d0 <= dmax; d0 += J) {
    const int nj = std::min(J, dmax - d0 + 1);
    for (long long x_b = 0; x_b < N; x_b += L) {
      const long long x_e = std::min<long long>(N, x_b + L);
      if ((err = stripe_pass(input, row_stride, Tr, N, d0, nj, x_b, x_e, Lp, buf, top, nparts, num_sms, stream,
                             status)) != cudaSuccess)
        return err;
    }
  }
  return cudaGetLastError();
}

// First level of the default one-level split (SETICORE_B200_LEVEL_FIRST overrides it for
// tuning: 16, 1016 or 1017).
int default_first_level() {
  static const int v = [] {
    const char* e = getenv("SETICORE_B200_LEVEL_FIRST");
    const long x = e ? strtol(e, nullptr, 10) : 0;
    return (x == 16 || x == kStreamEmit16 || x == kStreamEmit16One) ? (int)x : kStreamEmit16;
  }();
  return v;
}

}  // namespace

void set_level_stripe_bytes(long long bytes) { g_stripe_bytes.store(bytes < 0 ? -1 : bytes); }
long long level_stripe_bytes() { return g_stripe_bytes.load(); }

cudaError_t levels_search(const void* input_v, long long row_stride, int Tr, int N, int dmin, int dmax,
                          float* scratch_a, float* scratch_b, float* top, int num_sms,
                          cudaStream_t stream, const LevelPlan& plan, int elem, int* status) {
  int sizes[12];
  int nlev = 0;
  int final_rows = 16;
  const float* input = static_cast<const float*>(input_v);
  if (elem != kElemF32 && plan.n > 0) return cudaErrorInvalidValue;  // 16-bit input: default split only
  if (plan.n > 0) {
    int prod = plan.final_rows;
    for (int l = 0; l < plan.n; ++l) {
      const int M = plan.m[l];
      const bool emit = (M == kStreamEmit16 || M == kStreamEmit16One) && l == 0;
      if (M != 2 && M != 4 && M != 8 && M != 16 && !emit) return cudaErrorInvalidValue;
      sizes[nlev++] = M;
      prod *= emit ? 16 : M;
    }
    final_rows = plan.final_rows;
    if (prod != Tr || (final_rows != 2 && final_rows != 4 && final_rows != 8 && final_rows != 16))
      return cudaErrorInvalidValue;
  } else {
    // Default: the 16-row level, then 4s and 2s down to at most 16 rows.  A single 16-row
    // level (Tr <= 256) of float rows takes the emitting tree in stripe passes; 16-bit rows
    // and deeper splits the four-channels-per-thread level kernel (the emitting tree
    // converts 16-bit rows with per-thread loads as it stages them: 0.79x on 256-row beams).
    int tp = Tr / 16;
    sizes[nlev++] = (tp <= 16 && elem == kElemF32) ? default_first_level() : 16;
    while (tp > 16) {
      const int M = (tp / 4 >= 16) ? 4 : 2;
      sizes[nlev++] = M;
      tp /= M;
    }
    final_rows = tp;
  }
  // scratch_b lies in the same allocation as scratch_a, which holds 2 * (scratch_b -
  // scratch_a) floats: one level buffer for the ping-pong of multi-level plans, or room for
  // the planes of several drift blocks at once.
  const long long half = scratch_b - scratch_a;
  const long long Np = level_row_length(N);  // plane row length
  const long long per_db = (long long)Tr * Np;
  cudaError_t err;
  if (nlev == 1 && (sizes[0] == kStreamEmit16 || sizes[0] == kStreamEmit16One))  // float rows (checked above)
    return stripes_search(input, row_stride, Tr, N, dmin, dmax, scratch_a, 2 * half, top,
                          sizes[0] == kStreamEmit16One ? 1 : 2, num_sms, stream, status);
  if (nlev == 1 && (sizes[0] == 16 || sizes[0] == kStreamEmit16)) {
    // One level, then the last: the planes of up to J drift blocks per pair of launches.
    long long J = 2 * half / per_db;
    if (J > kMaxBatch) J = kMaxBatch;
    if (J < 1) return cudaErrorInvalidValue;
    const int nb = Tr / 16;
    for (int db = dmin; db <= dmax; db += (int)J) {
      const int nj = (int)std::min<long long>(J, dmax - db + 1);
      {
        dim3 grid((N + 511) / 512, (unsigned)(nj * nb));
        if (elem == kElemBF16)
          direct16x4_kernel<<<grid, 128, 0, stream>>>(static_cast<const __nv_bfloat16*>(input_v), row_stride, 0, Tr, db,
                                                      scratch_a, Np, N);
        else if (elem == kElemF16)
          direct16x4_kernel<<<grid, 128, 0, stream>>>(static_cast<const __half*>(input_v), row_stride, 0, Tr, db,
                                                      scratch_a, Np, N);
        else
          direct16x4_kernel<<<grid, 128, 0, stream>>>(input, row_stride, 0, Tr, db, scratch_a, Np, N);
      }
      TreeBatch tb;
      tb.count = nj;
      tb.n_items = 0;
      for (int j = 0; j < nj; ++j) {
        tb.g[j] = final_group(scratch_a + j * per_db, Np, N, final_rows, 16, 16, db + j, Tr, top);
        tb.g[j].status = status;
      }
      if ((err = tree_max_batch(tb, final_rows, num_sms, stream)) != cudaSuccess) return err;
    }
    return cudaGetLastError();
  }
  if (half < per_db) return cudaErrorInvalidValue;
  for (int db = dmin; db <= dmax; ++db) {
    const float* src = input;
    long long stride = row_stride;
    float* dst = scratch_a;
    int P = 1, Tp = Tr;
    long long dscale = 1;  // product of the level sizes so far
    for (int l = 0; l < nlev; ++l) {
      int M = sizes[l];
      const int D0 = (int)(dscale * db);
      if (M == kStreamEmit16 || M == kStreamEmit16One) {
        M = 16;
        if ((err = emit16(src, stride, Tp, N, Np, db, 1, dst, per_db, num_sms, stream, status)) != cudaSuccess) return err;
      } else if (M == 16) {
        dim3 grid((N + 511) / 512, (unsigned)(P * (Tp / M)));
        if (l == 0 && elem == kElemBF16) {
          direct16x4_kernel<<<grid, 128, 0, stream>>>(static_cast<const __nv_bfloat16*>(input_v), stride, Tp, Tp, D0,
                                                      dst, Np, N);
        } else if (l == 0 && elem == kElemF16) {
          direct16x4_kernel<<<grid, 128, 0, stream>>>(static_cast<const __half*>(input_v), stride, Tp, Tp, D0, dst, Np,
                                                      N);
        } else {
          direct16x4_kernel<<<grid, 128, 0, stream>>>(src, stride, Tp, Tp, D0, dst, Np, N);
        }
      } else if (M == 8) {
        dim3 grid((N + 127) / 128, (unsigned)(P * (Tp / M)));
        direct_kernel<8><<<grid, 128, 0, stream>>>(src, stride, Tp, Tp, D0, dst, Np, N);
      } else {
        dim3 grid((N + 255) / 256, (unsigned)(P * (Tp / M)));
        if (M == 4) emit_kernel<4><<<grid, 256, 0, stream>>>(src, stride, Tp, D0, dst, Np, N);
        else emit_kernel<2><<<grid, 256, 0, stream>>>(src, stride, Tp, D0, dst, Np, N);
      }
      src = dst;
      stride = Np;
      dst = (dst == scratch_a) ? scratch_b : scratch_a;
      P *= M;
      Tp /= M;
      dscale *= M;
    }
    TreeBatch tb;
    tb.count = 1;
    tb.n_items = 0;
    tb.g[0] = final_group(src, Np, N, final_rows, P, dscale, db, Tr, top);
    tb.g[0].status = status;
    if ((err = tree_max_batch(tb, final_rows, num_sms, stream)) != cudaSuccess) return err;
  }
  return cudaGetLastError();
}

}  // namespace scb
