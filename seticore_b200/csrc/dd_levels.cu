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
// Each emit level reads and writes Tr*N floats per drift block; the pairing of the adds
// is the tree's own, so every path sum is bit-identical to the reference's
// twoStageTaylorTree (taylor.cu:298-327).
#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

__device__ __forceinline__ float ld_or_zero(const float* row, long long c, int N) {
  return (c >= 0 && c < N) ? __ldg(row + c) : 0.0f;
}

// One level of M in {2, 4} rows for every problem.  blockIdx.y = p*(Tp/M) + q.
template <int M>
__global__ void emit_kernel(const float* __restrict__ src, long long src_stride, int Tp, int D0,
                            float* __restrict__ dst, int N) {
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
  for (int o = 0; o < M; ++o) dst[(((long long)p * M + o) * nb + q) * N + c] = out[o];
}

}  // namespace

cudaError_t levels_search(const float* input, long long row_stride, int Tr, int N, int dmin, int dmax,
                          float* scratch_a, float* scratch_b, float* top, int num_sms,
                          cudaStream_t stream, const LevelPlan& plan) {
  int sizes[12];
  int nlev = 0;
  int final_rows = 16;
  if (plan.n > 0) {
    int prod = plan.final_rows;
    for (int l = 0; l < plan.n; ++l) {
      if (plan.m[l] != 2 && plan.m[l] != 4) return cudaErrorInvalidValue;
      sizes[nlev++] = plan.m[l];
      prod *= plan.m[l];
    }
    final_rows = plan.final_rows;
    if (prod != Tr || (final_rows != 2 && final_rows != 4 && final_rows != 8 && final_rows != 16))
      return cudaErrorInvalidValue;
  } else {
    for (int tp = Tr; tp > 16;) {
      const int M = (tp / 4 >= 16) ? 4 : 2;
      sizes[nlev++] = M;
      tp /= M;
    }
  }
  for (int db = dmin; db <= dmax; ++db) {
    const float* src = input;
    long long stride = row_stride;
    float* dst = scratch_a;
    int P = 1, Tp = Tr;
    long long dscale = 1;  // product of the level sizes so far
    for (int l = 0; l < nlev; ++l) {
      const int M = sizes[l];
      dim3 grid((N + 255) / 256, (unsigned)(P * (Tp / M)));
      const int D0 = (int)(dscale * db);
      if (M == 4) emit_kernel<4><<<grid, 256, 0, stream>>>(src, stride, Tp, D0, dst, N);
      else emit_kernel<2><<<grid, 256, 0, stream>>>(src, stride, Tp, D0, dst, N);
      src = dst;
      stride = N;
      dst = (dst == scratch_a) ? scratch_b : scratch_a;
      P *= M;
      Tp /= M;
      dscale *= M;
    }
    TreeBatch tb;
    tb.count = 1;
    tb.n_items = 0;
    TreeGroup& tp = tb.g[0];
    tp = TreeGroup{};
    tp.rows = src;
    tp.row_stride = N;
    tp.job_row_stride = (long long)final_rows * N;
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
    cudaError_t err = tree_max_batch(tb, final_rows, num_sms, stream);
    if (err != cudaSuccess) return err;
  }
  return cudaGetLastError();
}

}  // namespace scb
