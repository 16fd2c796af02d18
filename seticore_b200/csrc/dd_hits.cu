// Hit selection on the GPU.
//
// window_kernel: the reference's window de-duplication (dedoppler.cu:264-303).  Channels
//   are cut into non-overlapping windows of window_size; a window's candidate is the
//   first channel holding its largest top sum, if that sum is strictly above the
//   threshold; it survives if no channel in [c - window_size + 1, c + window_size) has a
//   strictly larger top sum.  One warp per window.
// resolve_kernel: recovers the drift of each survivor.  The reference keeps, per channel,
//   the first (drift block, offset) in scan order whose sum beat the running maximum
//   (dedoppler.cu:49-53); that is the first eligible path, in (drift block, offset)
//   order, whose sum equals the final top sum.  The fused tree kernel keeps only the top
//   value, so the few survivors recompute their paths here, bit-identically (the tree's
//   pairing): one thread per (survivor, drift block) up to 16 rows (resolve_direct_kernel),
//   one thread per (survivor, path) beyond; the host decodes the packed best and checks its
//   sum against the stored top sum.
// path_values_kernel: addIncoherentPower (dedoppler.cu:139-176): the path sum along a
//   hit's path; the drift block is floor((float)drift_steps / (Tr-1)) in float, as there.
#include <algorithm>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

__global__ void window_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ top = sd.top;
  const int N = sd.N, w = sd.window_size, cap = sd.cand_cap;
  SearchHeader* hdr = sd.hdr;
  Candidate* cands = sd.cands;
  const float thr = hdr->threshold;
  const int lane = threadIdx.x & 31;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  const long long nwin = ((long long)N + w - 1) / w;
  for (long long i = gw; i < nwin; i += nw) {
    const long long start = i * w;
    const long long end = min((long long)N, start + w);
    float best = thr;
    long long bidx = -1;
    for (long long f = start + lane; f < end; f += 32) {
      const float v = top[f];
      if (v > best) {
        best = v;
        bidx = f;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, best, o);
      const long long oi = __shfl_xor_sync(0xffffffffu, bidx, o);
      if (oi >= 0 && (bidx < 0 || ov > best || (ov == best && oi < bidx))) {
        best = ov;
        bidx = oi;
      }
    }
    if (bidx < 0) continue;
    const long long lo = max(0ll, bidx - w + 1);
    const long long hi = min((long long)N, bidx + w);
    bool larger = false;
    for (long long f = lo + lane; f < hi && !larger; f += 32) larger = top[f] > best;
    if (__any_sync(0xffffffffu, larger)) continue;
    if (lane == 0) {
      const int slot = atomicAdd(&hdr->num_candidates, 1);
      if (slot < cap) cands[slot] = Candidate{(int)bidx, 0, best, 0, 0ull};
    }
  }
}

// One thread per (candidate, path): every eligible path of every surviving channel is
// summed in tree order and folded into the candidate's packed best with atomicMax.
__global__ void resolve_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ in = sd.input;
  const long long stride = sd.row_stride;
  const int Tr = sd.Tr, N = sd.N, dmin = sd.dmin, dmax = sd.dmax, cap = sd.cand_cap;
  const SearchHeader* hdr = sd.hdr;
  Candidate* cands = sd.cands;
  const long long n = min(hdr->num_candidates, cap);
  const long long npaths = (long long)(dmax - dmin + 1) * Tr;
  const long long total = n * npaths;
  const int levels = 31 - __clz(Tr);  // Tr is a power of two
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx / npaths;
    const int p = (int)(idx - i * npaths);
    const long long c = cands[i].index;
    const int db = dmin + p / Tr;
    const int off = p - (p / Tr) * Tr;
    const long long e = (long long)(Tr - 1) * db;
    if (c + e < 0 || c + e + off >= N) continue;
    const float v = path_sum_pow2(levels, off, [&](int t, int pos) {
      return __ldg(in + (long long)t * stride + c + (long long)db * t + pos);
    });
    if (v > 0.0f) {  // the reference's top sums start at zero and update on strict >
      const unsigned long long key = ((unsigned long long)float_key(v) << 32) | (unsigned long long)(~(uint32_t)p);
      atomicMax(&cands[i].best, key);
    }
  }
}

__global__ void path_values_kernel(const float* __restrict__ in, long long stride, int Tr, int N,
                                   const int* index, const int* drift_steps, float* out, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int shift = Tr - 1;
  const int ds = drift_steps[i];
  const int db = (int)floorf((float)ds / (float)shift);
  const int off = ds - db * shift;
  const long long c = index[i];
  const long long first = c, last = c + (long long)db * shift + off;
  if (off < 0 || off >= Tr || first < 0 || first >= N || last < 0 || last >= N) {
    out[i] = __int_as_float(0x7fc00000);
    return;
  }
  out[i] = path_sum_pow2(31 - __clz(Tr), off, [&](int t, int pos) {  // Tr is a power of two
    return __ldg(in + (long long)t * stride + c + (long long)db * t + pos);
  });
}

#include "generated/taylor_direct_gen.cuh"

// Up to 16 rows: one thread per (survivor, drift block) computes all Tr offsets of the
// block from the subtree's leaves (taylor_direct_M, the tree's pairing; leaves outside
// [0, N) read as zero, which only ineligible paths touch) and merges its best packed key.
template <int M>
__global__ void resolve_direct_kernel(const __grid_constant__ SearchBatch b) {
  const SearchDesc& sd = b.s[blockIdx.y];
  const float* __restrict__ in = sd.input;
  const long long stride = sd.row_stride;
  const int N = sd.N, dmin = sd.dmin, ndb = sd.dmax - sd.dmin + 1, cap = sd.cand_cap;
  Candidate* cands = sd.cands;
  const long long n = min(sd.hdr->num_candidates, cap);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n * ndb;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long i = idx / ndb;
    const int j = (int)(idx - i * ndb);
    const int db = dmin + j;
    const long long c = cands[i].index;
    const long long e = (long long)(M - 1) * db;
    if (c + e < 0) continue;  // no offset of this drift block is eligible
    auto ld = [&](int t, int pos) {
      const long long x = c + (long long)db * t + pos;
      return (x >= 0 && x < N) ? __ldg(in + t * stride + x) : 0.0f;
    };
    float out[M];
    if constexpr (M == 16) taylor_direct_16(ld, out);
    else if constexpr (M == 8) taylor_direct_8(ld, out);
    else if constexpr (M == 4) taylor_direct_4(ld, out);
    else taylor_direct_2(ld, out);
    unsigned long long best = 0;
#pragma unroll
    for (int off = 0; off < M; ++off) {
      if (c + e + off >= N || !(out[off] > 0.0f)) continue;  // eligible, and above the zero start
      const uint32_t p = (uint32_t)(j * M + off);
      const unsigned long long key = ((unsigned long long)float_key(out[off]) << 32) | (unsigned long long)(~p);
      best = key > best ? key : best;
    }
    if (best) atomicMax(&cands[i].best, best);
  }
}

}  // namespace

cudaError_t search_hits_batch(const SearchBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  long long nwin = 1;
  for (int k = 0; k < b.count; ++k) {
    const long long n = ((long long)b.s[k].N + b.s[k].window_size - 1) / b.s[k].window_size;
    if (n > nwin) nwin = n;
  }
  long long wblocks = (nwin + 7) / 8;  // 8 warps per block, one window per warp
  const long long wcap = (8ll * num_sms + b.count - 1) / b.count;
  if (wblocks > wcap) wblocks = wcap;
  if (wblocks < 1) wblocks = 1;
  window_kernel<<<dim3((unsigned)wblocks, b.count), 256, 0, stream>>>(b);
  int rblocks = (4 * num_sms + b.count - 1) / b.count;
  if (rblocks < 4) rblocks = 4;
  // Drift recovery, one launch per row count: the direct form up to 16 rows, one path per
  // thread beyond.
  for (int R : {2, 4, 8, 16, 0}) {
    SearchBatch q;
    q.count = 0;
    q.maxN = 0;
    for (int k = 0; k < b.count; ++k)
      if (R ? b.s[k].Tr == R : b.s[k].Tr > 16) {
        q.s[q.count++] = b.s[k];
        q.maxN = std::max(q.maxN, b.s[k].N);
      }
    if (!q.count) continue;
    const dim3 grid(rblocks, q.count);
    switch (R) {
      case 2: resolve_direct_kernel<2><<<grid, 128, 0, stream>>>(q); break;
      case 4: resolve_direct_kernel<4><<<grid, 128, 0, stream>>>(q); break;
      case 8: resolve_direct_kernel<8><<<grid, 128, 0, stream>>>(q); break;
      case 16: resolve_direct_kernel<16><<<grid, 128, 0, stream>>>(q); break;
      default: resolve_kernel<<<grid, 256, 0, stream>>>(q); break;
    }
  }
  return cudaGetLastError();
}

cudaError_t path_values(const float* input, long long row_stride, int Tr, int N, const int* index,
                        const int* drift_steps, float* out, int n, cudaStream_t stream) {
  if (n <= 0) return cudaSuccess;
  path_values_kernel<<<(n + 127) / 128, 128, 0, stream>>>(input, row_stride, Tr, N, index, drift_steps,
                                                          out, n);
  return cudaGetLastError();
}

}  // namespace scb
