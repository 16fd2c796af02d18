// Hit selection on the GPU.
//
// window_kernel: the reference's window de-duplication (dedoppler.cu:353-383).  Channels
//   are cut into non-overlapping windows of window_size; a window's candidate is the
//   first channel holding its largest top sum, if that sum is strictly above the
//   threshold; it survives if no channel in [c - window_size + 1, c + window_size) has a
//   strictly larger top sum.  One warp per window.
// resolve_kernel: recovers the drift of each survivor.  The reference keeps, per channel,
//   the first (drift block, offset) in scan order whose sum beat the running maximum
//   (dedoppler.cu:49-53); that is the first eligible path, in (drift block, offset)
//   order, whose sum equals the final top sum.  The fused tree kernel keeps only the top
//   value, so the few survivors recompute their paths here, bit-identically (pairwise
//   tree order), and check the maximum against the stored top sum.
// path_values_kernel: addIncoherentPower (dedoppler.cu:139-176): the path sum along a
//   hit's path; the drift block is floor((float)drift_steps / (Tr-1)) in float, as there.
#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

__global__ void window_kernel(const float* __restrict__ top, int N, int w, SearchHeader* hdr,
                              Candidate* cands, int cap) {
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
      if (slot < cap) cands[slot] = Candidate{(int)bidx, 0, best, 0};
    }
  }
}

__global__ void resolve_kernel(const float* __restrict__ in, long long stride, int Tr, int N, int dmin,
                               int dmax, SearchHeader* hdr, Candidate* cands, int cap) {
  const int n = min(hdr->num_candidates, cap);
  const int lane = threadIdx.x & 31;
  const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int npaths = (dmax - dmin + 1) * Tr;
  for (int i = gw; i < n; i += nw) {
    const long long c = cands[i].index;
    float best = 0.0f;  // the reference's top sums start at zero
    int bp = -1;
    for (int p = lane; p < npaths; p += 32) {
      const int db = dmin + p / Tr;
      const int off = p - (p / Tr) * Tr;
      const long long e = (long long)(Tr - 1) * db;
      if (c + e < 0 || c + e + off >= N) continue;
      const float v = path_sum_pairwise(Tr, off, [&](int t, int pos) {
        return __ldg(in + (long long)t * stride + c + (long long)db * t + pos);
      });
      if (v > best) {
        best = v;
        bp = p;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, best, o);
      const int op = __shfl_xor_sync(0xffffffffu, bp, o);
      if (op >= 0 && (bp < 0 || ov > best || (ov == best && op < bp))) {
        best = ov;
        bp = op;
      }
    }
    if (lane == 0) {
      if (bp >= 0) {
        const int db = dmin + bp / Tr;
        const int off = bp - (bp / Tr) * Tr;
        cands[i].drift_steps = db * (Tr - 1) + off;
        cands[i].flags = 1;
        if (__float_as_int(best) != __float_as_int(cands[i].power)) atomicOr(&hdr->error, 1);
      } else {
        cands[i].drift_steps = 0;
        cands[i].flags = 0;
      }
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
  out[i] = path_sum_pairwise(Tr, off, [&](int t, int pos) {
    return __ldg(in + (long long)t * stride + c + (long long)db * t + pos);
  });
}

}  // namespace

cudaError_t search_hits(const float* input, long long row_stride, int Tr, int N, const float* top,
                        int window_size, int dmin, int dmax, SearchHeader* hdr, Candidate* cands,
                        int cand_capacity, int num_sms, cudaStream_t stream) {
  const long long nwin = ((long long)N + window_size - 1) / window_size;
  long long wblocks = (nwin + 7) / 8;
  if (wblocks > 8 * num_sms) wblocks = 8 * num_sms;
  if (wblocks < 1) wblocks = 1;
  window_kernel<<<(int)wblocks, 256, 0, stream>>>(top, N, window_size, hdr, cands, cand_capacity);
  resolve_kernel<<<2 * num_sms, 256, 0, stream>>>(input, row_stride, Tr, N, dmin, dmax, hdr, cands,
                                                   cand_capacity);
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
