// The precision form: searches over normalised 16-bit spectra with exact hits.
//
//   1. norm_moments_kernel: per search, the FP64 mean and standard deviation of the
//      unrounded rows of the original float32 power (zero-padded rows excluded).
//   2. normalize_kernel: y = (x - mean) / std, rounded to BF16 or FP16 (padded rows stay
//      0), into a dense [Tr][N] 16-bit copy -- half the bytes of the float32 input.
//   3. (dd_tree.cu) the fused tree over y, accumulating in FP32, gives approximate tops.
//      A path sum of y equals (P - T*mean) / std for the path sum P of x, so the order of
//      path sums is preserved up to the 16-bit rounding.
//   4. flag_tiles_kernel: a tile is flagged if any of its channels has an approximate
//      top at or above 0.9 x the threshold in SNR units: P >= median + 0.9 * snr * std.
//   5. (dd_tree.cu) the FP32 tree runs again over the flagged tiles only, from the
//      original power, writing exact tops (bit-identical to the plain form) there.
//      Every other channel keeps top 0: its approximate top is below 0.9 x threshold, so
//      its exact top is below the threshold and it can neither become a window
//      candidate nor beat one (dedoppler.cu:353-383 compares only with values above
//      the threshold).  The hit list is therefore the plain form's.
// The statistics (median, standard deviation, threshold) always come from the float32
// column sums, exactly as in the plain form.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

__global__ void norm_moments_kernel(const __grid_constant__ PrecisionBatch b) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  __shared__ double r1[32], r2[32];
  __shared__ bool last_block;
  const long long total = (long long)d.T * d.N;
  double s1 = 0.0, s2 = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long t = i / d.N, c = i - t * d.N;
    const double v = (double)__ldg(d.input + t * d.row_stride + c);
    s1 += v;
    s2 += v * v;
  }
  for (int o = 16; o > 0; o >>= 1) {
    s1 += __shfl_down_sync(0xffffffffu, s1, o);
    s2 += __shfl_down_sync(0xffffffffu, s2, o);
  }
  if ((threadIdx.x & 31) == 0) {
    r1[threadIdx.x >> 5] = s1;
    r2[threadIdx.x >> 5] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, q = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += r1[w];
      q += r2[w];
    }
    d.moments[blockIdx.x] = a;
    d.moments[kVarChunks + blockIdx.x] = q;
    __threadfence();
    last_block = (atomicAdd(d.ticket, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last_block) return;
  __threadfence();
  double a = 0.0, q = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
    a += __ldcg(d.moments + k);
    q += __ldcg(d.moments + kVarChunks + k);
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    q += __shfl_down_sync(0xffffffffu, q, o);
  }
  __syncthreads();
  if ((threadIdx.x & 31) == 0) {
    r1[threadIdx.x >> 5] = a;
    r2[threadIdx.x >> 5] = q;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  a = 0.0;
  q = 0.0;
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    a += r1[w];
    q += r2[w];
  }
  const double n = (double)total;
  const double mean = a / n;
  double var = q / n - mean * mean;
  if (!(var > 0.0)) var = 1.0;  // constant input: any positive scale keeps the order
  d.moments[2 * kVarChunks] = mean;
  d.moments[2 * kVarChunks + 1] = sqrt(var);
  *d.ticket = 0;
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

template <typename E>
__global__ void normalize_kernel(const __grid_constant__ PrecisionBatch b) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  const double mean = d.moments[2 * kVarChunks];
  const double inv = 1.0 / d.moments[2 * kVarChunks + 1];
  E* out = static_cast<E*>(d.norm);
  const long long total = (long long)d.Tr * d.N;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const long long t = i / d.N, c = i - t * d.N;
    float y = 0.0f;
    if (t < d.T) y = (float)(((double)__ldg(d.input + t * d.row_stride + c) - mean) * inv);
    out[i] = from_float<E>(y);
  }
}

__global__ void flag_tiles_kernel(const __grid_constant__ PrecisionBatch b, int tile_width) {
  const PrecisionDesc& d = b.s[blockIdx.y];
  __shared__ int any;
  const int n_tiles = (d.N + tile_width - 1) / tile_width;
  // Loose threshold in SNR units (0.9 x), mapped to normalised path-sum units.
  const double median = (double)d.hdr->median, sd = (double)d.hdr->std_dev;
  const double mean = d.moments[2 * kVarChunks], scale = d.moments[2 * kVarChunks + 1];
  const double thr_x = median + 0.9 * d.snr_threshold * sd;
  const float thr_y = (float)((thr_x - (double)d.T * mean) / scale);
  for (int tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    const int c0 = tile * tile_width, c1 = min(d.N, c0 + tile_width);
    bool hit = false;
    for (int c = c0 + threadIdx.x; c < c1; c += blockDim.x) hit |= !(d.top16[c] < thr_y);
    if (__any_sync(0xffffffffu, hit) && (threadIdx.x & 31) == 0) any = 1;
    __syncthreads();
    if (threadIdx.x == 0 && any) d.tile_list[atomicAdd(d.tile_count, 1)] = tile;
    __syncthreads();
  }
}

}  // namespace

cudaError_t normalize_batch(const PrecisionBatch& b, int num_sms, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  int blocks = (4 * num_sms + b.count - 1) / b.count;
  if (blocks < 8) blocks = 8;
  if (blocks > kVarChunks) blocks = kVarChunks;
  norm_moments_kernel<<<dim3(blocks, b.count), 256, 0, stream>>>(b);
  int nb = (8 * num_sms + b.count - 1) / b.count;
  if (nb < 8) nb = 8;
  if (b.elem == kElemBF16) normalize_kernel<__nv_bfloat16><<<dim3(nb, b.count), 256, 0, stream>>>(b);
  else normalize_kernel<__half><<<dim3(nb, b.count), 256, 0, stream>>>(b);
  return cudaGetLastError();
}

cudaError_t flag_tiles_batch(const PrecisionBatch& b, int tile_width, cudaStream_t stream) {
  if (b.count <= 0) return cudaSuccess;
  const int n_tiles = (b.maxN + tile_width - 1) / tile_width;
  int blocks = n_tiles < 1024 ? n_tiles : 1024;
  flag_tiles_kernel<<<dim3(blocks, b.count), 256, 0, stream>>>(b, tile_width);
  return cudaGetLastError();
}

}  // namespace scb
