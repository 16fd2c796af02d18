// The GPU halves of loading a coarse channel and of recording hits.
//
// sc_dd_prepare_coarse_channels: what H5Reader::loadCoarseChannel does to a buffer after
// the read (h5_reader.cpp:190-209), on the device and for many coarse channels at once:
// rows [num_timesteps, rounded_timesteps) become zero, and with a DC spike the middle
// column of every loaded row becomes the mean of its neighbours.
//
// sc_dd_gather_columns: the filterbank slices a .hits file stores with each hit
// (hit_file_writer.cpp:81-96: rows [0, num_timesteps), columns [begin, end)), gathered by
// one launch into a packed device buffer.
#include <string>

#include "seticore_b200.h"
#include "dd_internal.h"

namespace scb {
int api_fail(int code, const std::string& msg);
}

namespace {

__global__ void prepare_kernel(float* base, long long item_stride, long long row_stride, int T, int Tr, int N,
                               int dc_spike) {
  float* x = base + (long long)blockIdx.y * item_stride;
  const long long pad = (long long)(Tr - T) * N;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < pad; i += (long long)gridDim.x * blockDim.x) {
    const long long r = T + i / N;
    x[r * row_stride + i % N] = 0.0f;
  }
  if (dc_spike && N >= 3) {
    const int mid = N / 2;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
      float* row = x + (long long)t * row_stride;
      // (row[mid-1] + row[mid+1]) / 2.0 in the reference: a float sum, halved exactly.
      row[mid] = (row[mid - 1] + row[mid + 1]) * 0.5f;
    }
  }
}

__global__ void gather_kernel(const float* __restrict__ in, long long row_stride, int T, const int* __restrict__ ranges,
                              const long long* __restrict__ offsets, float* __restrict__ out) {
  const int k = blockIdx.x;
  const int b = ranges[2 * k], w = ranges[2 * k + 1] - ranges[2 * k];
  float* o = out + offsets[k];
  const long long n = (long long)T * w;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    const long long t = i / w;
    o[i] = __ldg(in + t * row_stride + b + (i - t * w));
  }
}

}  // namespace

extern "C" {

int sc_dd_prepare_coarse_channels(float* dev_base, int count, long long item_stride, long long row_stride,
                                  int num_timesteps, int rounded_timesteps, int num_channels, int has_dc_spike,
                                  void* stream) {
  if (!dev_base || count < 0 || count > 65535 || num_timesteps < 1 || rounded_timesteps < num_timesteps ||
      num_channels < 1 || row_stride < num_channels)
    return scb::api_fail(SC_DD_EINVAL, "sc_dd_prepare_coarse_channels: bad arguments");
  if (count == 0) return SC_DD_OK;
  const long long pad = (long long)(rounded_timesteps - num_timesteps) * num_channels;
  long long work = pad > num_timesteps ? pad : num_timesteps;
  int gx = (int)((work + 255) / 256);
  if (gx > 1024) gx = 1024;
  if (gx < 1) gx = 1;
  prepare_kernel<<<dim3(gx, count), 256, 0, (cudaStream_t)stream>>>(dev_base, item_stride, row_stride, num_timesteps,
                                                                      rounded_timesteps, num_channels, has_dc_spike);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    return scb::api_fail(SC_DD_ECUDA, std::string("sc_dd_prepare_coarse_channels: ") + cudaGetErrorString(e));
  return SC_DD_OK;
}

int sc_dd_gather_columns(const float* dev_input, long long row_stride, int num_timesteps, int num_channels,
                         const int* dev_ranges, const long long* dev_offsets, int count, float* dev_out,
                         void* stream) {
  if (count < 0 || count > 2147483647 / 2 || num_timesteps < 1 || num_channels < 1 || row_stride < num_channels)
    return scb::api_fail(SC_DD_EINVAL, "sc_dd_gather_columns: bad arguments");
  if (count == 0) return SC_DD_OK;
  if (!dev_input || !dev_ranges || !dev_offsets || !dev_out)
    return scb::api_fail(SC_DD_EINVAL, "sc_dd_gather_columns: null pointer");
  gather_kernel<<<count, 256, 0, (cudaStream_t)stream>>>(dev_input, row_stride, num_timesteps, dev_ranges,
                                                          dev_offsets, dev_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return scb::api_fail(SC_DD_ECUDA, std::string("sc_dd_gather_columns: ") + cudaGetErrorString(e));
  return SC_DD_OK;
}

}  // extern "C"
