// C ABI of the B200 dedoppler search (declared in include/seticore_b200.h).
//
// sc_dd mirrors the reference's Dedopplerer (dedoppler.h:15-79): it is built for one
// (timesteps, channels, foff, tsamp) shape and owns every scratch buffer, reused across
// searches (dedoppler.cu:76-111).  A search queues, on the caller's stream:
//   memset(top) -> column sums + order statistics + moments (dd_stats.cu)
//   -> fused tree/top kernel (dd_tree.cu, or the level path of dd_levels.cu for Tr > 16)
//   -> window de-duplication + drift recovery (dd_hits.cu)
// and then copies one small block (statistics + candidates) to pinned host memory.
// Only the hit list crosses to the host, not the reference's four N-length arrays.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t err, const char* what) {
  return fail(SC_DD_ECUDA, std::string(what) + ": " + cudaGetErrorString(err));
}

constexpr int kHostCands = 1024;

int round_up_pow2(int n) {  // util.cpp:16-22
  int r = 1;
  while (r < n) r *= 2;
  return r;
}

// Saves and restores the caller's current device around a call.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

struct sc_dd {
  int T = 0, Tr = 0, N = 0;
  double foff = 0, tsamp = 0;
  int has_dc_spike = 0;
  int device = 0, num_sms = 148;
  float* top = nullptr;
  float* colsum = nullptr;
  scb::SelectState* sel = nullptr;
  scb::MomentPartial* partials = nullptr;
  int n_partials = 0;
  double* var_scratch = nullptr;
  void* result = nullptr;  // SearchHeader followed by Candidate[cand_cap]
  int cand_cap = 0;
  float* scratch_a = nullptr;
  float* scratch_b = nullptr;
  void* host_result = nullptr;  // pinned: SearchHeader + kHostCands candidates
  int* inc_index = nullptr;
  int* inc_steps = nullptr;
  float* inc_vals = nullptr;
  int inc_cap = 0;
  size_t device_bytes = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // search start, tree start/end, search end
  sc_dd_stats last{};
  bool have_last = false;

  scb::SearchHeader* hdr() { return static_cast<scb::SearchHeader*>(result); }
  scb::Candidate* cands() {
    return reinterpret_cast<scb::Candidate*>(static_cast<char*>(result) + sizeof(scb::SearchHeader));
  }
};

namespace {

void free_all(sc_dd* d) {
  cudaFree(d->top);
  cudaFree(d->colsum);
  cudaFree(d->sel);
  cudaFree(d->partials);
  cudaFree(d->var_scratch);
  cudaFree(d->result);
  cudaFree(d->scratch_a);
  cudaFree(d->scratch_b);
  cudaFree(d->inc_index);
  cudaFree(d->inc_steps);
  cudaFree(d->inc_vals);
  if (d->host_result) cudaFreeHost(d->host_result);
  for (cudaEvent_t& e : d->ev)
    if (e) cudaEventDestroy(e);
}

template <typename T>
cudaError_t dalloc(sc_dd* d, T** p, size_t bytes) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
  if (e == cudaSuccess) d->device_bytes += bytes;
  return e;
}

int ensure_inc(sc_dd* d, int n) {
  if (n <= d->inc_cap) return SC_DD_OK;
  cudaFree(d->inc_index);
  cudaFree(d->inc_steps);
  cudaFree(d->inc_vals);
  d->device_bytes -= (size_t)d->inc_cap * 12;
  d->inc_cap = 0;
  const int cap = std::max(n, 4096);
  cudaError_t e;
  if ((e = dalloc(d, &d->inc_index, sizeof(int) * cap)) != cudaSuccess ||
      (e = dalloc(d, &d->inc_steps, sizeof(int) * cap)) != cudaSuccess ||
      (e = dalloc(d, &d->inc_vals, sizeof(float) * cap)) != cudaSuccess)
    return cuda_fail(e, "incoherent staging allocation");
  d->inc_cap = cap;
  return SC_DD_OK;
}

}  // namespace

extern "C" {

const char* sc_dd_last_error(void) { return g_last_error.c_str(); }

const char* sc_dd_version(void) { return "seticore-b200 0.1 (dedoppler; reference seticore 1.0.6)"; }

int sc_dd_create(int num_timesteps, int num_channels, double foff_mhz, double tsamp_s,
                 int has_dc_spike, sc_dd** out) {
  g_last_error.clear();
  if (!out) return fail(SC_DD_EINVAL, "sc_dd_create: out is null");
  *out = nullptr;
  if (num_timesteps < 2) return fail(SC_DD_EINVAL, "sc_dd_create: num_timesteps must be > 1");
  if (num_timesteps > 2048) return fail(SC_DD_EINVAL, "sc_dd_create: num_timesteps above 2048");
  if (num_channels < 64) return fail(SC_DD_EINVAL, "sc_dd_create: num_channels must be >= 64");
  if (!(tsamp_s > 0) || !(foff_mhz != 0) || !std::isfinite(foff_mhz))
    return fail(SC_DD_EINVAL, "sc_dd_create: foff must be nonzero and tsamp positive");
  sc_dd* d = new (std::nothrow) sc_dd();
  if (!d) return fail(SC_DD_ENOMEM, "sc_dd_create: host allocation failed");
  d->T = num_timesteps;
  d->Tr = round_up_pow2(num_timesteps);
  d->N = num_channels;
  d->foff = foff_mhz;
  d->tsamp = tsamp_s;
  d->has_dc_spike = has_dc_spike;
  cudaError_t e = cudaGetDevice(&d->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&d->num_sms, cudaDevAttrMultiProcessorCount, d->device);
  if (e != cudaSuccess) {
    delete d;
    return cuda_fail(e, "sc_dd_create: no CUDA device");
  }
  const size_t N = (size_t)num_channels;
  d->n_partials = 4 * d->num_sms;
  d->cand_cap = num_channels / 2 + 2;
  const size_t result_bytes = sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * d->cand_cap;
  if ((e = dalloc(d, &d->top, sizeof(float) * N)) != cudaSuccess ||
      (e = dalloc(d, &d->colsum, sizeof(float) * N)) != cudaSuccess ||
      (e = dalloc(d, &d->sel, sizeof(scb::SelectState))) != cudaSuccess ||
      (e = dalloc(d, &d->partials, sizeof(scb::MomentPartial) * d->n_partials)) != cudaSuccess ||
      (e = dalloc(d, &d->var_scratch, sizeof(double) * 2 * scb::kVarChunks)) != cudaSuccess ||
      (e = dalloc(d, &d->result, result_bytes)) != cudaSuccess ||
      (d->Tr > 16 && (e = dalloc(d, &d->scratch_a, sizeof(float) * N * d->Tr)) != cudaSuccess) ||
      (d->Tr > 16 && (e = dalloc(d, &d->scratch_b, sizeof(float) * N * d->Tr)) != cudaSuccess) ||
      (e = cudaMallocHost(&d->host_result,
                          sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * kHostCands)) != cudaSuccess) {
    free_all(d);
    delete d;
    return fail(e == cudaErrorMemoryAllocation ? SC_DD_ENOMEM : SC_DD_ECUDA,
                std::string("sc_dd_create: allocation failed: ") + cudaGetErrorString(e));
  }
  e = cudaMemset(d->sel, 0, sizeof(scb::SelectState));
  for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&d->ev[i]);
  if (e != cudaSuccess) {
    free_all(d);
    delete d;
    return cuda_fail(e, "sc_dd_create: memset");
  }
  *out = d;
  return SC_DD_OK;
}

int sc_dd_destroy(sc_dd* dd) {
  if (!dd) return SC_DD_OK;
  DeviceGuard g(dd->device);
  free_all(dd);
  delete dd;
  return SC_DD_OK;
}

size_t sc_dd_memory_usage(const sc_dd* dd) { return dd ? dd->device_bytes : 0; }

int sc_dd_rounded_timesteps(const sc_dd* dd) { return dd ? dd->Tr : 0; }

int sc_dd_search(sc_dd* dd, const float* dev_input, long long row_stride, int beam,
                 int coarse_channel, double max_drift, double min_drift, double snr_threshold,
                 sc_dd_hit* out, int capacity, int* num_hits, void* stream_ptr) {
  g_last_error.clear();
  if (!dd || !dev_input || !num_hits || (capacity > 0 && !out))
    return fail(SC_DD_EINVAL, "sc_dd_search: null argument");
  if (row_stride < dd->N) return fail(SC_DD_ESHAPE, "sc_dd_search: row_stride smaller than num_channels");
  DeviceGuard guard(dd->device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const int Tr = dd->Tr, N = dd->N;

  // dedoppler.cu:165-167 and 274-278, 354: the same double arithmetic.
  const int drift_timesteps = Tr - 1;
  const double res = 1e6 * dd->foff / (drift_timesteps * dd->tsamp);
  const double diag = res * drift_timesteps;
  const double nmax = max_drift / std::fabs(diag);
  const int dmin = (int)std::floor(-nmax);
  const int dmax = (int)std::floor(nmax);
  const int window_size = (int)(2 * std::ceil(nmax * drift_timesteps));
  if (!(window_size >= 1) || dmax < dmin)
    return fail(SC_DD_EINVAL, "sc_dd_search: max_drift gives no drift range (window size < 1)");
  if ((long long)(dmax - dmin + 1) * Tr > (1ll << 30))
    return fail(SC_DD_EINVAL, "sc_dd_search: drift range too large");

  cudaError_t e;
  if ((e = cudaEventRecord(dd->ev[0], stream)) != cudaSuccess) return cuda_fail(e, "sc_dd_search: event");
  if ((e = cudaMemsetAsync(dd->top, 0, sizeof(float) * N, stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(dd->result, 0, sizeof(scb::SearchHeader), stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search: memset");
  if ((e = scb::search_stats(dev_input, row_stride, Tr, N, dd->colsum, dd->sel, dd->partials,
                             dd->n_partials, dd->var_scratch, snr_threshold, dd->hdr(), dd->num_sms,
                             stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search: statistics kernels");
  cudaEventRecord(dd->ev[1], stream);
  if (Tr <= 16) {
    scb::TreeParams tp{};
    tp.rows = dev_input;
    tp.row_stride = row_stride;
    tp.job_row_stride = 0;
    tp.N = N;
    tp.d_first = dmin;
    tp.d_step = 1;
    tp.n_jobs = dmax - dmin + 1;
    tp.db_first = dmin;
    tp.db_step = 1;
    tp.off_base = 0;
    tp.off_step = 0;
    tp.elig_T1 = Tr - 1;
    tp.top = dd->top;
    e = scb::tree_max(tp, Tr, dd->num_sms, stream);
  } else {
    e = scb::levels_search(dev_input, row_stride, Tr, N, dmin, dmax, dd->scratch_a, dd->scratch_b, dd->top,
                           dd->num_sms, stream);
  }
  if (e != cudaSuccess) return cuda_fail(e, "sc_dd_search: tree kernels");
  cudaEventRecord(dd->ev[2], stream);
  if ((e = scb::search_hits(dev_input, row_stride, Tr, N, dd->top, window_size, dmin, dmax, dd->hdr(),
                            dd->cands(), dd->cand_cap, dd->num_sms, stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search: hit kernels");
  cudaEventRecord(dd->ev[3], stream);
  const int head_cands = std::min(kHostCands, dd->cand_cap);
  const size_t head = sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * head_cands;
  if ((e = cudaMemcpyAsync(dd->host_result, dd->result, head, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search: result copy");
  const scb::SearchHeader h = *static_cast<scb::SearchHeader*>(dd->host_result);
  if (h.error) return fail(SC_DD_EINTERNAL, "sc_dd_search: drift recovery did not reproduce a top sum");
  const int ncand = std::min(h.num_candidates, dd->cand_cap);
  std::vector<scb::Candidate> cands(ncand);
  const scb::Candidate* hc = reinterpret_cast<const scb::Candidate*>(
      static_cast<const char*>(dd->host_result) + sizeof(scb::SearchHeader));
  std::copy(hc, hc + std::min(ncand, head_cands), cands.begin());
  if (ncand > head_cands) {
    if ((e = cudaMemcpyAsync(cands.data() + head_cands, dd->cands() + head_cands,
                             sizeof(scb::Candidate) * (ncand - head_cands), cudaMemcpyDeviceToHost,
                             stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
      return cuda_fail(e, "sc_dd_search: candidate copy");
  }
  std::sort(cands.begin(), cands.end(),
            [](const scb::Candidate& a, const scb::Candidate& b) { return a.index < b.index; });

  dd->last.median = h.median;
  dd->last.std_dev = h.std_dev;
  dd->last.mean = h.mean;
  dd->last.threshold = h.threshold;
  dd->last.window_size = window_size;
  dd->last.min_drift_block = dmin;
  dd->last.max_drift_block = dmax;
  dd->last.num_candidates = ncand;
  cudaEventElapsedTime(&dd->last.tree_ms, dd->ev[1], dd->ev[2]);
  cudaEventElapsedTime(&dd->last.search_ms, dd->ev[0], dd->ev[3]);
  dd->have_last = true;

  int n = 0;
  for (const scb::Candidate& c : cands) {
    // dedoppler.cu:385-396
    const int drift_bins = c.drift_steps;
    const double drift_rate = drift_bins * res;
    const float snr = (c.power - h.median) / h.std_dev;
    if (std::fabs(drift_rate) >= min_drift) {
      if (n < capacity) {
        sc_dd_hit& o = out[n];
        o.index = c.index;
        o.drift_steps = drift_bins;
        o.drift_rate = drift_rate;
        o.snr = snr;
        o.power = c.power;
        o.incoherent_power = 0.0f;
        o.coarse_channel = coarse_channel;
        o.beam = beam;
        o.num_timesteps = dd->T;
      }
      ++n;
    }
  }
  *num_hits = n;
  if (n > capacity) return fail(SC_DD_ETRUNC, "sc_dd_search: more hits than capacity");
  return SC_DD_OK;
}

int sc_dd_add_incoherent_power(sc_dd* dd, const float* dev_input, long long row_stride,
                               sc_dd_hit* hits, int num_hits, void* stream_ptr) {
  g_last_error.clear();
  if (!dd || !dev_input || (num_hits > 0 && !hits)) return fail(SC_DD_EINVAL, "sc_dd_add_incoherent_power: null argument");
  if (row_stride < dd->N) return fail(SC_DD_ESHAPE, "sc_dd_add_incoherent_power: row_stride smaller than num_channels");
  if (num_hits <= 0) return SC_DD_OK;
  DeviceGuard guard(dd->device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  int rc = ensure_inc(dd, num_hits);
  if (rc != SC_DD_OK) return rc;
  std::vector<int> idx(num_hits), steps(num_hits);
  std::vector<float> vals(num_hits);
  for (int i = 0; i < num_hits; ++i) {
    idx[i] = hits[i].index;
    steps[i] = hits[i].drift_steps;
  }
  cudaError_t e;
  if ((e = cudaMemcpyAsync(dd->inc_index, idx.data(), sizeof(int) * num_hits, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(dd->inc_steps, steps.data(), sizeof(int) * num_hits, cudaMemcpyHostToDevice, stream)) != cudaSuccess ||
      (e = scb::path_values(dev_input, row_stride, dd->Tr, dd->N, dd->inc_index, dd->inc_steps, dd->inc_vals,
                            num_hits, stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(vals.data(), dd->inc_vals, sizeof(float) * num_hits, cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_add_incoherent_power");
  for (int i = 0; i < num_hits; ++i) hits[i].incoherent_power = vals[i];
  return SC_DD_OK;
}

int sc_dd_last_stats(const sc_dd* dd, sc_dd_stats* out) {
  if (!dd || !out) return fail(SC_DD_EINVAL, "sc_dd_last_stats: null argument");
  if (!dd->have_last) return fail(SC_DD_EINVAL, "sc_dd_last_stats: no search has completed");
  *out = dd->last;
  return SC_DD_OK;
}

int sc_dd_copy_channel_array(sc_dd* dd, int which, float* dst, void* stream_ptr) {
  if (!dd || !dst || (which != 0 && which != 1)) return fail(SC_DD_EINVAL, "sc_dd_copy_channel_array: bad argument");
  DeviceGuard guard(dd->device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const float* src = which == 0 ? dd->top : dd->colsum;
  cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(float) * dd->N, cudaMemcpyDefault, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "sc_dd_copy_channel_array");
  return SC_DD_OK;
}

}  // extern "C"
