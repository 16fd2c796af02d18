// sc_dd_search_static: the dedoppler search without any allocation.
//
// Some callers cannot allocate device memory at the point where they search: a real-time
// capture or beamforming pipeline that reserved the GPU's memory up front and must not
// call cudaMalloc (which can synchronise the device) inside its processing loop, or a
// host framework whose allocator owns all device memory.  This entry point serves them.
// It runs the same kernels as sc_dd_search, but its scratch (top path sums, column sums,
// order-statistic state, variance partials, the exact statistics' work array and pair
// lists, and the candidate block) lives in the
// fixed-size device array below instead of an engine's cudaMalloc'd buffers, and its
// host side allocates nothing either: the statistics and candidates come back through a
// small stack buffer, and the hits are written straight into the caller's array.
//
// Limits: at most kStaticMaxChannels channels, at most 16 rounded timesteps, and at most
// kStaticMaxCands windows per search.  The array is shared by every call on a device and
// keeps the last call's contents; each call clears what must start at zero.  Calls that
// overlap on the GPU (different streams, or different host threads) race on it.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <mutex>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace {

constexpr int kStaticMaxChannels = SC_DD_STATIC_MAX_CHANNELS;
constexpr int kStaticMaxCands = 65536;
constexpr int kStaticPartials = 1024;
constexpr int kMaxDevices = 64;
constexpr int kHostChunk = 256;

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Byte offsets of each scratch region inside the static array.
constexpr size_t kOffTop = 0;
constexpr size_t kOffColsum = kOffTop + align256(sizeof(float) * kStaticMaxChannels);
constexpr size_t kOffSelect = kOffColsum + align256(sizeof(float) * kStaticMaxChannels);
constexpr size_t kOffPartials = kOffSelect + align256(sizeof(scb::SelectState));
constexpr size_t kOffVar = kOffPartials + align256(sizeof(scb::MomentPartial) * kStaticPartials);
constexpr size_t kOffWork = kOffVar + align256(sizeof(double) * 2 * scb::kVarChunks);
constexpr size_t kOffLists = kOffWork + align256(sizeof(float) * scb::order_work_floats(kStaticMaxChannels));
constexpr size_t kOffResult = kOffLists + align256(sizeof(int) * scb::order_list_entries(kStaticMaxChannels));
constexpr size_t kScratchBytes =
    kOffResult + align256(sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * kStaticMaxCands);

// The scratch.  Every GPU that loads this library holds these bytes until the process
// exits.  Host code must not use this name as an address (it is a host-side stand-in);
// it uses the device address looked up with cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_dd_static_scratch[kScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[kMaxDevices] = {};
int g_num_sms[kMaxDevices] = {};

// Failures are reported by status code only: this path keeps no message string, since
// building one could allocate.  The message argument documents the cause in the source.
int fail(int code, const char* /*message*/) { return code; }
int cuda_fail(cudaError_t /*e*/, const char* /*what*/) { return SC_DD_ECUDA; }

// Once per device, with that device current: the array's device address and SM count.
int setup_device(int dev, void** addr, int* num_sms) {
  if (dev < 0 || dev >= kMaxDevices) return fail(SC_DD_EINVAL, "sc_dd_search_static: device ordinal too large");
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_dd_static_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "sc_dd_search_static: cudaGetSymbolAddress");
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "sc_dd_search_static: cudaDeviceGetAttribute");
    g_num_sms[dev] = sms;
    g_scratch_addr[dev] = p;
  }
  *addr = g_scratch_addr[dev];
  *num_sms = g_num_sms[dev];
  return SC_DD_OK;
}

}  // namespace

extern "C" {

int sc_dd_search_static(const float* dev_input, long long row_stride, int num_timesteps, int num_channels,
                        double foff_mhz, double tsamp_s, int beam, int coarse_channel, double max_drift,
                        double min_drift, double snr_threshold, sc_dd_hit* out, int capacity, int* num_hits,
                        void* stream_ptr) {
  if (!dev_input || !num_hits || (capacity > 0 && !out)) return fail(SC_DD_EINVAL, "sc_dd_search_static: null argument");
  if (num_timesteps < 2) return fail(SC_DD_EINVAL, "sc_dd_search_static: num_timesteps must be > 1");
  int Tr = 1;
  while (Tr < num_timesteps) Tr *= 2;
  if (Tr > 16) return fail(SC_DD_ELIMIT, "sc_dd_search_static: at most 16 rounded timesteps");
  if (num_channels > kStaticMaxChannels)
    return fail(SC_DD_ELIMIT, "sc_dd_search_static: more than SC_DD_STATIC_MAX_CHANNELS channels");
  if (num_channels < 64) return fail(SC_DD_EINVAL, "sc_dd_search_static: num_channels must be >= 64");
  if (row_stride < num_channels) return fail(SC_DD_ESHAPE, "sc_dd_search_static: row_stride smaller than num_channels");
  if (!(tsamp_s > 0) || !(foff_mhz != 0) || !std::isfinite(foff_mhz))
    return fail(SC_DD_EINVAL, "sc_dd_search_static: foff must be nonzero and tsamp positive");
  const int N = num_channels;

  // dedoppler.cu:84-87, 194-198, 274: the same double arithmetic as sc_dd_search.
  const int drift_timesteps = Tr - 1;
  const double res = 1e6 * foff_mhz / (drift_timesteps * tsamp_s);
  const double nmax = max_drift / std::fabs(res * drift_timesteps);
  // The same bound on the drift range as sc_dd_search, checked before any int conversion.
  if (!std::isfinite(max_drift) || !std::isfinite(nmax) || nmax * drift_timesteps > (double)(1 << 30))
    return fail(SC_DD_EINVAL, "sc_dd_search_static: max_drift is not finite or too large");
  const int dmin = (int)std::floor(-nmax);
  const int dmax = (int)std::floor(nmax);
  const int window_size = (int)(2 * std::ceil(nmax * drift_timesteps));
  if (!(window_size >= 1) || dmax < dmin)
    return fail(SC_DD_EINVAL, "sc_dd_search_static: max_drift gives no drift range (window size < 1)");
  if ((long long)(dmax - dmin + 1) * Tr > (1ll << 30))
    return fail(SC_DD_EINVAL, "sc_dd_search_static: drift range too large");
  if ((long long)(N + window_size - 1) / window_size > kStaticMaxCands)
    return fail(SC_DD_ELIMIT, "sc_dd_search_static: more than 65536 windows; use sc_dd_search");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "sc_dd_search_static: cudaGetDevice");
  void* base = nullptr;
  int num_sms = 0;
  int rc = setup_device(dev, &base, &num_sms);
  if (rc != SC_DD_OK) return rc;
  char* b = static_cast<char*>(base);
  float* top = reinterpret_cast<float*>(b + kOffTop);
  float* colsum = reinterpret_cast<float*>(b + kOffColsum);
  scb::SelectState* sel = reinterpret_cast<scb::SelectState*>(b + kOffSelect);
  scb::MomentPartial* partials = reinterpret_cast<scb::MomentPartial*>(b + kOffPartials);
  double* var = reinterpret_cast<double*>(b + kOffVar);
  float* work = reinterpret_cast<float*>(b + kOffWork);
  int* lists = reinterpret_cast<int*>(b + kOffLists);
  scb::SearchHeader* hdr = reinterpret_cast<scb::SearchHeader*>(b + kOffResult);
  scb::Candidate* cands = reinterpret_cast<scb::Candidate*>(b + kOffResult + sizeof(scb::SearchHeader));
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);

  // Clear what must start at zero; the order-statistic state is reset by the first kernel.
  if ((e = cudaMemsetAsync(top, 0, sizeof(float) * N, stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(hdr, 0, sizeof(scb::SearchHeader), stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search_static: memset");
  // One-search batches; the descriptors travel as kernel parameters (no device copy).
  // (About 15 KB of descriptors on the stack.)
  scb::SearchBatch batch;
  batch.count = 1;
  batch.maxN = N;
  scb::SearchDesc& sd = batch.s[0];
  sd = scb::SearchDesc{};
  sd.input = dev_input;
  sd.row_stride = row_stride;
  sd.Tr = Tr;
  sd.N = N;
  sd.dmin = dmin;
  sd.dmax = dmax;
  sd.window_size = window_size;
  sd.first = (int)std::ceil(0.05 * N);
  sd.mid = N / 2;
  sd.last = (int)std::floor(0.95 * N);
  sd.snr_threshold = snr_threshold;
  sd.top = top;
  sd.colsum = colsum;
  sd.sel = sel;
  sd.partials = partials;
  sd.var = var;
  sd.work = work;
  sd.lists = lists;
  sd.hdr = hdr;
  sd.cands = cands;
  sd.cand_cap = kStaticMaxCands;
  if (kStaticPartials < 2 * num_sms) return fail(SC_DD_EINTERNAL, "sc_dd_search_static: too many SMs for the partials");
  if ((e = scb::column_sums_batch(batch, stream)) != cudaSuccess ||
      (e = scb::search_stats_batch(batch, num_sms, stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search_static: statistics kernels");
  scb::TreeBatch tb;
  tb.count = 1;
  tb.n_items = 0;
  scb::TreeGroup& tp = tb.g[0];
  tp = scb::TreeGroup{};
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
  tp.top = top;
  tp.status = &hdr->error;  // an address inside the device array, not a host read
  if ((e = scb::tree_max_batch(tb, Tr, num_sms, stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search_static: tree kernel");
  if ((e = scb::search_hits_batch(batch, num_sms, stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search_static: hit kernels");

  // Results through a stack buffer: the header, then the candidates in chunks.
  scb::SearchHeader h;
  if ((e = cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(stream)) != cudaSuccess)
    return cuda_fail(e, "sc_dd_search_static: result copy");
  if (h.error) return fail(SC_DD_EINTERNAL, "sc_dd_search_static: a tree kernel gave up a wait");
  const int ncand = std::min(h.num_candidates, kStaticMaxCands);
  scb::Candidate chunk[kHostChunk];
  int n = 0;
  for (int c0 = 0; c0 < ncand; c0 += kHostChunk) {
    const int k = std::min(kHostChunk, ncand - c0);
    if ((e = cudaMemcpyAsync(chunk, cands + c0, sizeof(scb::Candidate) * k, cudaMemcpyDeviceToHost, stream)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
      return cuda_fail(e, "sc_dd_search_static: candidate copy");
    for (int i = 0; i < k; ++i) {
      const scb::Candidate& c = chunk[i];
      int drift_steps = 0;
      if (!scb::decode_candidate(c, dmin, Tr, &drift_steps))
        return fail(SC_DD_EINTERNAL, "sc_dd_search_static: drift recovery did not reproduce a top sum");
      const double drift_rate = drift_steps * res;  // dedoppler.cu:305-317
      const float snr = (c.power - h.median) / h.std_dev;
      if (std::fabs(drift_rate) >= min_drift) {
        if (n < capacity) {
          sc_dd_hit& o = out[n];
          o.index = c.index;
          o.drift_steps = drift_steps;
          o.drift_rate = drift_rate;
          o.snr = snr;
          o.power = c.power;
          o.incoherent_power = 0.0f;
          o.coarse_channel = coarse_channel;
          o.beam = beam;
          o.num_timesteps = num_timesteps;
        }
        ++n;
      }
    }
  }
  // Increasing index order, as sc_dd_search returns them (sorting in place allocates nothing).
  std::sort(out, out + std::min(n, capacity), [](const sc_dd_hit& a, const sc_dd_hit& x) { return a.index < x.index; });
  *num_hits = n;
  if (n > capacity) return fail(SC_DD_ETRUNC, "sc_dd_search_static: more hits than capacity");
  return SC_DD_OK;
}

}  // extern "C"
