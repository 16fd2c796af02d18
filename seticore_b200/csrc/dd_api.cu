// C ABI of the B200 dedoppler search (declared in include/seticore_b200.h).
//
// sc_dd mirrors the reference's Dedopplerer (dedoppler.h:15-79): it is built for one
// (timesteps, channels, foff, tsamp) shape and owns every scratch buffer, reused across
// searches (dedoppler.cu:76-111).  It keeps one scratch "slot" per search of the largest
// batch it has run.  A call queues, on the caller's stream, for up to kMaxBatch searches
// at a time, through exec_queue (dd_exec.cu):
//   clear -> fused tree/top kernel over every search's work items, which also forms the
//   column sums (dd_tree.cu; for Tr > 32 the level path of dd_levels.cu, one search at a
//   time) -> order statistics + variance (dd_stats.cu) -> window de-duplication + drift
//   recovery (dd_hits.cu)
// then copies the headers and the first candidates of every search to pinned host memory
// in two copies and synchronises once.  Only hit lists cross to the host, not the
// reference's four N-length arrays per search.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <unordered_map>
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

}  // namespace

namespace scb {
// Sets the calling thread's sc_dd_last_error message (for the other ABI translation units).
int api_fail(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace scb

namespace {

constexpr int kHostCands = 256;  // candidates per search fetched with the headers

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

// The drift range and window of a search (dedoppler.cu:84-87, 194-198, 274).
struct DriftPlan {
  double res;
  int dmin, dmax, window_size;
};

DriftPlan plan_drift(int Tr, double foff, double tsamp, double max_drift) {
  DriftPlan p;
  const int drift_timesteps = Tr - 1;
  p.res = 1e6 * foff / (drift_timesteps * tsamp);
  const double diag = p.res * drift_timesteps;
  const double nmax = max_drift / std::fabs(diag);
  p.dmin = (int)std::floor(-nmax);
  p.dmax = (int)std::floor(nmax);
  p.window_size = (int)(2 * std::ceil(nmax * drift_timesteps));
  return p;
}

}  // namespace

struct sc_dd {
  int T = 0, Tr = 0, N = 0;
  double foff = 0, tsamp = 0;
  int has_dc_spike = 0;
  int device = 0, num_sms = 148;
  int n_partials = 0;
  // Per-slot scratch, slot k at offset k * (per-slot size) in each array.
  int slots = 0;
  int cand_cap = 0;  // candidates per slot
  float* top = nullptr;
  float* colsum = nullptr;
  scb::SelectState* sel = nullptr;
  scb::MomentPartial* partials = nullptr;
  double* var = nullptr;
  float* work = nullptr;  // [slot][order_work_floats(N)] column sums in nth_element order
  int* lists = nullptr;   // [slot][order_list_entries(N)] partition pairs
  scb::SearchHeader* hdrs = nullptr;
  scb::Candidate* cands = nullptr;
  float* scratch_a = nullptr;  // Tr > 32 level buffers (one search at a time), one allocation
  float* scratch_b = nullptr;  // = scratch_a + level_buffer_floats(Tr, N)
  // The side streams' pairs (scratch_a + 2 + 2i and 3 + 2i level_buffer_floats, the same
  // allocation) with their streams and events: a batch deals its level searches over them.
  scb::LevelSide side;
  int level_pairs = 1;  // pairs of level buffers in scratch_a
  void* host = nullptr;  // pinned: slots * (header + kHostCands candidates)
  int* inc_index = nullptr;
  int* inc_steps = nullptr;
  float* inc_vals = nullptr;
  int inc_cap = 0;
  // Precision form (16-bit normalised storage), per slot.
  int precision = SC_DD_PRECISION_FP32;
  int prec_slots = 0;
  void* norm16 = nullptr;        // [slot] normalised copies of norm_buffer_bytes(Tr, N)
  float* top16 = nullptr;        // [slot][N]
  int* flags = nullptr;          // [slot][N] flagged channels
  int* flag_counts = nullptr;    // [slot]
  double* norm_moments = nullptr;  // [slot][kNormMomentsDoubles]
  unsigned* norm_tickets = nullptr;  // [slot]
  int* host_flag_counts = nullptr;   // pinned [slot]
  double* host_norm = nullptr;       // pinned [2]: mean, std of search 0
  size_t device_bytes = 0;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // call start, tree start/end, call end
  sc_dd_stats last{};
  bool have_last = false;
  // CUDA graphs of repeated batches (same inputs, drift plan, threshold, form and settings):
  // captured on the second sight, replayed afterwards.  Any reallocation of the scratch bumps
  // `generation`, which is part of the key, and drops the graphs.
  struct Graph {
    uint64_t key;
    cudaGraphExec_t exec;
    unsigned long long last_use;
  };
  std::vector<Graph> graphs;
  std::unordered_map<uint64_t, int> seen;  // sightings per key; -1: not capturable
  unsigned long long clock = 0;
  unsigned generation = 0;
  cudaStream_t cap_stream = nullptr;
  cudaEvent_t evj = nullptr;

  scb::SearchHeader* host_hdrs() { return static_cast<scb::SearchHeader*>(host); }
  scb::Candidate* host_cands() {
    return reinterpret_cast<scb::Candidate*>(static_cast<char*>(host) + sizeof(scb::SearchHeader) * slots);
  }
};

namespace {

template <typename T>
cudaError_t dalloc(sc_dd* d, T** p, size_t bytes) {
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), bytes);
  if (e == cudaSuccess) d->device_bytes += bytes;
  return e;
}

template <typename T>
void dfree(sc_dd* d, T** p, size_t bytes) {
  if (*p) {
    cudaFree(*p);
    d->device_bytes -= bytes;
    *p = nullptr;
  }
}

void drop_graphs(sc_dd* d) {
  for (auto& g : d->graphs) cudaGraphExecDestroy(g.exec);
  d->graphs.clear();
  d->seen.clear();
  ++d->generation;
}

void free_slots(sc_dd* d) {
  const size_t N = d->N, S = d->slots;
  dfree(d, &d->top, sizeof(float) * N * S);
  dfree(d, &d->colsum, sizeof(float) * N * S);
  dfree(d, &d->sel, sizeof(scb::SelectState) * S);
  dfree(d, &d->partials, sizeof(scb::MomentPartial) * d->n_partials * S);
  dfree(d, &d->var, sizeof(double) * 2 * scb::kVarChunks * S);
  dfree(d, &d->work, sizeof(float) * scb::order_work_floats(d->N) * S);
  dfree(d, &d->lists, sizeof(int) * scb::order_list_entries(d->N) * S);
  dfree(d, &d->hdrs, sizeof(scb::SearchHeader) * S);
  dfree(d, &d->cands, sizeof(scb::Candidate) * d->cand_cap * S);
  if (d->host) cudaFreeHost(d->host);
  d->host = nullptr;
  d->slots = 0;
}

void free_prec(sc_dd* d) {
  const size_t S = d->prec_slots, N = d->N;
  dfree(d, &d->norm16, scb::norm_buffer_bytes(d->Tr, (int)N) * S);
  dfree(d, &d->top16, sizeof(float) * N * S);
  dfree(d, &d->flags, sizeof(int) * N * S);
  dfree(d, &d->flag_counts, sizeof(int) * S);
  dfree(d, &d->norm_moments, sizeof(double) * scb::kNormMomentsDoubles * S);
  dfree(d, &d->norm_tickets, sizeof(unsigned) * S);
  if (d->host_flag_counts) cudaFreeHost(d->host_flag_counts);
  if (d->host_norm) cudaFreeHost(d->host_norm);
  d->host_flag_counts = nullptr;
  d->host_norm = nullptr;
  d->prec_slots = 0;
}

int ensure_prec(sc_dd* d, int slots) {
  if (slots <= d->prec_slots) return SC_DD_OK;
  cudaDeviceSynchronize();
  drop_graphs(d);
  free_prec(d);
  const size_t S = slots, N = d->N;
  cudaError_t e;
  if ((e = dalloc(d, &d->norm16, scb::norm_buffer_bytes(d->Tr, (int)N) * S)) != cudaSuccess ||
      (e = dalloc(d, &d->top16, sizeof(float) * N * S)) != cudaSuccess ||
      (e = dalloc(d, &d->flags, sizeof(int) * N * S)) != cudaSuccess ||
      (e = dalloc(d, &d->flag_counts, sizeof(int) * S)) != cudaSuccess ||
      (e = dalloc(d, &d->norm_moments, sizeof(double) * scb::kNormMomentsDoubles * S)) != cudaSuccess ||
      (e = dalloc(d, &d->norm_tickets, sizeof(unsigned) * S)) != cudaSuccess ||
      (e = cudaMallocHost(&d->host_flag_counts, sizeof(int) * S)) != cudaSuccess ||
      (e = cudaMallocHost(&d->host_norm, sizeof(double) * 2)) != cudaSuccess) {
    d->prec_slots = slots;
    free_prec(d);
    return fail(e == cudaErrorMemoryAllocation ? SC_DD_ENOMEM : SC_DD_ECUDA,
                std::string("precision scratch allocation failed: ") + cudaGetErrorString(e));
  }
  d->prec_slots = slots;
  if ((e = cudaMemset(d->norm_tickets, 0, sizeof(unsigned) * S)) != cudaSuccess) return cuda_fail(e, "memset");
  return SC_DD_OK;
}

void free_all(sc_dd* d) {
  drop_graphs(d);
  if (d->cap_stream) cudaStreamDestroy(d->cap_stream);
  if (d->evj) cudaEventDestroy(d->evj);
  d->cap_stream = nullptr;
  d->evj = nullptr;
  free_slots(d);
  free_prec(d);
  d->scratch_b = nullptr;  // inside scratch_a's allocation
  dfree(d, &d->scratch_a, 2 * (size_t)d->level_pairs * sizeof(float) * scb::level_buffer_floats(d->Tr, d->N));
  for (int i = 0; i < scb::kLevelSides; ++i) {
    if (d->side.stream[i]) cudaStreamDestroy(d->side.stream[i]);
    if (d->side.join[i]) cudaEventDestroy(d->side.join[i]);
  }
  if (d->side.fork) cudaEventDestroy(d->side.fork);
  d->side = scb::LevelSide{};
  dfree(d, &d->inc_index, sizeof(int) * d->inc_cap);
  dfree(d, &d->inc_steps, sizeof(int) * d->inc_cap);
  dfree(d, &d->inc_vals, sizeof(float) * d->inc_cap);
  for (cudaEvent_t& e : d->ev)
    if (e) cudaEventDestroy(e);
}

// Makes room for `slots` searches with `cand_cap` candidates each (never shrinks).
int ensure_slots(sc_dd* d, int slots, int cand_cap) {
  if (slots <= d->slots && cand_cap <= d->cand_cap) return SC_DD_OK;
  const int ns = std::max(slots, d->slots);
  const int nc = std::max(cand_cap, d->cand_cap);
  cudaDeviceSynchronize();  // the old slots may still be in use by queued work
  drop_graphs(d);
  free_slots(d);
  d->cand_cap = nc;
  const size_t N = d->N, S = ns;
  cudaError_t e;
  if ((e = dalloc(d, &d->top, sizeof(float) * N * S)) != cudaSuccess ||
      (e = dalloc(d, &d->colsum, sizeof(float) * N * S)) != cudaSuccess ||
      (e = dalloc(d, &d->sel, sizeof(scb::SelectState) * S)) != cudaSuccess ||
      (e = dalloc(d, &d->partials, sizeof(scb::MomentPartial) * d->n_partials * S)) != cudaSuccess ||
      (e = dalloc(d, &d->var, sizeof(double) * 2 * scb::kVarChunks * S)) != cudaSuccess ||
      (e = dalloc(d, &d->work, sizeof(float) * scb::order_work_floats(d->N) * S)) != cudaSuccess ||
      (e = dalloc(d, &d->lists, sizeof(int) * scb::order_list_entries(d->N) * S)) != cudaSuccess ||
      (e = dalloc(d, &d->hdrs, sizeof(scb::SearchHeader) * S)) != cudaSuccess ||
      (e = dalloc(d, &d->cands, sizeof(scb::Candidate) * (size_t)nc * S)) != cudaSuccess ||
      (e = cudaMallocHost(&d->host, (sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * kHostCands) * S)) !=
          cudaSuccess) {
    d->slots = ns;
    free_slots(d);
    return fail(e == cudaErrorMemoryAllocation ? SC_DD_ENOMEM : SC_DD_ECUDA,
                std::string("scratch allocation failed: ") + cudaGetErrorString(e));
  }
  d->slots = ns;
  if ((e = cudaMemset(d->sel, 0, sizeof(scb::SelectState) * S)) != cudaSuccess) return cuda_fail(e, "scratch memset");
  return SC_DD_OK;
}

int ensure_inc(sc_dd* d, int n) {
  if (n <= d->inc_cap) return SC_DD_OK;
  dfree(d, &d->inc_index, sizeof(int) * d->inc_cap);
  dfree(d, &d->inc_steps, sizeof(int) * d->inc_cap);
  dfree(d, &d->inc_vals, sizeof(float) * d->inc_cap);
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

// Queues n <= kMaxBatch searches into slots 0..n-1.
struct EventHooks {
  sc_dd* dd;
  bool record;
};

int queue_batch(sc_dd* dd, int n, const float* const* inputs, const long long* strides, const DriftPlan& p,
                double snr_threshold, cudaStream_t stream, bool first_batch) {
  scb::ExecSearch es[scb::kMaxBatch];
  const bool prec = dd->precision != SC_DD_PRECISION_FP32;
  const int elem = !prec ? scb::kElemF32
                         : (dd->precision == SC_DD_PRECISION_BF16 ? scb::kElemBF16 : scb::kElemF16);
  for (int k = 0; k < n; ++k) {
    scb::ExecSearch& q = es[k];
    q = scb::ExecSearch{};
    q.input = inputs[k];
    q.row_stride = strides[k];
    q.T = dd->T;
    q.Tr = dd->Tr;
    q.N = dd->N;
    q.dmin = p.dmin;
    q.dmax = p.dmax;
    q.window_size = p.window_size;
    q.snr_threshold = snr_threshold;
    q.elem = elem;
    q.cand_cap = dd->cand_cap;
    const size_t N = dd->N;
    q.top = dd->top + N * k;
    q.colsum = dd->colsum + N * k;
    q.sel = dd->sel + k;
    q.partials = dd->partials + (size_t)dd->n_partials * k;
    q.var = dd->var + (size_t)2 * scb::kVarChunks * k;
    q.work = dd->work + scb::order_work_floats(dd->N) * k;
    q.lists = dd->lists + scb::order_list_entries(dd->N) * k;
    q.hdr = dd->hdrs + k;
    q.cands = dd->cands + (size_t)dd->cand_cap * k;
    if (prec) {
      q.norm16 = static_cast<char*>(dd->norm16) + scb::norm_buffer_bytes(dd->Tr, dd->N) * k;
      q.top16 = dd->top16 + N * k;
      q.flags = dd->flags + N * k;
      q.flag_count = dd->flag_counts + k;
      q.norm_moments = dd->norm_moments + (size_t)scb::kNormMomentsDoubles * k;
      q.norm_ticket = dd->norm_tickets + k;
    }
  }
  EventHooks eh{dd, first_batch};
  scb::ExecHooks hooks;
  hooks.ctx = &eh;
  // External event-record nodes when captured into a graph, so that the tree's time stays
  // measurable from the host on every replay.
  hooks.before_tree = [](void* c, cudaStream_t st) {
    EventHooks* h = static_cast<EventHooks*>(c);
    if (h->record && cudaEventRecordWithFlags(h->dd->ev[1], st, cudaEventRecordExternal) != cudaSuccess)
      cudaGetLastError();
  };
  hooks.after_tree = [](void* c, cudaStream_t st) {
    EventHooks* h = static_cast<EventHooks*>(c);
    if (h->record && cudaEventRecordWithFlags(h->dd->ev[2], st, cudaEventRecordExternal) != cudaSuccess)
      cudaGetLastError();
  };
  cudaError_t e = scb::exec_queue(es, n, dd->scratch_a, dd->scratch_b, dd->num_sms, stream, hooks,
                                  dd->side.n > 0 ? &dd->side : nullptr);
  if (e != cudaSuccess) return cuda_fail(e, "search kernels");
  return SC_DD_OK;
}

uint64_t fnv_mix(uint64_t h, const void* p, size_t n) {
  const unsigned char* c = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
  return h;
}

constexpr int kEngineGraphs = 8;

// queue_batch through a CUDA graph when the same batch was queued before: the key covers the
// inputs and strides, the drift plan, the threshold, the storage form, the process-wide
// settings that change the launches, and the scratch generation.  Second sight: capture on
// the engine's capture stream (ordered after `stream`) and launch; later: replay.  A batch
// whose capture fails is queued directly from then on.
int queue_batch_graphed(sc_dd* dd, int n, const float* const* inputs, const long long* strides, const DriftPlan& p,
                        double snr_threshold, cudaStream_t stream, bool first_batch) {
  uint64_t key = 1469598103934665603ull;
  key = fnv_mix(key, &n, sizeof(n));
  key = fnv_mix(key, inputs, sizeof(*inputs) * n);
  key = fnv_mix(key, strides, sizeof(*strides) * n);
  const int v[9] = {p.dmin, p.dmax, p.window_size, dd->precision, first_batch ? 1 : 0,
                    scb::exact_statistics_always() ? 1 : 0, scb::stage_wait_tries(), (int)dd->generation,
                    scb::paired_fp16() ? 1 : 0};
  key = fnv_mix(key, v, sizeof(v));
  const long long stripe = scb::level_stripe_bytes();
  key = fnv_mix(key, &stripe, sizeof(stripe));
  key = fnv_mix(key, &snr_threshold, sizeof(snr_threshold));
  cudaError_t e;
  auto it = std::find_if(dd->graphs.begin(), dd->graphs.end(), [&](const sc_dd::Graph& g) { return g.key == key; });
  if (it != dd->graphs.end()) {
    it->last_use = ++dd->clock;
    if ((e = cudaGraphLaunch(it->exec, stream)) != cudaSuccess) return cuda_fail(e, "graph launch");
    return SC_DD_OK;
  }
  if (dd->seen.size() > 4096) dd->seen.clear();  // many different batches: forget old sightings
  int& seen = dd->seen[key];
  if (seen < 0 || ++seen < 2 || !dd->cap_stream) return queue_batch(dd, n, inputs, strides, p, snr_threshold, stream, first_batch);
  if ((e = cudaEventRecord(dd->evj, stream)) != cudaSuccess ||
      (e = cudaStreamWaitEvent(dd->cap_stream, dd->evj, 0)) != cudaSuccess)
    return cuda_fail(e, "capture ordering");
  if ((e = cudaStreamBeginCapture(dd->cap_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return cuda_fail(e, "begin capture");
  const int rc = queue_batch(dd, n, inputs, strides, p, snr_threshold, dd->cap_stream, first_batch);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(dd->cap_stream, &g);
  cudaGraphExec_t ex = nullptr;
  if (rc == SC_DD_OK && e == cudaSuccess) e = cudaGraphInstantiate(&ex, g, 0);
  if (g) cudaGraphDestroy(g);
  if (rc != SC_DD_OK || e != cudaSuccess || !ex) {
    // not capturable: run it directly, now and from now on
    cudaGetLastError();
    seen = -1;
    return queue_batch(dd, n, inputs, strides, p, snr_threshold, stream, first_batch);
  }
  if ((int)dd->graphs.size() >= kEngineGraphs) {
    auto lru = std::min_element(dd->graphs.begin(), dd->graphs.end(),
                                [](const sc_dd::Graph& a, const sc_dd::Graph& b) { return a.last_use < b.last_use; });
    cudaGraphExecDestroy(lru->exec);
    dd->graphs.erase(lru);
  }
  dd->graphs.push_back({key, ex, ++dd->clock});
  if ((e = cudaGraphLaunch(ex, stream)) != cudaSuccess) return cuda_fail(e, "graph launch");
  return SC_DD_OK;
}

// Runs `count` searches; hits of search k land in out[off_k ...], off_k = sum of earlier counts.
int run_searches(sc_dd* dd, int count, const float* const* inputs, const long long* strides, const int* beams,
                 const int* coarse, double max_drift, double min_drift, double snr_threshold, sc_dd_hit* out,
                 int capacity, int* num_hits, cudaStream_t stream) {
  const int Tr = dd->Tr, N = dd->N;
  const DriftPlan p = plan_drift(Tr, dd->foff, dd->tsamp, max_drift);
  if (!(p.window_size >= 1) || p.dmax < p.dmin)
    return fail(SC_DD_EINVAL, "max_drift gives no drift range (window size < 1)");
  if ((long long)(p.dmax - p.dmin + 1) * Tr > (1ll << 30)) return fail(SC_DD_EINVAL, "drift range too large");
  const long long nwin = ((long long)N + p.window_size - 1) / p.window_size;
  int rc = ensure_slots(dd, std::min(count, scb::kMaxBatch), (int)std::min<long long>(nwin + 1, N / 2 + 2));
  if (rc != SC_DD_OK) return rc;
  const bool prec = dd->precision != SC_DD_PRECISION_FP32;
  if (prec && (rc = ensure_prec(dd, std::min(count, scb::kMaxBatch))) != SC_DD_OK) return rc;
  cudaError_t e;
  if ((e = cudaEventRecord(dd->ev[0], stream)) != cudaSuccess) return cuda_fail(e, "event");
  int total = 0;
  long long d2h = 0;
  for (int k0 = 0; k0 < count; k0 += scb::kMaxBatch) {
    const int n = std::min(scb::kMaxBatch, count - k0);
    rc = queue_batch_graphed(dd, n, inputs + k0, strides + k0, p, snr_threshold, stream, k0 == 0);
    if (rc != SC_DD_OK) return rc;
    if (k0 == 0) cudaEventRecord(dd->ev[3], stream);
    // Headers of all n searches, then the first kHostCands candidates of each (strided copy).
    const int head = std::min(kHostCands, dd->cand_cap);
    if ((e = cudaMemcpyAsync(dd->host_hdrs(), dd->hdrs, sizeof(scb::SearchHeader) * n, cudaMemcpyDeviceToHost,
                             stream)) != cudaSuccess ||
        (e = cudaMemcpy2DAsync(dd->host_cands(), sizeof(scb::Candidate) * kHostCands, dd->cands,
                               sizeof(scb::Candidate) * dd->cand_cap, sizeof(scb::Candidate) * head, n,
                               cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
        (prec && (e = cudaMemcpyAsync(dd->host_flag_counts, dd->flag_counts, sizeof(int) * n, cudaMemcpyDeviceToHost,
                                      stream)) != cudaSuccess) ||
        (prec && k0 == 0 &&
         (e = cudaMemcpyAsync(dd->host_norm, dd->norm_moments + 2 * scb::kVarChunks, sizeof(double) * 2,
                              cudaMemcpyDeviceToHost, stream)) != cudaSuccess) ||
        (e = cudaStreamSynchronize(stream)) != cudaSuccess)
      return cuda_fail(e, "result copy");
    d2h += (long long)(sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * head) * n +
           (prec ? (long long)sizeof(int) * n + (k0 == 0 ? 2 * (long long)sizeof(double) : 0) : 0);
    for (int k = 0; k < n; ++k) {
      const scb::SearchHeader h = dd->host_hdrs()[k];
      if (h.error) return fail(SC_DD_EINTERNAL, "a tree kernel gave up waiting for its staged rows");
      const int ncand = std::min(h.num_candidates, dd->cand_cap);
      std::vector<scb::Candidate> cands(ncand);
      const scb::Candidate* hc = dd->host_cands() + (size_t)kHostCands * k;
      std::copy(hc, hc + std::min(ncand, head), cands.begin());
      if (ncand > head) {
        if ((e = cudaMemcpyAsync(cands.data() + head, dd->cands + (size_t)dd->cand_cap * k + head,
                                 sizeof(scb::Candidate) * (ncand - head), cudaMemcpyDeviceToHost, stream)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
          return cuda_fail(e, "candidate copy");
        d2h += (long long)sizeof(scb::Candidate) * (ncand - head);
      }
      std::sort(cands.begin(), cands.end(),
                [](const scb::Candidate& a, const scb::Candidate& b) { return a.index < b.index; });
      if (k0 + k == 0) {
        dd->last.median = h.median;
        dd->last.std_dev = h.std_dev;
        dd->last.mean = h.mean;
        dd->last.threshold = h.threshold;
        dd->last.window_size = p.window_size;
        dd->last.min_drift_block = p.dmin;
        dd->last.max_drift_block = p.dmax;
        dd->last.num_candidates = ncand;
        dd->last.precision = dd->precision;
        dd->last.total_channels = N;
        dd->last.recomputed_channels = prec ? dd->host_flag_counts[0] : N;
        dd->last.norm_mean = prec ? dd->host_norm[0] : 0.0;
        dd->last.norm_std = prec ? dd->host_norm[1] : 0.0;
        dd->last.order_exact = h.order_exact;
      }
      int nk = 0;
      for (const scb::Candidate& c : cands) {
        int drift_bins = 0;
        if (!scb::decode_candidate(c, p.dmin, Tr, &drift_bins))
          return fail(SC_DD_EINTERNAL, "drift recovery did not reproduce a top sum");
        // dedoppler.cu:305-317
        const double drift_rate = drift_bins * p.res;
        const float snr = (c.power - h.median) / h.std_dev;
        if (std::fabs(drift_rate) >= min_drift) {
          if (total < capacity) {
            sc_dd_hit& o = out[total];
            o.index = c.index;
            o.drift_steps = drift_bins;
            o.drift_rate = drift_rate;
            o.snr = snr;
            o.power = c.power;
            o.incoherent_power = 0.0f;
            o.coarse_channel = coarse[k0 + k];
            o.beam = beams[k0 + k];
            o.num_timesteps = dd->T;
          }
          ++total;
          ++nk;
        }
      }
      num_hits[k0 + k] = nk;
    }
  }
  dd->last.d2h_bytes = (int)std::min<long long>(d2h, INT_MAX);
  // Timing is informational: a failed query leaves -1 and no pending error behind.
  if (cudaEventElapsedTime(&dd->last.tree_ms, dd->ev[1], dd->ev[2]) != cudaSuccess) {
    dd->last.tree_ms = -1.0f;
    cudaGetLastError();
  }
  if (cudaEventElapsedTime(&dd->last.search_ms, dd->ev[0], dd->ev[3]) != cudaSuccess) {
    dd->last.search_ms = -1.0f;
    cudaGetLastError();
  }
  dd->have_last = true;
  if (total > capacity) return fail(SC_DD_ETRUNC, "more hits than capacity");
  return SC_DD_OK;
}

}  // namespace

extern "C" {

const char* sc_dd_last_error(void) { return g_last_error.c_str(); }

const char* sc_dd_version(void) { return "seticore-b200 0.2 (dedoppler; reference seticore 1.0.6)"; }

int sc_dd_set_stage_wait_limit(int tries) {
  scb::set_stage_wait_tries(tries);
  return SC_DD_OK;
}

int sc_dd_set_level_stripe_bytes(long long bytes) {
  scb::set_level_stripe_bytes(bytes);
  return SC_DD_OK;
}

int sc_dd_set_exact_statistics(int mode) {
  if (mode != 0 && mode != 1) return fail(SC_DD_EINVAL, "sc_dd_set_exact_statistics: mode must be 0 or 1");
  scb::set_exact_statistics_always(mode == 1);
  return SC_DD_OK;
}

int sc_dd_set_paired_fp16(int on) {
  if (on != 0 && on != 1) return fail(SC_DD_EINVAL, "sc_dd_set_paired_fp16: on must be 0 or 1");
  scb::set_paired_fp16(on == 1);
  return SC_DD_OK;
}

int sc_dd_create(int num_timesteps, int num_channels, double foff_mhz, double tsamp_s, int has_dc_spike,
                 sc_dd** out) {
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
  d->n_partials = 2 * d->num_sms;
  // One slot; candidates for windows of 16 channels or more (grown when a call needs more).
  int rc = ensure_slots(d, 1, std::min(num_channels / 2 + 2, num_channels / 16 + 2));
  if (rc == SC_DD_OK && d->Tr > 32) {
    // All pairs of level buffers in one allocation: the emitting level addresses a pair as
    // one array; pair 0 serves the main stream, pair 1 + i side stream i.
    const size_t L = scb::level_buffer_floats(d->Tr, num_channels);
    const int sides = scb::level_sides(true);
    d->level_pairs = 1 + sides;
    if ((e = dalloc(d, &d->scratch_a, 2 * (size_t)d->level_pairs * sizeof(float) * L)) != cudaSuccess) {
      d->level_pairs = 1;
      rc = fail(e == cudaErrorMemoryAllocation ? SC_DD_ENOMEM : SC_DD_ECUDA, "sc_dd_create: level buffers");
    } else {
      d->scratch_b = d->scratch_a + L;
      if (sides > 0 && (e = cudaEventCreateWithFlags(&d->side.fork, cudaEventDisableTiming)) != cudaSuccess)
        rc = cuda_fail(e, "sc_dd_create: level stream");
      for (int i = 0; i < sides && rc == SC_DD_OK; ++i) {
        d->side.lvl_a[i] = d->scratch_a + (2 + 2 * i) * L;
        d->side.lvl_b[i] = d->scratch_a + (3 + 2 * i) * L;
        if ((e = cudaStreamCreateWithFlags(&d->side.stream[i], cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&d->side.join[i], cudaEventDisableTiming)) != cudaSuccess)
          rc = cuda_fail(e, "sc_dd_create: level stream");
        else
          d->side.n = i + 1;
      }
    }
  }

  for (int i = 0; i < 4 && rc == SC_DD_OK; ++i)
    if ((e = cudaEventCreate(&d->ev[i])) != cudaSuccess) rc = cuda_fail(e, "sc_dd_create: event");
  if (rc == SC_DD_OK && ((e = cudaStreamCreateWithFlags(&d->cap_stream, cudaStreamNonBlocking)) != cudaSuccess ||
                         (e = cudaEventCreateWithFlags(&d->evj, cudaEventDisableTiming)) != cudaSuccess))
    rc = cuda_fail(e, "sc_dd_create: capture stream");
  if (rc != SC_DD_OK) {
    free_all(d);
    delete d;
    return rc;
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

int sc_dd_search(sc_dd* dd, const float* dev_input, long long row_stride, int beam, int coarse_channel,
                 double max_drift, double min_drift, double snr_threshold, sc_dd_hit* out, int capacity,
                 int* num_hits, void* stream) {
  g_last_error.clear();
  if (!dd || !dev_input || !num_hits || (capacity > 0 && !out)) return fail(SC_DD_EINVAL, "sc_dd_search: null argument");
  if (row_stride < dd->N) return fail(SC_DD_ESHAPE, "sc_dd_search: row_stride smaller than num_channels");
  DeviceGuard guard(dd->device);
  return run_searches(dd, 1, &dev_input, &row_stride, &beam, &coarse_channel, max_drift, min_drift, snr_threshold,
                      out, capacity, num_hits, static_cast<cudaStream_t>(stream));
}

int sc_dd_search_batch(sc_dd* dd, int count, const float* const* dev_inputs, const long long* row_strides,
                       const int* beams, const int* coarse_channels, double max_drift, double min_drift,
                       double snr_threshold, sc_dd_hit* out, int capacity, int* num_hits, void* stream) {
  g_last_error.clear();
  if (!dd || count < 0 || (count > 0 && (!dev_inputs || !row_strides || !beams || !coarse_channels || !num_hits)) ||
      (capacity > 0 && !out))
    return fail(SC_DD_EINVAL, "sc_dd_search_batch: null argument");
  for (int k = 0; k < count; ++k) {
    if (!dev_inputs[k]) return fail(SC_DD_EINVAL, "sc_dd_search_batch: null input");
    if (row_strides[k] < dd->N) return fail(SC_DD_ESHAPE, "sc_dd_search_batch: row_stride smaller than num_channels");
  }
  if (count == 0) return SC_DD_OK;
  DeviceGuard guard(dd->device);
  return run_searches(dd, count, dev_inputs, row_strides, beams, coarse_channels, max_drift, min_drift,
                      snr_threshold, out, capacity, num_hits, static_cast<cudaStream_t>(stream));
}

int sc_dd_add_incoherent_power(sc_dd* dd, const float* dev_input, long long row_stride, sc_dd_hit* hits,
                               int num_hits, void* stream_ptr) {
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

int sc_dd_set_precision(sc_dd* dd, int precision) {
  g_last_error.clear();
  if (!dd) return fail(SC_DD_EINVAL, "sc_dd_set_precision: null engine");
  if (precision != SC_DD_PRECISION_FP32 && precision != SC_DD_PRECISION_BF16 && precision != SC_DD_PRECISION_FP16)
    return fail(SC_DD_EINVAL, "sc_dd_set_precision: unknown precision");
  dd->precision = precision;
  return SC_DD_OK;
}

int sc_dd_last_stats(const sc_dd* dd, sc_dd_stats* out) {
  if (!dd || !out) return fail(SC_DD_EINVAL, "sc_dd_last_stats: null argument");
  if (!dd->have_last) return fail(SC_DD_EINVAL, "sc_dd_last_stats: no search has completed");
  *out = dd->last;
  return SC_DD_OK;
}

int sc_dd_copy_channel_array(sc_dd* dd, int which, float* dst, void* stream_ptr) {
  if (!dd || !dst || which < 0 || which > 2) return fail(SC_DD_EINVAL, "sc_dd_copy_channel_array: bad argument");
  if (dd->slots < 1) return fail(SC_DD_EINVAL, "sc_dd_copy_channel_array: no scratch");
  if (which == 2 && dd->prec_slots < 1) return fail(SC_DD_EINVAL, "sc_dd_copy_channel_array: no 16-bit search yet");
  DeviceGuard guard(dd->device);
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  const float* src = which == 0 ? dd->top : (which == 1 ? dd->colsum : dd->top16);
  cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(float) * dd->N, cudaMemcpyDefault, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) return cuda_fail(e, "sc_dd_copy_channel_array");
  return SC_DD_OK;
}

}  // extern "C"
