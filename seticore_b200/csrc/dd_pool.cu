// sc_dd_pool: many searches of different shapes in one pass over the GPU.
//
// A pool owns a device scratch arena of a stated budget.  A call takes a list of search
// requests (each with its own timesteps, channels, frequency resolution, drift range,
// threshold and precision), admits them into sub-batches whose scratch fits the arena,
// and for each sub-batch queues one fixed sequence of launches through exec_queue: every
// kernel runs once for up to 64 searches, and the tree kernel's persistent CTAs pull work
// items (tile x drift-block chunk) from all searches of the same row count.
//
// Autotuning: the first time a tree launch of a given class (rows, element type, and the
// power-of-two buckets of its largest drift-block count and total channels) is seen, it is
// timed with each candidate launch shape -- tile width (1056 or 352 channels) and
// shared-memory budget (which sets how many drift blocks share a staged trapezoid and how
// many CTAs share an SM) -- and the fastest is kept; likewise, each
// class of more than 32 rows (rows, buckets of channels and drift blocks) times the
// candidate level splits (stage-fusion depth).  Timing reruns are harmless: the tree
// kernel only raises per-channel maxima, so repeating it is idempotent.
//
// CUDA graphs: a sub-batch seen before (same requests, same arena layout) is replayed
// from a captured graph that also holds the copies of the results to pinned host memory.
#include <algorithm>
#include <cstddef>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace {

thread_local std::string g_pool_error;

int pfail(int code, const std::string& m) {
  g_pool_error = m;
  return code;
}
int pcuda(cudaError_t e, const char* what) { return pfail(SC_DD_ECUDA, std::string(what) + ": " + cudaGetErrorString(e)); }

constexpr int kHostCands = 256;
constexpr int kMaxGraphs = 16;

uint64_t fnv(uint64_t h, const void* p, size_t n) {
  const unsigned char* c = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) h = (h ^ c[i]) * 1099511628211ull;
  return h;
}

int round_up_pow2(int n) {
  int r = 1;
  while (r < n) r *= 2;
  return r;
}

struct Planned {
  scb::ExecSearch es;
  double res;
  double min_drift;
  int beam, coarse;
  size_t bytes;
};

}  // namespace

struct sc_dd_pool {
  int device = 0, num_sms = 148, n_partials = 0;
  size_t budget = 0;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  float* lvl_a = nullptr;
  float* lvl_b = nullptr;
  size_t lvl_floats = 0;
  scb::LevelSide side;  // side stream i's buffers: lvl_a + 2 + 2i and 3 + 2i lvl_floats
  char* host = nullptr;  // pinned: headers + candidate heads of the largest sub-batch
  size_t host_bytes = 0;
  cudaStream_t cap_stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evj = nullptr, t0 = nullptr, t1 = nullptr;
  struct Graph {
    uint64_t key;
    cudaGraphExec_t exec;
    uint64_t last_use;
  };
  std::vector<Graph> graphs;
  std::unordered_map<uint64_t, int> seen;  // sub-batch key -> times seen
  std::unordered_map<uint64_t, scb::TreeLaunch> tuned_launch;
  std::unordered_map<uint64_t, scb::LevelPlan> tuned_plan;
  uint64_t clock = 0;
  int tuning = 1, use_graphs = 1;
  bool tuning_now = false;
  sc_dd_pool_stats st{};
};

namespace {

// Power-of-two bucket of a positive count (tuning keys describe a launch's class, not
// its exact composition, so a mix of shapes is tuned a few times rather than per batch).
int bucket(long long v) {
  int b = 0;
  while ((1ll << b) < v) ++b;
  return b;
}

scb::TreeLaunch pool_tree_launch(void* ctx, const scb::TreeBatch& tb, int R, int elem) {
  sc_dd_pool* p = static_cast<sc_dd_pool*>(ctx);
  // The launch shape decides how many drift blocks share a staged tile, how wide the tile is
  // and how many CTAs fit an SM: the key is the rows, the element type, the largest
  // drift-block count and the launch's total channels, each bucketed.
  int max_jobs = 1;
  long long channels = 0;
  for (int k = 0; k < tb.count; ++k) {
    max_jobs = std::max(max_jobs, tb.g[k].n_jobs);
    channels += tb.g[k].N;
  }
  const int v[5] = {R, elem, bucket(max_jobs), bucket(channels), tb.pair16};
  const uint64_t key = fnv(1469598103934665603ull, v, sizeof(v));
  auto it = p->tuned_launch.find(key);
  if (it != p->tuned_launch.end()) return it->second;
  if (!p->tuning || !p->tuning_now) return scb::TreeLaunch{};
  // Time each candidate on the stream the search runs on (idempotent reruns): shared-memory
  // budgets with 1056-channel tiles, and 352-channel tiles.  The 32-row tree runs one CTA per
  // SM with long strips only: its candidates are the budgets from 200 KB up.
  cudaStream_t s = p->cap_stream;
  const scb::TreeLaunch cands16[5] = {{110, 1056}, {160, 1056}, {200, 1056}, {110, 352}, {48, 352}};
  const scb::TreeLaunch cands32[2] = {{200, 1056}, {226, 1056}};
  const scb::TreeLaunch* cands = R == 32 ? cands32 : cands16;
  const int n_cands = R == 32 ? 2 : 5;
  scb::TreeLaunch best{};
  float best_ms = 1e30f;
  for (int ci = 0; ci < n_cands; ++ci) {
    const scb::TreeLaunch& c = cands[ci];
    scb::TreeBatch copy = tb;
    cudaEventRecord(p->t0, s);
    if (scb::tree_max_batch(copy, R, p->num_sms, s, elem, c) != cudaSuccess) continue;
    cudaEventRecord(p->t1, s);
    cudaEventSynchronize(p->t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, p->t0, p->t1);
    if (ms < best_ms) {
      best_ms = ms;
      best = c;
    }
  }
  p->tuned_launch[key] = best;
  p->st.tuned_launches++;
  return best;
}

std::vector<scb::LevelPlan> level_candidates(int Tr) {
  std::vector<scb::LevelPlan> out;
  // a 16-row first level (one thread per channel, or the emitting fused tree with two
  // drift blocks per staged read), then 4s / 2s down to at most 16 rows
  if (Tr >= 32) {
    for (int first : {16, scb::kStreamEmit16}) {
      scb::LevelPlan pl{};
      pl.m[pl.n++] = first;
      int rem = Tr / 16;
      while (rem > 16 && pl.n < 12) {
        const int m = (rem / 4 >= 16) ? 4 : 2;
        pl.m[pl.n++] = m;
        rem /= m;
      }
      pl.final_rows = rem;
      out.push_back(pl);
    }
    // the one-thread-per-channel 8-row level first, finishing in 16 or fewer rows
    if (Tr / 8 <= 16) {
      scb::LevelPlan pl{};
      pl.m[pl.n++] = 8;
      pl.final_rows = Tr / 8;
      out.push_back(pl);
    }
  }
  // emit levels of 4s then 2s (or 2s then 4s) down to a final of 16 or 8 rows
  for (int fin : {16, 8}) {
    for (int order = 0; order < 2; ++order) {
      scb::LevelPlan pl{};
      pl.final_rows = fin;
      int rem = Tr / fin;
      if (rem < 2) continue;
      std::vector<int> ms;
      while (rem > 1) {
        const int m = (rem % 4 == 0) ? 4 : 2;
        ms.push_back(m);
        rem /= m;
      }
      if (order == 1) std::reverse(ms.begin(), ms.end());
      if ((int)ms.size() > 12) continue;
      pl.n = (int)ms.size();
      for (int i = 0; i < pl.n; ++i) pl.m[i] = ms[i];
      bool dup = false;
      for (auto& q : out)
        if (q.n == pl.n && q.final_rows == pl.final_rows && std::equal(q.m, q.m + q.n, pl.m)) dup = true;
      if (!dup) out.push_back(pl);
    }
  }
  return out;
}

scb::LevelPlan pool_level_plan(void* ctx, const scb::ExecSearch& s, float* la, float* lb, cudaStream_t st) {
  sc_dd_pool* p = static_cast<sc_dd_pool*>(ctx);
  const int v[3] = {s.Tr, bucket(s.N), bucket(s.dmax - s.dmin + 1)};
  const uint64_t key = fnv(1469598103934665603ull, v, sizeof(v));
  auto it = p->tuned_plan.find(key);
  if (it != p->tuned_plan.end()) return it->second;
  if (!p->tuning || !p->tuning_now) return scb::LevelPlan{};
  scb::LevelPlan best{};
  float best_ms = 1e30f;
  for (const scb::LevelPlan& pl : level_candidates(s.Tr)) {
    cudaEventRecord(p->t0, st);
    int* status = reinterpret_cast<int*>(reinterpret_cast<char*>(s.hdr) + offsetof(scb::SearchHeader, error));
    if (scb::levels_search(s.input, s.row_stride, s.Tr, s.N, s.dmin, s.dmax, la, lb, s.top, p->num_sms, st, pl,
                           scb::kElemF32, status) != cudaSuccess)
      continue;
    cudaEventRecord(p->t1, st);
    cudaEventSynchronize(p->t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, p->t0, p->t1);
    if (ms < best_ms) {
      best_ms = ms;
      best = pl;
    }
  }
  p->tuned_plan[key] = best;
  p->st.tuned_launches++;
  return best;
}

// Grows the arena and the level buffers in stream order on `stream` (cudaFreeAsync /
// cudaMallocAsync): every earlier call of this pool has finished with them (a call
// synchronises its stream before it returns), and work of other streams -- another pool's,
// another server worker's -- is not waited for, as a device-wide synchronisation or a plain
// cudaFree would.  Graphs captured over the old buffers are dropped.
int ensure_device(sc_dd_pool* p, size_t arena, size_t lvl, cudaStream_t stream) {
  cudaError_t e;
  if (arena > p->arena_bytes || lvl > p->lvl_floats) {
    for (auto& g : p->graphs) cudaGraphExecDestroy(g.exec);
    p->graphs.clear();
    p->seen.clear();
  }
  if (arena > p->arena_bytes) {
    if (p->arena) cudaFreeAsync(p->arena, stream);
    p->arena = nullptr;
    p->arena_bytes = 0;
    if ((e = cudaMallocAsync(reinterpret_cast<void**>(&p->arena), arena, stream)) != cudaSuccess)
      return pfail(SC_DD_ENOMEM, std::string("pool arena: ") + cudaGetErrorString(e));
    if ((e = cudaMemsetAsync(p->arena, 0, arena, stream)) != cudaSuccess) return pcuda(e, "pool arena memset");
    p->arena_bytes = arena;
  }
  if (lvl > p->lvl_floats) {
    if (p->lvl_a) cudaFreeAsync(p->lvl_a, stream);
    p->lvl_a = p->lvl_b = nullptr;
    for (int i = 0; i < scb::kLevelSides; ++i) p->side.lvl_a[i] = p->side.lvl_b[i] = nullptr;
    p->lvl_floats = 0;
    // All pairs of level buffers in one allocation: the emitting level addresses a pair as
    // one array; pair 0 serves the pool's stream, pair 1 + i side stream i.
    const size_t pairs = 1 + (size_t)p->side.n;
    if ((e = cudaMallocAsync(reinterpret_cast<void**>(&p->lvl_a), 2 * pairs * lvl * sizeof(float), stream)) !=
        cudaSuccess)
      return pfail(SC_DD_ENOMEM, std::string("pool level buffers: ") + cudaGetErrorString(e));
    p->lvl_b = p->lvl_a + lvl;
    for (int i = 0; i < p->side.n; ++i) {
      p->side.lvl_a[i] = p->lvl_a + (2 + 2 * i) * lvl;
      p->side.lvl_b[i] = p->lvl_a + (3 + 2 * i) * lvl;
    }
    p->lvl_floats = lvl;
  }
  return SC_DD_OK;
}

// Queues one sub-batch plus the copies of its results into p->host.
cudaError_t queue_sub(sc_dd_pool* p, std::vector<Planned>& sub, cudaStream_t s) {
  std::vector<scb::ExecSearch> es(sub.size());
  for (size_t k = 0; k < sub.size(); ++k) es[k] = sub[k].es;
  scb::ExecHooks hooks;
  hooks.ctx = p;
  hooks.tree_launch = pool_tree_launch;
  hooks.level_plan = pool_level_plan;
  // The tuner times one level search at a time on its own stream: no side stream then.
  cudaError_t e = scb::exec_queue(es.data(), (int)es.size(), p->lvl_a, p->lvl_b, p->num_sms, s, hooks,
                                  p->tuning_now || p->side.n == 0 ? nullptr : &p->side);
  if (e != cudaSuccess) return e;
  char* h = p->host;
  for (size_t k = 0; k < sub.size(); ++k) {
    const scb::ExecSearch& q = sub[k].es;
    const int head = std::min(kHostCands, q.cand_cap);
    if ((e = cudaMemcpyAsync(h, q.hdr, sizeof(scb::SearchHeader), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
    if ((e = cudaMemcpyAsync(h + sizeof(scb::SearchHeader), q.cands, sizeof(scb::Candidate) * head,
                             cudaMemcpyDeviceToHost, s)) != cudaSuccess)
      return e;
    h += sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * kHostCands;
  }
  return cudaSuccess;
}

}  // namespace

extern "C" {

const char* sc_dd_pool_last_error(void) { return g_pool_error.c_str(); }

int sc_dd_pool_create(size_t scratch_budget_bytes, sc_dd_pool** out) {
  g_pool_error.clear();
  if (!out) return pfail(SC_DD_EINVAL, "sc_dd_pool_create: out is null");
  *out = nullptr;
  sc_dd_pool* p = new (std::nothrow) sc_dd_pool();
  if (!p) return pfail(SC_DD_ENOMEM, "sc_dd_pool_create: host allocation");
  cudaError_t e = cudaGetDevice(&p->device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->cap_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess && scb::level_sides(false) > 0) e = cudaEventCreateWithFlags(&p->side.fork, cudaEventDisableTiming);
  for (int i = 0; i < scb::level_sides(false) && e == cudaSuccess; ++i) {
    if ((e = cudaStreamCreateWithFlags(&p->side.stream[i], cudaStreamNonBlocking)) == cudaSuccess &&
        (e = cudaEventCreateWithFlags(&p->side.join[i], cudaEventDisableTiming)) == cudaSuccess)
      p->side.n = i + 1;
  }
  for (cudaEvent_t* ev : {&p->ev0, &p->ev1, &p->evj, &p->t0, &p->t1})
    if (e == cudaSuccess) e = cudaEventCreate(ev);
  // The host buffer of the largest possible sub-batch, allocated once: pinned allocations
  // synchronise the device, which a pool serving beside other streams must not do per call.
  p->host_bytes = (size_t)4 * scb::kMaxBatch * (sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * kHostCands);
  if (e == cudaSuccess) e = cudaMallocHost(&p->host, p->host_bytes);
  if (e != cudaSuccess) {
    if (p->host) cudaFreeHost(p->host);
    for (cudaEvent_t ev : {p->ev0, p->ev1, p->evj, p->t0, p->t1, p->side.fork})
      if (ev) cudaEventDestroy(ev);
    if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
    for (int i = 0; i < scb::kLevelSides; ++i) {
      if (p->side.stream[i]) cudaStreamDestroy(p->side.stream[i]);
      if (p->side.join[i]) cudaEventDestroy(p->side.join[i]);
    }
    delete p;
    return pcuda(e, "sc_dd_pool_create");
  }
  p->n_partials = 2 * p->num_sms;
  p->budget = scratch_budget_bytes;
  *out = p;
  return SC_DD_OK;
}

int sc_dd_pool_destroy(sc_dd_pool* p) {
  if (!p) return SC_DD_OK;
  cudaDeviceSynchronize();
  for (auto& g : p->graphs) cudaGraphExecDestroy(g.exec);
  if (p->arena) cudaFreeAsync(p->arena, nullptr);
  if (p->lvl_a) cudaFreeAsync(p->lvl_a, nullptr);
  cudaDeviceSynchronize();
  if (p->host) cudaFreeHost(p->host);
  for (cudaEvent_t ev : {p->ev0, p->ev1, p->evj, p->t0, p->t1})
    if (ev) cudaEventDestroy(ev);
  if (p->cap_stream) cudaStreamDestroy(p->cap_stream);
  for (int i = 0; i < scb::kLevelSides; ++i) {
    if (p->side.stream[i]) cudaStreamDestroy(p->side.stream[i]);
    if (p->side.join[i]) cudaEventDestroy(p->side.join[i]);
  }
  if (p->side.fork) cudaEventDestroy(p->side.fork);
  delete p;
  return SC_DD_OK;
}

int sc_dd_pool_configure(sc_dd_pool* p, int autotune, int cuda_graphs) {
  if (!p) return pfail(SC_DD_EINVAL, "sc_dd_pool_configure: null pool");
  p->tuning = autotune ? 1 : 0;
  p->use_graphs = cuda_graphs ? 1 : 0;
  return SC_DD_OK;
}

int sc_dd_pool_stats_get(const sc_dd_pool* p, sc_dd_pool_stats* out) {
  if (!p || !out) return pfail(SC_DD_EINVAL, "sc_dd_pool_stats_get: null argument");
  *out = p->st;
  return SC_DD_OK;
}

size_t sc_dd_request_scratch_bytes(const sc_dd_request* r) {
  if (!r || r->num_timesteps < 2 || r->num_channels < 64) return 0;
  const int Tr = round_up_pow2(r->num_timesteps);
  const double res = 1e6 * r->foff_mhz / ((Tr - 1) * r->tsamp_s);
  const double nmax = r->max_drift / std::fabs(res * (Tr - 1));
  const int w = (int)(2 * std::ceil(nmax * (Tr - 1)));
  if (w < 1) return 0;
  const long long nwin = ((long long)r->num_channels + w - 1) / w;
  const int cap = (int)std::min<long long>(nwin + 1, r->num_channels / 2 + 2);
  int sms = 148;
  int dev = 0;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int elem = r->precision == SC_DD_PRECISION_BF16 ? scb::kElemBF16
                   : r->precision == SC_DD_PRECISION_FP16 ? scb::kElemF16 : scb::kElemF32;
  return scb::ExecSearch::scratch_bytes(Tr, r->num_channels, cap, 2 * sms, elem);
}

int sc_dd_pool_search(sc_dd_pool* p, const sc_dd_request* reqs, int count, sc_dd_hit* out, int capacity,
                      int* num_hits, void* stream_ptr) {
  g_pool_error.clear();
  if (!p || count < 0 || (count > 0 && (!reqs || !num_hits)) || (capacity > 0 && !out))
    return pfail(SC_DD_EINVAL, "sc_dd_pool_search: null argument");
  cudaStream_t stream = static_cast<cudaStream_t>(stream_ptr);
  // Plan every request.
  std::vector<Planned> plans(count);
  for (int i = 0; i < count; ++i) {
    const sc_dd_request& r = reqs[i];
    if (!r.dev_input || r.num_timesteps < 2 || r.num_timesteps > 2048 || r.num_channels < 64 ||
        r.row_stride < r.num_channels || !(r.tsamp_s > 0) || !(r.foff_mhz != 0))
      return pfail(SC_DD_EINVAL, "sc_dd_pool_search: bad request " + std::to_string(i));
    Planned& pl = plans[i];
    scb::ExecSearch& q = pl.es;
    q = scb::ExecSearch{};
    q.input = r.dev_input;
    q.row_stride = r.row_stride;
    q.T = r.num_timesteps;
    q.Tr = round_up_pow2(r.num_timesteps);
    q.N = r.num_channels;
    // dedoppler.cu:84-87, 194-198, 274
    const int dt = q.Tr - 1;
    pl.res = 1e6 * r.foff_mhz / (dt * r.tsamp_s);
    const double nmax = r.max_drift / std::fabs(pl.res * dt);
    q.dmin = (int)std::floor(-nmax);
    q.dmax = (int)std::floor(nmax);
    q.window_size = (int)(2 * std::ceil(nmax * dt));
    if (!(q.window_size >= 1) || q.dmax < q.dmin)
      return pfail(SC_DD_EINVAL, "sc_dd_pool_search: request " + std::to_string(i) + " has no drift range");
    q.snr_threshold = r.snr_threshold;
    q.elem = r.precision == SC_DD_PRECISION_BF16 ? scb::kElemBF16
             : r.precision == SC_DD_PRECISION_FP16 ? scb::kElemF16 : scb::kElemF32;
    const long long nwin = ((long long)q.N + q.window_size - 1) / q.window_size;
    q.cand_cap = (int)std::min<long long>(nwin + 1, q.N / 2 + 2);
    pl.min_drift = r.min_drift;
    pl.beam = r.beam;
    pl.coarse = r.coarse_channel;
    pl.bytes = scb::ExecSearch::scratch_bytes(q.Tr, q.N, q.cand_cap, p->n_partials, q.elem);
  }
  // Admission: consecutive requests while their scratch fits the budget (at least one).
  size_t arena_need = 0, lvl_need = 0;
  std::vector<std::pair<int, int>> subs;
  {
    int i = 0;
    while (i < count) {
      size_t used = 0;
      int j = i;
      while (j < count && (j == i || used + plans[j].bytes <= p->budget) && j - i < 4 * scb::kMaxBatch) {
        used += plans[j].bytes;
        ++j;
      }
      subs.push_back({i, j});
      arena_need = std::max(arena_need, used);
      i = j;
    }
    for (const Planned& pl : plans)
      if (pl.es.Tr > 32) lvl_need = std::max(lvl_need, scb::level_buffer_floats(pl.es.Tr, pl.es.N));
  }
  int rc = ensure_device(p, arena_need, lvl_need, stream);
  if (rc != SC_DD_OK) return rc;

  cudaError_t e;
  int total = 0;
  p->st.calls++;
  cudaEventRecord(p->ev0, stream);
  for (auto& sb : subs) {
    std::vector<Planned> sub(plans.begin() + sb.first, plans.begin() + sb.second);
    size_t off = 0;
    uint64_t key = 1469598103934665603ull;
    for (Planned& pl : sub) {
      pl.es.carve(p->arena + off, p->n_partials);
      off += pl.bytes;
      const sc_dd_request& r = reqs[sb.first + (&pl - sub.data())];
      key = fnv(key, &r, sizeof(r));
    }
    // and the process-wide settings that change the launches
    const long long settings[4] = {scb::exact_statistics_always() ? 1 : 0, scb::stage_wait_tries(),
                                   scb::paired_fp16() ? 1 : 0, scb::level_stripe_bytes()};
    key = fnv(key, settings, sizeof(settings));
    p->st.sub_batches++;
    auto git = std::find_if(p->graphs.begin(), p->graphs.end(), [&](const sc_dd_pool::Graph& g) { return g.key == key; });
    if (p->use_graphs && git != p->graphs.end()) {
      git->last_use = ++p->clock;
      if ((e = cudaGraphLaunch(git->exec, stream)) != cudaSuccess) return pcuda(e, "graph launch");
      p->st.graph_replays++;
    } else {
      const int seen = ++p->seen[key];
      if (p->use_graphs && seen >= 2) {
        // Capture on the pool's stream, ordered after the caller's stream.
        cudaEventRecord(p->evj, stream);
        cudaStreamWaitEvent(p->cap_stream, p->evj, 0);
        cudaGraph_t g = nullptr;
        if ((e = cudaStreamBeginCapture(p->cap_stream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
          return pcuda(e, "begin capture");
        p->tuning_now = false;
        cudaError_t qe = queue_sub(p, sub, p->cap_stream);
        e = cudaStreamEndCapture(p->cap_stream, &g);
        if (qe != cudaSuccess) return pcuda(qe, "capture");
        if (e != cudaSuccess) return pcuda(e, "end capture");
        cudaGraphExec_t ex = nullptr;
        e = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return pcuda(e, "instantiate");
        if ((int)p->graphs.size() >= kMaxGraphs) {
          auto lru = std::min_element(p->graphs.begin(), p->graphs.end(),
                                      [](const sc_dd_pool::Graph& a, const sc_dd_pool::Graph& b) {
                                        return a.last_use < b.last_use;
                                      });
          cudaGraphExecDestroy(lru->exec);
          p->graphs.erase(lru);
        }
        p->graphs.push_back({key, ex, ++p->clock});
        p->st.graph_captures++;
        if ((e = cudaGraphLaunch(ex, stream)) != cudaSuccess) return pcuda(e, "graph launch");
      } else {
        // First sight: run directly; tree launches and level splits not seen before are tuned.
        p->tuning_now = true;
        std::swap(p->cap_stream, stream);  // the tuning hooks time on p->cap_stream
        e = queue_sub(p, sub, p->cap_stream);
        std::swap(p->cap_stream, stream);
        p->tuning_now = false;
        if (e != cudaSuccess) return pcuda(e, "search kernels");
      }
    }
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return pcuda(e, "synchronise");
    // Results.
    const char* h = p->host;
    for (size_t k = 0; k < sub.size(); ++k, h += sizeof(scb::SearchHeader) + sizeof(scb::Candidate) * kHostCands) {
      const Planned& pl = sub[k];
      const scb::SearchHeader hd = *reinterpret_cast<const scb::SearchHeader*>(h);
      if (hd.error) return pfail(SC_DD_EINTERNAL, "a tree kernel gave up waiting for its staged rows");
      const int ncand = std::min(hd.num_candidates, pl.es.cand_cap);
      const int head = std::min(kHostCands, pl.es.cand_cap);
      std::vector<scb::Candidate> cands(ncand);
      const scb::Candidate* hc = reinterpret_cast<const scb::Candidate*>(h + sizeof(scb::SearchHeader));
      std::copy(hc, hc + std::min(ncand, head), cands.begin());
      if (ncand > head) {
        if ((e = cudaMemcpyAsync(cands.data() + head, pl.es.cands + head, sizeof(scb::Candidate) * (ncand - head),
                                 cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
          return pcuda(e, "candidate copy");
      }
      std::sort(cands.begin(), cands.end(),
                [](const scb::Candidate& a, const scb::Candidate& b) { return a.index < b.index; });
      int nk = 0;
      for (const scb::Candidate& c : cands) {
        int drift_bins = 0;
        if (!scb::decode_candidate(c, pl.es.dmin, pl.es.Tr, &drift_bins))
          return pfail(SC_DD_EINTERNAL, "drift recovery did not reproduce a top sum");
        const double drift_rate = drift_bins * pl.res;  // dedoppler.cu:305-317
        const float snr = (c.power - hd.median) / hd.std_dev;
        if (std::fabs(drift_rate) >= pl.min_drift) {
          if (total < capacity) {
            sc_dd_hit& o = out[total];
            o.index = c.index;
            o.drift_steps = drift_bins;
            o.drift_rate = drift_rate;
            o.snr = snr;
            o.power = c.power;
            o.incoherent_power = 0.0f;
            o.coarse_channel = pl.coarse;
            o.beam = pl.beam;
            o.num_timesteps = pl.es.T;
          }
          ++total;
          ++nk;
        }
      }
      num_hits[sb.first + k] = nk;
    }
  }
  cudaEventRecord(p->ev1, stream);
  cudaEventSynchronize(p->ev1);
  cudaEventElapsedTime(&p->st.last_call_ms, p->ev0, p->ev1);
  if (total > capacity) return pfail(SC_DD_ETRUNC, "more hits than capacity");
  return SC_DD_OK;
}

}  // extern "C"
