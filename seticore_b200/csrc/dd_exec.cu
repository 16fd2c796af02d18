// Queues the kernels of a list of searches of any shapes, drift ranges and precisions.
//
// Used by the engine (dd_api.cu, one shape) and by the pool (dd_pool.cu, mixed shapes).
// The searches travel in batches of up to kMaxBatch as kernel parameters, so a call is a
// fixed sequence of launches (capturable in a CUDA graph) whatever the mix:
//   clear -> [normalise] -> column sums (searches whose tree does not compute them) ->
//   tree launches grouped by (rows, element type), the float32 ones adding the column
//   sums -> levels for more than 32 rows, one search at a time -> statistics ->
//   [flag + FP32 recompute of the flagged channels] -> hits
#include <algorithm>
#include <cstddef>
#include <cstdlib>

#include "dd_common.cuh"
#include "dd_internal.h"

namespace scb {

namespace {

// Zeroes, per search of the batch: top (and the 16-bit tops), the result header, the
// order-statistic state and the flagged-channel count.
__global__ void clear_kernel(const __grid_constant__ SearchBatch b, const __grid_constant__ PrecisionBatch pb) {
  const SearchDesc& d = b.s[blockIdx.y];
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < d.N; c += gridDim.x * blockDim.x) d.top[c] = 0.0f;
  if (blockIdx.x == 0 && threadIdx.x < (int)(sizeof(SearchHeader) / 4))
    reinterpret_cast<int*>(d.hdr)[threadIdx.x] = 0;
  if (blockIdx.x == 0) reset_select(d.sel, d.first, d.mid, d.last);  // the order-statistic state
  if (pb.count > 0 && blockIdx.y < (unsigned)pb.count && pb.s[blockIdx.y].flag_count) {
    const PrecisionDesc& q = pb.s[blockIdx.y];
    float* t16 = const_cast<float*>(q.top16);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < q.N; c += gridDim.x * blockDim.x) t16[c] = 0.0f;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      *q.flag_count = 0;
      *q.ticket = 0;
    }
  }
}

SearchDesc to_desc(const ExecSearch& e) {
  SearchDesc s{};
  s.input = e.input;
  s.row_stride = e.row_stride;
  s.Tr = e.Tr;
  s.N = e.N;
  s.dmin = e.dmin;
  s.dmax = e.dmax;
  s.window_size = e.window_size;
  s.first = (int)ceil(0.05 * e.N);  // dedoppler.cu:247
  s.mid = e.N / 2;                   // dedoppler.cu:211
  s.last = (int)floor(0.95 * e.N);  // dedoppler.cu:248
  s.snr_threshold = e.snr_threshold;
  s.top = e.top;
  s.colsum = e.colsum;
  s.sel = e.sel;
  s.partials = e.partials;
  s.var = e.var;
  s.work = e.work;
  s.lists = e.lists;
  s.hdr = e.hdr;
  s.cands = e.cands;
  s.cand_cap = e.cand_cap;
  return s;
}

// 16-bit 16- and 32-row searches take the paired-FP16 tree when it is on (the flag bound must
// know).
bool pair16_search(const ExecSearch& e, bool on) { return on && e.elem != kElemF32 && pair_rows(e.Tr); }

PrecisionDesc to_pdesc(const ExecSearch& e, const SearchHeader* hdr, bool pair_on) {
  PrecisionDesc q{};
  q.input = e.input;
  q.row_stride = e.row_stride;
  q.T = e.T;
  q.Tr = e.Tr;
  q.N = e.N;
  q.norm = e.norm16;
  q.colsum = e.colsum;
  q.moments = e.norm_moments;
  q.ticket = e.norm_ticket;
  q.top16 = e.top16;
  q.hdr = hdr;
  q.snr_threshold = e.snr_threshold;
  q.dmin = e.dmin;
  q.dmax = e.dmax;
  q.top = e.top;
  q.flag_list = e.flags;
  q.flag_count = e.flag_count;
  q.pair16 = pair16_search(e, pair_on) ? 1 : 0;
  return q;
}

// Searches whose column sums come with another pass over the input: the float32 tree of up
// to 32 rows (its drift range always holds drift block 0: dmin <= 0 <= dmax), and the
// 16-bit forms' normalising pass.
bool tree_colsum(const ExecSearch& e) { return e.elem == kElemF32 && e.Tr <= 32 && e.dmin <= 0 && e.dmax >= 0; }
bool fused_colsum(const ExecSearch& e) { return tree_colsum(e) || e.elem != kElemF32; }

// The search's header word that a kernel sets when it gives up a wait.
int* header_status(const ExecSearch& e) {
  return reinterpret_cast<int*>(reinterpret_cast<char*>(e.hdr) + offsetof(SearchHeader, error));
}

TreeGroup tree_group(const ExecSearch& e, const void* rows, long long row_stride, float* top) {
  TreeGroup g{};
  g.rows = rows;
  g.row_stride = row_stride;
  g.job_row_stride = 0;
  g.N = e.N;
  g.d_first = e.dmin;
  g.d_step = 1;
  g.n_jobs = e.dmax - e.dmin + 1;
  g.db_first = e.dmin;
  g.db_step = 1;
  g.off_base = 0;
  g.off_step = 0;
  g.elig_T1 = e.Tr - 1;
  g.top = top;
  g.status = header_status(e);
  return g;
}

}  // namespace

int level_sides(bool engine) {
  static const long v = [] {
    const char* e = getenv("SETICORE_B200_LEVEL_SIDES");
    return e ? strtol(e, nullptr, 10) : -1L;
  }();
  // An engine holds one search shape, so its extra buffer pairs are small: three sides
  // (beams 194.5 -> 197.4 Gsamples/s).  A pool sizes its pairs for its largest search and
  // serves beside others: one.
  const long x = v >= 0 ? v : (engine ? 3 : 1);
  return (int)std::min<long>(kLevelSides, std::max<long>(0, x));
}

cudaError_t exec_queue(const ExecSearch* s, int n, float* lvl_a, float* lvl_b, int num_sms, cudaStream_t stream,
                       const ExecHooks& hooks, const LevelSide* side) {
  cudaError_t e = cudaSuccess;
  const bool pair_on = paired_fp16();  // read once: the trees and the flag bounds agree
  for (int k0 = 0; k0 < n && e == cudaSuccess; k0 += kMaxBatch) {
    const int m = std::min(kMaxBatch, n - k0);
    const ExecSearch* ss = s + k0;
    SearchBatch b;
    b.count = m;
    b.maxN = 0;
    for (int k = 0; k < m; ++k) {
      b.s[k] = to_desc(ss[k]);
      b.maxN = std::max(b.maxN, ss[k].N);
    }
    // Clear (one launch).
    PrecisionBatch clear_pb;
    clear_pb.count = m;
    clear_pb.maxN = b.maxN;
    clear_pb.elem = kElemBF16;
    for (int k = 0; k < m; ++k) {
      clear_pb.s[k] = PrecisionDesc{};
      if (ss[k].elem != kElemF32) clear_pb.s[k] = to_pdesc(ss[k], b.s[k].hdr, pair_on);
    }
    {
      int gx = (b.maxN + 1023) / 1024;
      if (gx > 64) gx = 64;
      clear_kernel<<<dim3(gx, m), 256, 0, stream>>>(b, clear_pb);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // Normalisation of the 16-bit searches (one launch per element type).
    for (int elem : {kElemBF16, kElemF16}) {
      PrecisionBatch q;
      q.count = 0;
      q.maxN = 0;
      q.elem = elem;
      for (int k = 0; k < m; ++k)
        if (ss[k].elem == elem) {
          q.s[q.count++] = to_pdesc(ss[k], b.s[k].hdr, pair_on);
          q.maxN = std::max(q.maxN, ss[k].N);
        }
      if (q.count && (e = normalize_batch(q, num_sms, stream)) != cudaSuccess) return e;
    }
    // Column sums: the float32 trees over up to 32 rows compute their own from the staged
    // rows and the 16-bit forms in their normalising pass; the level path reads the input
    // once here.
    {
      SearchBatch cb;
      cb.count = 0;
      cb.maxN = 0;
      for (int k = 0; k < m; ++k)
        if (!fused_colsum(ss[k])) {
          cb.s[cb.count++] = b.s[k];
          cb.maxN = std::max(cb.maxN, ss[k].N);
        }
      if ((e = column_sums_batch(cb, stream)) != cudaSuccess) return e;
    }
    if (hooks.before_tree) hooks.before_tree(hooks.ctx, stream);
    // Trees over up to 32 rows: one launch per (rows, element type).
    for (int R : {2, 4, 8, 16, 32}) {
      for (int elem : {kElemF32, kElemBF16, kElemF16}) {
        TreeBatch tb;
        tb.count = 0;
        tb.n_items = 0;
        tb.pair16 = (elem != kElemF32 && pair_rows(R) && pair_on) ? 1 : 0;
        for (int k = 0; k < m; ++k) {
          if (ss[k].Tr != R || ss[k].elem != elem) continue;
          if (elem == kElemF32) {
            TreeGroup g = tree_group(ss[k], ss[k].input, ss[k].row_stride, ss[k].top);
            if (tree_colsum(ss[k])) {
              g.colsum = ss[k].colsum;
              g.colsum_job = -ss[k].dmin;
            }
            tb.g[tb.count++] = g;
          } else if (tb.pair16) {
            // the paired copy: channel 0 of row 0 sits kPairPad words into the buffer
            TreeGroup g = tree_group(ss[k], static_cast<const uint32_t*>(ss[k].norm16) + kPairPad,
                                     pair_row_words(ss[k].N), ss[k].top16);
            g.pad = kPairPad;
            tb.g[tb.count++] = g;
          } else {
            tb.g[tb.count++] = tree_group(ss[k], ss[k].norm16, ss[k].N, ss[k].top16);
          }
        }
        if (tb.count && (e = tree_max_batch(tb, R, num_sms, stream, elem, hooks.tree_launch(hooks.ctx, tb, R, elem))) !=
                            cudaSuccess)
          return e;
      }
    }
    // More than 32 rows: the level path, one search at a time per level-buffer pair.  FP32
    // searches are dealt round-robin over the main stream and the side streams, when there are
    // any (two concurrent 16-bit level searches measured slower than one after the other: their
    // first level is bound by L1 throughput, not by latency); the 16-bit searches run it on
    // their normalised copy, with the default split, on the main stream.
    int n_level = 0;
    for (int k = 0; k < m; ++k) n_level += ss[k].Tr > 32 && ss[k].elem == kElemF32;
    const int lanes = (side && side->n > 0 && n_level >= 2) ? 1 + std::min(side->n, n_level - 1) : 1;
    if (lanes > 1) {
      if ((e = cudaEventRecord(side->fork, stream)) != cudaSuccess) return e;
      for (int i = 0; i + 1 < lanes; ++i)
        if ((e = cudaStreamWaitEvent(side->stream[i], side->fork, 0)) != cudaSuccess) return e;
    }
    int j = 0;
    for (int k = 0; k < m; ++k) {
      if (ss[k].Tr <= 32) continue;
      const int lane = (lanes > 1 && ss[k].elem == kElemF32) ? (j++ % lanes) : 0;  // 0: the main stream
      cudaStream_t st = lane ? side->stream[lane - 1] : stream;
      float* la = lane ? side->lvl_a[lane - 1] : lvl_a;
      float* lb = lane ? side->lvl_b[lane - 1] : lvl_b;
      if (ss[k].elem != kElemF32) {
        if ((e = levels_search(ss[k].norm16, ss[k].N, ss[k].Tr, ss[k].N, ss[k].dmin, ss[k].dmax, la, lb, ss[k].top16,
                               num_sms, st, LevelPlan{}, ss[k].elem, header_status(ss[k]))) != cudaSuccess)
          return e;
        continue;
      }
      const LevelPlan plan = hooks.level_plan ? hooks.level_plan(hooks.ctx, ss[k], la, lb, st) : ss[k].level_plan;
      if ((e = levels_search(ss[k].input, ss[k].row_stride, ss[k].Tr, ss[k].N, ss[k].dmin, ss[k].dmax, la, lb,
                             ss[k].top, num_sms, st, plan, kElemF32, header_status(ss[k]))) != cudaSuccess)
        return e;
    }
    for (int i = 0; i + 1 < lanes; ++i) {
      if ((e = cudaEventRecord(side->join[i], side->stream[i])) != cudaSuccess ||
          (e = cudaStreamWaitEvent(stream, side->join[i], 0)) != cudaSuccess)
        return e;
    }
    if (hooks.after_tree) hooks.after_tree(hooks.ctx, stream);
    if ((e = search_stats_batch(b, num_sms, stream)) != cudaSuccess) return e;
    // The 16-bit searches: list the channels near the threshold, recompute them exactly
    // in FP32 from the original power.
    {
      PrecisionBatch q;
      q.count = 0;
      q.maxN = 0;
      q.elem = kElemBF16;
      for (int k = 0; k < m; ++k)
        if (ss[k].elem != kElemF32) {
          q.s[q.count++] = to_pdesc(ss[k], b.s[k].hdr, pair_on);
          q.maxN = std::max(q.maxN, ss[k].N);
        }
      if (q.count) {
        if ((e = flag_channels_batch(q, num_sms, stream)) != cudaSuccess) return e;
        if ((e = recompute_batch(q, num_sms, stream)) != cudaSuccess) return e;
      }
    }
    if ((e = search_hits_batch(b, num_sms, stream)) != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

size_t ExecSearch::scratch_bytes(int Tr, int N, int cand_cap, int n_partials, int elem) {
  auto a = [](size_t x) { return (x + 255) & ~size_t(255); };
  size_t b = a(sizeof(float) * N) * 2 + a(sizeof(SelectState)) + a(sizeof(MomentPartial) * n_partials) +
             a(sizeof(double) * 2 * kVarChunks) + a(sizeof(float) * order_work_floats(N)) +
             a(sizeof(int) * order_list_entries(N)) + a(sizeof(SearchHeader)) + a(sizeof(Candidate) * cand_cap);
  if (elem != kElemF32) {
    b += a(norm_buffer_bytes(Tr, N)) + a(sizeof(float) * N) + a(sizeof(int) * N) + a(sizeof(int)) +
         a(sizeof(double) * kNormMomentsDoubles) + a(sizeof(unsigned));
  }
  return b;
}

void ExecSearch::carve(char* base, int n_partials) {
  auto a = [](size_t x) { return (x + 255) & ~size_t(255); };
  char* p = base;
  top = reinterpret_cast<float*>(p);
  p += a(sizeof(float) * N);
  colsum = reinterpret_cast<float*>(p);
  p += a(sizeof(float) * N);
  sel = reinterpret_cast<SelectState*>(p);
  p += a(sizeof(SelectState));
  partials = reinterpret_cast<MomentPartial*>(p);
  p += a(sizeof(MomentPartial) * n_partials);
  var = reinterpret_cast<double*>(p);
  p += a(sizeof(double) * 2 * kVarChunks);
  work = reinterpret_cast<float*>(p);
  p += a(sizeof(float) * order_work_floats(N));
  lists = reinterpret_cast<int*>(p);
  p += a(sizeof(int) * order_list_entries(N));
  hdr = reinterpret_cast<SearchHeader*>(p);
  p += a(sizeof(SearchHeader));
  cands = reinterpret_cast<Candidate*>(p);
  p += a(sizeof(Candidate) * cand_cap);
  if (elem != kElemF32) {
    norm16 = p;
    p += a(norm_buffer_bytes(Tr, N));
    top16 = reinterpret_cast<float*>(p);
    p += a(sizeof(float) * N);
    flags = reinterpret_cast<int*>(p);
    p += a(sizeof(int) * N);
    flag_count = reinterpret_cast<int*>(p);
    p += a(sizeof(int));
    norm_moments = reinterpret_cast<double*>(p);
    p += a(sizeof(double) * kNormMomentsDoubles);
    norm_ticket = reinterpret_cast<unsigned*>(p);
  }
}

}  // namespace scb
