// Internal host/device interfaces between the seticore-b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace scb {

constexpr int kMaxSeg = 4;       // staged windows per tree work item when jobs have their own rows
constexpr int kMaxBatch = 64;    // searches per batched launch (descriptors travel as kernel parameters)
constexpr int kVarChunks = 1024; // variance-emulation chunks per search, at most
// The 16-bit forms' moments buffer per search (doubles): per-block sums [0, K), sums of
// squares [K, 2K), then the normalisation's mean and standard deviation and the minimum and
// maximum of the unrounded rows at 2K .. 2K + 3, then per-block (minimum, maximum) pairs
// from 2K + 4.
constexpr int kNormMomentsDoubles = 4 * kVarChunks + 4;

// Element types of a tree launch's input.
constexpr int kElemF32 = 0;
constexpr int kElemBF16 = 1;
constexpr int kElemF16 = 2;

constexpr int kSelBins = 4096;   // histogram bins per order-statistic pass
constexpr int kSelCands = 4096;  // candidates kept per order statistic for the exact pick

// Order-statistic state for the three column-sum ranks (first, mid, last).  Each target's
// key range narrows by histogram passes until it holds one key (mode 2) or at most kSelCands
// values (mode 1), which a compaction pass collects for an exact pick.  Keys are the
// order-preserving unsigned images of the floats (sel_key: -0 keyed as +0).
struct SelectState {
  uint32_t prefix[3];  // the selected keys, once known (read by the variance kernels)
  uint32_t lo[3];      // current range of each target: [lo, lo + 2^wshift)
  uint32_t wshift[3];
  uint32_t rank[3];    // rank of the target inside its range
  uint32_t count[3];   // values inside the range
  uint32_t mode[3];    // 0: narrow further, 1: pick from candidates, 2: exact (one key)
  uint32_t ncand[3];
  uint32_t kmin, kmax;
  unsigned ticket;
  // filled by the order-statistic finaliser for the variance kernels
  float mean;
  int pad;
  long long n_lo, n_hi, n;
  unsigned hist[3][kSelBins];
  uint32_t cand[3][kSelCands];
};

#ifdef __CUDACC__
// Resets the order-statistic state of one search; run by every thread of one block.
__device__ __forceinline__ void reset_select(SelectState* st, int first, int mid, int last) {
  if (threadIdx.x < 3) {
    const int j = threadIdx.x;
    st->prefix[j] = 0;
    st->lo[j] = 0;
    st->wshift[j] = 0;
    st->rank[j] = (uint32_t)(j == 0 ? first : (j == 1 ? mid : last));
    st->count[j] = 0;
    st->mode[j] = 0;
    st->ncand[j] = 0;
  }
  if (threadIdx.x == 0) {
    st->kmin = 0xffffffffu;
    st->kmax = 0u;
    st->ticket = 0;
  }
  for (int i = threadIdx.x; i < 3 * kSelBins; i += blockDim.x) (&st->hist[0][0])[i] = 0;
}
#endif

struct MomentPartial {
  double s1, s2;  // s2 unused (kept for layout)
  unsigned long long lt_first, eq_first, lt_last, eq_last;
};

// A confirmed window maximum: channel and top sum, plus the best path found by the resolve
// kernel, packed as (order key of the sum) << 32 | ~(path number) so that one 64-bit
// atomicMax keeps the largest sum and, among equal sums, the first path.
struct Candidate {
  int index;
  int drift_steps;  // decoded from `best` on the host
  float power;
  int flags;
  unsigned long long best;
};

// Device-side result block of one search; the candidates follow it in memory.
struct SearchHeader {
  int num_candidates;
  int error;  // nonzero: a kernel of the search gave up a wait (the results are invalid)
  int order_exact;  // 1: the statistics were formed in the reference's nth_element order
  int ties;         // most copies of one value among the three order statistics' values
  float median, std_dev, mean, threshold;
};

// Everything the batched kernels need to know about one search.
struct SearchDesc {
  const float* input;
  long long row_stride;
  int Tr, N;
  int dmin, dmax, window_size;
  int first, mid, last;  // order-statistic ranks: ceil(0.05 N), N/2, floor(0.95 N)
  double snr_threshold;
  float* top;
  float* colsum;
  SelectState* sel;
  MomentPartial* partials;  // at least as many as the statistics grid's x dimension
  double* var;              // 2 * kVarChunks
  float* work;              // order_work_floats(N): the column sums in nth_element order
  int* lists;               // order_list_entries(N): the swap pairs of a partition step
  SearchHeader* hdr;
  Candidate* cands;
  int cand_cap;
  int pad;
};

struct SearchBatch {
  int count;
  int maxN;
  SearchDesc s[kMaxBatch];
};

// One group of tree jobs (normally the drift blocks of one search): job k reads R rows
// starting at rows + k*job_row_stride (row stride row_stride), sheared by
// d_first + k*d_step channels per row; it is drift block db_first + k*db_step of its
// search and its in-block offset r is path offset off_base + k*off_step + r; eligibility
// uses elig_T1 = rounded timesteps - 1.  The launcher fills the scheduling fields.
struct TreeGroup {
  const void* rows;          // elements of the launch's element type
  long long row_stride;
  long long job_row_stride;  // 0: all jobs read the same rows (one shared trapezoid)
  int N;
  int d_first;
  int d_step;
  int n_jobs;
  int db_first;
  int db_step;
  int off_base;
  int off_step;
  int elig_T1;
  float* top;
  // Optional column sums (sumColumns, dedoppler.cu:63-72): the CTA staging the chunk that
  // holds job colsum_job -- the job whose shear is zero, so its window of every row covers
  // the tile's own channels -- writes colsum[c] = x[0][c] + x[1][c] + ... in row order.
  float* colsum;
  int colsum_job;
  // Emitting launches (tree_emit_batch): root offset r of job k at channel c goes to
  // emit_out[k * emit_job_stride + r * emit_plane_stride + c]; top is unused.
  float* emit_out;
  long long emit_job_stride;
  long long emit_plane_stride;
  // Optional channel range of the group's tiles: the tiles that cover [x_begin, x_end), with
  // x_begin a multiple of the launch's tile width (x_end == 0: every tile of [0, N); x_end < 0:
  // none).
  int x_begin;
  int x_end;
  int jobs_per_chunk;
  int n_chunks;
  int n_tiles;
  int tile_first;
  int item_begin;  // first work item of this group in the launch
  // Optional: set to 1 if a staging wait of the tree gave up (its results are then invalid).
  int* status;
  // Elements before channel 0 that the rows hold (read as data, not as zeros): kPairPad for
  // the paired-FP16 copy, 0 otherwise.
  int pad;
};

struct TreeBatch {
  int count;
  int n_items;
  // Polls of the staging wait before a CTA gives up (negative: the default, about a second).
  // The launcher fills it from stage_wait_tries().
  int stage_wait_tries = -1;
  // L2 hints of the bulk copies: 0 none; 1 (stripe passes' first level) staged input rows
  // evict-first and emitted planes evict-last, so the planes stay in L2 for the last level.
  int cache_mode = 0;
  // 1: the groups are the paired copies of 16-bit 16- or 32-row searches, run by the
  // paired-FP16 tree (two drift blocks per unit, FP16 sums; the precision form's flag bound
  // then takes FP16 adds).
  int pair16 = 0;
  TreeGroup g[kMaxBatch];
};

// Whether 16-bit 16- and 32-row searches queued from now on take the paired-FP16 tree (default
// on; off: the float-accumulating 16-bit tree).  The hit lists are the same either way.
void set_paired_fp16(bool on);
bool paired_fp16();

// The staging-wait poll limit of tree launches queued from now on (negative: the default).
// Tests set 0 to make every staged item give up, which exercises the give-up path (the
// search then reports SC_DD_EINTERNAL) without any fault.
void set_stage_wait_tries(int tries);
int stage_wait_tries();

// Launch shape of a tree launch.  smem_kb bounds the shared memory of a CTA (0: the
// default), which sets how many drift blocks share a staged trapezoid and how many CTAs fit
// an SM; tile is the channels per work item, 1056 or 352 (0: 1056 for jobs that share their
// rows, 352 for jobs with their own rows).
struct TreeLaunch {
  int smem_kb = 0;
  int tile = 0;
};

// Fused tree + per-channel top for the groups (all of R rows, elements of type `elem`).
// The launcher fills the scheduling fields of `b` in place.
cudaError_t tree_max_batch(TreeBatch& b, int R, int num_sms, cudaStream_t stream, int elem = kElemF32,
                           TreeLaunch how = TreeLaunch{});

// The same staged tree for 16 rows, writing every root value (all 16 in-block offsets of
// every channel) to the groups' emit planes instead of folding maxima: the first level of
// a tree of more than 32 rows.  Values of paths that leave [0, N) are sums with zeros.
// Every 352-channel tile is stored whole, so plane rows must hold level_row_length(N)
// floats.  nparts: the offsets in two halves of eight (2) or all sixteen in one warp (1).
// Float rows only.
cudaError_t tree_emit_batch(TreeBatch& b, int num_sms, cudaStream_t stream, int smem_budget_kb = 0, int nparts = 2);

// Channels per tree work item (the tile a flag refers to).
int tree_tile_width();

// Row length of the level planes (N rounded up to whole tiles) and the floats one level
// buffer holds for a search of Tr rounded timesteps: levels_search needs two such buffers
// in one allocation (scratch_b = scratch_a + level_buffer_floats).
inline long long level_row_length(int N) {
  const long long w = tree_tile_width();
  return (N + w - 1) / w * w;
}
// The slack of each row covers the stripe passes' per-row channel origins and shears (up to
// four drift blocks of a last level of up to 16 rows, dd_levels.cu), so the two level
// buffers hold a whole-row pass of two drift blocks.
constexpr long long kLevelRowSlack = 2048;
// The paired-FP16 copy of a 16- or 32-row search (the 16-bit forms' paired tree): row t
// holds, for channel x in [-kPairPad, N), the word (y[t][x], y[t][x + t]) as two FP16 values
// (0 outside [0, N)), kPairPad words before channel 0 (at least the largest shift, 31) and
// rows pair_row_words(N) words apart.
constexpr int kPairPad = 32;
inline long long pair_row_words(int N) { return ((long long)N + kPairPad + 3) / 4 * 4; }
inline bool pair_rows(int Tr) { return Tr == 16 || Tr == 32; }
// Bytes of a search's normalised copy: the dense 16-bit [Tr][N] copy, or for 16 and 32 rows
// room for the paired copy as well (whichever the paired-FP16 setting picks at launch).
inline size_t norm_buffer_bytes(int Tr, int N) {
  const size_t dense = (size_t)2 * Tr * N;
  const size_t paired = pair_rows(Tr) ? (size_t)4 * Tr * (size_t)pair_row_words(N) : 0;
  return dense > paired ? dense : paired;
}

inline size_t level_buffer_floats(int Tr, int N) {
  return (size_t)Tr * (size_t)(level_row_length(N) + kLevelRowSlack);
}

// Precision form (dd_precision.cu), per search of a batch:
struct PrecisionDesc {
  const float* input;   // original float32 power [Tr][N], row stride row_stride
  long long row_stride;
  int T, Tr, N;         // unrounded and rounded timesteps, channels
  void* norm;           // normalised 16-bit copy [Tr][N] (dense)
  float* colsum;        // column sums of the float32 power, formed by the normalising pass
  double* moments;      // kNormMomentsDoubles: partials, [mean, std, min, max], partial extremes
  unsigned* ticket;
  const float* top16;   // tops of the 16-bit tree (normalised units)
  const SearchHeader* hdr;
  double snr_threshold;
  int dmin, dmax;       // drift blocks
  float* top;           // exact float32 tops of the flagged channels (others stay 0)
  int* flag_list;       // flagged channels (capacity N)
  int* flag_count;
  int pair16;           // 1: norm holds the paired-FP16 copy and the tops come from the
                        // paired-FP16 tree (FP16 adds)
};
struct PrecisionBatch {
  int count;
  int maxN;
  int elem;             // kElemBF16 or kElemF16
  PrecisionDesc s[kMaxBatch];
};
// FP64 mean and standard deviation of the unrounded rows, then the normalised copy.
cudaError_t normalize_batch(const PrecisionBatch& b, int num_sms, cudaStream_t stream);
// Lists every channel whose 16-bit top reaches the threshold less the rounding bound
// (dd_precision.cu, flag_threshold): every channel whose exact top can reach it.
cudaError_t flag_channels_batch(const PrecisionBatch& b, int num_sms, cudaStream_t stream);
// The exact float32 top of every listed channel: each eligible path summed from the
// original power in the tree's pairing, the maximum floored at 0.
cudaError_t recompute_batch(const PrecisionBatch& b, int num_sms, cudaStream_t stream);

// Column sums of each search (searches whose tree computes them skip this); also resets
// each search's order-statistic state.
cudaError_t column_sums_batch(const SearchBatch& b, cudaStream_t stream);
// Order statistics, mean, standard deviation and threshold of each search, from its column
// sums and a reset select state (column_sums_batch or exec_queue's clear launch): the
// order statistics exactly and the float variance emulated in channel order (dd_stats.cu),
// then, for the searches whose order statistics sit on repeated values, everything again
// in the reference's own nth_element order, bit-identical (dd_order.cu).
cudaError_t search_stats_batch(const SearchBatch& b, int num_sms, cudaStream_t stream);
cudaError_t search_stats_emulated(const SearchBatch& b, int num_sms, cudaStream_t stream);
cudaError_t search_stats_exact(const SearchBatch& b, int num_sms, cudaStream_t stream);
// The exact statistics run for a search whose three order statistics' values include one
// held by at least this many column sums (automatic mode), or for every search.
constexpr int kExactStatsTies = 8;
void set_exact_statistics_always(bool always);
bool exact_statistics_always();
// Scratch of the exact statistics per search of N channels: the work array (N floats,
// padded so that 16-byte loads of a range's last group stay inside it) and the pair lists
// (two halves, one per end of the array, for the two nth_element calls that run side by side).
#ifdef __CUDACC__
#define SCB_HD __host__ __device__
#else
#define SCB_HD
#endif
SCB_HD constexpr size_t order_work_floats(int N) { return ((size_t)N + 7) & ~(size_t)3; }
// One std::nth_element call of the exact statistics while its range is partitioned by
// multi-CTA rounds (dd_order.cu); three per search, after the pair lists.
constexpr int kOrderMaxSegs = 2048;  // counting segments of one partition step
struct OrderTask {
  int first, last, nth, depth;  // the call's current range, its target and depth budget
  int sfirst, slast;            // the range of the partition step in progress
  int active;                   // 1: the rounds partition this call; 0: its finisher does the rest
  int error;
  int K, cut, lk, rk;           // pairs, cut, K-th value >= pivot, (K-1)-th value <= pivot
  unsigned ticket;              // CTAs of a round done so far
  float pivot;
  int nseg, seglen;
  int seg_ge[kOrderMaxSegs + 1];  // per segment: values >= pivot, then the exclusive prefix
  int seg_le[kOrderMaxSegs + 1];
};
SCB_HD constexpr size_t order_pair_entries(int N) { return 8 * ((size_t)N / 4 + 2); }
SCB_HD constexpr size_t order_list_entries(int N) {
  return order_pair_entries(N) + 3 * (sizeof(OrderTask) / sizeof(int)) + 64;
}

// Window de-duplication (dedoppler.cu:264-303) and drift recovery of the survivors.
cudaError_t search_hits_batch(const SearchBatch& b, int num_sms, cudaStream_t stream);

// Path sums along the given (index, drift_steps) paths: addIncoherentPower.
cudaError_t path_values(const float* input, long long row_stride, int Tr, int N, const int* index,
                        const int* drift_steps, float* out, int n, cudaStream_t stream);

// How a tree of more than 32 rows is split: levels of m[0..n) rows each -- 2 or 4
// (emit_kernel), 8 or 16 (direct_kernel, one thread per channel) or, first only,
// kStreamEmit16 (the emitting form of the fused tree) -- then a fused max level of
// final_rows (2, 4, 8 or 16) rows.  n == 0: the default split.
constexpr int kStreamEmit16 = 1016;
constexpr int kStreamEmit16One = 1017;  // the emitting form with all sixteen offsets in one warp
struct LevelPlan {
  int n;
  int m[12];
  int final_rows;
};

// L2 budget of one stripe pass of the one-level split (bytes; negative: the default).
void set_level_stripe_bytes(long long bytes);
long long level_stripe_bytes();  // the value set (negative: none)

// Multi-level tree for Tr > 32 (one search): level kernels write the partial planes of
// every sub-problem, then the fused max kernel finishes them (see dd_levels.cu).
// scratch_a / scratch_b: level_buffer_floats(Tr, N) floats each, in one allocation.
// `input` holds elements of type `elem` (float, or the precision form's 16-bit copy, which
// only the default plan reads: its first level converts on load).
cudaError_t levels_search(const void* input, long long row_stride, int Tr, int N, int dmin, int dmax,
                          float* scratch_a, float* scratch_b, float* top, int num_sms,
                          cudaStream_t stream, const LevelPlan& plan = LevelPlan{}, int elem = kElemF32,
                          int* status = nullptr);

// A fully planned search for exec_queue: the request, its drift plan and its scratch.
struct ExecSearch {
  const float* input;
  long long row_stride;
  int T, Tr, N;
  int dmin, dmax, window_size;
  double snr_threshold;
  int elem;  // kElemF32, or the 16-bit storage of the precision form
  LevelPlan level_plan;
  int cand_cap;
  // scratch (carve() lays it out from one base pointer)
  float* top;
  float* colsum;
  SelectState* sel;
  MomentPartial* partials;
  double* var;
  float* work;
  int* lists;
  SearchHeader* hdr;
  Candidate* cands;
  void* norm16;
  float* top16;
  int* flags;       // flagged channels (N)
  int* flag_count;
  double* norm_moments;
  unsigned* norm_ticket;
  static size_t scratch_bytes(int Tr, int N, int cand_cap, int n_partials, int elem);
  void carve(char* base, int n_partials);
};

// Callbacks of exec_queue: the launch shape of each tree launch (autotuning) and points at
// which the caller may record events.
struct ExecHooks {
  void* ctx = nullptr;
  TreeLaunch (*tree_launch)(void* ctx, const TreeBatch& tb, int R, int elem) = [](void*, const TreeBatch&, int,
                                                                                   int) { return TreeLaunch{}; };
  // The level split of a search with more than 32 rows (may time alternatives first).
  LevelPlan (*level_plan)(void* ctx, const ExecSearch& s, float* lvl_a, float* lvl_b, cudaStream_t st) = nullptr;
  void (*before_tree)(void* ctx, cudaStream_t s) = nullptr;
  void (*after_tree)(void* ctx, cudaStream_t s) = nullptr;
};

// Up to kLevelSides more streams, each with its own pair of level buffers (the same size as
// the first pair, in one allocation), a fork event and join events: exec_queue then deals the
// FP32 searches of more than 32 rows round-robin over the main stream and the side streams,
// forked from and joined back into the main stream, so that the level kernels of several
// searches share the SMs (they are bound by latency, with shared memory and registers the
// respective limits).
constexpr int kLevelSides = 3;
struct LevelSide {
  int n = 0;  // side streams in use
  cudaStream_t stream[kLevelSides] = {};
  float* lvl_a[kLevelSides] = {};
  float* lvl_b[kLevelSides] = {};
  cudaEvent_t fork = nullptr;
  cudaEvent_t join[kLevelSides] = {};
};
// Side streams an engine (engine = true) or a pool creates: SETICORE_B200_LEVEL_SIDES, 0 to 3;
// by default 3 for an engine and 1 for a pool.
int level_sides(bool engine);

// Queues every kernel of n searches (any mix) on `stream`; no synchronisation.
// lvl_a / lvl_b: level buffers of level_buffer_floats(Tr, N) floats for every search with
// Tr > 32, in one allocation.  side: optional side streams for the level path.
cudaError_t exec_queue(const ExecSearch* s, int n, float* lvl_a, float* lvl_b, int num_sms, cudaStream_t stream,
                       const ExecHooks& hooks, const LevelSide* side = nullptr);

// Decodes a resolved candidate: returns false if the recovered path sum does not equal the
// stored top sum (a consistency failure).  Paths are numbered (db - dmin) * Tr + off.
inline bool decode_candidate(const Candidate& c, int dmin, int Tr, int* drift_steps) {
  if (c.best == 0ull) {  // no path sum above zero: the reference keeps no drift for it
    *drift_steps = 0;
    return true;
  }
  const uint32_t hi = (uint32_t)(c.best >> 32);
  const uint32_t p = ~(uint32_t)(c.best & 0xffffffffull);
  const uint32_t fbits = (hi & 0x80000000u) ? (hi & 0x7fffffffu) : ~hi;
  uint32_t pbits;
  __builtin_memcpy(&pbits, &c.power, 4);
  const int db = dmin + (int)(p / (uint32_t)Tr);
  const int off = (int)(p % (uint32_t)Tr);
  *drift_steps = db * (Tr - 1) + off;
  return fbits == pbits;
}

}  // namespace scb
