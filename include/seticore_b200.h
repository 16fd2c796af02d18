/*
 * seticore-b200: C ABI of the B200 dedoppler search.
 *
 * Every entry point returns an int status (SC_DD_OK on success) and never exits the
 * process; sc_dd_last_error() gives the message of the calling thread's last failure.
 * Pointers named dev_* are device-accessible (cudaMalloc'd, managed, or a view into a
 * larger device buffer); other pointers are host memory.  Streams are cudaStream_t
 * values passed as void*; NULL means the legacy default stream, which is the stream
 * the reference runs everything on.
 *
 * Reference interface replaced (lacker/seticore 1.0.6):
 *   class Dedopplerer, dedoppler.h:15-79 and dedoppler.cu:79-320.
 * A header-only C++ class with the reference's signatures sits on top of this ABI in
 * include/seticore_b200/dedoppler.hpp.
 */
#ifndef SETICORE_B200_H
#define SETICORE_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SC_DD_OK = 0,
  SC_DD_EINVAL = 1,    /* bad argument (null pointer, T < 2, N < 64, window size 0) */
  SC_DD_ECUDA = 2,     /* a CUDA runtime call failed */
  SC_DD_ENOMEM = 3,    /* device or pinned allocation failed */
  SC_DD_ETRUNC = 4,    /* more hits than the caller's capacity; *num_hits is the total */
  SC_DD_EINTERNAL = 5, /* a device-side consistency check failed, or a kernel gave up a bounded
                          wait for its staged rows (the results of that call are invalid) */
  SC_DD_ESHAPE = 6,    /* input shape differs from the engine's (dedoppler.cu:191-192) */
  SC_DD_ELIMIT = 7     /* a size exceeds the stated maximum of sc_dd_search_static */
};

#define SC_DD_NO_BEAM (-1) /* dedoppler_hit.h:9 */

/* One hit (dedoppler_hit.h:11-66 without the metadata-derived frequency). */
typedef struct sc_dd_hit {
  int index;              /* start channel within the coarse channel */
  int drift_steps;        /* channels drifted over the rounded-up timesteps */
  double drift_rate;      /* Hz/s: drift_steps * drift_rate_resolution */
  float snr;              /* (power - median) / std_dev of the column sums */
  float power;            /* the path sum */
  float incoherent_power; /* filled by sc_dd_add_incoherent_power, else 0 */
  int coarse_channel;
  int beam;               /* the beam argument of the search */
  int num_timesteps;      /* unrounded timesteps of the engine */
} sc_dd_hit;

/* Statistics of the last search (dedoppler.cu:242-273). */
typedef struct sc_dd_stats {
  float median;
  float std_dev;
  float mean;
  float threshold;
  int window_size;
  int min_drift_block;
  int max_drift_block;
  int num_candidates; /* window maxima above threshold, before the min_drift filter */
  float tree_ms;      /* device time of the Taylor-tree kernel(s), CUDA events on the stream */
  float search_ms;    /* device time of the whole search, first memset to last kernel */
  int precision;          /* SC_DD_PRECISION_* of the search */
  int recomputed_channels; /* precision form: channels whose top was recomputed in FP32 */
  int total_channels;      /* channels of the search */
  int d2h_bytes;           /* bytes the whole call copied device -> host (headers, candidates) */
  double norm_mean;       /* precision form: the FP64 mean that normalised the power (of the
                             first, middle and last unrounded rows) */
  double norm_std;        /* precision form: the FP64 standard deviation used with it */
  int order_exact;        /* 1: median, mean and std_dev were formed in the order the
                             reference's std::nth_element calls leave the column sums, so they
                             are bit-identical to the reference's (searches whose 5 %, 50 % or
                             95 % order statistic sits on a value held by 8 or more column sums,
                             or every search after sc_dd_set_exact_statistics(1)); 0: median and
                             mean exact, the float variance emulated in channel order */
  int pad2;
} sc_dd_stats;

/* Storage of the spectra the tree reads.  FP32: the input as given (the reference's
 * form).  BF16 / FP16: each search first normalises its input per coarse channel,
 * (x - mean) / std with an FP64 mean and std (the arithmetic in float), into a 16-bit copy;
 * the tree accumulates in FP32 over that copy (for 16 and 32 rounded timesteps in FP16
 * pairs of two drift blocks, see sc_dd_set_paired_fp16), every channel whose top could reach
 * the threshold (its 16-bit top reaches the threshold less a bound on the rounding of the
 * normalised values and of the tree's sums) is then recomputed in FP32 from the original
 * power, and the hit list equals the FP32 form's. */
enum { SC_DD_PRECISION_FP32 = 0, SC_DD_PRECISION_BF16 = 1, SC_DD_PRECISION_FP16 = 2 };

typedef struct sc_dd sc_dd;

/* Dedopplerer::Dedopplerer (dedoppler.cu:79-111).  num_timesteps is NOT rounded; the
 * engine processes roundUpToPowerOfTwo(num_timesteps) rows.  Allocates all scratch. */
int sc_dd_create(int num_timesteps, int num_channels, double foff_mhz, double tsamp_s,
                 int has_dc_spike, sc_dd** out);

/* Dedopplerer::~Dedopplerer (dedoppler.cu:113-124). */
int sc_dd_destroy(sc_dd* dd);

/* Dedopplerer::memoryUsage (dedoppler.cu:127-130): device bytes the engine holds. */
size_t sc_dd_memory_usage(const sc_dd* dd);

/* Rounded timesteps (rows the input must have). */
int sc_dd_rounded_timesteps(const sc_dd* dd);

/* Dedopplerer::search (dedoppler.cu:186-320).  dev_input is [rounded T][N] row-major
 * float32; row_stride is the element distance between rows (N for a dense buffer; a
 * larger stride searches a window of a wider buffer in place).  Writes up to
 * `capacity` hits in increasing index order and stores the total in *num_hits
 * (SC_DD_ETRUNC when it exceeds capacity).  Work is ordered on `stream` after what
 * is already queued there; the call returns once the hits are on the host. */
int sc_dd_search(sc_dd* dd, const float* dev_input, long long row_stride, int beam,
                 int coarse_channel, double max_drift, double min_drift,
                 double snr_threshold, sc_dd_hit* out, int capacity, int* num_hits,
                 void* stream);

/* Dedopplerer::search (dedoppler.cu:186-320) for `count` inputs of the engine's shape at
 * once -- e.g. every coarse channel of a band or every beam -- sharing max_drift,
 * min_drift and snr_threshold.  Search k reads dev_inputs[k] with row_strides[k] and
 * reports beams[k] / coarse_channels[k].  Up to 64 searches share each launch of every
 * kernel, and the hits come back with one synchronisation per 64 searches.  Hits are
 * written search after search (each search's in increasing index order); num_hits[k]
 * receives search k's count.  The engine keeps scratch for the largest batch it has run
 * (the first call with a larger count, up to 64, allocates more).
 *
 * Both calls keep CUDA graphs of repeated batches: a batch queued for the second time with the
 * same input pointers and row strides, drift range, threshold, storage form and process-wide
 * settings is captured (on a private stream ordered after `stream`) and later replayed on
 * `stream`, which saves the per-kernel launch cost.  A replay reads the buffers' current
 * contents; at most 8 graphs are kept, and growing the scratch drops them.  The calls
 * synchronise `stream`, so they cannot themselves be captured into a caller's graph. */
int sc_dd_search_batch(sc_dd* dd, int count, const float* const* dev_inputs,
                       const long long* row_strides, const int* beams,
                       const int* coarse_channels, double max_drift, double min_drift,
                       double snr_threshold, sc_dd_hit* out, int capacity, int* num_hits,
                       void* stream);

/* Dedopplerer::addIncoherentPower (dedoppler.cu:139-176) for hits in place: each
 * hit's incoherent_power becomes the path sum of dev_input along the hit's path.
 * Unlike the reference this does not reorder the array (the C++ layer sorts by
 * drift_steps first, as the reference does). */
int sc_dd_add_incoherent_power(sc_dd* dd, const float* dev_input, long long row_stride,
                               sc_dd_hit* hits, int num_hits, void* stream);

/* Selects the storage form of later searches (SC_DD_PRECISION_*).  The 16-bit forms store
 * the normalised power as BF16 or FP16, sum it (in FP32, or in FP16 pairs for 16 and 32
 * rounded timesteps), and recompute in FP32, from the original power, the top of every
 * channel that the rounding bound cannot exclude from the threshold, so their hit lists
 * equal the FP32 form's.  They allocate their scratch on first use. */
int sc_dd_set_precision(sc_dd* dd, int precision);

/* Statistics of the first search of the engine's last completed call; tree_ms and
 * search_ms time its first batch of up to 64 searches. */
int sc_dd_last_stats(const sc_dd* dd, sc_dd_stats* out);

/* Copies an internal per-channel array of the first search of the last call into dst
 * (any memory cudaMemcpy can reach): which = 0 top path sums, 1 column sums, 2 the 16-bit
 * form's approximate tops in normalised units.  N floats. */
int sc_dd_copy_channel_array(sc_dd* dd, int which, float* dst, void* stream);

/* Message of the calling thread's last failed call ("" if none). */
const char* sc_dd_last_error(void);

/* Library version string. */
const char* sc_dd_version(void);

/* Test hook, no counterpart in the reference.  Every tree launch queued after this call
 * polls the mbarrier of its staged rows at most `tries` times before it gives up (tries < 0
 * restores the default, about a second).  A CTA that gives up waits for its copies to land
 * and leaves, and the search reports SC_DD_EINTERNAL.  With 0, every search whose tree
 * stages rows by bulk copies gives up: the tests use this to exercise the give-up path
 * without a fault.  Process-wide; a CUDA graph keeps the limit it was captured with. */
int sc_dd_set_stage_wait_limit(int tries);

/* Tuning and test hook, no counterpart in the reference.  A search of 64 to 256 rounded
 * timesteps runs its first (16-row) level and its last level in stripe passes: each pass
 * writes the planes of a range of channels and a few drift blocks.  bytes > 0 bounds the
 * planes of one pass (narrower passes, which keep their planes in L2 with eviction hints);
 * 0 lets a pass cover whole rows; bytes < 0 restores the default (whole rows, or
 * SETICORE_B200_LEVEL_L2_MB).  Results do not depend on it.  Process-wide; a CUDA graph
 * keeps the passes it was captured with. */
int sc_dd_set_level_stripe_bytes(long long bytes);

/* No counterpart in the reference (which always forms its statistics in one order).
 * mode 0 (the default): a search whose 5 %, 50 % or 95 % order statistic sits on a value held
 * by 8 or more column sums -- integer-valued power, where the order of the reference's float
 * variance sum moves the deviation by up to a few 1e-4 -- gets its statistics in the
 * reference's own std::nth_element order, bit-identical; the others emulate the float sum in
 * channel order (measured 2e-5 to 4e-5 relative on distinct-valued column sums, up to 3e-4
 * on heavy-tailed ones).  mode 1: every search takes the exact order (about 4 ms per batch of
 * 64 searches of 2^20 channels).  Process-wide; launches queued after the call follow it (a
 * CUDA graph keeps the mode it was captured with).  Other modes: SC_DD_EINVAL. */
int sc_dd_set_exact_statistics(int mode);

/* No counterpart in the reference (which has no 16-bit form).  on 1 (the default): the BF16
 * and FP16 forms' searches of 16 or 32 rounded timesteps run their approximate tree in FP16 pairs,
 * two drift blocks per instruction; the flag bound then covers FP16 adds, so a few more
 * channels are recomputed in float32.  on 0: that tree accumulates in float32.  The hit
 * lists are identical either way.  Process-wide; launches queued after the call follow it (a
 * CUDA graph keeps the form it was captured with).  Other values: SC_DD_EINVAL. */
int sc_dd_set_paired_fp16(int on);

/* The device half of H5Reader::loadCoarseChannel (h5_reader.cpp:190-209) for `count`
 * coarse channels laid out item_stride floats apart, each [rounded_timesteps][row_stride]:
 * rows num_timesteps .. rounded_timesteps-1 become zero and, if has_dc_spike, column
 * num_channels/2 of every loaded row becomes (left + right) / 2.  Stream-ordered, one
 * launch, no synchronisation.  The reference does both on the host after the read. */
int sc_dd_prepare_coarse_channels(float* dev_base, int count, long long item_stride, long long row_stride,
                                  int num_timesteps, int rounded_timesteps, int num_channels,
                                  int has_dc_spike, void* stream);

/* The filterbank slices stored with hits in .hits files (hit_file_writer.cpp:81-96):
 * for k < count, rows [0, num_timesteps) and columns [dev_ranges[2k], dev_ranges[2k+1])
 * of dev_input go, row-major, to dev_out + dev_offsets[k].  All arrays are device memory;
 * one launch, no synchronisation.  The reference copies each slice on the host. */
int sc_dd_gather_columns(const float* dev_input, long long row_stride, int num_timesteps, int num_channels,
                         const int* dev_ranges, const long long* dev_offsets, int count, float* dev_out,
                         void* stream);

/* ---- Heterogeneous batches: many searches of different shapes at once ---- */

/* One search request: its input, the shape sc_dd_create would take, and the arguments
 * of Dedopplerer::search (dedoppler.h:42-45), plus its storage precision. */
typedef struct sc_dd_request {
  const float* dev_input; /* [rounded T][N] float32, row_stride elements between rows */
  long long row_stride;
  int num_timesteps;      /* unrounded */
  int num_channels;
  double foff_mhz;
  double tsamp_s;
  double max_drift;
  double min_drift;
  double snr_threshold;
  int beam;
  int coarse_channel;
  int precision;          /* SC_DD_PRECISION_* */
  int pad;
} sc_dd_request;

typedef struct sc_dd_pool_stats {
  long long calls;
  long long sub_batches;     /* admitted groups of requests that fit the scratch budget */
  long long graph_replays;   /* sub-batches replayed from a captured CUDA graph */
  long long graph_captures;
  long long tuned_launches;  /* autotuning decisions taken (tree launches, level splits) */
  float last_call_ms;        /* device time of the last call, CUDA events */
  int pad;
} sc_dd_pool_stats;

typedef struct sc_dd_pool sc_dd_pool;

/* A pool runs lists of requests of any mix of shapes: requests are admitted in order
 * into sub-batches whose scratch fits scratch_budget_bytes (one request always fits:
 * the pool grows its arena for a larger one), every kernel runs once per sub-batch of up
 * to 64 searches, tree launches and level splits are autotuned on first sight, and a
 * sub-batch seen again is replayed from a captured CUDA graph.  No counterpart in the
 * reference (which runs one search at a time). */
int sc_dd_pool_create(size_t scratch_budget_bytes, sc_dd_pool** out);
int sc_dd_pool_destroy(sc_dd_pool* pool);
/* autotune / cuda_graphs: 1 (default) or 0. */
int sc_dd_pool_configure(sc_dd_pool* pool, int autotune, int cuda_graphs);
/* Runs the requests; hits are written request after request (each in increasing index
 * order) and num_hits[i] receives request i's count.  Returns after the hits are on the
 * host; work is ordered on `stream`. */
int sc_dd_pool_search(sc_dd_pool* pool, const sc_dd_request* requests, int count,
                      sc_dd_hit* out, int capacity, int* num_hits, void* stream);
int sc_dd_pool_stats_get(const sc_dd_pool* pool, sc_dd_pool_stats* out);
/* Device scratch bytes one request needs in a pool (0 for an invalid request). */
size_t sc_dd_request_scratch_bytes(const sc_dd_request* request);
/* Message of the calling thread's last failed pool call. */
const char* sc_dd_pool_last_error(void);

/* Largest channel count sc_dd_search_static accepts. */
#define SC_DD_STATIC_MAX_CHANNELS 1048576

/* The search, for callers that cannot allocate device memory where they search -- e.g. a
 * real-time capture or beamforming pipeline that reserved the GPU's memory up front and
 * must not call cudaMalloc (which can synchronise the device) in its processing loop, or a
 * host framework whose allocator owns all device memory.  No counterpart in the
 * reference; it has no engine object.
 *
 * Same inputs, results and ordering as sc_dd_search, plus the shape (unrounded
 * num_timesteps, num_channels, foff in MHz, tsamp in s) that sc_dd_create would take.
 * It calls no cudaMalloc, cudaFree, cudaMallocHost or other allocating routine: its scratch
 * is one fixed device array inside the library (22.8 MB, held by every GPU that loads
 * the library until the process exits) and its host side uses the stack and `out`.
 * Limits (SC_DD_ELIMIT beyond them): num_channels <= SC_DD_STATIC_MAX_CHANNELS, rounded
 * timesteps <= 16, at most 65536 windows (num_channels / window_size).  A max_drift that is
 * not finite, or whose drift range exceeds sc_dd_search's bound, is SC_DD_EINVAL.  Errors are status
 * codes only (sc_dd_last_error is not updated).
 *
 * The array is shared by every call on a device and keeps the last call's contents; each
 * call clears what must start at zero.  Calls that overlap on the GPU -- on different
 * streams, or from different host threads -- race on it and must be serialised by the
 * caller.  The first call on each device looks up the array's device address (with that
 * device current) and caches it; make that first call before any stream capture.  Every
 * call copies its results to the host and synchronizes `stream` before it returns.  On
 * SC_DD_ETRUNC, *num_hits is the total and the hits written are not necessarily the
 * lowest-index ones. */
int sc_dd_search_static(const float* dev_input, long long row_stride, int num_timesteps,
                        int num_channels, double foff_mhz, double tsamp_s, int beam,
                        int coarse_channel, double max_drift, double min_drift,
                        double snr_threshold, sc_dd_hit* out, int capacity, int* num_hits,
                        void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SETICORE_B200_H */
