// Internal host/device interfaces between the seticore-b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace scb {

// One fused tree launch: jobs k = 0..n_jobs-1 read R rows starting at
// rows + k*job_row_stride (row stride row_stride elements), sheared by d_first + k*d_step
// channels per row.  Job k is drift
// block db_first + k*db_step of the search and its in-block offset r is path offset
// off_base + k*off_step + r; eligibility uses elig_T1 = rounded timesteps - 1.
constexpr int kMaxSeg = 4;

struct TreeParams {
  const float* rows;
  long long row_stride;
  long long job_row_stride;  // 0: all jobs read the same rows; else job k reads rows + k*this
  int N;
  int d_first;
  int d_step;                // job k is sheared by d_first + k*d_step channels per row
  int n_jobs;
  int db_first;
  int db_step;
  int off_base;
  int off_step;
  int elig_T1;
  float* top;
  // filled by the launcher
  int jobs_per_chunk;
  int n_chunks;
  int n_tiles;
};

cudaError_t tree_max(const TreeParams& p, int R, int num_sms, cudaStream_t stream);

}  // namespace scb

namespace scb {

// Radix-select state for the three column-sum order statistics (first, mid, last).
struct SelectState {
  uint32_t prefix[3];
  uint32_t mask[3];
  uint32_t rank[3];
  unsigned ticket;
  unsigned hist[3][256];
  // filled by moments_kernel for the variance kernels
  float mean;
  int pad;
  long long n_lo, n_hi, n;
};

// Variance emulation scratch: per-chunk sums of the squared deviations and per-chunk
// emulated contributions (kVarChunks entries each).
constexpr int kVarChunks = 1024;

struct MomentPartial {
  double s1, s2;  // s2 unused (kept for layout)
  unsigned long long lt_first, eq_first, lt_last, eq_last;
};

// A confirmed window maximum: channel, drift (filled by the resolve kernel), power.
struct Candidate {
  int index;
  int drift_steps;
  float power;
  int flags;  // 1 = drift resolved
};

// Device-side result block of one search; the candidates follow it in memory.
struct SearchHeader {
  int num_candidates;
  int error;  // nonzero: a device-side consistency check failed
  int pad0, pad1;
  float median, std_dev, mean, threshold;
};

cudaError_t search_stats(const float* input, long long row_stride, int Tr, int N, float* colsum,
                         SelectState* st, MomentPartial* partials, int n_partials, double* var_scratch,
                         double snr_threshold, SearchHeader* hdr, int num_sms, cudaStream_t stream);

// Window de-duplication (dedoppler.cu:353-383) and drift recovery of the survivors.
cudaError_t search_hits(const float* input, long long row_stride, int Tr, int N, const float* top,
                        int window_size, int dmin, int dmax, SearchHeader* hdr, Candidate* cands,
                        int cand_capacity, int num_sms, cudaStream_t stream);

// Path sums along the given (index, drift_steps) paths: addIncoherentPower.
cudaError_t path_values(const float* input, long long row_stride, int Tr, int N, const int* index,
                        const int* drift_steps, float* out, int n, cudaStream_t stream);

// Multi-level tree for Tr > 16: level kernels write the partial planes of every
// problem, then the last level runs the fused max kernel (see dd_levels.cu).
cudaError_t levels_search(const float* input, long long row_stride, int Tr, int N, int dmin, int dmax,
                          float* scratch_a, float* scratch_b, float* top, int num_sms,
                          cudaStream_t stream);

}  // namespace scb
