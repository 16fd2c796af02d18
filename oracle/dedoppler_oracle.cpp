// Oracle for the seticore dedoppler search.  TEST INFRASTRUCTURE ONLY.
//
// This file restates, on the CPU, the algorithm of seticore's Dedopplerer::search
// (dedoppler.cu:186-320), its Taylor tree (taylor.cu:116-156 schedule, recursion
// taylor.h:30-86), findTopPathSums (dedoppler.cu:32-55), sumColumns (dedoppler.cu:63-72)
// and addIncoherentPower (dedoppler.cu:139-176).  It is used only by the test suite,
// by __graft_entry__.smoke() to check its result, and by bench.py's CPU-baseline leg.
// The product path (seticore_b200/) never links, loads or calls it.
//
// Built two ways (oracle/Makefile):
//   * liboracle.so    -- every step restated here (the "port").
//   * libref_cpu.so   -- ORACLE_USE_REFERENCE_TAYLOR: each tree step calls the
//                        reference's own __host__ __device__ taylorOneStepOneChannel
//                        (taylor.h:30-86) compiled for the host from the reference
//                        sources; the remaining host logic is the restatement below.
//
// Parity pins: tests/test_oracle.py checks this code against the reference's own unit
// tests (taylor_test.cu:8-51 and dedoppler_test.cpp:9-33) and against golden vectors
// produced by the reference's own code (tests/golden/make_golden.py).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <numeric>
#include <type_traits>
#include <vector>

#ifdef ORACLE_USE_REFERENCE_TAYLOR
#include <cuda_runtime.h>
#include "taylor.h"   // the reference's header, from the reference tree
#endif

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// util.cpp:16-22 (roundUpToPowerOfTwo)
int round_up_pow2(int n) {
  int r = 1;
  while (r < n) r *= 2;
  return r;
}

// One recursion step of the Taylor tree for every channel (taylor.h:30-86 restated,
// looping channel-innermost so the compiler vectorises it).  Writes only the entries
// whose second operand is in range; others keep their previous contents.
template <typename F>
void tree_step(const F* src, F* tgt, int T, int N, int L, int db) {
#ifdef ORACLE_USE_REFERENCE_TAYLOR
  if constexpr (std::is_same<F, float>::value) {
#pragma omp parallel for schedule(static)
    for (int chan = 0; chan < N; ++chan) {
      taylorOneStepOneChannel(src, tgt, chan, T, N, N, L, db);
    }
    return;
  }
#endif
  const int num_blocks = T / L;
  for (int tb = 0; tb < num_blocks; ++tb) {
    for (int off = 0; off < L; ++off) {
      const int half = off / 2;
      const int shift = (off + 1) / 2 + db * L / 2;
      const F* a = src + (size_t)(tb * L + half) * N;
      const F* b = src + (size_t)(tb * L + half + L / 2) * N;
      F* o = tgt + (size_t)(tb * L + off) * N;
      const int c0 = std::max(0, -shift);
      const int c1 = std::min(N, N - shift);
#pragma omp parallel for schedule(static)
      for (int c = c0; c < c1; ++c) o[c] = a[c] + b[c + shift];
    }
  }
}

// basicTaylorTree (taylor.cu:116-156): returns the buffer holding out[off][c].
template <typename F>
const F* taylor_tree(const F* input, F* buf1, F* buf2, int T, int N, int db) {
  const F* src = input;
  F* tgt = buf1;
  for (int L = 2; L <= T; L *= 2) {
    tree_step<F>(src, tgt, T, N, L, db);
    src = tgt;
    tgt = (tgt == buf1) ? buf2 : buf1;
  }
  return src;
}

// Path geometry of the recursion: channel offset at row t of the path with
// in-block offset `off` over L rows (taylor.h:48-54: halves share off/2, the second
// half starts (off+1)/2 to the right).
int path_pos(int off, int L, int t) {
  int p = 0;
  while (L > 1) {
    const int half = L / 2;
    if (t >= half) {
      p += (off + 1) / 2;
      t -= half;
    }
    off /= 2;
    L = half;
  }
  return p;
}

}  // namespace

extern "C" {

typedef struct oracle_hit {
  int index;
  int drift_steps;
  double drift_rate;
  float snr;
  float power;
} oracle_hit;

typedef struct oracle_stats {
  float median;
  float std_dev;
  float mean;
  float threshold;
  int window_size;
  int min_drift_block;
  int max_drift_block;
  double drift_rate_resolution;
} oracle_stats;

void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

int oracle_max_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Full Taylor tree for one drift block: out[off*N + c].  Entries for invalid paths
// (last channel out of range, taylor.h:17-22) are NaN.
void oracle_taylor_f32(const float* input, int T, int N, int db, float* out) {
  std::vector<float> b1((size_t)T * N, std::numeric_limits<float>::quiet_NaN());
  std::vector<float> b2((size_t)T * N, std::numeric_limits<float>::quiet_NaN());
  if (T == 1) {
    std::memcpy(out, input, sizeof(float) * N);
    return;
  }
  const float* r = taylor_tree<float>(input, b1.data(), b2.data(), T, N, db);
  for (int off = 0; off < T; ++off)
    for (int c = 0; c < N; ++c) {
      const long last = (long)(T - 1) * db + off + c;
      out[(size_t)off * N + c] =
          (last < 0 || last >= N) ? std::numeric_limits<float>::quiet_NaN()
                                  : r[(size_t)off * N + c];
    }
}

// FP64 twin: the same geometry and tree order with double accumulation.
void oracle_taylor_f64(const float* input, int T, int N, int db, double* out) {
  std::vector<double> in((size_t)T * N);
  for (size_t i = 0; i < in.size(); ++i) in[i] = input[i];
  std::vector<double> b1(in.size(), std::numeric_limits<double>::quiet_NaN());
  std::vector<double> b2(in.size(), std::numeric_limits<double>::quiet_NaN());
  const double* r = taylor_tree<double>(in.data(), b1.data(), b2.data(), T, N, db);
  for (int off = 0; off < T; ++off)
    for (int c = 0; c < N; ++c) {
      const long last = (long)(T - 1) * db + off + c;
      out[(size_t)off * N + c] =
          (last < 0 || last >= N) ? std::numeric_limits<double>::quiet_NaN()
                                  : r[(size_t)off * N + c];
    }
}

// One path sum, pairwise in tree order (bit-identical to the tree's value).
float oracle_path_sum(const float* input, int T, int N, int db, int off, int c) {
  float stack[32];
  int depth = 0;
  for (int t = 0; t < T; ++t) {
    float v = input[(size_t)t * N + c + db * t + path_pos(off, T, t)];
    int k = t;
    while (k & 1) {
      v = stack[--depth] + v;
      k >>= 1;
    }
    stack[depth++] = v;
  }
  return stack[0];
}

// Dedopplerer::search restated.  input is [Tr][N] row-major, Tr = rounded timesteps.
// Optional outputs (may be null): top_sums/top_db/top_off/colsums of length N.
// Returns the number of hits (all of them; at most `cap` are written), or -1 for an
// argument the reference cannot handle (window size 0 makes its scan loop forever).
int oracle_search(const float* input, int Tr, int N, double foff, double tsamp,
                  double max_drift, double min_drift, double snr_threshold,
                  oracle_hit* hits, int cap, float* top_sums_out, int* top_db_out,
                  int* top_off_out, float* colsums_out, oracle_stats* stats) {
  const int drift_timesteps = Tr - 1;                                   // dedoppler.cu:165
  const double res = 1e6 * foff / (drift_timesteps * tsamp);            // dedoppler.cu:87
  const double diag = res * drift_timesteps;                            // dedoppler.cu:195
  const double nmax = max_drift / std::abs(diag);                       // dedoppler.cu:196
  const int dmin = (int)std::floor(-nmax);
  const int dmax = (int)std::floor(nmax);

  // sumColumns (dedoppler.cu:63-72): sequential float sum in row order.
  std::vector<float> colsum(N);
  for (int c = 0; c < N; ++c) {
    float s = 0.0f;
    for (int t = 0; t < Tr; ++t) s += input[(size_t)t * N + c];
    colsum[c] = s;
  }

  // findTopPathSums (dedoppler.cu:32-55), top sums reset to 0 (dedoppler.cu:205).
  std::vector<float> top(N, 0.0f);
  std::vector<int> topdb(N, 0), topoff(N, 0);
  std::vector<float> b1((size_t)Tr * N), b2((size_t)Tr * N);
  for (int db = dmin; db <= dmax; ++db) {
    const float* sums = (Tr == 1) ? input : taylor_tree<float>(input, b1.data(), b2.data(), Tr, N, db);
#pragma omp parallel for schedule(static)
    for (int c = 0; c < N; ++c) {
      for (int off = 0; off < Tr; ++off) {
        const long last = (long)(Tr - 1) * db + off + c;
        if (last < 0 || last >= N) break;  // early return, dedoppler.cu:40-46
        const float v = sums[(size_t)off * N + c];
        if (v > top[c]) {
          top[c] = v;
          topdb[c] = db;
          topoff[c] = off;
        }
      }
    }
  }

  // Host statistics (dedoppler.cu:242-262), same library calls in the same order.
  std::vector<float> cs(colsum);
  const int mid = N / 2;
  std::nth_element(cs.begin(), cs.begin() + mid, cs.end());
  const int first = (int)std::ceil(0.05 * N);
  const int last = (int)std::floor(0.95 * N);
  std::nth_element(cs.begin(), cs.begin() + first, cs.begin() + mid - 1);
  std::nth_element(cs.begin() + mid + 1, cs.begin() + last, cs.end());
  const float median = cs[mid];
  const float sum = std::accumulate(cs.begin() + first, cs.begin() + last + 1, 0.0);
  const float m = sum / (last + 1 - first);
  float accum = 0.0f;
  std::for_each(cs.begin() + first, cs.begin() + last + 1,
                [&](const float f) { accum += (f - m) * (f - m); });
  const float std_dev = std::sqrt(accum / (last + 1 - first));

  // Window de-duplication (dedoppler.cu:264-319).
  const float thr = snr_threshold * std_dev + median;
  const int window_size = 2 * std::ceil(nmax * drift_timesteps);
  if (stats) {
    stats->median = median;
    stats->std_dev = std_dev;
    stats->mean = m;
    stats->threshold = thr;
    stats->window_size = window_size;
    stats->min_drift_block = dmin;
    stats->max_drift_block = dmax;
    stats->drift_rate_resolution = res;
  }
  if (top_sums_out) std::copy(top.begin(), top.end(), top_sums_out);
  if (top_db_out) std::copy(topdb.begin(), topdb.end(), top_db_out);
  if (top_off_out) std::copy(topoff.begin(), topoff.end(), top_off_out);
  if (colsums_out) std::copy(colsum.begin(), colsum.end(), colsums_out);
  if (window_size <= 0) return -1;

  int n = 0;
  for (int i = 0; (long)i * window_size < N; ++i) {
    int cand = -1;
    float cand_sum = thr;
    for (int j = 0; j < window_size; ++j) {
      const long f = (long)i * window_size + j;
      if (f >= N) break;
      if (top[f] > cand_sum) {
        cand = (int)f;
        cand_sum = top[f];
      }
    }
    if (cand < 0) continue;
    const int wend = std::min(N, cand + window_size);
    bool larger = false;
    for (int f = std::max(0, cand - window_size + 1); f < wend; ++f) {
      if (top[f] > cand_sum) {
        larger = true;
        break;
      }
    }
    if (larger) continue;
    const int drift_bins = topdb[cand] * drift_timesteps + topoff[cand];
    const double drift_rate = drift_bins * res;
    const float snr = (cand_sum - median) / std_dev;
    if (std::abs(drift_rate) >= min_drift) {
      if (n < cap) {
        hits[n].index = cand;
        hits[n].drift_steps = drift_bins;
        hits[n].drift_rate = drift_rate;
        hits[n].snr = snr;
        hits[n].power = cand_sum;
      }
      ++n;
    }
  }
  return n;
}

// addIncoherentPower (dedoppler.cu:139-176) for one hit: the drift block is
// floor((float) drift_steps / (Tr-1)) computed in float as the reference does.
float oracle_incoherent_power(const float* input, int Tr, int N, int drift_steps, int index) {
  const int drift_shift = Tr - 1;
  const int db = (int)std::floor((float)drift_steps / drift_shift);
  const int off = drift_steps - db * drift_shift;
  return oracle_path_sum(input, Tr, N, db, off, index);
}

}  // extern "C"
