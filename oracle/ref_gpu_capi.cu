// C entry points around the reference's own GPU dedoppler classes, compiled from the
// reference sources (dedoppler.cu, taylor.cu, filterbank_buffer.cu, cuda_util.cu,
// dedoppler_hit.cpp, filterbank_metadata.cpp) by oracle/Makefile into
// oracle/_ref/libref_gpu.so.  TEST INFRASTRUCTURE ONLY: the GPU parity tests call it
// to compare this project's search with the reference's on the same inputs, and
// bench.py reports its timing beside ours.  Nothing in seticore_b200/ uses it.
#include <chrono>
#include <cstring>
#include <vector>

#include "dedoppler.h"
#include "filterbank_buffer.h"
#include "filterbank_metadata.h"
#include "taylor.h"
#include "util.h"

extern "C" {

typedef struct ref_hit {
  int index;
  int drift_steps;
  double drift_rate;
  float snr;
  float power;
  float incoherent_power;
  int coarse_channel;
  int beam;
  int num_timesteps;
  double frequency;
} ref_hit;

static void copy_hit(const DedopplerHit& h, ref_hit* o) {
  o->index = h.index;
  o->drift_steps = h.drift_steps;
  o->drift_rate = h.drift_rate;
  o->snr = h.snr;
  o->power = h.power;
  o->incoherent_power = h.incoherent_power;
  o->coarse_channel = h.coarse_channel;
  o->beam = h.beam;
  o->num_timesteps = h.num_timesteps;
  o->frequency = h.frequency;
}

// A persistent reference search context: one Dedopplerer plus one managed input buffer.
struct RefCtx {
  Dedopplerer dd;
  FilterbankBuffer buf;
  FilterbankMetadata meta;
  RefCtx(int T, int N, double foff, double tsamp)
      : dd(T, N, foff, tsamp, false), buf(roundUpToPowerOfTwo(T), N) {
    meta.fch1 = 0.0;
    meta.foff = foff;
    meta.coarse_channel_size = N;
  }
};

void* ref_gpu_create(int T, int N, double foff_mhz, double tsamp) {
  return new RefCtx(T, N, foff_mhz, tsamp);
}

void ref_gpu_destroy(void* h) { delete static_cast<RefCtx*>(h); }

// Copies [Tr][N] host floats into the managed input buffer.
void ref_gpu_load(void* h, const float* host) {
  RefCtx* c = static_cast<RefCtx*>(h);
  cudaMemcpy(c->buf.data, host, c->buf.bytes, cudaMemcpyDefault);
  cudaDeviceSynchronize();
}

// Dedopplerer::search on the loaded buffer.  Returns the hit count (<= cap written).
int ref_gpu_search(void* h, int beam, int coarse_channel, double max_drift,
                   double min_drift, double snr, ref_hit* out, int cap) {
  RefCtx* c = static_cast<RefCtx*>(h);
  std::vector<DedopplerHit> hits;
  c->dd.search(c->buf, c->meta, beam, coarse_channel, max_drift, min_drift, snr, &hits);
  for (int i = 0; i < (int)hits.size() && i < cap; ++i) copy_hit(hits[i], &out[i]);
  return (int)hits.size();
}

// Times `iters` back-to-back searches (each one returns only after its hits are on the
// host, as the reference's search does).  Returns milliseconds per search.
double ref_gpu_time_search(void* h, double max_drift, double min_drift, double snr, int iters) {
  RefCtx* c = static_cast<RefCtx*>(h);
  std::vector<DedopplerHit> hits;
  c->dd.search(c->buf, c->meta, NO_BEAM, 0, max_drift, min_drift, snr, &hits);
  cudaDeviceSynchronize();
  auto t0 = std::chrono::steady_clock::now();
  for (int i = 0; i < iters; ++i) {
    hits.clear();
    c->dd.search(c->buf, c->meta, NO_BEAM, 0, max_drift, min_drift, snr, &hits);
  }
  cudaDeviceSynchronize();
  auto t1 = std::chrono::steady_clock::now();
  return std::chrono::duration<double, std::milli>(t1 - t0).count() / iters;
}

// addIncoherentPower on the loaded buffer for hits given as (index, drift_steps).
// Hits come back in the reference's post-call order (sorted by drift_steps).
int ref_gpu_add_incoherent(void* h, ref_hit* hits_io, int n) {
  RefCtx* c = static_cast<RefCtx*>(h);
  std::vector<DedopplerHit> hits;
  for (int i = 0; i < n; ++i) {
    DedopplerHit hit(c->meta, hits_io[i].index, hits_io[i].drift_steps, hits_io[i].drift_rate,
                     hits_io[i].snr, hits_io[i].beam, hits_io[i].coarse_channel,
                     hits_io[i].num_timesteps, hits_io[i].power);
    hits.push_back(hit);
  }
  c->dd.addIncoherentPower(c->buf, hits);
  for (int i = 0; i < n; ++i) copy_hit(hits[i], &hits_io[i]);
  return n;
}

// optimizedTaylorTree for one drift block: out[off][c] for all offsets and channels
// (entries of invalid paths are whatever the reference leaves there).
int ref_gpu_taylor(const float* host_in, int Tr, int N, int drift_block, float* host_out) {
  FilterbankBuffer in(Tr, N), b1(Tr, N), b2(Tr, N);
  cudaMemcpy(in.data, host_in, in.bytes, cudaMemcpyDefault);
  cudaDeviceSynchronize();
  const float* r = optimizedTaylorTree(in.data, b1.data, b2.data, Tr, N, drift_block);
  cudaDeviceSynchronize();
  cudaMemcpy(host_out, r, in.bytes, cudaMemcpyDefault);
  cudaDeviceSynchronize();
  return (int)cudaGetLastError();
}

}  // extern "C"
