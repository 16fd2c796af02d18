// Header-only C++ drop-in for seticore's dedoppler API, over the C ABI in
// seticore_b200.h.  Class and member names, argument meanings and error behaviour
// follow the reference:
//   FilterbankBuffer   -- filterbank_buffer.h:11-48 / filterbank_buffer.cu:13-78
//   FilterbankMetadata -- filterbank_metadata.h:17-62 (the fields a search reads)
//   DedopplerHit       -- dedoppler_hit.h:11-66 / dedoppler_hit.cpp:11-73
//   Dedopplerer        -- dedoppler.h:15-79 / dedoppler.cu:79-320
// As in the reference, a CUDA or shape error prints a message and exits with status 2
// (cuda_util.cu:8-15); call the C ABI directly to get status codes instead.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "seticore_b200.h"

namespace seticore_b200 {

const int NO_BEAM = SC_DD_NO_BEAM;

inline void checkStatus(int rc, const char* tag) {
  if (rc != SC_DD_OK) {
    std::fprintf(stderr, "%s: seticore_b200 error %d: %s\n", tag, rc, sc_dd_last_error());
    std::exit(2);
  }
}

inline int roundUpToPowerOfTwo(int n) {
  int r = 1;
  while (r < n) r *= 2;
  return r;
}

class FilterbankMetadata {
 public:
  bool has_dc_spike = false;
  std::string source_name;
  std::vector<std::string> source_names;
  long num_timesteps = 0, num_channels = 0, coarse_channel_size = 0, num_coarse_channels = 0;
  double fch1 = 0, foff = 0, tstart = 0, tsamp = 0;
  virtual ~FilterbankMetadata() {}
  bool isCoherentBeam(int beam) const { return 0 <= beam && beam < (int)source_names.size(); }
};

class FilterbankBuffer {
 public:
  const int num_timesteps;
  const int num_channels;
  const bool managed;
  const int size;
  const size_t bytes;
  float* data;
  // Row stride in floats (num_channels for an owning buffer; a view may be wider).
  long long row_stride;

  FilterbankBuffer(int num_timesteps, int num_channels)
      : num_timesteps(num_timesteps), num_channels(num_channels), managed(true),
        size(num_timesteps * num_channels), bytes(sizeof(float) * (size_t)size),
        data(nullptr), row_stride(num_channels) {
    if (cudaMallocManaged(&data, bytes) != cudaSuccess) {
      std::fprintf(stderr, "FilterbankBuffer: cuda error allocating %zu bytes\n", bytes);
      std::exit(2);
    }
  }
  FilterbankBuffer(int num_timesteps, int num_channels, float* data, long long row_stride = 0)
      : num_timesteps(num_timesteps), num_channels(num_channels), managed(false),
        size(num_timesteps * num_channels), bytes(sizeof(float) * (size_t)size), data(data),
        row_stride(row_stride ? row_stride : num_channels) {}
  ~FilterbankBuffer() {
    if (managed) cudaFree(data);
  }
  FilterbankBuffer(const FilterbankBuffer&) = delete;
  FilterbankBuffer& operator=(FilterbankBuffer&) = delete;

  void zero() {
    cudaDeviceSynchronize();
    for (int t = 0; t < num_timesteps; ++t) std::memset(data + t * row_stride, 0, sizeof(float) * num_channels);
  }
  void set(int time, int channel, float value) { data[time * row_stride + channel] = value; }
  float get(int time, int channel) const {
    cudaDeviceSynchronize();
    return data[time * row_stride + channel];
  }
};

// filterbank_buffer.cu:71-78
inline void makeNoisyBuffer(FilterbankBuffer& buffer) {
  buffer.zero();
  for (int chan = 0; chan < buffer.num_channels; ++chan)
    buffer.set(0, chan, 0.1 * chan / buffer.num_channels);
}

class DedopplerHit {
 public:
  double frequency;
  int index;
  int drift_steps;
  double drift_rate;
  float snr;
  int coarse_channel;
  int beam;
  int num_timesteps;
  float power;
  float incoherent_power;

  DedopplerHit(const FilterbankMetadata& metadata, int _index, int _drift_steps, double _drift_rate,
               float _snr, int _beam, int _coarse_channel, int _num_timesteps, float _power)
      : index(_index), drift_steps(_drift_steps), drift_rate(_drift_rate), snr(_snr),
        coarse_channel(_coarse_channel), beam(metadata.isCoherentBeam(_beam) ? _beam : NO_BEAM),
        num_timesteps(_num_timesteps), power(_power), incoherent_power(0.0) {
    const long global_index = (long)coarse_channel * metadata.coarse_channel_size + index;
    frequency = metadata.fch1 + global_index * metadata.foff;
  }
  std::string toString() const {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "coarse channel = %d, index = %d, snr = %.5f, drift rate = %.5f (%d %s)",
                  coarse_channel, index, snr, drift_rate, drift_steps,
                  (drift_steps == 1 || drift_steps == -1) ? "bin" : "bins");
    return buf;
  }
  int lowIndex() const { return std::min(index, index + drift_steps); }
  int highIndex() const { return std::max(index, index + drift_steps); }
  int expectedIndex(int timesteps) const {
    const double per = ((double)drift_steps) / ((double)(num_timesteps - 1));
    return index + (int)std::round(timesteps * per);
  }
  float score() const { return incoherent_power > 0 ? power / incoherent_power : -1.0 / (1.0 + snr); }
};

inline bool operator<(const DedopplerHit& lhs, const DedopplerHit& rhs) {
  if (lhs.coarse_channel != rhs.coarse_channel) return lhs.coarse_channel < rhs.coarse_channel;
  if (lhs.lowIndex() != rhs.lowIndex()) return lhs.lowIndex() < rhs.lowIndex();
  return lhs.highIndex() < rhs.highIndex();
}

inline bool driftStepsLessThan(const DedopplerHit& lhs, const DedopplerHit& rhs) {
  return lhs.drift_steps < rhs.drift_steps;
}

class Dedopplerer {
 public:
  const int num_timesteps;
  const int num_channels;
  const double foff;
  const double tsamp;
  const bool has_dc_spike;
  bool print_hits;
  // The stream every call is ordered on (0: the legacy default stream, as the reference).
  cudaStream_t stream = 0;

  Dedopplerer(int num_timesteps, int num_channels, double foff, double tsamp, bool has_dc_spike)
      : num_timesteps(num_timesteps), num_channels(num_channels), foff(foff), tsamp(tsamp),
        has_dc_spike(has_dc_spike), print_hits(false) {
    checkStatus(sc_dd_create(num_timesteps, num_channels, foff, tsamp, has_dc_spike, &engine_),
                "Dedopplerer");
  }
  ~Dedopplerer() { sc_dd_destroy(engine_); }
  Dedopplerer(const Dedopplerer&) = delete;
  Dedopplerer& operator=(Dedopplerer&) = delete;

  void search(const FilterbankBuffer& input, const FilterbankMetadata& metadata, int beam,
              int coarse_channel, double max_drift, double min_drift, double snr_threshold,
              std::vector<DedopplerHit>* output) {
    checkShape(input);
    std::vector<sc_dd_hit> raw(256);
    int n = 0;
    int rc = sc_dd_search(engine_, input.data, input.row_stride, beam, coarse_channel, max_drift, min_drift,
                          snr_threshold, raw.data(), (int)raw.size(), &n, stream);
    if (rc == SC_DD_ETRUNC) {
      raw.resize(n);
      rc = sc_dd_search(engine_, input.data, input.row_stride, beam, coarse_channel, max_drift, min_drift,
                        snr_threshold, raw.data(), (int)raw.size(), &n, stream);
    }
    checkStatus(rc, "Dedopplerer::search");
    for (int i = 0; i < n; ++i) {
      DedopplerHit hit(metadata, raw[i].index, raw[i].drift_steps, raw[i].drift_rate, raw[i].snr, beam,
                       coarse_channel, num_timesteps, raw[i].power);
      if (print_hits) std::printf("hit: %s\n", hit.toString().c_str());
      output->push_back(hit);
    }
  }

  // Sorts hits by drift_steps (as dedoppler.cu:144 does) and fills incoherent_power.
  void addIncoherentPower(const FilterbankBuffer& input, std::vector<DedopplerHit>& hits) {
    checkShape(input);
    std::sort(hits.begin(), hits.end(), &driftStepsLessThan);
    std::vector<sc_dd_hit> raw(hits.size());
    for (size_t i = 0; i < hits.size(); ++i) {
      raw[i] = sc_dd_hit{};
      raw[i].index = hits[i].index;
      raw[i].drift_steps = hits[i].drift_steps;
    }
    checkStatus(sc_dd_add_incoherent_power(engine_, input.data, input.row_stride, raw.data(), (int)raw.size(),
                                           stream),
                "Dedopplerer::addIncoherentPower");
    for (size_t i = 0; i < hits.size(); ++i) hits[i].incoherent_power = raw[i].incoherent_power;
  }

  size_t memoryUsage() const { return sc_dd_memory_usage(engine_); }

 private:
  void checkShape(const FilterbankBuffer& input) const {
    if (input.num_timesteps != roundUpToPowerOfTwo(num_timesteps) || input.num_channels != num_channels) {
      std::fprintf(stderr, "Dedopplerer: input is %d x %d, expected %d x %d\n", input.num_timesteps,
                   input.num_channels, roundUpToPowerOfTwo(num_timesteps), num_channels);
      std::exit(2);
    }
  }
  sc_dd* engine_ = nullptr;
};

}  // namespace seticore_b200
