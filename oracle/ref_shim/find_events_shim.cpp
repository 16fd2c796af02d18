// Stand-ins that let the reference's own find_events.cpp (findEvents, findHit,
// removeZeroDriftHits) link as a test oracle.  TEST INFRASTRUCTURE ONLY: oracle/Makefile
// builds it into oracle/_ref/libref_gpu.so next to the reference's Dedopplerer, and the
// GPU tests compare this package's cadence matching with the reference's on the same
// synthetic files.
//
// * loadFilterbankFile: the file names handed to findEvents name in-memory files that the
//   caller registered (metadata plus [timesteps][coarse channels x channels] float rows).
//   Their loadCoarseChannel does what H5Reader::loadCoarseChannel does after its read
//   (h5_reader.cpp:195-209): rows past the file's timesteps are zeroed and, with a DC spike,
//   the middle column becomes the mean of its neighbours.
// * EventFileWriter: records each event -- per file, the hit findEvents passed or none --
//   instead of writing Cap'n Proto (the reference's writer needs capnp, absent here).
#include <cstring>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "event_file_writer.h"
#include "filterbank_file_reader.h"
#include "find_events.h"
#include "util.h"

namespace {

struct MemFile {
  FilterbankMetadata meta;
  const float* rows;  // [num_timesteps][num_coarse_channels * coarse_channel_size]
};
std::map<std::string, MemFile> g_files;

struct EventHit {
  int present, index, drift_steps;
  float snr, power;
};
std::vector<std::vector<EventHit>> g_events;

class MemReader : public FilterbankFileReader {
 public:
  MemReader(const std::string& name, const MemFile& f) : FilterbankFileReader(name), f_(f) {
    static_cast<FilterbankMetadata&>(*this) = f.meta;
  }
  void loadCoarseChannel(int i, FilterbankBuffer* buffer) const override {
    const long T = num_timesteps, N = coarse_channel_size, width = num_coarse_channels * coarse_channel_size;
    for (long t = 0; t < T; ++t) std::memcpy(buffer->data + t * N, f_.rows + t * width + (long)i * N, sizeof(float) * N);
    if (T < buffer->num_timesteps) std::memset(buffer->data + T * N, 0, sizeof(float) * (buffer->num_timesteps - T) * N);
    if (has_dc_spike) {
      const long mid = N / 2;
      for (long t = 0; t < T; ++t) {
        float* row = buffer->data + t * N;
        row[mid] = (row[mid - 1] + row[mid + 1]) / 2.0;
      }
    }
  }

 private:
  MemFile f_;
};

}  // namespace

void FilterbankFileReader::loadCoarseChannel(int, FilterbankBuffer*) const {
  throw std::runtime_error("loadCoarseChannel on a base FilterbankFileReader");
}

unique_ptr<FilterbankFileReader> loadFilterbankFile(const string& filename) {
  return unique_ptr<FilterbankFileReader>(new MemReader(filename, g_files.at(filename)));
}

EventFileWriter::EventFileWriter(const string& filename, const vector<shared_ptr<FilterbankFileReader> >& metadatas)
    : metadatas(metadatas), fd(-1), tmp_filename(filename + ".tmp"), final_filename(filename) {}

EventFileWriter::~EventFileWriter() {}

void EventFileWriter::write(const vector<DedopplerHit*>& hits, const vector<shared_ptr<FilterbankBuffer> >&) {
  std::vector<EventHit> ev;
  for (const DedopplerHit* h : hits)
    ev.push_back(h ? EventHit{1, h->index, h->drift_steps, h->snr, h->power} : EventHit{0, -1, 0, 0.0f, 0.0f});
  g_events.push_back(ev);
}

extern "C" {

typedef struct ref_event_hit {
  int present;
  int index;
  int drift_steps;
  float snr;
  float power;
} ref_event_hit;

// findEvents (find_events.cpp:65-226) over n in-memory files of one shape.  rows[k] holds
// file k's [num_timesteps][num_coarse * coarse_size] floats.  Writes up to `cap` events of
// n hits each into out (event-major) and returns the number of events (-1 on an error).
int ref_find_events(int n, const char* const* source_names, const double* tstarts, const float* const* rows,
                    int num_timesteps, int coarse_size, int num_coarse, double fch1, double foff, double tsamp,
                    int has_dc_spike, double max_drift, double snr_on, double snr_off, ref_event_hit* out, int cap) {
  g_files.clear();
  g_events.clear();
  std::vector<std::string> names;
  for (int k = 0; k < n; ++k) {
    MemFile f;
    f.meta.has_dc_spike = has_dc_spike != 0;
    f.meta.source_name = source_names[k];
    f.meta.num_timesteps = num_timesteps;
    f.meta.num_channels = (long)coarse_size * num_coarse;
    f.meta.coarse_channel_size = coarse_size;
    f.meta.num_coarse_channels = num_coarse;
    f.meta.fch1 = fch1;
    f.meta.foff = foff;
    f.meta.tstart = tstarts[k];
    f.meta.tsamp = tsamp;
    f.meta.telescope_id = 6;
    f.rows = rows[k];
    names.push_back("file" + std::to_string(k) + ".mem");
    g_files[names.back()] = f;
  }
  try {
    findEvents(names, "events.mem", max_drift, snr_on, snr_off);
  } catch (const std::exception&) {
    return -1;
  }
  int e = 0;
  for (const auto& ev : g_events) {
    if (e >= cap) break;
    for (int k = 0; k < n; ++k) {
      const EventHit& h = ev[k];
      out[e * n + k] = ref_event_hit{h.present, h.index, h.drift_steps, h.snr, h.power};
    }
    ++e;
  }
  return (int)g_events.size();
}

}  // extern "C"
