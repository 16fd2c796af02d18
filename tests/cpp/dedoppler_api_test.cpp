// The reference's dedoppler_test.cpp:9-33 ("basic functionality") and a drift-sorted
// addIncoherentPower check, written against the header-only C++ drop-in
// (include/seticore_b200/dedoppler.hpp).  Exit status 0 = pass.
#include <cstdio>
#include <vector>

#include "seticore_b200/dedoppler.hpp"

using namespace seticore_b200;

#define REQUIRE(x)                                                   \
  do {                                                               \
    if (!(x)) {                                                      \
      std::fprintf(stderr, "REQUIRE failed: %s (line %d)\n", #x, __LINE__); \
      return 1;                                                      \
    }                                                                \
  } while (0)

int main() {
  int num_timesteps = 8;
  int num_channels = 1000;
  FilterbankBuffer buffer(num_timesteps, num_channels);
  makeNoisyBuffer(buffer);
  FilterbankMetadata metadata;
  buffer.set(0, 70, 1.0);
  buffer.set(1, 70, 1.0);
  buffer.set(2, 71, 1.0);
  buffer.set(3, 71, 1.0);
  buffer.set(4, 72, 1.0);
  buffer.set(5, 72, 1.0);
  buffer.set(6, 73, 1.0);
  buffer.set(7, 73, 1.0);

  Dedopplerer dedopplerer(num_timesteps, num_channels, 1.0, 1.0, false);
  std::vector<DedopplerHit> hits;
  dedopplerer.search(buffer, metadata, NO_BEAM, 555, 0.01, 0.01, 200.0, &hits);
  REQUIRE(hits.size() == 1);
  REQUIRE(hits[0].index == 70);
  REQUIRE(hits[0].drift_steps == 3);
  REQUIRE(hits[0].beam == NO_BEAM);
  REQUIRE(hits[0].coarse_channel == 555);

  // The incoherent beam here is the same buffer: incoherent power equals the hit power.
  dedopplerer.addIncoherentPower(buffer, hits);
  REQUIRE(hits[0].incoherent_power == hits[0].power);
  REQUIRE(dedopplerer.memoryUsage() > 0);
  std::printf("dedoppler_api_test: ok (%s)\n", hits[0].toString().c_str());
  return 0;
}
