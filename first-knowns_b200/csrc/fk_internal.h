// fk_internal.h -- engine internals shared between libfk's translation
// units (not part of the public C ABI).
#pragma once
#include <cstdint>
#include <cstdio>

#include "../../include/fk.h"
#include "fk_types.h"

namespace fk {

// What another translation unit needs to launch the sieve for an engine.
struct EngineView {
  DevEngine dev;      // device-resident tables (pointers into HBM)
  uint32_t P0;        // pattern family: first pattern prime index
  uint64_t M;         // wheel period
  uint32_t L;         // lanes
  uint32_t NP;        // sieve primes
  int device;         // CUDA device the tables were uploaded to
};

EngineView engine_view(const fk_engine* e);

// Records msg as this thread's last error (fk_last_error) and returns s.
fk_status set_error(fk_status s, const char* msg);

// The domain checks every sweep entry point applies to [lo, hi) (two
// little-endian limbs each; hi > lo): width below 2^63 and every chain
// value of the interval within three 64-bit limbs (cap = the longest chain
// asked for, 0 for a pre-primality stream).  FK_OK or FK_ERR_DOMAIN with
// the message set.
fk_status check_interval(const fk_engine* e, const uint64_t lo[2],
                         const uint64_t hi[2], uint32_t cap, bool dense);

// Periods one device item spans at most for a wheel of period M: every
// offset u*M + R of the item stays below 2^55 (the candidate key), rounded
// down to whole 64-period words, at least one word, at most 2^36.
inline uint64_t item_periods_max(uint64_t M) {
  uint64_t u = (uint64_t)(((unsigned __int128)1 << 55) / M);
  u = u / 64 * 64;
  if (u < 64) u = 64;
  if (u > (1ull << 36)) u = 1ull << 36;
  return u;
}

// A call that launches on the current device with an engine's tables must
// run where those tables live: a kernel given another GPU's pointers
// faults there or reads that GPU's memory over the interconnect.  FK_OK
// when the devices agree, else FK_ERR_DEVICE with a message in msg.
inline fk_status check_engine_device(int engine_device, int current_device,
                                     char* msg, size_t msg_size) {
  if (engine_device == current_device) return FK_OK;
  std::snprintf(msg, msg_size,
                "the engine's tables live on CUDA device %d but device %d is "
                "current; make device %d current (fk_set_device) first",
                engine_device, current_device, engine_device);
  return FK_ERR_DEVICE;
}

}  // namespace fk
