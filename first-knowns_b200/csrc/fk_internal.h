// fk_internal.h -- engine internals shared between libfk's translation
// units (not part of the public C ABI).
#pragma once
#include <cstdint>

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
};

EngineView engine_view(const fk_engine* e);

// Records msg as this thread's last error (fk_last_error) and returns s.
fk_status set_error(fk_status s, const char* msg);

}  // namespace fk
