// Host-only driver for fk::check_engine_device (csrc/fk_internal.h), the
// rule fk_sieve_noalloc applies before any launch: an engine's tables may
// only be used with the device they were uploaded to current.  Prints one
// line per case: "<engine> <current> <status> <message>".
#include <cstdio>

#include "../../first-knowns_b200/csrc/fk_internal.h"

int main() {
  const int cases[][2] = {{0, 0}, {0, 1}, {3, 2}, {7, 7}};
  for (const auto& c : cases) {
    char msg[192] = {0};
    const fk_status s = fk::check_engine_device(c[0], c[1], msg, sizeof msg);
    std::printf("%d %d %d %s\n", c[0], c[1], (int)s, msg);
  }
  return 0;
}
