// Checks ffb::DeviceOnce (flagfft_b200/csrc/device_once.hpp): a setting done
// on one device id is recorded for that id only, ids 64 and above are never
// recorded (their setting is repeated), negative ids are ignored.
#include <cstdio>

#include "device_once.hpp"

#define CHECK(c)                                          \
  do {                                                    \
    if (!(c)) {                                           \
      std::fprintf(stderr, "check failed: %s\n", #c);     \
      return 1;                                           \
    }                                                     \
  } while (0)

int main() {
  ffb::DeviceOnce once;
  CHECK(!once.done(0) && !once.done(1));
  once.mark(0);
  CHECK(once.done(0));
  CHECK(!once.done(1));  // device 1 still needs its own setting
  once.mark(1);
  CHECK(once.done(1) && once.mask() == 3u);
  once.mark(63);
  CHECK(once.done(63) && !once.done(62));
  once.mark(64);
  CHECK(!once.done(64));
  once.mark(-1);
  CHECK(!once.done(-1) && once.mask() == (3u | (uint64_t{1} << 63)));
  std::puts("device_once ok");
  return 0;
}
