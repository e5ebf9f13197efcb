// Per-device "done once" flags for CUDA settings that belong to a device.
//
// A kernel's dynamic shared-memory limit (cudaFuncAttributeMaxDynamicShared-
// MemorySize) is set per device: a process that launches the same kernel on
// two GPUs has to set it on each.  DeviceOnce keeps one bit per device id
// (0..63) so a launcher sets the attribute the first time it runs on each
// device and skips the call afterwards.  Devices 64 and above are never
// marked: their setting is simply repeated on every launch.  Two threads that
// race on the same device both set the attribute, which is harmless.
#pragma once

#include <atomic>
#include <cstdint>

namespace ffb {

class DeviceOnce {
 public:
  bool done(int dev) const {
    return dev >= 0 && dev < 64 && (mask_.load(std::memory_order_acquire) >> dev & 1u) != 0;
  }
  void mark(int dev) {
    if (dev >= 0 && dev < 64) mask_.fetch_or(uint64_t{1} << dev, std::memory_order_release);
  }
  uint64_t mask() const { return mask_.load(std::memory_order_acquire); }

 private:
  std::atomic<uint64_t> mask_{0};
};

}  // namespace ffb
