// One-time set-up per CUDA device.
//
// Some set-up belongs to a device rather than to the process: a kernel's
// shared-memory limit (cudaFuncSetAttribute) applies to the device that is
// current when it is set, and the SM count differs between GPU models.  A
// process-wide "done" flag would skip the set-up on the second device a process
// uses, and an unsynchronised one races between host threads (the request
// server's worker thread and its callers).  PerDeviceOnce runs the set-up once
// per device index, on the first call for that device, and returns the stored
// result on every later call; concurrent first calls for one device wait for
// the one that runs it.  Plain C++ (no CUDA headers) so it is unit-tested on
// the CPU.
#pragma once
#include <mutex>

namespace nqpu {

constexpr int kMaxDevices = 64;

template <typename R>
class PerDeviceOnce {
 public:
  // Result of f() for device `dev`, running f only on the first call for that
  // device; `invalid` for a device index outside [0, kMaxDevices).
  template <typename F>
  R get(int dev, F&& f, R invalid) {
    if (dev < 0 || dev >= kMaxDevices) return invalid;
    std::call_once(flags_[dev], [&] { result_[dev] = f(); });
    return result_[dev];
  }

 private:
  std::once_flag flags_[kMaxDevices];
  R result_[kMaxDevices] = {};
};

}  // namespace nqpu
