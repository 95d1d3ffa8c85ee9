// CPU check of PerDeviceOnce (nqpu_b200/csrc/device_once.h): many host threads
// ask for the set-up of a few devices at once; each device's set-up must run
// exactly once, every caller must see that run's result, and an out-of-range
// device index must get the `invalid` value without running anything.
#include <atomic>
#include <thread>
#include <vector>

#include "device_once.h"

extern "C" int per_device_once_check(int threads, int devices, int rounds) {
  if (devices < 1 || devices > nqpu::kMaxDevices) return -1;
  nqpu::PerDeviceOnce<int> once;
  std::vector<std::atomic<int>> runs(static_cast<size_t>(devices));
  for (auto& r : runs) r.store(0);
  std::atomic<int> bad{0};
  std::atomic<bool> go{false};
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t)
    th.emplace_back([&, t] {
      while (!go.load()) {
      }
      for (int i = 0; i < rounds; ++i) {
        const int dev = (t + i) % devices;
        const int v = once.get(dev, [&, dev] {
          runs[size_t(dev)].fetch_add(1);
          std::this_thread::yield();  // widen the window for concurrent first calls
          return 1000 + dev;
        }, -7);
        if (v != 1000 + dev) bad.fetch_add(1);
      }
      if (once.get(-1, [] { return 1; }, -7) != -7) bad.fetch_add(1);
      if (once.get(nqpu::kMaxDevices, [] { return 1; }, -7) != -7) bad.fetch_add(1);
    });
  go.store(true);
  for (auto& x : th) x.join();
  if (bad.load() != 0) return 1;
  for (auto& r : runs)
    if (r.load() != 1) return 2;
  return 0;
}
