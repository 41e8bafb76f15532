// device_memo.hpp -- per-device memo for launch set-up (host only).
//
// Function attributes (the dynamic shared-memory opt-in, the carveout),
// occupancy and the SM count belong to one device.  A process may drive
// solvers on several GPUs (fp_config.device) from several host threads, so
// launch set-up is memoised per device ordinal, under a lock, rather than
// once per process.
#pragma once

#include <mutex>

#include <cuda_runtime.h>

namespace fp {

class DeviceMemo {
  public:
    static constexpr int kMaxDevices = 64;

    // The value for the current device: compute(dev) runs on the first call
    // on that device.  A result of 0 means failure and is not memoised.
    template <class F>
    int get(F&& compute) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return 0;
        if (dev < 0 || dev >= kMaxDevices) return compute(dev);
        std::lock_guard<std::mutex> lock(m_);
        if (!v_[dev]) v_[dev] = compute(dev);
        return v_[dev];
    }

  private:
    std::mutex m_;
    int v_[kMaxDevices] = {};
};

}  // namespace fp
