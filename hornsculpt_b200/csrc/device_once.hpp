// Once-per-device initialisation. __constant__ tables live separately on each
// device, so an upload done on device 0 leaves device 1's copy all zero: the
// flag must be per device ordinal, and the check-and-set must be serialised
// because sessions on several host threads may upload at the same time.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <stdexcept>
#include <string>

namespace hsb {

inline int currentDevice() {
    int device = 0;
    const cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess)
        throw std::runtime_error(std::string("CUDA current device: ") + cudaGetErrorString(e));
    if (device < 0 || device >= 256)
        throw std::runtime_error("CUDA device ordinal out of range.");
    return device;
}

class PerDeviceOnce {
  public:
    // Runs `init` unless it has already completed on the current device. A
    // throwing `init` leaves the device unmarked, so the next call retries.
    template <class F> void run(F &&init) {
        const int device = currentDevice();
        std::lock_guard<std::mutex> lock(mutex_);
        if (done_[device])
            return;
        init();
        done_[device] = true;
    }

  private:
    static constexpr int kMaxDevices = 256;
    std::mutex mutex_;
    bool done_[kMaxDevices] = {};
};

// A per-device value computed once by `make` (a device attribute, a schedulable
// cluster size); a thrown `make` leaves the device unset.
template <class V> class PerDeviceValue {
  public:
    template <class F> V get(F &&make) {
        const int device = currentDevice();
        std::lock_guard<std::mutex> lock(mutex_);
        if (!set_[device]) {
            value_[device] = make();
            set_[device] = true;
        }
        return value_[device];
    }

  private:
    std::mutex mutex_;
    bool set_[256] = {};
    V value_[256] = {};
};

// Largest dynamic shared-memory opt-in already applied to one kernel on each
// device: raise() returns true when `bytes` exceeds it (the caller then sets
// the kernel attribute) and records the new value.
class PerDeviceHighWater {
  public:
    bool raise(size_t bytes) {
        const int device = currentDevice();
        std::lock_guard<std::mutex> lock(mutex_);
        if (bytes <= level_[device])
            return false;
        level_[device] = bytes;
        return true;
    }

  private:
    std::mutex mutex_;
    size_t level_[256] = {};
};

}  // namespace hsb
