// egg_perdevice.h -- one value per GPU, set up once on each device that uses it.
//
// The library's device-resident tables (the binomial table the closed-form DP and the sieve read,
// the fixed scratch of the entry point that allocates nothing) are module globals: every GPU that
// loads the library has its own copy, at its own device address.  A host pointer to one device's
// copy must never reach a kernel on another device.  PerDevice keeps one slot per device index,
// filled by a set-up function that runs with that device current, the first time that device
// asks, under a lock.  A set-up that fails caches nothing, so the next call retries it.
//
// Host-only and free of CUDA headers, so that the per-device bookkeeping can be exercised on a
// machine without a GPU by driving it with device indices directly.
#pragma once

#include <mutex>

namespace egg {

constexpr int kMaxDevices = 64;

template <class T>
class PerDevice {
public:
    // Returned by get() for a device index outside [0, kMaxDevices).
    static constexpr int kBadDevice = -1;

    // The value of device dev in *out.  `init(dev, &value)` returns a status (0 is success) and runs
    // at most once per device until it succeeds.  Returns init's status, or kBadDevice.
    template <class Init>
    int get(int dev, T *out, Init &&init)
    {
        if (dev < 0 || dev >= kMaxDevices) return kBadDevice;
        std::lock_guard<std::mutex> lk(mu_);
        if (!set_[dev]) {
            T v{};
            const int rc = init(dev, &v);
            if (rc) return rc;
            val_[dev] = v;
            set_[dev] = true;
        }
        *out = val_[dev];
        return 0;
    }

    // Whether device dev has been set up (for tests).
    bool has(int dev)
    {
        std::lock_guard<std::mutex> lk(mu_);
        return dev >= 0 && dev < kMaxDevices && set_[dev];
    }

private:
    std::mutex mu_;
    T val_[kMaxDevices]{};
    bool set_[kMaxDevices]{};
};

}  // namespace egg
