// Per-kernel-family device timing with CUDA events on the launching stream.
// Disabled timers cost one branch per launch.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace hsb {

class KernelTimer {
  public:
    ~KernelTimer() {
        for (auto &p : pending_) {
            cudaEventDestroy(p.start);
            cudaEventDestroy(p.stop);
        }
        for (auto e : pool_)
            cudaEventDestroy(e);
    }
    void enable(bool on) { enabled_ = on; }
    bool enabled() const { return enabled_; }
    void reset() {
        collect();
        totals_.clear();
    }
    // Records a start event and returns its interval; stop() closes it.
    size_t start(const char *family, cudaStream_t stream) {
        if (!enabled_)
            return SIZE_MAX;
        Pending p{family, event(), event()};
        cudaEventRecord(p.start, stream);
        pending_.push_back(p);
        return pending_.size() - 1;
    }
    void stop(size_t interval, cudaStream_t stream) {
        if (!enabled_ || interval >= pending_.size())
            return;
        cudaEventRecord(pending_[interval].stop, stream);
    }
    // Synchronises on recorded events and folds them into per-family totals.
    void collect() {
        for (auto &p : pending_) {
            float ms = 0;
            if (cudaEventSynchronize(p.stop) == cudaSuccess && cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
                auto &t = totals_[p.family];
                t.ms += ms;
                t.launches += 1;
            }
            pool_.push_back(p.start);
            pool_.push_back(p.stop);
        }
        pending_.clear();
    }
    struct Total {
        double ms = 0;
        unsigned long long launches = 0;
    };
    const std::map<std::string, Total> &totals() const { return totals_; }

  private:
    struct Pending {
        std::string family;
        cudaEvent_t start, stop;
    };
    cudaEvent_t event() {
        if (!pool_.empty()) {
            cudaEvent_t e = pool_.back();
            pool_.pop_back();
            return e;
        }
        cudaEvent_t e{};
        cudaEventCreate(&e);
        return e;
    }
    bool enabled_ = false;
    std::vector<Pending> pending_;
    std::vector<cudaEvent_t> pool_;
    std::map<std::string, Total> totals_;
};

// RAII scope around one launch.
struct TimedScope {
    TimedScope(KernelTimer *t, const char *family, cudaStream_t s) : timer(t), stream(s) {
        if (timer)
            interval = timer->start(family, stream);
    }
    ~TimedScope() {
        if (timer)
            timer->stop(interval, stream);
    }
    KernelTimer *timer;
    cudaStream_t stream;
    size_t interval = SIZE_MAX;
};

}  // namespace hsb
