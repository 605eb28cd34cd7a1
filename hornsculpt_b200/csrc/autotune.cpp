#include "autotune.hpp"

#include <sstream>
#include <stdexcept>

namespace hsb {

Autotuner &Autotuner::instance() {
    static Autotuner tuner;
    return tuner;
}

int Autotuner::choice(const std::string &key) const {
    std::lock_guard<std::mutex> lock(mutex_);
    const auto it = table_.find(key);
    return it == table_.end() ? -1 : it->second.index;
}

void Autotuner::record(const std::string &key, int index, const std::vector<double> &ms) {
    std::lock_guard<std::mutex> lock(mutex_);
    table_[key] = Entry{index, ms};
}

void Autotuner::setEnabled(bool enabled) {
    std::lock_guard<std::mutex> lock(mutex_);
    enabled_ = enabled;
}

bool Autotuner::enabled() const {
    std::lock_guard<std::mutex> lock(mutex_);
    return enabled_;
}

void Autotuner::clear() {
    std::lock_guard<std::mutex> lock(mutex_);
    table_.clear();
}

std::string Autotuner::report() const {
    std::lock_guard<std::mutex> lock(mutex_);
    std::ostringstream out;
    for (const auto &[key, e] : table_) {
        out << key << '=' << e.index << ':';
        for (size_t i = 0; i < e.ms.size(); ++i)
            out << (i ? "/" : "") << e.ms[i];
        out << ';';
    }
    return out.str();
}

int Autotuner::tune(const std::string &key, int candidates, cudaStream_t stream, const std::function<void(int)> &launch) {
    struct Events {
        std::vector<cudaEvent_t> e;
        ~Events() {
            for (auto x : e)
                cudaEventDestroy(x);
        }
    } ev;
    ev.e.resize(size_t(candidates) + 1, nullptr);
    for (auto &x : ev.e)
        if (cudaEventCreate(&x) != cudaSuccess)
            throw std::runtime_error("autotuner event creation failed");
    launch(0);  // warm-up
    cudaEventRecord(ev.e[0], stream);
    for (int i = 0; i < candidates; ++i) {
        launch(i);
        cudaEventRecord(ev.e[size_t(i) + 1], stream);
    }
    if (cudaEventSynchronize(ev.e.back()) != cudaSuccess)
        throw std::runtime_error("autotuner timing failed");
    std::vector<double> ms(static_cast<size_t>(candidates), 0.0);
    int best = 0;
    for (int i = 0; i < candidates; ++i) {
        float t = 0;
        cudaEventElapsedTime(&t, ev.e[size_t(i)], ev.e[size_t(i) + 1]);
        ms[size_t(i)] = t;
        if (t < ms[size_t(best)])
            best = i;
    }
    // every candidate computes the same results, so the last launch's stand
    record(key, best, ms);
    return best;
}

bool capturing(cudaStream_t stream) {
    cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(stream, &status) == cudaSuccess && status != cudaStreamCaptureStatusNone;
}

}  // namespace hsb
