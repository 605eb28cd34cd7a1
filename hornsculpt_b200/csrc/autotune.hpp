// Launch-shape autotuner. For a kernel family and a size class it times each
// candidate shape once, with CUDA events on the launching stream, the first
// time the class is met outside a stream capture, and keeps the fastest for the
// rest of the process. Candidates of one family differ only in how the same
// work is spread over the grid (a grid-stride loop over independent items, or
// the support-tree leaf size of the fast-multipole form), never in the
// arithmetic of an item, so a choice changes speed, not results.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace hsb {

class Autotuner {
  public:
    static Autotuner &instance();
    // Index of the candidate chosen for `key`, or -1 when the class is not tuned yet.
    int choice(const std::string &key) const;
    // Times `launch(i)` for every candidate i on `stream` (each once, in order,
    // after one untimed launch of candidate 0 that warms caches and code),
    // stores and returns the fastest. The last launch leaves its results in
    // place, so the caller's work is done. Must not run inside a stream capture.
    int tune(const std::string &key, int candidates, cudaStream_t stream, const std::function<void(int)> &launch);
    // Records an externally measured choice (e.g. a tree parameter timed by its owner).
    void record(const std::string &key, int index, const std::vector<double> &ms);
    void setEnabled(bool enabled);
    bool enabled() const;
    // "key=choice:ms0/ms1/...;" for every tuned class.
    std::string report() const;
    void clear();

  private:
    struct Entry {
        int index;
        std::vector<double> ms;
    };
    mutable std::mutex mutex_;
    std::map<std::string, Entry> table_;
    bool enabled_ = true;
};

// True while `stream` is being captured into a graph (no tuning then).
bool capturing(cudaStream_t stream);

}  // namespace hsb
