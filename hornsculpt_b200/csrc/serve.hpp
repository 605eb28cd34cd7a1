// Serving form: a persistent request loop over solver sessions on one GPU.
//
// Requests (mesh + BemRequest) arrive at any time. Worker threads, each with
// its own CUDA stream, take them in arrival order as device memory allows
// (admission by the estimated footprint of the solve), so requests on
// different meshes run concurrently on the device. Sessions (geometry, plan,
// workspaces) stay resident per mesh for reuse, least recently used evicted.
// Queued requests on the same mesh with the same solve settings are merged
// into one session call, their frequencies batched together. With a fixed
// planning frequency every request on a mesh uses the same interaction plan,
// so a result does not depend on what it was batched with.
#pragma once

#include "hs_bem.h"
#include "session.hpp"

#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <exception>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace hsb {

// Owned copy of an hs_request (the caller's arrays may go away after submit).
struct RequestCopy {
    hs_request base{};
    std::vector<double> frequencies, raster, observers, velocities;
    std::vector<size_t> offsets;
    std::vector<uint32_t> faceIds;
    explicit RequestCopy(const hs_request &r);
    hs_request view(const std::vector<double> &freqs, const std::vector<double> &planRaster) const;
    bool compatible(const RequestCopy &o) const;  // everything but the frequencies equal (planning raster too)
};

class Server {
  public:
    explicit Server(const hs_serve_options &options);
    ~Server();
    uint64_t submit(MeshInput mesh, const hs_request &request);
    // Blocks until the request is done; rethrows its error.
    std::unique_ptr<Result> wait(uint64_t ticket, hs_serve_timing &timing);

  private:
    using Clock = std::chrono::steady_clock;
    struct Job {
        uint64_t ticket;
        uint64_t meshKey;
        std::shared_ptr<const MeshInput> mesh;
        RequestCopy request;
        Clock::time_point arrival, start, finish;
        size_t footprint = 0;
        uint32_t batched = 1;
        bool done = false;
        std::unique_ptr<Result> result;
        std::exception_ptr error;
    };
    struct Resident {
        std::unique_ptr<Session> session;
        bool busy = false;
        uint64_t lastUse = 0;
    };
    void worker(int index);
    std::vector<std::shared_ptr<Job>> takeGroup(size_t &footprint);
    size_t idleBytes(uint64_t keep) const;
    void evictIdle(size_t needed, uint64_t keep);
    bool evictOldestIdle(uint64_t keep);

    hs_serve_options options_;
    int device_ = 0;
    size_t budget_ = 0, reserved_ = 0;
    uint64_t nextTicket_ = 1, useClock_ = 0;
    bool stop_ = false;
    std::mutex mutex_;
    std::condition_variable work_, done_;
    std::deque<std::shared_ptr<Job>> queue_;
    std::map<uint64_t, std::shared_ptr<Job>> jobs_;
    std::map<uint64_t, Resident> sessions_;
    std::vector<std::thread> workers_;
};

}  // namespace hsb
