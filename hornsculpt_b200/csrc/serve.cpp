// Serving form: persistent request loop (see serve.hpp).
#include "serve.hpp"

#include "host_mesh.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <set>
#include <string>

namespace hsb {
namespace {

void cudaOk(cudaError_t e, const char *what) {
    if (e != cudaSuccess)
        throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

// FNV-1a over the mesh arrays: requests with the same mesh share a session.
uint64_t meshKey(const MeshInput &m) {
    uint64_t h = 1469598103934665603ull;
    const auto mix = [&h](const void *p, size_t n) {
        const auto *b = static_cast<const unsigned char *>(p);
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    };
    mix(m.vertices.data(), m.vertices.size() * sizeof(V3));
    mix(m.triangles.data(), m.triangles.size() * sizeof(uint32_t));
    mix(m.faces.data(), m.faces.size() * sizeof(uint32_t));
    mix(m.driven.data(), m.driven.size());
    return h;
}

double msBetween(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

RequestCopy::RequestCopy(const hs_request &r) : base(r) {
    frequencies.assign(r.frequencies, r.frequencies + r.frequency_count);
    if (r.plan_frequency_count)
        raster.assign(r.plan_frequencies, r.plan_frequencies + r.plan_frequency_count);
    observers.assign(r.observers, r.observers + 3 * r.observer_count);
    offsets.assign(r.excitation_face_offsets, r.excitation_face_offsets + r.excitation_count + 1);
    const size_t faces = offsets.back();
    faceIds.assign(r.excitation_face_ids, r.excitation_face_ids + faces);
    velocities.assign(r.excitation_velocities, r.excitation_velocities + 2 * faces);
    base.frequencies = nullptr;
    base.plan_frequencies = nullptr;
    base.plan_frequency_count = 0;
}

hs_request RequestCopy::view(const std::vector<double> &freqs, const std::vector<double> &planRaster) const {
    hs_request r = base;
    r.frequencies = freqs.data();
    r.frequency_count = freqs.size();
    r.plan_frequencies = planRaster.empty() ? nullptr : planRaster.data();
    r.plan_frequency_count = planRaster.size();
    r.observers = observers.empty() ? nullptr : observers.data();
    r.excitation_face_offsets = offsets.data();
    r.excitation_face_ids = faceIds.empty() ? nullptr : faceIds.data();
    r.excitation_velocities = velocities.empty() ? nullptr : velocities.data();
    return r;
}

bool RequestCopy::compatible(const RequestCopy &o) const {
    return base.density == o.base.density && base.sound_speed == o.base.sound_speed &&
           base.excitation_count == o.base.excitation_count && base.observer_count == o.base.observer_count &&
           base.far_field == o.base.far_field && std::memcmp(base.far_origin, o.base.far_origin, sizeof base.far_origin) == 0 &&
           base.far_reference_distance == o.base.far_reference_distance &&
           std::memcmp(&base.numerics, &o.base.numerics, sizeof base.numerics) == 0 && observers == o.observers &&
           offsets == o.offsets && faceIds == o.faceIds && velocities == o.velocities && raster == o.raster;
}

Server::Server(const hs_serve_options &options) : options_(options) {
    if (options_.workers < 1 || options_.workers > 64 || !(options_.memory_fraction > 0) ||
        options_.memory_fraction > 0.95 || options_.resident_meshes < 1 || !std::isfinite(options_.planning_frequency) ||
        options_.planning_frequency < 0 || options_.max_batch_frequencies < 1 || options_.max_batch_frequencies > 32)
        throw InvalidArgument("Invalid serving options.");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        throw CudaError("No CUDA device is available.");
    cudaOk(cudaGetDevice(&device_), "CUDA device");
    size_t free = 0, total = 0;
    cudaOk(cudaMemGetInfo(&free, &total), "CUDA memory query");
    budget_ = size_t(double(free) * options_.memory_fraction);
    for (uint32_t i = 0; i < options_.workers; ++i)
        workers_.emplace_back([this, i] { worker(int(i)); });
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        stop_ = true;
        for (auto &job : queue_) {
            job->error = std::make_exception_ptr(Cancelled());
            job->done = true;
        }
        queue_.clear();
    }
    work_.notify_all();
    done_.notify_all();
    for (auto &t : workers_)
        t.join();
}

uint64_t Server::submit(MeshInput mesh, const hs_request &request) {
    validateExteriorSurface(mesh);  // reject bad meshes at the door, not on a worker
    auto job = std::make_shared<Job>(Job{0, meshKey(mesh), std::make_shared<const MeshInput>(std::move(mesh)),
                                         RequestCopy(request)});
    const double limit = options_.planning_frequency;
    const auto &raster = job->request.raster;
    for (double f : job->request.frequencies) {
        if (!std::isfinite(f) || f <= 0 || (limit > 0 && f > limit))
            throw InvalidArgument("Served frequencies must be finite, positive and at most the planning frequency.");
        if (!raster.empty() && std::find(raster.begin(), raster.end(), f) == raster.end())
            throw InvalidArgument("Solved frequency is invalid or absent from its interaction planning raster.");
    }
    std::lock_guard<std::mutex> lock(mutex_);
    if (stop_)
        throw Cancelled();
    job->ticket = nextTicket_++;
    job->arrival = Clock::now();
    jobs_[job->ticket] = job;
    queue_.push_back(job);
    work_.notify_one();
    return job->ticket;
}

std::unique_ptr<Result> Server::wait(uint64_t ticket, hs_serve_timing &timing) {
    std::unique_lock<std::mutex> lock(mutex_);
    auto it = jobs_.find(ticket);
    if (it == jobs_.end())
        throw InvalidArgument("Unknown or already collected serving ticket.");
    auto job = it->second;
    done_.wait(lock, [&] { return job->done; });
    jobs_.erase(it);
    timing = hs_serve_timing{};
    timing.queue_ms = msBetween(job->arrival, job->start);
    timing.run_ms = msBetween(job->start, job->finish);
    timing.latency_ms = msBetween(job->arrival, job->finish);
    timing.footprint_bytes = job->footprint;
    timing.batched_requests = job->batched;
    if (job->error)
        std::rethrow_exception(job->error);
    return std::move(job->result);
}

// Under the lock: the oldest queued request whose mesh is idle, with the
// compatible queued requests on the same mesh, if its footprint fits.
std::vector<std::shared_ptr<Server::Job>> Server::takeGroup(size_t &footprint) {
    for (auto it = queue_.begin(); it != queue_.end(); ++it) {
        const auto &head = *it;
        auto s = sessions_.find(head->meshKey);
        if (s != sessions_.end() && s->second.busy)
            continue;  // another worker is on this mesh; later requests on other meshes may go
        std::vector<std::shared_ptr<Job>> group{head};
        std::set<double> freqs(head->request.frequencies.begin(), head->request.frequencies.end());
        if (options_.planning_frequency > 0 || !head->request.raster.empty())
            for (auto jt = std::next(it); jt != queue_.end(); ++jt)
                if ((*jt)->meshKey == head->meshKey && (*jt)->request.compatible(head->request)) {
                    std::set<double> merged = freqs;
                    merged.insert((*jt)->request.frequencies.begin(), (*jt)->request.frequencies.end());
                    if (merged.size() > 4 * size_t(options_.max_batch_frequencies))
                        break;
                    freqs = std::move(merged);
                    group.push_back(*jt);
                }
        const auto &mesh = *head->mesh;
        const size_t T = mesh.faces.size(), N = mesh.vertices.size();
        const hs_numerics &o = head->request.base.numerics;
        const bool mixed = o.precision == HS_PRECISION_MIXED;
        const uint32_t E = uint32_t(head->request.base.excitation_count), O = uint32_t(head->request.base.observer_count);
        uint32_t B = uint32_t(std::min<size_t>(freqs.size(), options_.max_batch_frequencies));
        const bool fmm = o.acceleration == HS_FAST_MULTIPOLE;
        size_t need = fmm ? fmmSolveFootprint(T, N, E, O, o.fmm_restart_length)
                          : solveFootprint(T, N, E, O, B, mixed, o.fmm_restart_length);
        while (!fmm && B > 1 && need > budget_) {
            B = (B + 1) / 2;
            need = solveFootprint(T, N, E, O, B, mixed, o.fmm_restart_length);
        }
        if (need > budget_) {
            // cannot run even alone: fail it here
            for (auto &job : group) {
                job->error = std::make_exception_ptr(OutOfMemory("Served request needs " + std::to_string(need >> 20) +
                                                                 " MiB of device memory; the serving budget is " +
                                                                 std::to_string(budget_ >> 20) + " MiB."));
                job->done = true;
            }
            for (auto &job : group)
                queue_.erase(std::find(queue_.begin(), queue_.end(), job));
            done_.notify_all();
            return takeGroup(footprint);
        }
        // other idle resident sessions hold memory too; the head's own session is covered by `need`
        if (reserved_ + idleBytes(head->meshKey) + need > budget_) {
            evictIdle(reserved_ + idleBytes(head->meshKey) + need - budget_, head->meshKey);
            if (reserved_ + idleBytes(head->meshKey) + need > budget_)
                return {};  // wait: oldest-first admission, nothing jumps a request that does not fit yet
        }
        for (auto &job : group)
            queue_.erase(std::find(queue_.begin(), queue_.end(), job));
        footprint = need;
        return group;
    }
    return {};
}

// Device bytes held by idle resident sessions other than `keep`'s.
size_t Server::idleBytes(uint64_t keep) const {
    size_t bytes = 0;
    for (const auto &[key, r] : sessions_)
        if (!r.busy && r.session && key != keep)
            bytes += r.session->residentBytes();
    return bytes;
}

// Frees idle resident sessions other than `keep`'s, least recently used
// first, until `needed` bytes are released or none is left.
void Server::evictIdle(size_t needed, uint64_t keep) {
    std::vector<std::pair<uint64_t, uint64_t>> idle;  // (last use, key)
    for (auto &[key, r] : sessions_)
        if (!r.busy && key != keep)
            idle.emplace_back(r.lastUse, key);
    std::sort(idle.begin(), idle.end());
    size_t freed = 0;
    for (auto &[use, key] : idle) {
        if (freed >= needed)
            break;
        auto it = sessions_.find(key);
        freed += it->second.session ? it->second.session->residentBytes() : 0;
        sessions_.erase(it);
    }
}

// Drops the least recently used idle resident session other than `keep`'s.
bool Server::evictOldestIdle(uint64_t keep) {
    auto oldest = sessions_.end();
    for (auto it = sessions_.begin(); it != sessions_.end(); ++it)
        if (!it->second.busy && it->first != keep && (oldest == sessions_.end() || it->second.lastUse < oldest->second.lastUse))
            oldest = it;
    if (oldest == sessions_.end())
        return false;
    sessions_.erase(oldest);
    return true;
}

void Server::worker(int index) {
    (void)index;
    cudaSetDevice(device_);
    cudaStream_t stream = nullptr;
    if (cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess)
        stream = nullptr;
    for (;;) {
        std::vector<std::shared_ptr<Job>> group;
        size_t footprint = 0;
        {
            std::unique_lock<std::mutex> lock(mutex_);
            work_.wait(lock, [&] {
                if (stop_)
                    return true;
                group = takeGroup(footprint);
                return !group.empty();
            });
            if (stop_ && group.empty())
                break;
            reserved_ += footprint;
            if (!sessions_.count(group.front()->meshKey)) {
                // a new resident mesh: keep at most resident_meshes, dropping the least recently used idle one
                while (sessions_.size() >= options_.resident_meshes && evictOldestIdle(group.front()->meshKey)) {
                }
            }
            auto &resident = sessions_[group.front()->meshKey];
            resident.busy = true;
            resident.lastUse = ++useClock_;
            const auto now = Clock::now();
            for (auto &job : group) {
                job->start = now;
                job->footprint = footprint;
                job->batched = uint32_t(group.size());
            }
        }
        const Job &head = *group.front();
        std::map<double, FrequencyResult> solved;  // results of the call so far, by frequency
        std::unique_ptr<Result> merged;
        std::exception_ptr error;
        std::vector<double> freqs;
        try {
            Session *session = nullptr;
            {
                std::lock_guard<std::mutex> lock(mutex_);
                session = sessions_[head.meshKey].session.get();
            }
            if (!session) {
                auto created = std::make_unique<Session>(*head.mesh, HS_RESIDENCY_DEVICE);
                std::lock_guard<std::mutex> lock(mutex_);
                sessions_[head.meshKey].session = std::move(created);
                session = sessions_[head.meshKey].session.get();
            }
            std::set<double> unique;
            for (auto &job : group)
                unique.insert(job->request.frequencies.begin(), job->request.frequencies.end());
            freqs.assign(unique.begin(), unique.end());
            // planning raster: the request's own (a client sweeping one mesh keeps its
            // plan), else the server's planning frequency, else the solved frequencies
            std::vector<double> raster;
            if (!head.request.raster.empty() || options_.planning_frequency > 0) {
                std::set<double> r(unique);
                r.insert(head.request.raster.begin(), head.request.raster.end());
                if (options_.planning_frequency > 0)
                    r.insert(options_.planning_frequency);
                raster.assign(r.begin(), r.end());
            }
            const size_t T = head.mesh->faces.size(), N = head.mesh->vertices.size();
            const size_t resident = solveFootprint(T, N, 0, 0, 0, false, 0);
            session->setMemoryBudget(footprint > resident ? footprint - resident : footprint);
            session->setStream(stream);
            const hs_request r = head.request.view(freqs, raster);
            // Continuous batching. With the server's fixed planning frequency every
            // request on a mesh shares one interaction plan, so while this call runs,
            // compatible requests on the mesh that arrive join its next frequency
            // batch (ahead of the call's remaining frequencies), and every request is
            // completed as soon as its last frequency is solved, not when the call ends.
            SolveHooks hooks;
            std::set<double> scheduled(unique);
            if (options_.planning_frequency > 0) {
                hooks.more = [&]() {
                    std::vector<double> extra;
                    std::lock_guard<std::mutex> lock(mutex_);
                    if (stop_)
                        return extra;
                    const auto now = Clock::now();
                    for (auto it = queue_.begin(); it != queue_.end();) {
                        const auto job = *it;
                        if (job->meshKey != head.meshKey || !job->request.compatible(head.request)) {
                            ++it;
                            continue;
                        }
                        job->start = now;
                        job->footprint = footprint;
                        for (double f : job->request.frequencies)
                            if (scheduled.insert(f).second)
                                extra.push_back(f);
                        group.push_back(job);
                        it = queue_.erase(it);
                    }
                    return extra;
                };
            }
            hooks.done = [&](const FrequencyResult &fr) {
                solved.emplace(fr.frequency, fr);
                std::lock_guard<std::mutex> lock(mutex_);
                bool any = false;
                for (auto &job : group) {
                    if (job->done || !std::all_of(job->request.frequencies.begin(), job->request.frequencies.end(),
                                                  [&](double f) { return solved.count(f) != 0; }))
                        continue;
                    auto result = std::make_unique<Result>();
                    result->T = head.mesh->faces.size();
                    result->N = head.mesh->vertices.size();
                    result->O = job->request.base.observer_count;
                    result->E = job->request.base.excitation_count;
                    result->peakDeviceBytes = session->residentBytes();
                    for (double f : job->request.frequencies)
                        result->frequencies.push_back(solved.at(f));
                    job->result = std::move(result);
                    job->finish = Clock::now();
                    job->batched = uint32_t(group.size());
                    job->done = true;
                    any = true;
                }
                if (any)
                    done_.notify_all();
            };
            std::lock_guard<std::mutex> solveLock(session->mutex);
            merged = session->solve(r, nullptr, nullptr, nullptr, &hooks);
        } catch (...) {
            error = std::current_exception();
        }
        {
            std::lock_guard<std::mutex> lock(mutex_);
            const auto now = Clock::now();
            for (auto &job : group) {
                if (job->done)  // completed early by the continuous-batching hook
                    continue;
                job->finish = now;
                job->batched = uint32_t(group.size());
                if (error) {
                    job->error = error;
                } else {
                    auto result = std::make_unique<Result>();
                    result->T = merged->T;
                    result->N = merged->N;
                    result->O = merged->O;
                    result->E = merged->E;
                    result->peakDeviceBytes = merged->peakDeviceBytes;
                    for (const auto &fr : merged->frequencies)
                        solved.emplace(fr.frequency, fr);
                    for (double f : job->request.frequencies)
                        result->frequencies.push_back(solved.at(f));
                    job->result = std::move(result);
                }
                job->done = true;
            }
            reserved_ -= footprint;
            auto it = sessions_.find(head.meshKey);
            if (it != sessions_.end())
                it->second.busy = false;
        }
        done_.notify_all();
        work_.notify_all();
    }
    if (stream)
        cudaStreamDestroy(stream);
}

}  // namespace hsb
