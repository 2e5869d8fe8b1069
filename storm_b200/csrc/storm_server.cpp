// Serving loop: many independent IMC problems advanced concurrently on one GPU.
//
// Requests (a problem descriptor, a step count and a time step) queue on the
// host.  A request is admitted when a slot is free and its estimated device
// memory fits the HBM budget; it then owns a StormHandle, whose census bank
// and material state stay on the device until its last step.  Worker threads
// take active problems round-robin and issue one time step at a time; every
// handle has its own non-blocking stream, so the kernels and copies of
// different problems overlap on the device while each worker waits on its
// own problem's host round trips.  Problems share no device state and each
// draws from its own seeded streams, so a problem's result does not depend on
// what else is running (up to the summation order of its FP64 tally atomics).
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "storm_cuda.h"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

double percentile(std::vector<double> v, double q) {
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const double pos = q * static_cast<double>(v.size() - 1);
    const size_t lo = static_cast<size_t>(pos);
    const size_t hi = std::min(lo + 1, v.size() - 1);
    const double f = pos - static_cast<double>(lo);
    return v[lo] * (1.0 - f) + v[hi] * f;
}

// A request with its own copy of every array the descriptor points to.
struct Request {
    uint64_t ticket = 0;
    StormProblemDesc desc{};
    std::vector<double> xe, ye, ze, T, mass, eint, ceint, sa, ss, rho;
    uint32_t steps = 0;
    double dt = 0.0;
    double *temperatureOut = nullptr;
    uint64_t estimate = 0;
    Clock::time_point submitted, admitted;
    // while active
    StormHandle *h = nullptr;
    uint64_t bytes = 0;
    uint32_t done = 0;
    bool busy = false;
    int status = STORM_OK;
    uint64_t segments = 0;
    double deviceMs = 0.0;
    std::vector<double> stepMs;
};

template <class T>
const T *copy_array(std::vector<T> &dst, const T *src, size_t n) {
    if (!src) return nullptr;
    dst.assign(src, src + n);
    return dst.data();
}

// Device bytes a problem will hold: the handle's particle buffers at its
// starting capacity plus per-cell arrays and the Random Walk tables.
uint64_t estimate_bytes(const StormProblemDesc &d) {
    const uint64_t N = static_cast<uint64_t>(d.nx) * d.ny * d.nz;
    uint64_t facePackets = 0;
    const uint64_t faceCells[6] = {static_cast<uint64_t>(d.ny) * d.nz, static_cast<uint64_t>(d.ny) * d.nz,
                                   static_cast<uint64_t>(d.nx) * d.nz, static_cast<uint64_t>(d.nx) * d.nz,
                                   static_cast<uint64_t>(d.nx) * d.ny, static_cast<uint64_t>(d.nx) * d.ny};
    for (int f = 0; f < 6; ++f)
        if (d.faces[f].source_temperature > 0.0) facePackets += d.faces[f].packets_per_face * faceCells[f];
    uint64_t cap = d.capacity ? d.capacity : std::max<uint64_t>(1u << 20, N * d.new_photons_per_cell * 4 + facePackets * 2);
    cap += cap / 4;
    return cap * 360 + N * 256 + (4u << 20);
}

}  // namespace

struct StormServer {
    StormServerConfig cfg{};
    std::mutex m;
    std::condition_variable cv;
    std::deque<std::unique_ptr<Request>> pending;
    std::vector<std::unique_ptr<Request>> active;
    std::deque<StormRequestResult> results;
    uint32_t admitting = 0;        // requests being created outside the lock
    uint32_t finishing = 0;        // requests being copied out and freed outside the lock
    uint64_t reserved = 0;         // device bytes held or reserved by admitted requests
    uint64_t peakBytes = 0;
    uint64_t nextTicket = 1;
    uint64_t submitted = 0, completed = 0, failed = 0, segments = 0;
    size_t rr = 0;                 // round-robin position in `active`
    bool stop = false;
    bool started = false;
    Clock::time_point first, last;
    std::vector<double> allStepMs;
    std::vector<std::thread> threads;

    void worker();
    bool admit_one(std::unique_lock<std::mutex> &lk);
    void finish(std::unique_lock<std::mutex> &lk, size_t idx);
};

// Admit the oldest pending request if a slot and the budget allow; the handle
// is created with the lock released.  Returns true if it admitted one.
bool StormServer::admit_one(std::unique_lock<std::mutex> &lk) {
    if (pending.empty()) return false;
    if (active.size() + admitting >= cfg.max_active) return false;
    Request *front = pending.front().get();
    if (reserved + front->estimate > cfg.hbm_budget_bytes && !(active.empty() && admitting == 0)) return false;
    std::unique_ptr<Request> r = std::move(pending.front());
    pending.pop_front();
    reserved += r->estimate;
    ++admitting;
    lk.unlock();
    r->admitted = Clock::now();
    r->status = storm_cuda_create(&r->desc, &r->h);
    if (r->status == STORM_OK) storm_cuda_memory_bytes(r->h, &r->bytes);
    lk.lock();
    --admitting;
    if (!started) {
        started = true;
        first = r->admitted;
    }
    if (r->status == STORM_OK) {
        reserved = reserved - r->estimate + r->bytes;
        peakBytes = std::max(peakBytes, reserved);
        active.push_back(std::move(r));
    } else {
        reserved -= r->estimate;
        StormRequestResult res{};
        res.ticket = r->ticket;
        res.status = r->status;
        res.queued_ms = ms_between(r->submitted, r->admitted);
        results.push_back(res);
        ++failed;
        last = Clock::now();
    }
    cv.notify_all();
    return true;
}

// Completion of active[idx] (not busy): copy results out, free the handle.
void StormServer::finish(std::unique_lock<std::mutex> &lk, size_t idx) {
    std::unique_ptr<Request> r = std::move(active[idx]);
    active.erase(active.begin() + static_cast<std::ptrdiff_t>(idx));
    ++finishing;
    lk.unlock();
    if (r->status == STORM_OK && r->temperatureOut)
        r->status = storm_cuda_get_cell_arrays(r->h, r->temperatureOut, nullptr, nullptr, nullptr, nullptr, nullptr,
                                               nullptr);
    storm_cuda_destroy(r->h);
    r->h = nullptr;
    const Clock::time_point now = Clock::now();
    StormRequestResult res{};
    res.ticket = r->ticket;
    res.status = r->status;
    res.steps = r->done;
    res.segments = r->segments;
    res.device_bytes = r->bytes;
    res.queued_ms = ms_between(r->submitted, r->admitted);
    res.active_ms = ms_between(r->admitted, now);
    res.step_ms_p50 = percentile(r->stepMs, 0.50);
    res.step_ms_p99 = percentile(r->stepMs, 0.99);
    res.step_ms_max = r->stepMs.empty() ? 0.0 : *std::max_element(r->stepMs.begin(), r->stepMs.end());
    res.device_ms = r->deviceMs;
    lk.lock();
    --finishing;
    reserved -= r->bytes;
    results.push_back(res);
    if (r->status == STORM_OK) ++completed; else ++failed;
    segments += r->segments;
    allStepMs.insert(allStepMs.end(), r->stepMs.begin(), r->stepMs.end());
    last = now;
    cv.notify_all();
}

void StormServer::worker() {
    std::unique_lock<std::mutex> lk(m);
    for (;;) {
        while (admit_one(lk)) {
        }
        // next idle active problem, round-robin
        Request *r = nullptr;
        size_t idx = 0;
        for (size_t k = 0; k < active.size(); ++k) {
            size_t q = (rr + k) % active.size();
            if (!active[q]->busy) {
                r = active[q].get();
                idx = q;
                break;
            }
        }
        if (!r) {
            if (stop && pending.empty() && active.empty() && admitting == 0 && finishing == 0) return;
            cv.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        rr = idx + 1;
        r->busy = true;
        lk.unlock();
        const Clock::time_point t0 = Clock::now();
        StormStepStats st{};
        const int rc = storm_cuda_step(r->h, r->dt, &st);
        const double wall = ms_between(t0, Clock::now());
        lk.lock();
        r->busy = false;
        if (rc == STORM_OK) {
            ++r->done;
            r->segments += st.segments;
            r->deviceMs += st.step_ms;
            r->stepMs.push_back(wall);
        } else {
            r->status = rc;
        }
        if (rc != STORM_OK || r->done >= r->steps) {
            // find its current index (other workers may have reordered `active`)
            for (size_t q = 0; q < active.size(); ++q)
                if (active[q].get() == r) {
                    finish(lk, q);
                    break;
                }
        }
        cv.notify_all();
    }
}

extern "C" {

int storm_server_create(const StormServerConfig *cfg, StormServer **out) {
    if (!cfg || !out || cfg->max_active == 0 || cfg->workers == 0 || cfg->workers > 256) return STORM_ERR_INVALID_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return STORM_ERR_NO_DEVICE;
    if (cfg->device < 0 || cfg->device >= ndev) return STORM_ERR_INVALID_ARG;
    auto s = std::make_unique<StormServer>();
    s->cfg = *cfg;
    if (s->cfg.hbm_budget_bytes == 0) {
        size_t freeB = 0, totalB = 0;
        cudaSetDevice(cfg->device);
        cudaMemGetInfo(&freeB, &totalB);
        s->cfg.hbm_budget_bytes = static_cast<uint64_t>(freeB * 0.9);
    }
    for (uint32_t w = 0; w < cfg->workers; ++w) {
        s->threads.emplace_back([srv = s.get(), dev = cfg->device] {
            cudaSetDevice(dev);
            srv->worker();
        });
    }
    *out = s.release();
    return STORM_OK;
}

int storm_server_submit(StormServer *s, const StormProblemDesc *d, uint32_t steps, double dt, double *temperature_out,
                        uint64_t *ticket) {
    if (!s || !d || steps == 0 || !(dt > 0.0)) return STORM_ERR_INVALID_ARG;
    if (d->abi_version != STORM_CUDA_ABI_VERSION || !d->x_edges || !d->y_edges || !d->z_edges || !d->temperature ||
        !d->mass || !d->internal_energy)
        return STORM_ERR_INVALID_ARG;
    auto r = std::make_unique<Request>();
    r->desc = *d;
    const size_t N = static_cast<size_t>(d->nx) * d->ny * d->nz;
    r->desc.x_edges = copy_array(r->xe, d->x_edges, d->nx + 1);
    r->desc.y_edges = copy_array(r->ye, d->y_edges, d->ny + 1);
    r->desc.z_edges = copy_array(r->ze, d->z_edges, d->nz + 1);
    r->desc.temperature = copy_array(r->T, d->temperature, N);
    r->desc.mass = copy_array(r->mass, d->mass, N);
    r->desc.internal_energy = copy_array(r->eint, d->internal_energy, N);
    r->desc.cell_internal_energy = copy_array(r->ceint, d->cell_internal_energy, N);
    r->desc.sigma_a = copy_array(r->sa, d->sigma_a, N);
    r->desc.sigma_s = copy_array(r->ss, d->sigma_s, N);
    r->desc.density_factor = copy_array(r->rho, d->density_factor, N);
    r->desc.device = s->cfg.device;
    r->steps = steps;
    r->dt = dt;
    r->temperatureOut = temperature_out;
    r->estimate = estimate_bytes(r->desc);
    r->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(s->m);
    if (s->stop) return STORM_ERR_INVALID_ARG;
    r->ticket = s->nextTicket++;
    if (ticket) *ticket = r->ticket;
    ++s->submitted;
    s->pending.push_back(std::move(r));
    s->cv.notify_all();
    return STORM_OK;
}

int storm_server_poll(StormServer *s, StormRequestResult *res, uint32_t capacity, uint32_t *count) {
    if (!s || !count || (capacity && !res)) return STORM_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->m);
    uint32_t n = 0;
    while (n < capacity && !s->results.empty()) {
        res[n++] = s->results.front();
        s->results.pop_front();
    }
    *count = n;
    return STORM_OK;
}

int storm_server_drain(StormServer *s) {
    if (!s) return STORM_ERR_INVALID_ARG;
    std::unique_lock<std::mutex> lk(s->m);
    s->cv.wait(lk, [s] { return s->pending.empty() && s->active.empty() && s->admitting == 0 && s->finishing == 0; });
    return STORM_OK;
}

int storm_server_stats(StormServer *s, StormServerStats *o) {
    if (!s || !o) return STORM_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->m);
    *o = StormServerStats{};
    o->submitted = s->submitted;
    o->completed = s->completed;
    o->failed = s->failed;
    o->active = s->active.size();
    o->queued = s->pending.size();
    o->segments = s->segments;
    o->busy_ms = s->started ? ms_between(s->first, s->last) : 0.0;
    o->step_ms_p50 = percentile(s->allStepMs, 0.50);
    o->step_ms_p99 = percentile(s->allStepMs, 0.99);
    o->peak_device_bytes = s->peakBytes;
    o->budget_bytes = s->cfg.hbm_budget_bytes;
    return STORM_OK;
}

int storm_server_destroy(StormServer *s) {
    if (!s) return STORM_ERR_INVALID_ARG;
    {
        std::lock_guard<std::mutex> lk(s->m);
        s->stop = true;
        s->cv.notify_all();
    }
    for (auto &t : s->threads) t.join();
    delete s;
    return STORM_OK;
}

}  // extern "C"
