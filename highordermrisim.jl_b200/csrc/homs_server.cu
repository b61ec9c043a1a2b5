// Serving loop of libhoms: continuous batching of independent simulations.
//
// The reference keeps one persistent worker per device and runs prepared
// simulations one after another (src/simulation/PreparedSimulation.jl:144-258).
// Here a server owns `slots` contexts -- each with its own CUDA stream and its
// own cached device workspace -- one worker thread per slot, and a dispatcher
// thread with a stream of its own.  Requests wait in submission order; the
// request at the head of the queue is admitted as soon as a worker is free and
// its estimated device footprint fits in the byte budget beside the requests
// already in flight.
//
// A split-mode request is prepared by its worker (phantom and sequence on the
// device, initial state, split tables) and then joins the dispatcher's
// rounds.  A round issues, for every request in it, the work up to its next
// fused job (RF blocks, the next segment's prologue), then ONE persistent
// launch of the split kernel over all those jobs per output width (the jobs'
// (tile x chunk) work items in one device-side item space), then every
// request's finalize.  Requests that arrive join at the next round, so small
// requests share the GPU's SMs instead of each launching a partly empty grid.
// When a request's last job is done its worker copies the results out.
// Plain-mode requests run homs_simulate on their worker's context.  Either way
// a request computes exactly what homs_simulate computes for it: each job's
// work items and integer accumulators are its own, and their sums are exact,
// so its result does not depend on what runs beside it.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/homs.h"
#include "homs_internal.cuh"
#include "homs_split.cuh"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
    homs_phantom phantom;
    const homs_resident *resident = nullptr;  // set: run on this device-resident phantom
    homs_sequence seq;
    homs_run_options opts;
    homs_state state;
    bool has_state = false;
    void *sig = nullptr;
    homs_memory sig_memory = HOMS_HOST;
    size_t bytes = 0;  // admission estimate of the device footprint
    bool done = false;
    homs_status status = HOMS_EBUSY;
    std::string error;
    double t_submit = 0, t_start = 0, t_finish = 0;
};

// Upper estimate of the device memory one simulation needs (inputs, state,
// signal, staging of host sensitivities, and the path's work buffers).
// With `resident` the phantom's arrays, basis and pre-split sensitivities are
// already on the device and are left out.
size_t estimate_bytes(int64_t nspins, int32_t ncoils, homs_dtype dtype, const homs_sequence &q,
                      const homs_run_options &o, bool resident) {
    const double es = (dtype == HOMS_F64 || o.mode == HOMS_SPLIT) ? 8.0 : 4.0;  // split mode is resident in FP64
    const double ns = (double)nspins, nc = (double)ncoils, nt = (double)q.nnodes;
    int64_t nadc = q.nnodes;
    if (q.memory == HOMS_HOST) homs_count_adc(&q, &nadc);
    double b = ns * 3 * es;                                // state
    if (!resident) b += ns * (7 * es + 4 * es * nc);       // phantom, csm rows + staging
    b += nt * (26 * es + 2);                               // sampled sequence
    b += (double)nadc * nc * 2 * es;                       // signal
    if (o.mode == HOMS_SPLIT) {
        if (!resident) b += ns * homs::split_bytes_per_spin(ncoils);  // basis, phase and coil digit operands
        b += ns * 12.0;                                               // per-segment spin parameters
        // coil accumulators: per tile of 128 samples and slot of 2^18 chunks, 128 x 64 int64;
        // plus the phase prefix, phase A tiles and sample rows
        const double nchunks = std::ceil(ns / 32.0), tiles = std::ceil((double)nadc / 128.0) + q.nblocks;
        const double slots = std::ceil(nchunks / 262144.0);
        b += tiles * slots * 128 * 64 * 8 + (double)nadc * (192.0 + 96.0 + 8.0);
    } else {
        const double grid = std::ceil(ns / 256.0);
        b += std::min(768.0 * (1 << 20), grid * nc * 2 * es * (double)nadc);  // split-K partials
    }
    return (size_t)(b + (64 << 20));
}

}  // namespace

struct homs_server {
    int device = 0;
    size_t budget = 0;
    size_t inflight_bytes = 0;
    Clock::time_point t0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::map<int64_t, std::unique_ptr<Request>> requests;
    int64_t next_ticket = 1;
    bool stopping = false;
    std::vector<homs_context *> contexts;
    std::vector<std::thread> workers;
    // Split-mode runs handed to the dispatcher, and those in its rounds.
    struct Active {
        homs::ServerRun *run = nullptr;
        bool finished = false;
        homs_status status = HOMS_OK;
    };
    std::deque<Active *> pending;
    std::condition_variable cv_dispatch, cv_run;
    bool stop_dispatch = false;
    std::thread dispatcher;
    int64_t rounds = 0;  // rounds issued (diagnostics)

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

    // The head of the queue may start: a worker is asking, and it fits.
    bool head_fits() const {
        return !queue.empty() && (inflight_bytes == 0 || inflight_bytes + queue.front()->bytes <= budget);
    }

    void work(homs_context *ctx) {
        for (;;) {
            Request *r = nullptr;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] { return head_fits() || (stopping && queue.empty()); });
                if (queue.empty()) return;  // stopping
                r = queue.front();
                queue.pop_front();
                inflight_bytes += r->bytes;
                r->t_start = now();
            }
            homs_state *st = r->has_state ? &r->state : nullptr;
            homs_status s;
            if (homs::server_run_eligible(r->resident ? nullptr : &r->phantom, &r->opts))
                s = run_in_rounds(ctx, r, st);
            else
                s = r->resident ? homs_simulate_resident(ctx, r->resident, &r->seq, &r->opts, st, r->sig, r->sig_memory)
                                : homs_simulate(ctx, &r->phantom, &r->seq, &r->opts, st, r->sig, r->sig_memory);
            {
                std::lock_guard<std::mutex> lk(mu);
                r->status = s;
                if (s != HOMS_OK) r->error = homs_last_error(ctx);
                r->t_finish = now();
                r->done = true;
                inflight_bytes -= r->bytes;
            }
            cv_done.notify_all();
            cv_work.notify_all();
        }
    }

    // A split-mode request: prepared here, its fused work done by the
    // dispatcher's rounds, its results copied out here.
    homs_status run_in_rounds(homs_context *ctx, Request *r, homs_state *st) {
        homs::ServerRun *run = nullptr;
        homs_status s = homs::server_run_prepare(ctx, r->resident ? nullptr : &r->phantom, r->resident, &r->seq,
                                                 &r->opts, st, &run);
        if (s != HOMS_OK) return s;
        Active a;
        a.run = run;
        {
            std::unique_lock<std::mutex> lk(mu);
            pending.push_back(&a);
            cv_dispatch.notify_all();
            cv_run.wait(lk, [&] { return a.finished; });
        }
        s = a.status;
        if (s == HOMS_OK) s = homs::server_run_finish(run, r->sig, r->sig_memory, st);
        homs::server_run_free(run);
        return s;
    }

    void dispatch() {
        cudaSetDevice(device);
        cudaStream_t ds = nullptr;
        cudaStreamCreateWithFlags(&ds, cudaStreamNonBlocking);
        // A run's own work (RF blocks, prologues, finalizes) goes on its
        // context's stream, so that the runs' small kernels overlap; the
        // round's fused launches go on `ds` after every run's prologue
        // (pre events), and each run's finalize after them (fused event).
        // At most two rounds ahead of the device.
        cudaEvent_t round_ev[2] = {nullptr, nullptr}, fused = nullptr;
        cudaEventCreateWithFlags(&round_ev[0], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&round_ev[1], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&fused, cudaEventDisableTiming);
        std::vector<Active *> act;
        std::map<Active *, cudaEvent_t> pre;
        int64_t k = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_dispatch.wait(lk, [&] { return !pending.empty() || !act.empty() || stop_dispatch; });
                if (act.empty() && pending.empty()) break;  // stopping
                for (Active *a : pending) {
                    act.push_back(a);
                    cudaEvent_t e = nullptr;
                    cudaEventCreateWithFlags(&e, cudaEventDisableTiming);
                    pre[a] = e;
                }
                pending.clear();
            }
            cudaEventSynchronize(round_ev[k & 1]);
            // The round: every run's work up to its next job, the jobs (by
            // output width, at most SPLIT_MAX_JOBS per launch), the finalizes.
            std::vector<std::pair<Active *, homs::SplitJobDesc>> jobs;
            std::vector<Active *> fin;
            for (Active *a : act) {
                homs::SplitJobDesc d;
                bool has = false;
                cudaStream_t rs = homs::server_run_stream(a->run);
                const homs_status s = homs::server_run_next(a->run, rs, &d, &has);
                if (s != HOMS_OK) {
                    a->status = s;
                    fin.push_back(a);
                } else if (has) {
                    jobs.emplace_back(a, d);
                    cudaEventRecord(pre[a], rs);
                    cudaStreamWaitEvent(ds, pre[a], 0);
                } else {
                    fin.push_back(a);
                }
            }
            std::stable_sort(jobs.begin(), jobs.end(),
                             [](const auto &x, const auto &y) { return x.second.n_mma < y.second.n_mma; });
            for (size_t b = 0; b < jobs.size();) {
                size_t e = b;
                std::vector<homs::SplitJobDesc> batch;
                while (e < jobs.size() && jobs[e].second.n_mma == jobs[b].second.n_mma &&
                       batch.size() < (size_t)homs::SPLIT_MAX_JOBS)
                    batch.push_back(jobs[e++].second);
                if (homs::split_launch(batch.data(), (int)batch.size(), ds) != cudaSuccess)
                    for (size_t q = b; q < e; ++q) jobs[q].first->status = HOMS_ECUDA;
                b = e;
            }
            cudaEventRecord(fused, ds);
            for (auto &ja : jobs) {
                Active *a = ja.first;
                cudaStream_t rs = homs::server_run_stream(a->run);
                cudaStreamWaitEvent(rs, fused, 0);
                if (a->status == HOMS_OK) a->status = homs::server_run_after(a->run, rs);
                if (a->status != HOMS_OK) fin.push_back(a);
            }
            for (Active *a : fin) homs::server_run_done(a->run, homs::server_run_stream(a->run));
            cudaEventRecord(round_ev[k & 1], ds);
            ++k;
            if (!fin.empty()) {
                std::lock_guard<std::mutex> lk(mu);
                for (Active *a : fin) {
                    a->finished = true;
                    act.erase(std::find(act.begin(), act.end(), a));
                    cudaEventDestroy(pre[a]);
                    pre.erase(a);
                }
                rounds = k;
                cv_run.notify_all();
            }
        }
        cudaStreamSynchronize(ds);
        cudaEventDestroy(round_ev[0]);
        cudaEventDestroy(round_ev[1]);
        cudaEventDestroy(fused);
        cudaStreamDestroy(ds);
    }
};

namespace {

homs_status enqueue(homs_server *srv, std::unique_ptr<Request> r, int64_t *ticket) {
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->stopping) return HOMS_ECLOSED;
    r->t_submit = srv->now();
    const int64_t id = srv->next_ticket++;
    Request *rp = r.get();
    srv->requests.emplace(id, std::move(r));
    if (rp->bytes > srv->budget) {
        // Larger than the whole admission budget: fail it here rather than block the queue.
        rp->status = HOMS_ENOMEM;
        rp->error = "the request's estimated device footprint exceeds the server's admission budget";
        rp->done = true;
        rp->t_start = rp->t_finish = rp->t_submit;
    } else {
        srv->queue.push_back(rp);
    }
    *ticket = id;
    srv->cv_work.notify_all();
    return HOMS_OK;
}

}  // namespace

extern "C" {

homs_status homs_server_create(const homs_server_options *opts, homs_server **out) {
    if (!opts || !out) return HOMS_EINVAL;
    *out = nullptr;
    const int slots = opts->slots > 0 ? opts->slots : 4;
    if (slots > 64 || opts->max_device_bytes < 0) return HOMS_EINVAL;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return HOMS_EUNSUPPORTED;
    }
    if (opts->device < 0 || opts->device >= ndev) return HOMS_EINVAL;
    auto srv = std::make_unique<homs_server>();
    srv->device = opts->device;
    srv->t0 = Clock::now();
    if (opts->max_device_bytes > 0) {
        srv->budget = (size_t)opts->max_device_bytes;
    } else {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(opts->device);
        size_t free_b = 0, total_b = 0;
        const cudaError_t e = cudaMemGetInfo(&free_b, &total_b);
        cudaSetDevice(prev);
        if (e != cudaSuccess) return HOMS_ECUDA;
        srv->budget = free_b / 4 * 3;
    }
    for (int k = 0; k < slots; ++k) {
        homs_context *ctx = nullptr;
        const homs_status s = homs_context_create(opts->device, nullptr, &ctx);
        if (s != HOMS_OK) {
            for (homs_context *c : srv->contexts) homs_context_destroy(c);
            return s;
        }
        srv->contexts.push_back(ctx);
    }
    homs_server *raw = srv.get();
    srv->dispatcher = std::thread([raw] { raw->dispatch(); });
    for (homs_context *ctx : srv->contexts) srv->workers.emplace_back([raw, ctx] { raw->work(ctx); });
    *out = srv.release();
    return HOMS_OK;
}


homs_status homs_server_submit(homs_server *srv, const homs_phantom *phantom, const homs_sequence *seq,
                               const homs_run_options *opts, homs_state *state, void *sig, homs_memory sig_memory,
                               int64_t *ticket) {
    if (!srv || !phantom || !seq || !opts || !ticket) return HOMS_EINVAL;
    auto r = std::make_unique<Request>();
    r->phantom = *phantom;
    r->seq = *seq;
    r->opts = *opts;
    if (state) {
        r->state = *state;
        r->has_state = true;
    }
    r->sig = sig;
    r->sig_memory = sig_memory;
    r->bytes = estimate_bytes(phantom->nspins, phantom->ncoils, phantom->dtype, *seq, *opts, false);
    return enqueue(srv, std::move(r), ticket);
}

homs_status homs_server_submit_resident(homs_server *srv, const homs_resident *res, const homs_sequence *seq,
                                        const homs_run_options *opts, homs_state *state, void *sig,
                                        homs_memory sig_memory, int64_t *ticket) {
    homs::ResidentShape shape;
    if (!srv || !seq || !opts || !ticket || !homs::resident_shape(res, &shape)) return HOMS_EINVAL;
    if (shape.device != srv->device) return HOMS_EINVAL;
    auto r = std::make_unique<Request>();
    r->resident = res;
    r->seq = *seq;
    r->opts = *opts;
    if (state) {
        r->state = *state;
        r->has_state = true;
    }
    r->sig = sig;
    r->sig_memory = sig_memory;
    r->bytes = estimate_bytes(shape.nspins, shape.ncoils, shape.compute, *seq, *opts, true);
    return enqueue(srv, std::move(r), ticket);
}

homs_status homs_server_poll(homs_server *srv, int64_t ticket) {
    if (!srv) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) return HOMS_EINVAL;
    return it->second->done ? it->second->status : HOMS_EBUSY;
}

homs_status homs_server_wait(homs_server *srv, int64_t ticket, double timeout_seconds) {
    if (!srv || !(timeout_seconds >= 0)) return HOMS_EINVAL;
    std::unique_lock<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) return HOMS_EINVAL;
    Request *r = it->second.get();
    const auto limit = std::chrono::duration<double>(std::min(timeout_seconds, 1e7));
    if (!srv->cv_done.wait_for(lk, limit, [r] { return r->done; })) return HOMS_ETIMEDOUT;
    return r->status;
}

homs_status homs_server_times(homs_server *srv, int64_t ticket, homs_request_times *out) {
    if (!srv || !out) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) return HOMS_EINVAL;
    out->submitted = it->second->t_submit;
    out->started = it->second->t_start;
    out->finished = it->second->t_finish;
    return it->second->done ? HOMS_OK : HOMS_EBUSY;
}

homs_status homs_server_estimate(homs_server *srv, int64_t ticket, int64_t *bytes) {
    if (!srv || !bytes) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) return HOMS_EINVAL;
    *bytes = (int64_t)it->second->bytes;
    return HOMS_OK;
}

const char *homs_server_error(homs_server *srv, int64_t ticket) {
    if (!srv) return "no server";
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) return "unknown ticket";
    return it->second->error.c_str();
}

homs_status homs_server_release(homs_server *srv, int64_t ticket) {
    if (!srv) return HOMS_EINVAL;
    std::lock_guard<std::mutex> lk(srv->mu);
    auto it = srv->requests.find(ticket);
    if (it == srv->requests.end()) return HOMS_EINVAL;
    if (!it->second->done) return HOMS_EBUSY;
    srv->requests.erase(it);
    return HOMS_OK;
}

homs_status homs_server_destroy(homs_server *srv) {
    if (!srv) return HOMS_EINVAL;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stopping = true;
    }
    srv->cv_work.notify_all();
    for (std::thread &t : srv->workers) t.join();
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop_dispatch = true;
    }
    srv->cv_dispatch.notify_all();
    srv->dispatcher.join();
    for (homs_context *c : srv->contexts) homs_context_destroy(c);
    delete srv;
    return HOMS_OK;
}

}  // extern "C"
