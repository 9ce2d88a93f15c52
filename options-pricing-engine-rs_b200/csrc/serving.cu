// Device-resident serving loop with continuous batching.
//
// No reference twin: the reference prices and calibrates synchronously, one
// call at a time (batch.rs:23-48, calibration.rs:204-210).  The server takes
// surface-repricing and calibration requests as they arrive and runs them on
// the GPU through the same kernels:
//
//  * submit() copies a request into host memory and queues it (non-blocking);
//  * two scheduler threads, one per request kind, form micro-batches from
//    everything pending whenever an in-flight slot and device memory are
//    free: all pending reprices of one model go into ONE multi-surface
//    persistent launch (each request is a surface with its own parameters),
//    pending calibrations into ONE batched device-LM run (one
//    conditional-WHILE graph).  The slow host part of a calibration batch
//    (graph capture and instantiation) runs on its own thread outside the
//    server lock, so it never delays a reprice launch;
//  * reprices run on high-priority streams; calibrations run one batch at a
//    time on low-priority streams with their kernels' grids capped at a share
//    of the GPU's block slots: a reprice's blocks are scheduled ahead of
//    queued calibration blocks and find free slots on every SM while a
//    calibration runs;
//  * admission is by device memory: at creation the server reserves a slab
//    of a configurable fraction of the FREE HBM (cudaMemGetInfo); a batch is
//    launched when its buffers fit in the slab, requests that can never fit
//    are rejected (OPE_ERR_REJECTED);
//  * several micro-batches are in flight at once on different streams, so
//    work admitted later overlaps work already running on the device;
//  * completion is detected with events; results are copied to the request,
//    its latency (submit -> results on the host) recorded, waiters woken.
//
// Every contract is priced by the same per-unit kernel code and every LM
// state machine is independent of the others in its batch, so a request's
// results are bit-identical whether it runs alone or mixed with others.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace ope {

namespace {

using Clock = std::chrono::steady_clock;

double ms_since(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

enum ReqState { RQ_PENDING = 0, RQ_RUNNING = 1, RQ_DONE = 2, RQ_FAILED = 3, RQ_CANCELLED = 4, RQ_REJECTED = 5 };
enum ReqKind { RK_PRICE = 0, RK_CALIB = 1 };

struct Request {
    uint64_t id = 0;
    int kind = RK_PRICE;
    int model = OPE_MODEL_HESTON;
    std::vector<ope_contract> con;
    std::vector<double> iv;      // calibration: market IVs
    std::vector<double> params;  // reprice: one parameter set; calibration: p0
    std::vector<double> prices;  // reprice result
    ope_calib_result calib{};    // calibration result
    int state = RQ_PENDING;
    int error = OPE_OK;
    std::string message;
    Clock::time_point t_submit, t_done;
};

// First-fit allocator over [0, cap) in 256-byte units.
class Slab {
   public:
    explicit Slab(size_t cap) : cap_(cap) { free_[0] = cap; }
    bool alloc(size_t bytes, size_t* off) {
        bytes = align_up(std::max<size_t>(bytes, 256), 256);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                const size_t rest = it->second - bytes;
                const size_t at = it->first + bytes;
                free_.erase(it);
                if (rest) free_[at] = rest;
                used_ += bytes;
                peak_ = std::max(peak_, used_);
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = align_up(std::max<size_t>(bytes, 256), 256);
        used_ -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
    size_t capacity() const { return cap_; }
    size_t peak() const { return peak_; }

   private:
    size_t cap_, used_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;
};

struct Job {
    int kind = RK_PRICE, model = 0;
    std::vector<std::shared_ptr<Request>> reqs;
    int slot = -1;
    size_t dev_off = 0, dev_bytes = 0, pin_off = 0, pin_bytes = 0;
    cudaEvent_t done = nullptr;
    CalibGraph* graph = nullptr;
    // result locations in pinned memory
    double* prices_h = nullptr;
    ope_calib_result* calib_h = nullptr;
};

}  // namespace

struct Server {
    ope_server_config cfg{};
    int device = 0;
    double tol = OPE_REF_TOL;
    void* dev_base = nullptr;
    char* pin_base = nullptr;
    std::unique_ptr<Slab> dev_slab, pin_slab;
    std::vector<cudaStream_t> streams_hi, streams_lo;  // per slot: reprice / calibration streams
    std::vector<bool> slot_busy;
    std::mutex mu;
    std::condition_variable cv_sched, cv_done;
    std::deque<std::shared_ptr<Request>> pending;
    std::map<uint64_t, std::shared_ptr<Request>> all;
    std::vector<Job> inflight;
    std::atomic<bool> stop{false};
    std::thread thr_price, thr_calib;
    uint64_t next_id = 1;
    ope_server_stats stats{};
    std::string fatal;
};

namespace {

size_t price_job_dev_bytes(size_t n, size_t ns, int dim) {
    return align_up(n * sizeof(ope_contract), 256) + align_up((ns + 1) * sizeof(int64_t), 256) +
           align_up(ns * dim * sizeof(double), 256) + align_up(n * sizeof(double), 256) + price_scratch_bytes(n);
}

// Form and launch one micro-batch of `kind` from the pending queue.  Called
// with `lk` held; the lock is released while the batch is packed and
// enqueued, and held again on return.  Returns true if something was launched.
bool launch_batch(Server& S, int kind, std::unique_lock<std::mutex>& lk) {
    if (S.pending.empty()) return false;
    // A free slot; calibration batches never take the last free one, so an
    // arriving reprice always finds a slot.
    int slot = -1;
    size_t n_free = 0;
    for (size_t i = 0; i < S.slot_busy.size(); ++i)
        if (!S.slot_busy[i]) { n_free += 1; if (slot < 0) slot = (int)i; }
    if (slot < 0) return false;
    if (kind == RK_CALIB) {
        // one calibration batch at a time (later ones join the next batch), and
        // never in the last free slot: with its grids capped, the rest of the
        // GPU's block slots and at least one stream stay free for reprices
        if (n_free < 2 && S.slot_busy.size() > 1) return false;
        for (const auto& j : S.inflight)
            if (j.kind == RK_CALIB) return false;
    }
    // The oldest pending request of this kind decides the model; every pending
    // request of that kind and model is taken, FIFO, while the batch still fits
    // the contract limit and the admission budget (the whole slab).
    const Request* lead = nullptr;
    for (const auto& r : S.pending)
        if (r->kind == kind) { lead = r.get(); break; }
    if (!lead) return false;
    const int model = lead->model;
    const int dim = param_stride(model);
    auto dev_need = [&](size_t n, size_t ns) {
        return kind == RK_PRICE ? price_job_dev_bytes(n, ns, dim) : calib_workspace_bytes(n, ns, dim);
    };
    auto pin_need = [&](size_t n, size_t ns) {
        size_t b = n * sizeof(ope_contract) + (ns + 1) * sizeof(int64_t) + ns * dim * sizeof(double) + 4096;
        return b + (kind == RK_PRICE ? n * sizeof(double)
                                     : n * sizeof(double) + calib_pinned_bytes(n, ns, dim) +
                                           ns * sizeof(ope_calib_result));
    };
    std::vector<std::shared_ptr<Request>> take;
    size_t n = 0;
    const size_t max_n = S.cfg.max_batch_contracts;
    for (auto it = S.pending.begin(); it != S.pending.end();) {
        Request& r = **it;
        const size_t n2 = n + r.con.size(), ns2 = take.size() + 1;
        const bool fits = dev_need(n2, ns2) <= S.dev_slab->capacity() && pin_need(n2, ns2) <= S.pin_slab->capacity();
        if (r.kind == kind && r.model == model && (take.empty() || (n2 <= max_n && fits))) {
            if (take.empty() && !fits) {  // can never be admitted
                r.state = RQ_REJECTED;
                r.error = OPE_ERR_REJECTED;
                r.message = "request needs more memory than the server's admission budget";
                r.t_done = Clock::now();
                S.stats.rejected += 1;
                S.cv_done.notify_all();
                it = S.pending.erase(it);
                return false;
            }
            take.push_back(*it);
            n = n2;
            it = S.pending.erase(it);
        } else {
            ++it;
        }
    }
    const size_t ns = take.size();
    const size_t dev_bytes = dev_need(n, ns), pin_bytes = pin_need(n, ns);
    size_t dev_off = 0, pin_off = 0;
    auto requeue = [&]() {  // not enough free memory now: keep arrival order, retry after a completion
        for (auto it = take.rbegin(); it != take.rend(); ++it) S.pending.push_front(*it);
    };
    if (!S.dev_slab->alloc(dev_bytes, &dev_off)) { requeue(); return false; }
    if (!S.pin_slab->alloc(pin_bytes, &pin_off)) {
        S.dev_slab->release(dev_off, dev_bytes);
        requeue();
        return false;
    }
    S.slot_busy[slot] = true;
    for (auto& r : take) r->state = RQ_RUNNING;
    Job J;
    J.kind = kind;
    J.model = model;
    J.reqs = take;
    J.slot = slot;
    J.dev_off = dev_off;
    J.dev_bytes = dev_bytes;
    J.pin_off = pin_off;
    J.pin_bytes = pin_bytes;
    cudaStream_t st = kind == RK_PRICE ? S.streams_hi[slot] : S.streams_lo[slot];
    char* dev = static_cast<char*>(S.dev_base) + dev_off;
    char* pin = S.pin_base + pin_off;
    const double tol = S.tol;
    const double calib_fraction = S.cfg.calib_sm_fraction;

    // The requests, slot, device and pinned regions now belong to this batch:
    // pack and enqueue without the lock.
    lk.unlock();
    OPE_RANGE(kind == RK_PRICE ? "ope.server.reprice_batch" : "ope.server.calibration_batch");
    char* p = pin;
    ope_contract* con_h = reinterpret_cast<ope_contract*>(p);
    p += align_up(n * sizeof(ope_contract), 256);
    int64_t* off_h = reinterpret_cast<int64_t*>(p);
    p += align_up((ns + 1) * sizeof(int64_t), 256);
    double* par_h = reinterpret_cast<double*>(p);
    p += align_up(ns * dim * sizeof(double), 256);
    size_t at = 0;
    off_h[0] = 0;
    for (size_t s = 0; s < ns; ++s) {
        Request& r = *take[s];
        std::memcpy(con_h + at, r.con.data(), r.con.size() * sizeof(ope_contract));
        std::memcpy(par_h + s * dim, r.params.data(), dim * sizeof(double));
        at += r.con.size();
        off_h[s + 1] = (int64_t)at;
    }
    int rc = OPE_OK;
    if (kind == RK_PRICE) {
        char* d = dev;
        ope_contract* d_con = reinterpret_cast<ope_contract*>(d);
        d += align_up(n * sizeof(ope_contract), 256);
        int64_t* d_off = reinterpret_cast<int64_t*>(d);
        d += align_up((ns + 1) * sizeof(int64_t), 256);
        double* d_par = reinterpret_cast<double*>(d);
        d += align_up(ns * dim * sizeof(double), 256);
        double* d_out = reinterpret_cast<double*>(d);
        d += align_up(n * sizeof(double), 256);
        J.prices_h = reinterpret_cast<double*>(p);
        rc = check_cuda(cudaMemcpyAsync(d_con, con_h, n * sizeof(ope_contract), cudaMemcpyHostToDevice, st), "h2d");
        if (rc == OPE_OK)
            rc = check_cuda(cudaMemcpyAsync(d_off, off_h, (ns + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st), "h2d");
        if (rc == OPE_OK)
            rc = check_cuda(cudaMemcpyAsync(d_par, par_h, ns * dim * sizeof(double), cudaMemcpyHostToDevice, st), "h2d");
        if (rc == OPE_OK)
            rc = launch_price_persistent(model, d_con, n, d_off, ns, nullptr, d_par, tol, d_out,
                                         carve_price_scratch(d, n), st);
        if (rc == OPE_OK)
            rc = check_cuda(cudaMemcpyAsync(J.prices_h, d_out, n * sizeof(double), cudaMemcpyDeviceToHost, st), "d2h");
    } else {
        double* iv_h = reinterpret_cast<double*>(p);
        p += align_up(n * sizeof(double), 256);
        at = 0;
        for (size_t s = 0; s < ns; ++s) {
            std::memcpy(iv_h + at, take[s]->iv.data(), take[s]->iv.size() * sizeof(double));
            at += take[s]->iv.size();
        }
        char* cpin = p;
        p += align_up(calib_pinned_bytes(n, ns, dim), 256);
        J.calib_h = reinterpret_cast<ope_calib_result*>(p);
        J.graph = calib_graph_new();
        // this thread's persistent launches (captured into the LM graph) leave
        // the rest of the block slots to reprices
        ThreadCtx& c = tctx();
        c.grid_fraction = calib_fraction;
        rc = calib_enqueue(model, con_h, iv_h, nullptr, n, off_h, off_h, ns, par_h, J.calib_h, tol,
                           cudaMemcpyHostToDevice, cudaMemcpyDeviceToHost, dev, cpin, st, J.graph);
        c.grid_fraction = 1.0;
    }
    if (rc == OPE_OK) rc = check_cuda(cudaEventCreateWithFlags(&J.done, cudaEventDisableTiming), "event");
    if (rc == OPE_OK) rc = check_cuda(cudaEventRecord(J.done, st), "event");
    const std::string err = rc != OPE_OK ? tctx().last_error : std::string();
    if (rc != OPE_OK) {
        cudaStreamSynchronize(st);
        cudaGetLastError();
        if (J.done) cudaEventDestroy(J.done);
        if (J.graph) calib_graph_delete(J.graph);
    }
    lk.lock();
    if (rc != OPE_OK) {
        for (auto& r : take) {
            r->state = RQ_FAILED;
            r->error = rc;
            r->message = err;
            r->t_done = Clock::now();
        }
        S.dev_slab->release(dev_off, dev_bytes);
        S.pin_slab->release(pin_off, pin_bytes);
        S.slot_busy[slot] = false;
        S.stats.failed += ns;
        S.cv_done.notify_all();
        return false;
    }
    S.stats.batches += 1;
    S.stats.batched_requests += ns;
    S.inflight.push_back(J);
    S.stats.max_inflight = std::max<uint64_t>(S.stats.max_inflight, S.inflight.size());
    return true;
}

// Retire finished micro-batches (caller holds mu).
bool retire(Server& S) {
    bool any = false;
    for (size_t j = 0; j < S.inflight.size();) {
        Job& J = S.inflight[j];
        const cudaError_t q = cudaEventQuery(J.done);
        if (q == cudaErrorNotReady) { ++j; continue; }
        const auto now = Clock::now();
        size_t at = 0;
        for (auto& rp : J.reqs) {
            Request& r = *rp;
            if (q != cudaSuccess) {
                r.state = RQ_FAILED;
                r.error = OPE_ERR_DEVICE;
                r.message = cudaGetErrorString(q);
                S.stats.failed += 1;
            } else {
                if (J.kind == RK_PRICE) {
                    r.prices.assign(J.prices_h + at, J.prices_h + at + r.con.size());
                    at += r.con.size();
                } else {
                    r.calib = J.calib_h[at++];
                }
                if (r.state == RQ_RUNNING) r.state = RQ_DONE;
                S.stats.completed += 1;
            }
            r.t_done = now;
        }
        if (q != cudaSuccess) cudaGetLastError();
        cudaEventDestroy(J.done);
        if (J.graph) calib_graph_delete(J.graph);
        S.dev_slab->release(J.dev_off, J.dev_bytes);
        S.pin_slab->release(J.pin_off, J.pin_bytes);
        S.slot_busy[J.slot] = false;
        S.inflight.erase(S.inflight.begin() + j);
        any = true;
    }
    if (any) S.cv_done.notify_all();
    return any;
}

// One scheduler thread per request kind: retire finished batches, launch
// batches of its kind while slots and memory allow, sleep briefly.
void scheduler(Server* S, int kind) {
    cudaSetDevice(S->device);
    ensure_device();
    std::unique_lock<std::mutex> lk(S->mu);
    while (!S->stop.load()) {
        retire(*S);
        while (!S->stop.load() && launch_batch(*S, kind, lk)) {
        }
        // sleep until a submit arrives, or briefly while work is in flight
        if (S->inflight.empty() && S->pending.empty())
            S->cv_sched.wait_for(lk, std::chrono::milliseconds(5));
        else
            S->cv_sched.wait_for(lk, std::chrono::microseconds(20));
    }
}

int submit(Server* S, int kind, int model, const ope_contract* con, size_t n, const double* iv, const void* params,
           uint64_t* out_id) {
    if (!S || !con || !params || !out_id || (kind == RK_CALIB && !iv)) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    if (model != OPE_MODEL_HESTON && model != OPE_MODEL_BATES) return set_error(OPE_ERR_INVALID_ARG, "bad model");
    if (n == 0) return set_error(OPE_ERR_INVALID_ARG, "empty request");
    auto r = std::make_shared<Request>();
    r->kind = kind;
    r->model = model;
    r->con.assign(con, con + n);
    if (iv) r->iv.assign(iv, iv + n);
    const int dim = param_stride(model);
    r->params.assign(static_cast<const double*>(params), static_cast<const double*>(params) + dim);
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> g(S->mu);
        if (!S->fatal.empty()) return set_error(OPE_ERR_DEVICE, S->fatal);
        r->id = S->next_id++;
        S->all[r->id] = r;
        S->pending.push_back(r);
        S->stats.submitted += 1;
    }
    S->cv_sched.notify_all();
    *out_id = r->id;
    return OPE_OK;
}

}  // namespace

}  // namespace ope

using namespace ope;

extern "C" {

int ope_server_create(const ope_server_config* cfg, ope_server** out) {
    if (!out) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    OPE_TRY(ensure_device());
    auto* S = new Server();
    if (cfg) S->cfg = *cfg;
    if (S->cfg.hbm_fraction <= 0.0 || S->cfg.hbm_fraction > 0.95) S->cfg.hbm_fraction = 0.5;
    if (S->cfg.max_inflight == 0) S->cfg.max_inflight = 4;
    if (S->cfg.max_batch_contracts == 0) S->cfg.max_batch_contracts = 1u << 20;
    if (S->cfg.pinned_bytes == 0) S->cfg.pinned_bytes = 256ull << 20;
    if (!(S->cfg.calib_sm_fraction > 0.0 && S->cfg.calib_sm_fraction <= 1.0)) S->cfg.calib_sm_fraction = 0.5;
    S->tol = S->cfg.tol > 0.0 ? S->cfg.tol : OPE_REF_TOL;
    cudaGetDevice(&S->device);
    size_t free_b = 0, total_b = 0;
    int rc = check_cuda(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (rc != OPE_OK) { delete S; return rc; }
    size_t budget = (size_t)(S->cfg.hbm_fraction * (double)free_b);
    if (S->cfg.hbm_cap_bytes && budget > S->cfg.hbm_cap_bytes) budget = S->cfg.hbm_cap_bytes;
    budget = align_up(std::max<size_t>(budget, 1 << 20), 1 << 20);
    rc = check_cuda(cudaMalloc(&S->dev_base, budget), "cudaMalloc(server slab)");
    if (rc != OPE_OK) { delete S; return rc; }
    void* pin = nullptr;
    rc = check_cuda(cudaMallocHost(&pin, S->cfg.pinned_bytes), "cudaMallocHost(server staging)");
    if (rc != OPE_OK) { cudaFree(S->dev_base); delete S; return rc; }
    S->pin_base = static_cast<char*>(pin);
    S->dev_slab.reset(new Slab(budget));
    S->pin_slab.reset(new Slab(S->cfg.pinned_bytes));
    S->streams_hi.resize(S->cfg.max_inflight);
    S->streams_lo.resize(S->cfg.max_inflight);
    S->slot_busy.assign(S->cfg.max_inflight, false);
    int prio_lo = 0, prio_hi = 0;  // numerically lower = higher priority
    cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi);
    for (auto& st : S->streams_hi) cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_hi);
    for (auto& st : S->streams_lo) cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio_lo);
    S->stats.hbm_budget_bytes = budget;
    S->thr_price = std::thread(scheduler, S, (int)RK_PRICE);
    S->thr_calib = std::thread(scheduler, S, (int)RK_CALIB);
    *out = reinterpret_cast<ope_server*>(S);
    return OPE_OK;
}

int ope_server_destroy(ope_server* srv) {
    auto* S = reinterpret_cast<Server*>(srv);
    if (!S) return OPE_OK;
    S->stop.store(true);
    S->cv_sched.notify_all();
    if (S->thr_price.joinable()) S->thr_price.join();
    if (S->thr_calib.joinable()) S->thr_calib.join();
    {  // drain what is still in flight
        std::unique_lock<std::mutex> lk(S->mu);
        while (!S->inflight.empty()) {
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(50));
            lk.lock();
            retire(*S);
        }
    }
    for (auto& st : S->streams_hi) cudaStreamDestroy(st);
    for (auto& st : S->streams_lo) cudaStreamDestroy(st);
    cudaFree(S->dev_base);
    cudaFreeHost(S->pin_base);
    delete S;
    return OPE_OK;
}

int ope_server_submit_price(ope_server* srv, int32_t model, const ope_contract* contracts, size_t n,
                            const void* params, uint64_t* out_id) {
    return submit(reinterpret_cast<Server*>(srv), RK_PRICE, model, contracts, n, nullptr, params, out_id);
}

int ope_server_submit_calibrate(ope_server* srv, int32_t model, const ope_contract* quotes, const double* iv_market,
                                size_t n, const void* p0, uint64_t* out_id) {
    return submit(reinterpret_cast<Server*>(srv), RK_CALIB, model, quotes, n, iv_market, p0, out_id);
}

int ope_server_wait(ope_server* srv, uint64_t id, double timeout_ms, double* out_prices, ope_calib_result* out_calib,
                    double* out_latency_ms) {
    auto* S = reinterpret_cast<Server*>(srv);
    if (!S) return set_error(OPE_ERR_INVALID_ARG, "NULL server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return set_error(OPE_ERR_NOT_FOUND, "unknown request id");
    std::shared_ptr<Request> r = it->second;
    const auto deadline = Clock::now() + std::chrono::microseconds((long long)(timeout_ms * 1000.0));
    while (r->state == RQ_PENDING || r->state == RQ_RUNNING) {
        if (timeout_ms >= 0.0) {
            if (S->cv_done.wait_until(lk, deadline) == std::cv_status::timeout &&
                (r->state == RQ_PENDING || r->state == RQ_RUNNING))
                return set_error(OPE_ERR_TIMEOUT, "request not finished within the timeout");
        } else {
            S->cv_done.wait(lk);
        }
    }
    S->all.erase(id);
    if (out_latency_ms) *out_latency_ms = ms_since(r->t_submit, r->t_done);
    switch (r->state) {
        case RQ_DONE:
            if (r->kind == RK_PRICE && out_prices) std::memcpy(out_prices, r->prices.data(), r->prices.size() * sizeof(double));
            if (r->kind == RK_CALIB && out_calib) *out_calib = r->calib;
            return OPE_OK;
        case RQ_CANCELLED: return set_error(OPE_ERR_CANCELLED, "request cancelled");
        case RQ_REJECTED: return set_error(OPE_ERR_REJECTED, r->message);
        default: return set_error(r->error ? r->error : OPE_ERR_DEVICE, r->message);
    }
}

int ope_server_cancel(ope_server* srv, uint64_t id) {
    auto* S = reinterpret_cast<Server*>(srv);
    if (!S) return set_error(OPE_ERR_INVALID_ARG, "NULL server");
    std::lock_guard<std::mutex> g(S->mu);
    auto it = S->all.find(id);
    if (it == S->all.end()) return set_error(OPE_ERR_NOT_FOUND, "unknown request id");
    Request& r = *it->second;
    if (r.state == RQ_PENDING) {
        for (auto p = S->pending.begin(); p != S->pending.end(); ++p)
            if ((*p)->id == id) { S->pending.erase(p); break; }
        r.state = RQ_CANCELLED;
        r.t_done = Clock::now();
        S->stats.cancelled += 1;
        S->cv_done.notify_all();
        return OPE_OK;
    }
    return set_error(OPE_ERR_INVALID_ARG, "request already running or finished");
}

int ope_server_get_stats(ope_server* srv, ope_server_stats* out) {
    auto* S = reinterpret_cast<Server*>(srv);
    if (!S || !out) return set_error(OPE_ERR_INVALID_ARG, "NULL argument");
    std::lock_guard<std::mutex> g(S->mu);
    *out = S->stats;
    out->hbm_peak_bytes = S->dev_slab->peak();
    out->pending = S->pending.size();
    out->inflight = S->inflight.size();
    return OPE_OK;
}

}  // extern "C"
