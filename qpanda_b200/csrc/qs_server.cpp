// qs_server.cpp - a request loop with continuous batching.
//
// The reference serves one program at a time (QPandaSDK::run, and its cloud
// mode ships QRunes text to a remote service, QuantumCloudHTTP.cpp:117-191).
// Here requests - a circuit plus "1024 shots" or "the full probability
// vector" - are submitted at any time and served concurrently on one GPU:
//  - `slots` worker threads, each with its own CUDA stream, take requests in
//    arrival order; a request is admitted when its HBM footprint (state,
//    scratch and, for probabilities, the output vector) fits the budget next
//    to the requests already on the device, so requests that arrive while
//    others run start as soon as a slot and memory free up, and their kernels
//    overlap on the GPU;
//  - states use stream-ordered memory (qs_create_async), so admitting and
//    retiring requests never synchronizes the device;
//  - probability vectors stay resident on the device until the caller
//    fetches or releases them; shots are written to the caller's buffer;
//  - every kernel's reductions run in a fixed order, so a request's result
//    does not depend on what else is running (tested alone and in the mix).
// Latency = submit -> result ready (shots on the host, probabilities on the
// device).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/qpanda_b200.h"
#include "qs_prim.h"

int qs_cuda_fail(cudaError_t e, const char *where);

namespace {

typedef std::chrono::steady_clock clk;

struct Request {
    uint64_t id = 0;
    int n = 0;
    int kind = 0;
    std::vector<qs_gate> gates;
    std::vector<double> u;
    size_t shots = 0;
    uint64_t *out_host = nullptr;
    size_t footprint = 0, result_bytes = 0;
    clk::time_point t_submit, t_start, t_done;
    bool done = false;
    int status = QS_OK;
    char error[256] = {0};
    double *probs_dev = nullptr;
    cudaStream_t stream = nullptr;     // stream the result lives on
};

size_t footprint_of(int n, int kind)
{
    const size_t state = 8ull << n;                   // complex64
    const size_t scratch = 64ull << 20;               // reductions, sampling tree, plan matrices
    return state + scratch + (kind == QS_REQ_PROBS ? (8ull << n) : 0);
}

}  // namespace

struct qs_server {
    qs_server_opts opts;
    int device = 0;
    size_t budget = 0, used = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    size_t running = 0, max_running = 0, served = 0;
    std::vector<std::thread> workers;
    std::vector<cudaStream_t> streams;
};

namespace {

// First request in arrival order that fits, looking at most `bypass` places
// past the head (0 = strict arrival order).
Request *pick(qs_server *S)
{
    const size_t look = std::min(S->queue.size(), (size_t)S->opts.bypass + 1);
    for (size_t i = 0; i < look; ++i) {
        Request *r = S->queue[i];
        if (S->used + r->footprint <= S->budget) {
            S->queue.erase(S->queue.begin() + (long)i);
            return r;
        }
    }
    return nullptr;
}

void serve(qs_server *S, Request *r, cudaStream_t st)
{
    qs_state *s = nullptr;
    qs_plan *p = nullptr;
    int rc = qs_create_async(r->n, QS_C64, st, &s);
    if (!rc) {
        if (r->n >= 12) {
            qs_plan_opts o;
            qs_plan_default_opts(&o);
            rc = qs_plan_create_ex(r->n, r->gates.data(), r->gates.size(), &o, &p);
            if (!rc) rc = qs_plan_apply(s, p);
            if (!rc) rc = qs_plan_status(s);
        } else {
            rc = qs_gates_apply(s, r->gates.data(), r->gates.size());
        }
    }
    std::vector<int> qs((size_t)r->n);
    for (int i = 0; i < r->n; ++i) qs[(size_t)i] = i;
    if (!rc && r->kind == QS_REQ_SHOTS) {
        rc = qs_sample(s, qs.data(), r->n, r->u.data(), r->shots, r->out_host);
    } else if (!rc) {
        cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&r->probs_dev), 8ull << r->n, st);
        if (e != cudaSuccess) rc = qs_cuda_fail(e, "server: probability buffer");
        if (!rc) rc = qs_probs_device(s, qs.data(), r->n, r->probs_dev);
        if (!rc) {
            e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = qs_cuda_fail(e, "server: request");
        }
    }
    if (rc) snprintf(r->error, sizeof(r->error), "%s", qs_last_error());
    if (p) qs_plan_destroy(p);
    if (s) qs_destroy(s);
    if (rc && r->probs_dev) {
        cudaFreeAsync(r->probs_dev, st);
        r->probs_dev = nullptr;
    }
    r->stream = st;
    r->status = rc;
}

void worker(qs_server *S, int slot)
{
    cudaSetDevice(S->device);
    cudaStream_t st = S->streams[(size_t)slot];
    std::unique_lock<std::mutex> lk(S->mu);
    while (true) {
        Request *r = nullptr;
        S->cv_work.wait(lk, [&] { return S->stop || ((r = pick(S)) != nullptr); });
        if (!r) break;                                   // stopping
        S->used += r->footprint;
        S->running++;
        S->max_running = std::max(S->max_running, S->running);
        r->t_start = clk::now();
        lk.unlock();
        serve(S, r, st);
        lk.lock();
        r->t_done = clk::now();
        r->done = true;
        S->running--;
        S->served++;
        // the state and scratch are released; a probability vector stays until released
        S->used -= r->footprint - (r->probs_dev ? r->result_bytes : 0);
        S->cv_done.notify_all();
        S->cv_work.notify_all();
    }
}

}  // namespace

extern "C" int qs_server_default_opts(qs_server_opts *o)
{
    if (!o) return qs_fail(QS_ERR_ARG, "qs_server_default_opts: null");
    o->hbm_budget_bytes = 96ull << 30;
    o->slots = 8;
    o->bypass = 0;
    return QS_OK;
}

extern "C" int qs_server_create(const qs_server_opts *opts, qs_server **out)
{
    if (!out) return qs_fail(QS_ERR_ARG, "qs_server_create: null output");
    *out = nullptr;
    qs_server_opts o;
    if (opts) o = *opts;
    else qs_server_default_opts(&o);
    if (o.slots < 1 || o.slots > 64 || o.bypass < 0 || o.hbm_budget_bytes == 0)
        return qs_fail(QS_ERR_ARG, "qs_server_create: slots 1..64, bypass >= 0, budget > 0");
    std::unique_ptr<qs_server> S(new qs_server());
    S->opts = o;
    S->budget = o.hbm_budget_bytes;
    cudaError_t e = cudaGetDevice(&S->device);
    if (e != cudaSuccess) return qs_cuda_fail(e, "qs_server_create");
    for (int i = 0; i < o.slots; ++i) {
        cudaStream_t st;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            for (cudaStream_t x : S->streams) cudaStreamDestroy(x);
            return qs_cuda_fail(e, "qs_server_create: stream");
        }
        S->streams.push_back(st);
    }
    for (int i = 0; i < o.slots; ++i) S->workers.emplace_back(worker, S.get(), i);
    *out = S.release();
    return QS_OK;
}

extern "C" int qs_server_submit(qs_server *S, int n_qubits, const qs_gate *gates, size_t count, int kind,
                                const double *uniforms, size_t shots, uint64_t *out_host, uint64_t *id)
{
    if (!S || !id || (count && !gates)) return qs_fail(QS_ERR_ARG, "qs_server_submit: null argument");
    if (n_qubits < 1 || n_qubits > QS_MAX_QUBITS_SERVED)
        return qs_fail(QS_ERR_ARG, "qs_server_submit: %d qubits (1..%d)", n_qubits, QS_MAX_QUBITS_SERVED);
    if (kind != QS_REQ_SHOTS && kind != QS_REQ_PROBS) return qs_fail(QS_ERR_ARG, "qs_server_submit: bad kind");
    if (kind == QS_REQ_SHOTS && (!uniforms || !out_host || shots == 0))
        return qs_fail(QS_ERR_ARG, "qs_server_submit: shots need uniforms and an output buffer");
    std::unique_ptr<Request> r(new Request());
    r->n = n_qubits;
    r->kind = kind;
    r->gates.assign(gates, gates + count);
    if (kind == QS_REQ_SHOTS) r->u.assign(uniforms, uniforms + shots * (size_t)n_qubits);
    r->shots = shots;
    r->out_host = out_host;
    r->footprint = footprint_of(n_qubits, kind);
    r->result_bytes = kind == QS_REQ_PROBS ? (8ull << n_qubits) : 0;
    if (r->footprint > S->budget)
        return qs_fail(QS_ERR_OOM, "qs_server_submit: request needs %zu bytes of HBM, budget is %zu",
                       r->footprint, S->budget);
    r->t_submit = clk::now();
    std::lock_guard<std::mutex> lk(S->mu);
    r->id = S->next_id++;
    *id = r->id;
    S->queue.push_back(r.get());
    S->reqs[r->id] = std::move(r);
    S->cv_work.notify_one();
    return QS_OK;
}

extern "C" int qs_server_wait(qs_server *S, uint64_t id, double *latency_s, double *service_s)
{
    if (!S) return qs_fail(QS_ERR_ARG, "qs_server_wait: null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return qs_fail(QS_ERR_ARG, "qs_server_wait: unknown request %llu", (unsigned long long)id);
    Request *r = it->second.get();
    S->cv_done.wait(lk, [&] { return r->done; });
    if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
    if (service_s) *service_s = std::chrono::duration<double>(r->t_done - r->t_start).count();
    if (r->status) return qs_fail(r->status, "request %llu: %s", (unsigned long long)id, r->error);
    return QS_OK;
}

extern "C" int qs_server_fetch_probs(qs_server *S, uint64_t id, double *host_out)
{
    if (!S || !host_out) return qs_fail(QS_ERR_ARG, "qs_server_fetch_probs: null argument");
    Request *r;
    {
        std::unique_lock<std::mutex> lk(S->mu);
        auto it = S->reqs.find(id);
        if (it == S->reqs.end()) return qs_fail(QS_ERR_ARG, "qs_server_fetch_probs: unknown request");
        r = it->second.get();
        S->cv_done.wait(lk, [&] { return r->done; });
        if (!r->probs_dev) return qs_fail(QS_ERR_ARG, "qs_server_fetch_probs: no probability vector held");
    }
    cudaError_t e = cudaMemcpyAsync(host_out, r->probs_dev, r->result_bytes, cudaMemcpyDeviceToHost, r->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(r->stream);
    if (e != cudaSuccess) return qs_cuda_fail(e, "qs_server_fetch_probs");
    return QS_OK;
}

// Drop a finished request: frees a held probability vector and forgets it.
extern "C" int qs_server_release(qs_server *S, uint64_t id)
{
    if (!S) return qs_fail(QS_ERR_ARG, "qs_server_release: null server");
    std::unique_lock<std::mutex> lk(S->mu);
    auto it = S->reqs.find(id);
    if (it == S->reqs.end()) return qs_fail(QS_ERR_ARG, "qs_server_release: unknown request");
    Request *r = it->second.get();
    S->cv_done.wait(lk, [&] { return r->done; });
    if (r->probs_dev) {
        cudaFreeAsync(r->probs_dev, r->stream);
        S->used -= r->result_bytes;
        r->probs_dev = nullptr;
    }
    S->reqs.erase(it);
    S->cv_work.notify_all();
    return QS_OK;
}

extern "C" int qs_server_stats(qs_server *S, size_t *served, size_t *max_concurrent, size_t *hbm_in_use)
{
    if (!S) return qs_fail(QS_ERR_ARG, "qs_server_stats: null server");
    std::lock_guard<std::mutex> lk(S->mu);
    if (served) *served = S->served;
    if (max_concurrent) *max_concurrent = S->max_running;
    if (hbm_in_use) *hbm_in_use = S->used;
    return QS_OK;
}

extern "C" int qs_server_destroy(qs_server *S)
{
    if (!S) return QS_OK;
    {
        // requests not yet started end with an error; running ones finish
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        for (Request *r : S->queue) {
            r->status = QS_ERR_STATE;
            snprintf(r->error, sizeof(r->error), "server stopped before the request started");
            r->t_start = r->t_done = clk::now();
            r->done = true;
        }
        S->queue.clear();
        S->cv_work.notify_all();
        S->cv_done.notify_all();
    }
    for (auto &t : S->workers) t.join();
    cudaSetDevice(S->device);
    for (auto &kv : S->reqs)
        if (kv.second->probs_dev) cudaFreeAsync(kv.second->probs_dev, kv.second->stream);
    for (cudaStream_t st : S->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    delete S;
    return QS_OK;
}
