// server.cu -- the serving loop: prove requests over resident circuits with
// continuous batching under a device-memory budget.
//
// The reference proves one circuit, once, per process (Groth16::Setup then
// Prove, groth16.cuh:48-222).  Here provers (circuit view + resident key
// tables) stay in HBM and a worker thread serves a request queue:
//   * admission: the oldest queued request whose circuit has an idle proof
//     context, or whose new context fits the budget (idle contexts of other
//     circuits are released to make room), is started; a request whose
//     context could never fit is rejected;
//   * each admitted request gets its own streams, so requests that arrive
//     while others run are admitted as contexts and memory free up and their
//     kernels overlap on the device;
//   * per request: witness copy host->device, the prove chain, proof copy
//     device->host, one completion event; the worker polls completions and
//     returns contexts to their circuit's idle list.
// Latency is measured on the host from submission to completion.
#include "prover.cuh"
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

using lzk::ProveCtx;
using Clock = std::chrono::steady_clock;

namespace {

enum ReqState { QUEUED, RUNNING, DONE, REJECTED, CANCELLED };

struct Request {
    uint64_t id = 0;
    uint32_t circuit = 0;
    const lzk_fr_t* z = nullptr;
    std::vector<lzk_fr_t> zcopy;   // when the caller's witness is not pinned and stable
    lzk_fr_t r{}, s{};
    ReqState state = QUEUED;
    ProveCtx* ctx = nullptr;
    lzk_groth16_proof proof{};
    Clock::time_point t_submit, t_done;
};

struct Circuit {
    lzk_prover* prover = nullptr;
    std::vector<ProveCtx*> idle;
    size_t ctx_bytes = 0;   // bytes of one context (0 until the first is made)
    size_t live = 0;        // contexts allocated (idle + running)
};

}  // namespace

struct lzk_server {
    lzk_server_cfg cfg{};
    int device = 0;
    std::vector<Circuit> circuits;
    size_t resident_bytes = 0, ctx_bytes = 0;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    std::deque<Request*> queue;
    std::vector<Request*> running;
    std::unordered_map<uint64_t, Request*> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    int fault = LZK_OK;
    std::thread worker;
    // statistics
    uint64_t submitted = 0, completed = 0, rejected = 0, cancelled = 0;
    std::vector<double> lat_ms;
    Clock::time_point t_first, t_last;
    bool have_first = false;
};

namespace {

size_t used(const lzk_server* s) { return s->resident_bytes + s->ctx_bytes; }

// release idle contexts of circuits other than `keep` until `need` more
// bytes fit; true if they do
bool make_room(lzk_server* s, uint32_t keep, size_t need)
{
    for (uint32_t c = 0; c < s->circuits.size() && used(s) + need > s->cfg.hbm_budget_bytes; c++) {
        if (c == keep) continue;
        Circuit& ci = s->circuits[c];
        while (!ci.idle.empty() && used(s) + need > s->cfg.hbm_budget_bytes) {
            ProveCtx* x = ci.idle.back();
            ci.idle.pop_back();
            s->ctx_bytes -= x->bytes;
            ci.live--;
            lzk::ctx_destroy(x);
        }
    }
    return used(s) + need <= s->cfg.hbm_budget_bytes;
}

// a context for circuit c, or nullptr when the budget does not allow one now
// (*never = true when it never will)
ProveCtx* get_ctx(lzk_server* s, uint32_t c, bool* never)
{
    Circuit& ci = s->circuits[c];
    *never = false;
    if (s->running.size() >= s->cfg.max_inflight) return nullptr;
    if (!ci.idle.empty()) {
        ProveCtx* x = ci.idle.back();
        ci.idle.pop_back();
        return x;
    }
    size_t need = ci.ctx_bytes;
    if (need && s->resident_bytes + need > s->cfg.hbm_budget_bytes) { *never = true; return nullptr; }
    if (need && !make_room(s, c, need)) return nullptr;
    ProveCtx* x = nullptr;
    if (lzk::ctx_create(ci.prover, true, &x) != LZK_OK) {
        cudaGetLastError();
        if (!ci.live && !s->ctx_bytes) *never = true;
        return nullptr;
    }
    if (!ci.ctx_bytes) ci.ctx_bytes = x->bytes;
    if (used(s) + x->bytes > s->cfg.hbm_budget_bytes && !make_room(s, c, x->bytes)) {
        bool alone = s->resident_bytes + x->bytes > s->cfg.hbm_budget_bytes;
        lzk::ctx_destroy(x);
        *never = alone;
        return nullptr;
    }
    s->ctx_bytes += x->bytes;
    ci.live++;
    return x;
}

int launch(lzk_server* s, Request* q)
{
    ProveCtx* x = q->ctx;
    const lzk_prover* p = s->circuits[q->circuit].prover;
    const void* src = q->zcopy.empty() ? static_cast<const void*>(q->z) : static_cast<const void*>(q->zcopy.data());
    LZK_CUDA(cudaMemcpyAsync(x->z, src, p->n_vars * sizeof(lzk_fr_t), cudaMemcpyHostToDevice, x->s0));
    LZK_TRY(lzk::prove_ctx(p, x, x->z, &q->r, &q->s, x->proof, x->s0));
    LZK_CUDA(cudaMemcpyAsync(x->proof_host, x->proof, sizeof(lzk_groth16_proof), cudaMemcpyDeviceToHost, x->s0));
    LZK_CUDA(cudaEventRecord(x->ev_done, x->s0));
    return LZK_OK;
}

void worker_main(lzk_server* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        bool progress = false;
        // admission, oldest first; a request that must wait does not block
        // requests of other circuits behind it
        for (auto it = s->queue.begin(); it != s->queue.end();) {
            Request* q = *it;
            bool never = false;
            ProveCtx* x = get_ctx(s, q->circuit, &never);
            if (!x) {
                if (never) {
                    q->state = REJECTED;
                    s->rejected++;
                    it = s->queue.erase(it);
                    s->done_cv.notify_all();
                    progress = true;
                    continue;
                }
                ++it;
                continue;
            }
            q->ctx = x;
            q->state = RUNNING;
            it = s->queue.erase(it);
            int rc = launch(s, q);
            if (rc != LZK_OK) {
                s->fault = rc;
                q->state = REJECTED;
                s->rejected++;
                s->circuits[q->circuit].idle.push_back(x);
                q->ctx = nullptr;
                s->done_cv.notify_all();
            }
            else s->running.push_back(q);
            progress = true;
        }
        // completions
        for (auto it = s->running.begin(); it != s->running.end();) {
            Request* q = *it;
            cudaError_t e = cudaEventQuery(q->ctx->ev_done);
            if (e == cudaErrorNotReady) { ++it; continue; }
            if (e != cudaSuccess) { s->fault = LZK_EDEVICE; cudaGetLastError(); }
            std::memcpy(&q->proof, q->ctx->proof_host, sizeof(lzk_groth16_proof));
            q->t_done = Clock::now();
            q->state = e == cudaSuccess ? DONE : REJECTED;
            s->circuits[q->circuit].idle.push_back(q->ctx);
            q->ctx = nullptr;
            if (q->state == DONE) {
                s->completed++;
                s->lat_ms.push_back(std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count());
                s->t_last = q->t_done;
            } else {
                s->rejected++;
            }
            it = s->running.erase(it);
            s->done_cv.notify_all();
            progress = true;
        }
        if (s->stop && s->running.empty()) break;
        if (!progress) {
            if (s->running.empty() && s->queue.empty()) s->cv.wait(lk, [s] { return s->stop || !s->queue.empty(); });
            else s->cv.wait_for(lk, std::chrono::microseconds(50));
        }
    }
}

}  // namespace

extern "C" {

int lzk_server_create(const lzk_server_cfg* cfg, lzk_server** out)
{
    if (!cfg || !out || !cfg->max_inflight || !cfg->hbm_budget_bytes) return LZK_EINVAL;
    *out = nullptr;
    lzk_server* s = new (std::nothrow) lzk_server();
    if (!s) return LZK_ENOMEM;
    s->cfg = *cfg;
    if (cudaGetDevice(&s->device) != cudaSuccess) { delete s; return LZK_EDEVICE; }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return LZK_OK;
}

int lzk_server_add_circuit(lzk_server* s, lzk_prover* prover, uint32_t* circuit_id)
{
    if (!s || !prover || !circuit_id) return LZK_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    size_t rb = lzk_prover_device_bytes(prover);
    if (s->resident_bytes + rb > s->cfg.hbm_budget_bytes) return LZK_EBUSY;
    s->resident_bytes += rb;
    Circuit c;
    c.prover = prover;
    s->circuits.push_back(c);
    *circuit_id = (uint32_t)(s->circuits.size() - 1);
    return LZK_OK;
}

int lzk_server_submit(lzk_server* s, uint32_t circuit_id, const lzk_fr_t* z, const lzk_fr_t* r, const lzk_fr_t* sv,
                      uint32_t flags, uint64_t* request_id)
{
    if (!s || !z || !r || !sv || !request_id) return LZK_EINVAL;
    Request* q = new (std::nothrow) Request();
    if (!q) return LZK_ENOMEM;
    {
        std::lock_guard<std::mutex> g(s->mu);
        if (circuit_id >= s->circuits.size()) { delete q; return LZK_EINVAL; }
        if (s->fault != LZK_OK) { delete q; return s->fault; }
        q->circuit = circuit_id;
        size_t nv = s->circuits[circuit_id].prover->n_vars;
        if (flags & LZK_REQ_WITNESS_PINNED) q->z = z;
        else q->zcopy.assign(z, z + nv);
        q->r = *r;
        q->s = *sv;
        q->id = s->next_id++;
        q->t_submit = Clock::now();
        if (!s->have_first) { s->t_first = q->t_submit; s->have_first = true; }
        s->reqs[q->id] = q;
        s->queue.push_back(q);
        s->submitted++;
        *request_id = q->id;
    }
    s->cv.notify_one();
    return LZK_OK;
}

int lzk_server_poll(lzk_server* s, uint64_t request_id, lzk_groth16_proof* proof, double* latency_ms)
{
    if (!s) return LZK_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return LZK_EINVAL;
    Request* q = it->second;
    if (q->state == QUEUED || q->state == RUNNING) return LZK_EBUSY;
    int rc = q->state == DONE ? LZK_OK : (q->state == CANCELLED ? LZK_ECANCELED : LZK_EREJECTED);
    if (q->state == DONE) {
        if (proof) *proof = q->proof;
        if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q->t_done - q->t_submit).count();
    }
    s->reqs.erase(it);
    delete q;
    return rc;
}

int lzk_server_cancel(lzk_server* s, uint64_t request_id)
{
    if (!s) return LZK_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->reqs.find(request_id);
    if (it == s->reqs.end()) return LZK_EINVAL;
    Request* q = it->second;
    if (q->state != QUEUED) return LZK_EBUSY;
    s->queue.erase(std::find(s->queue.begin(), s->queue.end(), q));
    q->state = CANCELLED;
    s->cancelled++;
    s->done_cv.notify_all();
    return LZK_OK;
}

int lzk_server_wait_idle(lzk_server* s, int timeout_ms)
{
    if (!s) return LZK_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    bool ok = s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms < 0 ? 0 : timeout_ms),
                                  [s] { return s->queue.empty() && s->running.empty(); });
    if (!ok) return LZK_ETIMEOUT;
    return s->fault;
}

int lzk_server_get_stats(lzk_server* s, lzk_server_stats* st)
{
    if (!s || !st) return LZK_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->submitted;
    st->completed = s->completed;
    st->rejected = s->rejected;
    st->cancelled = s->cancelled;
    st->queued = s->queue.size();
    st->running = s->running.size();
    st->device_bytes = used(s);
    if (!s->lat_ms.empty()) {
        std::vector<double> v = s->lat_ms;
        std::sort(v.begin(), v.end());
        auto pct = [&](double q) { return v[std::min(v.size() - 1, (size_t)(q * (v.size() - 1) + 0.5))]; };
        st->p50_ms = pct(0.50);
        st->p99_ms = pct(0.99);
        st->max_ms = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        st->mean_ms = sum / v.size();
        double span = std::chrono::duration<double>(s->t_last - s->t_first).count();
        st->proofs_per_s = span > 0 ? s->completed / span : 0.0;
    }
    return LZK_OK;
}

int lzk_server_reset_stats(lzk_server* s)
{
    if (!s) return LZK_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    s->submitted = s->completed = s->rejected = s->cancelled = 0;
    s->lat_ms.clear();
    s->have_first = false;
    return LZK_OK;
}

int lzk_server_destroy(lzk_server* s)
{
    if (!s) return LZK_EINVAL;
    {
        std::lock_guard<std::mutex> g(s->mu);
        for (Request* q : s->queue) { q->state = CANCELLED; }
        s->queue.clear();
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (auto& c : s->circuits)
        for (ProveCtx* x : c.idle) lzk::ctx_destroy(x);
    for (auto& kv : s->reqs) delete kv.second;
    delete s;
    return LZK_OK;
}

}  // extern "C"
