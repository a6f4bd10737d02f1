// Build server: continuous batching of whole phase-1 + phase-2 builds on one
// GPU.  No counterpart in the reference, which builds one collection per
// process.
//
// Requests (a host sequence batch + build parameters) arrive at any time.
// `slots` worker threads each own one engine (own CUDA stream, own device
// arena).  The admission gate (admission.hpp) reserves each request's device
// memory estimate against the server's HBM budget; an admitted request runs
// on a free worker with its grant as the engine's memory limit, so requests
// that arrive while others are on the GPU start as soon as a slot and memory
// free up, and their kernels overlap on the device (independent streams).
// Each request is built exactly as it would be alone (same engine code, its
// own class dictionary), so its outputs do not depend on what else runs.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cdbg_gpu.h"
#include "admission.hpp"

#include <cuda_runtime.h>

namespace {

thread_local std::string t_error;

// Page-locked host buffers recycled across requests (and servers) by
// power-of-two size class: pinning is slow and freeing pinned memory
// synchronizes the device, so neither happens per request once the pool has
// warmed up.  One pool per process; its buffers live until the process ends.
class pinned_pool {
public:
    static pinned_pool& instance() {
        static pinned_pool* p = new pinned_pool();  // never destroyed: freed with the process
        return *p;
    }
    void* take(size_t bytes, size_t& cls) {
        cls = size_t(1) << 20;
        while (cls < bytes) cls <<= 1;
        {
            std::lock_guard<std::mutex> lk(m_mu);
            auto& v = m_free[cls];
            if (!v.empty()) {
                void* p = v.back();
                v.pop_back();
                return p;
            }
        }
        void* p = nullptr;
        if (cudaHostAlloc(&p, cls, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("pinned host allocation of " + std::to_string(cls >> 20) + " MiB failed");
        }
        return p;
    }
    void give(void* p, size_t cls) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(m_mu);
        m_free[cls].push_back(p);
    }

private:
    std::mutex m_mu;
    std::unordered_map<size_t, std::vector<void*>> m_free;
};

struct host_buf {
    void* p = nullptr;
    size_t cls = 0;
};

struct request {
    uint64_t id = 0;
    cdbg_seq_batch batch{};
    cdbg_build_params params{};
    uint64_t need = 0, grant = 0;
    double t_submit = 0, t_start = 0, t_done = 0;
    bool done = false;
    int status = 0;
    std::string error;
    host_buf frag, words, offsets;  // from the server's pinned pool
    cdbg_build_result res{};
};

double now_s(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

struct cdbg_server {
    int device = 0;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    cdbg::serve::memory_model model;
    std::unique_ptr<cdbg::serve::admission_gate> gate;
    std::mutex mu;
    std::condition_variable cv;
    std::unordered_map<uint64_t, std::unique_ptr<request>> reqs;
    uint64_t next_id = 1;
    bool stop = false;
    std::vector<cdbg_engine*> engines;
    std::vector<std::thread> workers;
    pinned_pool& pinned = pinned_pool::instance();
    uint64_t completed = 0, failed = 0;
    uint64_t peak_reserved = 0;
    uint32_t peak_running = 0;

    void worker(cdbg_engine* e) {
        for (;;) {
            request* r = nullptr;
            uint64_t id = 0, grant = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                for (;;) {
                    if (gate->admit(id, grant)) break;
                    if (stop && gate->waiting() == 0) return;
                    cv.wait(lk);
                }
                r = reqs.at(id).get();
                r->grant = grant;
                r->t_start = now_s(t0);
                peak_reserved = std::max(peak_reserved, gate->reserved());
                peak_running = std::max(peak_running, gate->running());
            }
            cv.notify_all();  // another slot may admit the next request
            int rc = cdbg_engine_set_memory_limit(e, grant);
            cdbg_build_result res{};
            cdbg_build_params p = r->params;
            p.outputs_to_host = 0;  // outputs stay in HBM; copied below into the request's buffers
            if (rc == 0) rc = cdbg_gpu_build(e, &r->batch, &p, &res);
            std::string err;
            if (rc == 0) {
                try {
                    const uint64_t nw = (res.class_bits + 63) / 64;
                    r->frag.p = pinned.take(res.frag_nbytes + 1, r->frag.cls);
                    r->words.p = pinned.take(8 * nw + 8, r->words.cls);
                    r->offsets.p = pinned.take(8 * res.n_color_sets + 8, r->offsets.cls);
                    if (res.frag_nbytes) rc = cdbg_engine_copy_out(e, res.frag_bytes, r->frag.p, res.frag_nbytes);
                    if (rc == 0 && nw) rc = cdbg_engine_copy_out(e, res.class_words, r->words.p, 8 * nw);
                    if (rc == 0 && res.n_color_sets)
                        rc = cdbg_engine_copy_out(e, res.class_offsets, r->offsets.p, 8 * res.n_color_sets);
                    if (rc != 0) err = cdbg_last_error();
                } catch (std::exception const& ex) {
                    rc = -1;
                    err = ex.what();
                }
            } else {
                err = cdbg_last_error();
            }
            // the grant ends with the request: its memory goes back to the pool
            cdbg_engine_trim(e);
            {
                std::lock_guard<std::mutex> lk(mu);
                gate->finish(grant);
                r->res = res;
                r->status = rc;
                r->error = err;
                r->t_done = now_s(t0);
                r->done = true;
                if (rc == 0)
                    ++completed;
                else
                    ++failed;
            }
            cv.notify_all();
        }
    }
};

extern "C" {

const char* cdbg_server_last_error(void) { return t_error.c_str(); }

int cdbg_server_create(const cdbg_server_params* p, cdbg_server** out) {
    try {
        if (!p || !out) throw std::runtime_error("null argument");
        auto s = std::make_unique<cdbg_server>();
        s->device = p->device;
        const uint32_t slots = p->slots ? p->slots : 1;
        if (p->bytes_per_base > 0) s->model.per_base = p->bytes_per_base;
        if (p->floor_bytes) s->model.floor = p->floor_bytes;
        if (p->hbm_budget == 0) throw std::runtime_error("hbm_budget must be > 0");
        s->gate = std::make_unique<cdbg::serve::admission_gate>(p->hbm_budget, slots);
        for (uint32_t i = 0; i < slots; ++i) {
            cdbg_engine* e = nullptr;
            if (cdbg_engine_create(p->device, &e) != 0) {
                const std::string msg = cdbg_last_error();
                for (auto* x : s->engines) cdbg_engine_destroy(x);
                throw std::runtime_error("engine: " + msg);
            }
            s->engines.push_back(e);
        }
        cdbg_server* raw = s.get();
        for (auto* e : s->engines) s->workers.emplace_back([raw, e] { raw->worker(e); });
        *out = s.release();
        return 0;
    } catch (std::exception const& ex) {
        t_error = ex.what();
        return -1;
    }
}

int cdbg_server_submit(cdbg_server* s, const cdbg_seq_batch* b, const cdbg_build_params* p, uint64_t* id) {
    try {
        if (!s || !b || !p || !id) throw std::runtime_error("null argument");
        if (b->on_device) throw std::runtime_error("server requests take host sequence batches");
        auto r = std::make_unique<request>();
        r->batch = *b;
        r->params = *p;
        r->need = s->model.need(b->seq_bytes);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->stop) throw std::runtime_error("server is shutting down");
            r->id = s->next_id++;
            r->t_submit = now_s(s->t0);
            *id = r->id;
            s->gate->arrive(r->id, r->need);
            s->reqs.emplace(r->id, std::move(r));
        }
        s->cv.notify_all();
        return 0;
    } catch (std::exception const& ex) {
        t_error = ex.what();
        return -1;
    }
}

int cdbg_server_wait(cdbg_server* s, uint64_t id, cdbg_request_result* out) {
    try {
        if (!s || !out) throw std::runtime_error("null argument");
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) throw std::runtime_error("unknown request id");
        request* r = it->second.get();
        s->cv.wait(lk, [&] { return r->done; });
        cdbg_request_result o{};
        o.status = r->status;
        o.error = r->error.c_str();
        const bool ok = r->status == 0;
        o.frag_bytes = ok ? (const uint8_t*)r->frag.p : nullptr;
        o.frag_nbytes = ok ? r->res.frag_nbytes : 0;
        o.class_words = ok ? (const uint64_t*)r->words.p : nullptr;
        o.class_bits = ok ? r->res.class_bits : 0;
        o.class_offsets = ok ? (const uint64_t*)r->offsets.p : nullptr;
        o.n_color_sets = ok ? r->res.n_color_sets : 0;
        o.total_integers = r->res.total_integers;
        o.n_kmers = r->res.n_kmers;
        o.n_distinct = r->res.n_distinct;
        o.n_fragments = r->res.n_fragments;
        o.need_bytes = r->need;
        o.grant_bytes = r->grant;
        o.t_submit = r->t_submit;
        o.t_start = r->t_start;
        o.t_done = r->t_done;
        o.ms_device = r->res.ms_total;
        *out = o;
        return 0;
    } catch (std::exception const& ex) {
        t_error = ex.what();
        return -1;
    }
}

int cdbg_server_release(cdbg_server* s, uint64_t id) {
    if (!s) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end() || !it->second->done) {
        t_error = "unknown or unfinished request";
        return -1;
    }
    request* r = it->second.get();
    s->pinned.give(r->frag.p, r->frag.cls);
    s->pinned.give(r->words.p, r->words.cls);
    s->pinned.give(r->offsets.p, r->offsets.cls);
    s->reqs.erase(it);
    return 0;
}

int cdbg_server_stats(cdbg_server* s, cdbg_server_stats_t* out) {
    if (!s || !out) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    out->completed = s->completed;
    out->failed = s->failed;
    out->waiting = s->gate->waiting();
    out->running = s->gate->running();
    out->reserved_bytes = s->gate->reserved();
    out->peak_reserved_bytes = s->peak_reserved;
    out->peak_running = s->peak_running;
    out->clock_s = now_s(s->t0);
    return 0;
}

void cdbg_server_destroy(cdbg_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    for (auto& t : s->workers) t.join();
    for (auto* e : s->engines) cdbg_engine_destroy(e);
    for (auto& kv : s->reqs) {
        s->pinned.give(kv.second->frag.p, kv.second->frag.cls);
        s->pinned.give(kv.second->words.p, kv.second->words.cls);
        s->pinned.give(kv.second->offsets.p, kv.second->offsets.cls);
    }
    delete s;
}

}  // extern "C"
