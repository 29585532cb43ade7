// Serving engine behind gpj_serve_* (include/gpjson_b200.h): (corpus,
// JSONPath) requests against corpora kept resident in device memory with
// their structural indexes, under a byte budget.
//
// The reference has no serving mode: its query() reads, indexes and queries
// the file on every call (functions/QueryFunction.java:48-265); a host
// serving GPJSON sits behind the interop object of GPJSONLibrary.java:48-54
// and calls it once per request.
//
// Threads:
//  - `workers` serving threads, each with a context (its own CUDA stream)
//    and a batch.  A worker takes every pending request whose corpus is
//    resident (up to max_batch, in arrival order), evaluates them with one
//    gpj_batch_run (one find_value launch over every line of every corpus
//    involved) and hands each request its result.  Requests that arrive
//    while a batch is on the GPU are taken by the next free worker, whose
//    batch runs on its own stream beside the first one: continuous batching
//    with iterations overlapping on the device.
//  - one loader thread with a context of its own: loads cold corpora from
//    page-locked host memory (copy and index build pipelined,
//    gpj_file_from_host_indexed) and releases evicted ones.
// Admission: a corpus is loaded when a request needs it and its resident
// bytes fit the budget; least recently used corpora that no pending or
// running request needs are evicted to make room, and their bytes count
// against the budget until the loader has released them.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/gpjson_b200.h"

namespace {

int64_t now_ns(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - t0).count();
}

// Device bytes a corpus holds while resident: input, string index, ':'
// bitmap, leveled bitmaps and the first newline-index allocation.
int64_t resident_bytes(int64_t n, int levels) {
    const int64_t words = (n + 63) / 64;
    return n + 8 * words * (2 + levels) + 8 * (n / 256 + 1024);
}

enum class CorpusState { kCold, kLoading, kResident };

struct Corpus {
    const uint8_t* host = nullptr;
    int64_t n = 0;
    int64_t cost = 0;
    bool registered = false;  // host memory page-locked by us
    CorpusState state = CorpusState::kCold;
    gpj_file* file = nullptr;
    int pins = 0;            // batches using it
    uint64_t last_use = 0;   // admission clock
};

struct Request {
    uint64_t id = 0;
    int corpus = 0;
    std::vector<std::string> paths;
    int slots = 1;  // the largest num_results of its paths
    int64_t submit_ns = 0, done_ns = -1;
    int rc = GPJ_OK;
    std::string error;
    gpj_result* result = nullptr;
};

}  // namespace

struct gpj_server {
    gpj_server_config cfg{};
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
    std::mutex mu;
    std::condition_variable work_cv;  // pending requests, residency, stop
    std::condition_variable done_cv;  // completions
    std::condition_variable load_cv;  // the loader's queues
    std::vector<Corpus> corpora;
    std::deque<Request*> pending;
    std::unordered_map<uint64_t, Request*> requests;  // submitted, not yet handed back
    std::deque<int> load_queue;
    std::deque<std::pair<int, gpj_file*>> release_queue;
    int64_t used = 0;       // budget taken by resident and loading corpora and those not yet released
    int64_t releasing = 0;  // of which: evicted, release pending
    uint64_t next_id = 1, clock = 0;
    int max_batch = 1, max_inflight = 1, inflight = 0;
    bool stop = false;         // workers: finish
    bool loader_stop = false;  // loader: release everything and finish (after the workers)
    std::string fatal;  // a loader failure: every later request fails with it
    // counters
    int64_t served = 0, batches = 0, loads = 0, evictions = 0;
    std::vector<std::thread> workers;
    std::thread loader;
};

namespace {

// Starts the load of corpus c (lock held) when its bytes fit the budget,
// evicting least recently used corpora that no pending request and no
// running batch needs; false while it has to wait.
bool admit(gpj_server* s, int c) {
    Corpus& k = s->corpora[c];
    if (k.state != CorpusState::kCold) return false;
    const int64_t budget = s->cfg.budget_bytes;
    while (s->used - s->releasing + k.cost > budget) {
        std::vector<char> needed(s->corpora.size(), 0);
        for (const Request* r : s->pending) needed[r->corpus] = 1;
        int victim = -1;
        for (size_t i = 0; i < s->corpora.size(); i++) {
            const Corpus& v = s->corpora[i];
            if (v.state != CorpusState::kResident || v.pins > 0 || needed[i]) continue;
            if (victim < 0 || v.last_use < s->corpora[victim].last_use) victim = static_cast<int>(i);
        }
        if (victim < 0) return false;  // room comes when a running batch ends
        Corpus& v = s->corpora[victim];
        s->release_queue.emplace_back(victim, v.file);
        v.file = nullptr;
        v.state = CorpusState::kCold;
        s->releasing += v.cost;
        s->evictions++;
        s->load_cv.notify_all();
    }
    if (s->used + k.cost > budget) return false;  // wait for the releases
    s->used += k.cost;
    k.state = CorpusState::kLoading;
    s->load_queue.push_back(c);
    s->load_cv.notify_all();
    return false;
}

void finish(gpj_server* s, Request* r, int rc, const std::string& msg) {
    r->rc = rc;
    r->error = msg;
    r->done_ns = now_ns(s->t0);
}

void loader_loop(gpj_server* s) {
    gpj_ctx* ctx = nullptr;
    int rc = gpj_create(s->cfg.device, &ctx);
    std::unique_lock<std::mutex> lk(s->mu);
    if (rc) s->fatal = std::string("loader context: ") + gpj_last_error(nullptr);
    for (;;) {
        s->load_cv.wait(lk, [&] { return s->loader_stop || !s->release_queue.empty() || !s->load_queue.empty(); });
        if (!s->release_queue.empty()) {
            const auto job = s->release_queue.front();
            s->release_queue.pop_front();
            lk.unlock();
            gpj_file_release(job.second);
            lk.lock();
            // the budget is free again only now that the memory is released
            s->used -= s->corpora[job.first].cost;
            s->releasing -= s->corpora[job.first].cost;
            s->work_cv.notify_all();
            continue;
        }
        if (!s->load_queue.empty() && !s->loader_stop) {
            const int c = s->load_queue.front();
            s->load_queue.pop_front();
            const Corpus k = s->corpora[c];
            gpj_file* f = nullptr;
            std::string err;
            lk.unlock();
            int lrc = ctx ? gpj_file_from_host_indexed(ctx, k.host, k.n, s->cfg.num_levels, &f) : GPJ_ESTATE;
            if (lrc && ctx) err = gpj_last_error(ctx);
            lk.lock();
            Corpus& kk = s->corpora[c];
            if (lrc) {
                s->used -= kk.cost;
                kk.state = CorpusState::kCold;
                s->fatal = "loading corpus " + std::to_string(c) + " failed: " + err;
            } else {
                kk.file = f;
                kk.state = CorpusState::kResident;
                s->loads++;
            }
            s->work_cv.notify_all();
            continue;
        }
        if (s->loader_stop) break;
    }
    // the workers are gone: release every resident corpus (files of this context)
    std::vector<gpj_file*> files;
    for (Corpus& k : s->corpora) {
        if (k.file) files.push_back(k.file);
        k.file = nullptr;
        k.state = CorpusState::kCold;
    }
    s->load_queue.clear();
    lk.unlock();
    for (gpj_file* f : files) gpj_file_release(f);
    if (ctx) gpj_destroy(ctx);
}

void worker_loop(gpj_server* s) {
    gpj_ctx* ctx = nullptr;
    gpj_batch* batch = nullptr;
    int rc = gpj_create(s->cfg.device, &ctx);
    if (!rc) rc = gpj_batch_create(ctx, &batch);
    std::string setup_err = rc ? std::string(gpj_last_error(ctx)) : std::string();
    std::unique_lock<std::mutex> lk(s->mu);
    std::vector<Request*> take;
    for (;;) {
        take.clear();
        if (s->stop) break;
        const bool may_run = s->inflight < s->max_inflight;
        if (may_run) {
            for (auto it = s->pending.begin(); it != s->pending.end();) {
                Request* r = *it;
                Corpus& k = s->corpora[r->corpus];
                if (!s->fatal.empty() || rc) {
                    finish(s, r, rc ? rc : GPJ_ESTATE, rc ? setup_err : s->fatal);
                    it = s->pending.erase(it);
                    s->done_cv.notify_all();
                    continue;
                }
                if (k.state == CorpusState::kResident && static_cast<int>(take.size()) < s->max_batch) {
                    k.pins++;
                    k.last_use = ++s->clock;
                    take.push_back(r);
                    it = s->pending.erase(it);
                    continue;
                }
                if (k.state == CorpusState::kCold) admit(s, r->corpus);
                ++it;
            }
        }
        if (take.empty()) {
            s->work_cv.wait_for(lk, std::chrono::milliseconds(20));
            continue;
        }
        s->inflight++;
        std::vector<gpj_file*> files(take.size());
        for (size_t i = 0; i < take.size(); i++) files[i] = s->corpora[take[i]->corpus].file;
        lk.unlock();
        // one batch over every taken request
        gpj_batch_clear(batch);
        std::vector<int> items(take.size(), -1);
        for (size_t i = 0; i < take.size(); i++) {
            std::vector<const char*> ps;
            for (const auto& p : take[i]->paths) ps.push_back(p.c_str());
            const int arc = gpj_batch_add(batch, files[i], static_cast<int>(ps.size()), ps.data(), &items[i]);
            if (arc) {
                take[i]->rc = arc;
                take[i]->error = gpj_last_error(ctx);
            }
        }
        const int brc = gpj_batch_run(batch);
        const std::string berr = brc ? std::string(gpj_last_error(ctx)) : std::string();
        for (size_t i = 0; i < take.size(); i++) {
            Request* r = take[i];
            if (r->rc) continue;
            if (brc) {
                r->rc = brc;
                r->error = berr;
                continue;
            }
            const int grc = gpj_batch_result_ex(batch, items[i], r->slots, &r->result);
            if (grc) {
                r->rc = grc;
                r->error = gpj_last_error(ctx);
            }
        }
        lk.lock();
        s->inflight--;
        s->batches++;
        const int64_t t = now_ns(s->t0);
        for (Request* r : take) {
            s->corpora[r->corpus].pins--;
            r->done_ns = t;
            s->served++;
        }
        s->done_cv.notify_all();
        s->work_cv.notify_all();
    }
    lk.unlock();
    if (batch) gpj_batch_release(batch);
    if (ctx) gpj_destroy(ctx);
}

}  // namespace

extern "C" {

int gpj_serve_create(const gpj_server_config* cfg, gpj_server** out) {
    if (!cfg || !out) return GPJ_EINVAL;
    *out = nullptr;
    if (cfg->budget_bytes <= 0 || cfg->num_levels < 1 || cfg->num_levels > GPJ_MAX_LEVELS || cfg->max_batch < 1 ||
        cfg->workers < 1 || cfg->workers > 8)
        return GPJ_EINVAL;
    gpj_server* s = new (std::nothrow) gpj_server;
    if (!s) return GPJ_ENOMEM;
    s->cfg = *cfg;
    s->max_batch = cfg->max_batch;
    s->max_inflight = cfg->workers;
    try {
        s->loader = std::thread(loader_loop, s);
        for (int i = 0; i < cfg->workers; i++) s->workers.emplace_back(worker_loop, s);
    } catch (...) {
        gpj_serve_destroy(s);
        return GPJ_ENOMEM;
    }
    *out = s;
    return GPJ_OK;
}

int gpj_serve_add_corpus(gpj_server* s, const void* host, int64_t n, int* corpus) {
    if (!s || !corpus || n < 0 || (n > 0 && !host)) return GPJ_EINVAL;
    Corpus k;
    k.host = static_cast<const uint8_t*>(host);
    k.n = n;
    k.cost = resident_bytes(n, s->cfg.num_levels);
    if (k.cost > s->cfg.budget_bytes) return GPJ_ELIMIT;
    if (n > 0) {
        // page-locked, so that loads copy at full speed and overlap the index build
        const cudaError_t e = cudaHostRegister(const_cast<void*>(host), static_cast<size_t>(n),
                                               cudaHostRegisterReadOnly);
        if (e == cudaSuccess) {
            k.registered = true;
        } else if (e == cudaErrorHostMemoryAlreadyRegistered) {
            cudaGetLastError();  // already page-locked by the caller
        } else {
            cudaGetLastError();
            return e == cudaErrorMemoryAllocation ? GPJ_ENOMEM : GPJ_ECUDA;
        }
    }
    std::lock_guard<std::mutex> g(s->mu);
    s->corpora.push_back(k);
    *corpus = static_cast<int>(s->corpora.size() - 1);
    return GPJ_OK;
}

int gpj_serve_set_batching(gpj_server* s, int max_batch, int max_inflight) {
    if (!s || max_batch < 1 || max_inflight < 1) return GPJ_EINVAL;
    std::lock_guard<std::mutex> g(s->mu);
    s->max_batch = max_batch;
    s->max_inflight = std::min(max_inflight, s->cfg.workers);
    s->work_cv.notify_all();
    return GPJ_OK;
}

int gpj_serve_submit(gpj_server* s, int corpus, int nq, const char* const* paths, uint64_t* request) {
    if (!s || !request || nq < 1 || nq > GPJ_MAX_QUERIES || !paths) return GPJ_EINVAL;
    Request* r = new (std::nothrow) Request;
    if (!r) return GPJ_ENOMEM;
    // compile here: a path the reference rejects fails now, and one deeper
    // than the corpora's index is refused (evaluating it would rebuild a
    // corpus's index while other batches read it)
    for (int q = 0; q < nq; q++) {
        if (!paths[q]) {
            delete r;
            return GPJ_EINVAL;
        }
        uint8_t code[4096];
        size_t len = 0;
        int depth = 0, results = 0;
        std::vector<uint8_t> big;
        int crc = gpj_compile(paths[q], code, sizeof(code), &len, &depth, &results, nullptr, 0);
        if (crc == GPJ_ELIMIT && len > sizeof(code)) {
            big.resize(len);
            crc = gpj_compile(paths[q], big.data(), big.size(), &len, &depth, &results, nullptr, 0);
        }
        if (crc) {
            delete r;
            return crc;
        }
        if (depth > s->cfg.num_levels) {
            delete r;
            return GPJ_ELIMIT;
        }
        r->slots = std::max(r->slots, results);
        r->paths.emplace_back(paths[q]);
    }
    std::lock_guard<std::mutex> g(s->mu);
    if (corpus < 0 || corpus >= static_cast<int>(s->corpora.size())) {
        delete r;
        return GPJ_EINVAL;
    }
    r->corpus = corpus;
    r->id = s->next_id++;
    r->submit_ns = now_ns(s->t0);
    s->requests[r->id] = r;
    s->pending.push_back(r);
    s->work_cv.notify_all();
    *request = r->id;
    return GPJ_OK;
}

int gpj_serve_poll(gpj_server* s, uint64_t request, int timeout_ms, gpj_result** out, int64_t* submit_ns,
                   int64_t* done_ns) {
    if (!s || !out) return GPJ_EINVAL;
    *out = nullptr;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(request);
    if (it == s->requests.end()) return GPJ_EINVAL;
    Request* r = it->second;
    auto ready = [&] { return r->done_ns >= 0; };
    if (timeout_ms < 0)
        s->done_cv.wait(lk, ready);
    else if (timeout_ms > 0)
        s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready);
    if (!ready()) return GPJ_EAGAIN;
    s->requests.erase(it);
    lk.unlock();
    if (submit_ns) *submit_ns = r->submit_ns;
    if (done_ns) *done_ns = r->done_ns;
    const int rc = r->rc;
    *out = r->result;
    delete r;
    return rc;
}

int64_t gpj_serve_now_ns(const gpj_server* s) { return s ? now_ns(s->t0) : -1; }

int gpj_serve_stats(gpj_server* s, char* json, size_t cap, size_t* len) {
    if (!s || !len) return GPJ_EINVAL;
    std::string j;
    {
        std::lock_guard<std::mutex> g(s->mu);
        int64_t resident = 0;
        for (const Corpus& k : s->corpora) resident += k.state == CorpusState::kResident ? 1 : 0;
        j = "{\"served\": " + std::to_string(s->served) + ", \"batches\": " + std::to_string(s->batches) +
            ", \"loads\": " + std::to_string(s->loads) + ", \"evictions\": " + std::to_string(s->evictions) +
            ", \"resident_corpora\": " + std::to_string(resident) + ", \"budget_used_bytes\": " +
            std::to_string(s->used) + ", \"budget_bytes\": " + std::to_string(s->cfg.budget_bytes) +
            ", \"pending\": " + std::to_string(s->pending.size()) + "}";
    }
    *len = j.size();
    if (json && cap > 0) {
        const size_t k = std::min(cap - 1, j.size());
        std::memcpy(json, j.data(), k);
        json[k] = '\0';
    }
    return GPJ_OK;
}

void gpj_serve_destroy(gpj_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
        s->work_cv.notify_all();
    }
    for (auto& t : s->workers)
        if (t.joinable()) t.join();
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->loader_stop = true;
        s->load_cv.notify_all();
    }
    if (s->loader.joinable()) s->loader.join();
    for (Corpus& k : s->corpora)
        if (k.registered) cudaHostUnregister(const_cast<uint8_t*>(k.host));
    for (auto& kv : s->requests) {  // every request not handed back, pending ones included
        if (kv.second->result) gpj_result_release(kv.second->result);
        delete kv.second;
    }
    delete s;
}

}  // extern "C"
