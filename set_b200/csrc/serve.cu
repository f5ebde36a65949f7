// serve.cu -- a solve server: continuous batching of Cartesian MHD solves on one GPU.
// No counterpart in the reference (one grid per process).
//
// A server thread owns a setb_batch.  Clients submit requests from any thread; between chunks of
// `check_every` steps the thread admits queued requests in arrival order while their HBM
// footprint fits the budget (the head of the queue waits for room: no overtaking), advances the
// batch one chunk, runs the deterministic steady-state check and retires every solve that
// reached its tolerance or its step cap.  A solve's result depends only on its own request:
// chunk boundaries are at multiples of check_every steps of that solve.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "setb200.h"

namespace {

double now_s() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

struct Entry {
    int64_t id = 0;
    setb_request req{};
    setb_result res{};
    int slot = -1;
};

}  // namespace

struct setb_server {
    setb_batch* batch = nullptr;
    int max_slots = 0;
    int check_every = 50;
    std::thread th;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Entry> pending;
    std::map<int, Entry> active;          // slot -> entry
    std::map<int64_t, setb_result> done;  // id -> result (until collected)
    std::vector<setb_result> finished;    // completion order, for polling
    bool stop = false;
    int64_t next_id = 1;
    int64_t n_done = 0, n_failed = 0, chunks = 0;
    int32_t max_active = 0;
};

namespace {

void finish(setb_server* s, Entry& e, int status) {
    e.res.status = status;
    e.res.t_done = now_s();
    setb_diag d{};
    setb_batch_status(s->batch, e.slot, &d);
    e.res.diag = d;
    e.res.time_all = d.time_all;
    if (status == SETB_OK && e.req.result_U) {
        if (setb_batch_get_conserved(s->batch, e.slot, e.req.result_U) != SETB_OK) e.res.status = SETB_ECUDA;
    }
    setb_batch_remove(s->batch, e.slot);
}

void loop(setb_server* s) {
    std::vector<double> rel(s->max_slots);
    for (;;) {
        {
            std::unique_lock<std::mutex> lk(s->mu);
            // admission, in arrival order, while the footprint fits
            while (!s->pending.empty()) {
                Entry& e = s->pending.front();
                int slot = -1;
                const int rc = setb_batch_add(s->batch, &e.req.desc, &e.req.ic, &e.req.opts, &slot);
                if (rc == SETB_EBUSY && !s->active.empty()) break;   // wait for room
                if (rc != SETB_OK) {                                 // never fits, or invalid
                    e.res.status = rc;
                    e.res.t_admit = e.res.t_done = now_s();
                    s->done[e.id] = e.res;
                    s->finished.push_back(e.res);
                    s->n_failed++;
                    s->pending.pop_front();
                    s->cv_done.notify_all();
                    continue;
                }
                e.slot = slot;
                e.res.t_admit = now_s();
                s->active[slot] = e;
                s->pending.pop_front();
            }
            if (s->active.empty()) {
                if (s->stop && s->pending.empty()) return;
                s->cv_work.wait(lk, [&] { return s->stop || !s->pending.empty(); });
                continue;
            }
            s->max_active = std::max<int32_t>(s->max_active, (int32_t)s->active.size());
        }
        // one chunk for every active solve (outside the lock: clients keep submitting)
        int rc = setb_batch_step(s->batch, s->check_every);
        if (rc == SETB_OK) rc = setb_batch_check(s->batch, rel.data());
        s->chunks++;
        std::lock_guard<std::mutex> lk(s->mu);
        std::vector<int> retire;
        for (auto& kv : s->active) {
            Entry& e = kv.second;
            e.res.steps += s->check_every;
            e.res.last_change = rel[kv.first];
            const bool steady = e.req.steady_tol > 0.0 && rel[kv.first] >= 0.0 && rel[kv.first] < e.req.steady_tol;
            setb_diag d{};
            const int st = setb_batch_status(s->batch, kv.first, &d);
            if (rc != SETB_OK || st != SETB_OK || steady || e.res.steps >= e.req.max_steps) {
                finish(s, e, rc != SETB_OK ? rc : st);
                e.res.converged = steady ? 1 : 0;
                s->done[e.id] = e.res;
                s->finished.push_back(e.res);
                if (e.res.status == SETB_OK) s->n_done++;
                else s->n_failed++;
                retire.push_back(kv.first);
            }
        }
        for (int slot : retire) s->active.erase(slot);
        if (!retire.empty()) s->cv_done.notify_all();
    }
}

}  // namespace

extern "C" {

int32_t setb_server_create(setb_server** out, int32_t max_slots, int32_t precision, int64_t hbm_budget,
                           int32_t check_every) {
    if (!out || check_every < 1) return SETB_EINVAL;
    *out = nullptr;
    setb_server* s = new (std::nothrow) setb_server();
    if (!s) return SETB_ENOMEM;
    int rc = setb_batch_create(&s->batch, max_slots, precision, hbm_budget);
    if (rc) {
        delete s;
        return rc;
    }
    s->max_slots = max_slots;
    s->check_every = check_every;
    int dev = 0;
    cudaGetDevice(&dev);
    s->th = std::thread([s, dev] {
        cudaSetDevice(dev);
        loop(s);
    });
    *out = s;
    return SETB_OK;
}

int32_t setb_server_submit(setb_server* s, const setb_request* r, int64_t* id) {
    if (!s || !r || !id || r->max_steps < 1) return SETB_EINVAL;
    Entry e;
    e.req = *r;
    e.res.t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->stop) return SETB_EBUSY;
        e.id = s->next_id++;
        e.res.id = e.id;
        s->pending.push_back(e);
        *id = e.id;
    }
    s->cv_work.notify_one();
    return SETB_OK;
}

int32_t setb_server_wait(setb_server* s, int64_t id, setb_result* out, double timeout_s) {
    if (!s || !out) return SETB_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    const bool ok = s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                        [&] { return s->done.count(id) > 0; });
    if (!ok) return SETB_ETIMEOUT;
    *out = s->done[id];
    s->done.erase(id);
    return SETB_OK;
}

int32_t setb_server_poll(setb_server* s, setb_result* out, int32_t max, int32_t* n) {
    if (!s || !out || !n || max < 0) return SETB_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    const int k = std::min<int>(max, (int)s->finished.size());
    for (int i = 0; i < k; i++) out[i] = s->finished[i];
    s->finished.erase(s->finished.begin(), s->finished.begin() + k);
    *n = k;
    return SETB_OK;
}

int32_t setb_server_stats(setb_server* s, int32_t* pending, int32_t* active, int64_t* completed, int64_t* failed,
                          int32_t* max_active) {
    if (!s) return SETB_EINVAL;
    std::lock_guard<std::mutex> lk(s->mu);
    if (pending) *pending = (int32_t)s->pending.size();
    if (active) *active = (int32_t)s->active.size();
    if (completed) *completed = s->n_done;
    if (failed) *failed = s->n_failed;
    if (max_active) *max_active = s->max_active;
    return SETB_OK;
}

int32_t setb_server_destroy(setb_server* s) {
    if (!s) return SETB_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    setb_batch_destroy(s->batch);
    delete s;
    return SETB_OK;
}

}  // extern "C"
