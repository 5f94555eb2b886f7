// serve.cpp — batched execution of many plans and the serving loop.
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>

#include "plan.h"

namespace vq {
vexq_result_s* run_plan(Plan& p, int rg_start, int rg_end);
}  // namespace vq

using namespace vq;

namespace {

template <class F>
int32_t guard2(F&& f) {
    try {
        set_error("");
        return f();
    } catch (const Status& s) {
        set_error(s.what());
        return s.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return VEXQ_EINVAL;
    }
}

std::mutex& plan_mutex(Plan* p) {
    static std::mutex m;
    static std::map<Plan*, std::unique_ptr<std::mutex>> mus;
    std::lock_guard<std::mutex> lk(m);
    auto& u = mus[p];
    if (!u) u.reset(new std::mutex);
    return *u;
}

}  // namespace

struct vexq_server_s {
    int64_t budget;
    int max_inflight;
    std::mutex mu;
    std::condition_variable cv, done_cv;
    struct Ticket {
        vexq_plan_s* plan;
        std::chrono::steady_clock::time_point submitted, finished;
        vexq_result_s* result = nullptr;
        int32_t status = VEXQ_OK;
        std::string err;
        bool done = false;
        bool taken = false;
    };
    std::map<int64_t, Ticket> tickets;
    std::deque<int64_t> queue;
    int64_t next_id = 1;
    int64_t inflight_bytes = 0;
    int inflight = 0;
    bool stop = false;
    std::vector<std::thread> workers;
    int device = 0;
};

extern "C" {

int32_t vexq_batch_run(vexq_plan_t* plans, int32_t n, vexq_result_t* out_results) {
    return guard2([&]() -> int32_t {
        if (n < 0 || (n > 0 && (!plans || !out_results))) fail(VEXQ_EINVAL, "null argument");
        for (int i = 0; i < n; i++) out_results[i] = nullptr;
        if (n == 0) return VEXQ_OK;
        std::unique_ptr<Batch, void (*)(Batch*)> b(create_batch(plans, n, 0), destroy_batch);
        exec_batch(*b, out_results);
        return VEXQ_OK;
    });
}

int32_t vexq_server_start(int64_t hbm_budget_bytes, int32_t max_inflight, vexq_server_t* out) {
    return guard2([&]() -> int32_t {
        if (!out || max_inflight < 1 || hbm_budget_bytes <= 0) fail(VEXQ_EINVAL, "bad server parameters");
        auto* s = new vexq_server_s;
        s->budget = hbm_budget_bytes;
        s->max_inflight = max_inflight;
        cudaGetDevice(&s->device);
        for (int w = 0; w < max_inflight; w++) {
            s->workers.emplace_back([s]() {
                cudaSetDevice(s->device);
                for (;;) {
                    int64_t id;
                    vexq_plan_s* pl;
                    int64_t fp;
                    {
                        std::unique_lock<std::mutex> lk(s->mu);
                        // admission: the head of the queue starts when its footprint fits
                        s->cv.wait(lk, [&] {
                            if (s->stop) return true;
                            if (s->queue.empty()) return false;
                            auto& t = s->tickets[s->queue.front()];
                            return s->inflight == 0 || s->inflight_bytes + t.plan->footprint <= s->budget;
                        });
                        if (s->stop) return;
                        id = s->queue.front();
                        s->queue.pop_front();
                        pl = s->tickets[id].plan;
                        fp = pl->footprint;
                        s->inflight_bytes += fp;
                        s->inflight++;
                    }
                    vexq_result_s* r = nullptr;
                    int32_t st = VEXQ_OK;
                    std::string err;
                    try {
                        std::lock_guard<std::mutex> plk(plan_mutex(pl->p));
                        r = run_plan(*pl->p, 0, -1);
                    } catch (const Status& e) {
                        st = e.code;
                        err = e.what();
                    } catch (const std::exception& e) {
                        st = VEXQ_EINVAL;
                        err = e.what();
                    }
                    {
                        std::lock_guard<std::mutex> lk(s->mu);
                        auto& t = s->tickets[id];
                        t.result = r;
                        t.status = st;
                        t.err = err;
                        t.done = true;
                        t.finished = std::chrono::steady_clock::now();
                        s->inflight_bytes -= fp;
                        s->inflight--;
                    }
                    s->cv.notify_all();
                    s->done_cv.notify_all();
                }
            });
        }
        *out = s;
        return VEXQ_OK;
    });
}

int32_t vexq_server_submit(vexq_server_t s, vexq_plan_t p, int64_t* ticket) {
    return guard2([&]() -> int32_t {
        if (!s || !p || !ticket) fail(VEXQ_EINVAL, "null argument");
        if (p->footprint > s->budget) fail(VEXQ_EADMIT, "query footprint exceeds the server's HBM budget");
        {
            std::lock_guard<std::mutex> lk(s->mu);
            if (s->stop) fail(VEXQ_ECANCELED, "server stopped");
            int64_t id = s->next_id++;
            auto& t = s->tickets[id];
            t.plan = p;
            t.submitted = std::chrono::steady_clock::now();
            s->queue.push_back(id);
            *ticket = id;
        }
        s->cv.notify_all();
        return VEXQ_OK;
    });
}

int32_t vexq_server_poll(vexq_server_t s, int64_t ticket, int32_t* done, vexq_result_t* out) {
    return guard2([&]() -> int32_t {
        if (!s || !done || !out) fail(VEXQ_EINVAL, "null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) fail(VEXQ_EINVAL, "unknown ticket");
        *done = it->second.done;
        *out = nullptr;
        if (it->second.done) {
            if (it->second.status != VEXQ_OK) fail(it->second.status, it->second.err);
            if (it->second.taken) fail(VEXQ_EINVAL, "ticket result already taken");
            *out = it->second.result;
            it->second.taken = true;
        }
        return VEXQ_OK;
    });
}

int32_t vexq_server_wait(vexq_server_t s, int64_t ticket, int64_t timeout_ms, vexq_result_t* out) {
    return guard2([&]() -> int32_t {
        if (!s || !out) fail(VEXQ_EINVAL, "null argument");
        std::unique_lock<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end()) fail(VEXQ_EINVAL, "unknown ticket");
        bool ok = s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return it->second.done; });
        if (!ok) fail(VEXQ_ETIMEDOUT, "ticket did not finish within the timeout");
        if (it->second.status != VEXQ_OK) fail(it->second.status, it->second.err);
        if (it->second.taken) fail(VEXQ_EINVAL, "ticket result already taken");
        *out = it->second.result;
        it->second.taken = true;
        return VEXQ_OK;
    });
}

int32_t vexq_server_latency(vexq_server_t s, int64_t ticket, double* ms) {
    return guard2([&]() -> int32_t {
        if (!s || !ms) fail(VEXQ_EINVAL, "null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->tickets.find(ticket);
        if (it == s->tickets.end() || !it->second.done) fail(VEXQ_EINVAL, "ticket not finished");
        *ms = std::chrono::duration<double, std::milli>(it->second.finished - it->second.submitted).count();
        return VEXQ_OK;
    });
}

int32_t vexq_server_stop(vexq_server_t s) {
    return guard2([&]() -> int32_t {
        if (!s) return VEXQ_OK;
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
        }
        s->cv.notify_all();
        for (auto& w : s->workers) w.join();
        for (auto& kv : s->tickets)
            if (kv.second.result && !kv.second.taken) delete kv.second.result;
        delete s;
        return VEXQ_OK;
    });
}

}  // extern "C"
