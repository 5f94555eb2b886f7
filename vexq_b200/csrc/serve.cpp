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

}  // namespace

struct vexq_server_s {
    int64_t budget;
    int max_inflight;
    int nworkers = 1;
    bool batching = true;
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
    // launch statistics
    int64_t launches = 0, launched_queries = 0;
    int max_batch = 0, running = 0, max_running = 0;
};

namespace {

// Runs one admitted set: aggregate plans together in one direct batched
// execution on the worker's workspace, joins on their own (their plan owns the
// join-table buffers, so one run at a time per plan). A failing batch is rerun
// plan by plan so each ticket gets its own status.
void run_admitted(Batch* ws, const std::vector<vexq_plan_s*>& pls, std::vector<vexq_result_s*>& res,
                  std::vector<int32_t>& st, std::vector<std::string>& err, bool batching) {
    const size_t n = pls.size();
    res.assign(n, nullptr);
    st.assign(n, VEXQ_OK);
    err.assign(n, std::string());
    auto one = [&](size_t i) {
        try {
            std::lock_guard<std::mutex> plk(plan_mutex(pls[i]->p));
            res[i] = run_plan(*pls[i]->p, 0, -1);
        } catch (const Status& e) {
            st[i] = e.code;
            err[i] = e.what();
        } catch (const std::exception& e) {
            st[i] = VEXQ_EINVAL;
            err[i] = e.what();
        }
    };
    std::vector<size_t> aggs;
    for (size_t i = 0; i < n; i++) {
        if (batching && !pls[i]->p->is_join) aggs.push_back(i);
        else one(i);
    }
    if (aggs.empty()) return;
    std::vector<vexq_plan_s*> ap;
    for (size_t i : aggs) ap.push_back(pls[i]);
    std::vector<vexq_result_s*> out(ap.size(), nullptr);
    std::string first_err;
    try {
        run_batch_direct(*ws, ap.data(), (int)ap.size(), out.data());
        for (size_t k = 0; k < aggs.size(); k++) res[aggs[k]] = out[k];
        return;
    } catch (const std::exception& e) {
        first_err = e.what();
    }
    for (size_t i : aggs) {
        one(i);
        if (st[i] != VEXQ_OK) err[i] += " (the batched run failed first: " + first_err + ")";
    }
}

}  // namespace

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

int32_t vexq_server_start(int64_t hbm_budget_bytes, int32_t max_inflight, int32_t nworkers, uint32_t flags,
                          vexq_server_t* out) {
    return guard2([&]() -> int32_t {
        if (!out || max_inflight < 1 || hbm_budget_bytes <= 0 || nworkers < 1) fail(VEXQ_EINVAL, "bad server parameters");
        auto* s = new vexq_server_s;
        s->budget = hbm_budget_bytes;
        s->max_inflight = max_inflight;
        s->nworkers = nworkers;
        s->batching = !(flags & VEXQ_SERVE_NO_BATCH);
        cudaGetDevice(&s->device);
        for (int w = 0; w < nworkers; w++) {
            s->workers.emplace_back([s]() {
                cudaSetDevice(s->device);
                std::unique_ptr<Batch, void (*)(Batch*)> ws(nullptr, destroy_batch);
                try {
                    ws.reset(new_batch());
                } catch (...) {
                    return;
                }
                for (;;) {
                    std::vector<int64_t> ids;
                    std::vector<vexq_plan_s*> pls;
                    int64_t fp = 0;
                    {
                        std::unique_lock<std::mutex> lk(s->mu);
                        // admission: the head of the queue starts when a slot is free
                        // and its footprint fits the budget beside what is in flight
                        s->cv.wait(lk, [&] {
                            if (s->stop) return true;
                            if (s->queue.empty() || s->inflight >= s->max_inflight) return false;
                            auto& t = s->tickets[s->queue.front()];
                            return s->inflight == 0 || s->inflight_bytes + t.plan->footprint <= s->budget;
                        });
                        if (s->stop) return;
                        // continuous batching: queued aggregates that fit join this
                        // launch, up to an equal share of the slots so the other
                        // workers can launch beside it; a join is a launch of its own
                        const int cap = std::max(1, s->max_inflight / s->nworkers);
                        while (!s->queue.empty() && s->inflight < s->max_inflight && (int)ids.size() < cap) {
                            auto& t = s->tickets[s->queue.front()];
                            if (s->inflight > 0 && s->inflight_bytes + t.plan->footprint > s->budget) break;
                            const bool join = t.plan->p->is_join;
                            if (join && !ids.empty()) break;
                            ids.push_back(s->queue.front());
                            pls.push_back(t.plan);
                            fp += t.plan->footprint;
                            s->inflight_bytes += t.plan->footprint;
                            s->inflight++;
                            s->queue.pop_front();
                            if (!s->batching || join) break;
                        }
                        s->launches++;
                        s->launched_queries += (int64_t)ids.size();
                        s->max_batch = std::max(s->max_batch, (int)ids.size());
                        s->running++;
                        s->max_running = std::max(s->max_running, s->running);
                    }
                    std::vector<vexq_result_s*> res;
                    std::vector<int32_t> st;
                    std::vector<std::string> err;
                    run_admitted(ws.get(), pls, res, st, err, s->batching);
                    {
                        std::lock_guard<std::mutex> lk(s->mu);
                        auto now = std::chrono::steady_clock::now();
                        for (size_t k = 0; k < ids.size(); k++) {
                            auto& t = s->tickets[ids[k]];
                            t.result = res[k];
                            t.status = st[k];
                            t.err = err[k];
                            t.done = true;
                            t.finished = now;
                        }
                        s->inflight_bytes -= fp;
                        s->inflight -= (int)ids.size();
                        s->running--;
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

int32_t vexq_server_stats(vexq_server_t s, int64_t* launches, int64_t* queries, int32_t* max_batch,
                          int32_t* max_concurrent) {
    return guard2([&]() -> int32_t {
        if (!s) fail(VEXQ_EINVAL, "null argument");
        std::lock_guard<std::mutex> lk(s->mu);
        if (launches) *launches = s->launches;
        if (queries) *queries = s->launched_queries;
        if (max_batch) *max_batch = s->max_batch;
        if (max_concurrent) *max_concurrent = s->max_running;
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
