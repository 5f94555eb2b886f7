// tune.cpp — per-plan tuning of the launch-time choices, by timing the plan's
// own runs: for a join, the global build table against radix partitioning at
// several partition-bit counts; for a dense group table, the size of the
// block-private shared-memory group cache (the shared-versus-global table
// cutover). The fastest choice is kept in plan_tuning.json beside the kernel
// cache, keyed by the plan's shape and the sizes it ran on, so a later plan of
// the same shape takes it without timing.
//
// The reference fixes the partition bits from the build size alone
// (RadixBitsFor, exec/parallel_join.go:72-81, tuned once by its authors on one
// machine); here they are measured on the GPU the plan runs on.
#include <unistd.h>

#include <cstring>
#include <fstream>
#include <sstream>

#include "plan.h"

namespace vq {
vexq_result_s* run_plan(Plan& p, int rg_start, int rg_end);

namespace {

std::mutex g_tune_mu;

std::string tune_path() { return jit_cache_dir() + "/plan_tuning.json"; }

int lg2(long long v) {
    int l = 0;
    while (v > 1) { v >>= 1; l++; }
    return l;
}

// The plan's shape and sizes (log2 rows), the key of its stored choice.
std::string plan_key(const Plan& p) {
    std::ostringstream k;
    k << (p.is_join ? "join" : "agg") << "_" << (p.path == AggPath::Regs ? "regs" : p.path == AggPath::Dense ? "dense" : "hash")
      << "_s" << p.slots.size() << "_f" << p.nf << "_i" << p.ni << "_d" << lg2(std::max<int64_t>(p.domain, 1)) << "_r"
      << lg2(std::max<int64_t>(p.t->nrows, 1));
    if (p.is_join) k << "_b" << lg2(std::max<int64_t>(p.bt->nrows, 1)) << (p.join_gid ? "_gid" : "") << (p.rlocal ? "_local" : "");
    return k.str();
}

bool stored(const std::string& key, int& choice) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::ifstream f(tune_path());
    std::string line;
    const std::string want = "\"" + key + "\":";
    while (std::getline(f, line)) {
        const size_t at = line.find(want);
        if (at == std::string::npos) continue;
        const size_t c = line.find("\"choice\":", at);
        if (c == std::string::npos) return false;
        choice = std::atoi(line.c_str() + c + 9);
        return true;
    }
    return false;
}

void store(const std::string& key, int choice, double ms) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::vector<std::string> keep;
    {
        std::ifstream f(tune_path());
        std::string line;
        const std::string want = "\"" + key + "\":";
        while (std::getline(f, line))
            if (line.size() > 2 && line[0] == ' ' && line.find(want) == std::string::npos) {
                if (line.back() == ',') line.pop_back();
                keep.push_back(line);
            }
    }
    std::ostringstream e;
    e << "  \"" << key << "\": {\"choice\": " << choice << ", \"ms\": " << ms << "}";
    keep.push_back(e.str());
    const std::string tmp = tune_path() + ".tmp" + std::to_string(getpid());
    {
        std::ofstream f(tmp);
        f << "{\n";
        for (size_t i = 0; i < keep.size(); i++) f << keep[i] << (i + 1 < keep.size() ? ",\n" : "\n");
        f << "}\n";
    }
    std::rename(tmp.c_str(), tune_path().c_str());
}

// Applies one candidate: join → partition bits (0: the global table);
// dense aggregate → shared-memory group cache in KB.
void apply(Plan& p, int choice) {
    if (p.is_join) {
        p.radix_bits = choice;
        return;
    }
    p.smem_groups = dense_cache_groups(p, choice);
    const int smem = cache_bytes(p);
    p.smem = smem;
    p.k_main = jit_get(p.src_main, "vq_agg", p.block, smem);
}

double time_runs(Plan& p) {
    std::unique_ptr<vexq_result_s> w(run_plan(p, 0, -1));  // warm-up (and sizes from this run)
    double best = 1e30;
    for (int r = 0; r < 3; r++) {
        std::unique_ptr<vexq_result_s> x(run_plan(p, 0, -1));
        best = std::min(best, x->kernel_ms);
    }
    return best;
}

}  // namespace
}  // namespace vq

using namespace vq;

extern "C" int32_t vexq_plan_autotune(vexq_plan_t plan, uint32_t flags, int32_t* out_choice, double* out_ms) {
    try {
        set_error("");
        if (!plan) fail(VEXQ_EINVAL, "null argument");
        Plan& p = *plan->p;
        std::vector<int> cands;
        if (p.is_join) {
            cands = {0, 6, 8, 10, 12};
            if (!p.radix) cands = {0};
        } else if (p.path == AggPath::Dense) {
            cands = {0, 48, 96, 160};
        } else {
            if (out_choice) *out_choice = -1;  // nothing launch-time to choose on this path
            if (out_ms) *out_ms = 0;
            return VEXQ_OK;
        }
        std::lock_guard<std::mutex> lk(plan_mutex(&p));
        const std::string key = plan_key(p);
        int choice = 0;
        double best_ms = 0;
        if (!(flags & VEXQ_PLAN_RETUNE) && stored(key, choice)) {
            apply(p, choice);
        } else {
            best_ms = 1e30;
            for (int c : cands) {
                apply(p, c);
                double ms;
                try {
                    ms = time_runs(p);
                } catch (const Status& e) {
                    if (e.code == VEXQ_EDEVICE || e.code == VEXQ_ENOMEM) throw;
                    continue;  // a choice this plan cannot take (e.g. a skewed key for partitioning)
                }
                if (ms < best_ms) { best_ms = ms; choice = c; }
            }
            apply(p, choice);
            store(key, choice, best_ms);
        }
        const size_t at = p.explain.find(" tuned=");
        if (at != std::string::npos) {
            const size_t end = p.explain.find(' ', at + 1);
            p.explain.erase(at, end == std::string::npos ? std::string::npos : end - at);
        }
        p.explain += " tuned=" + std::string(p.is_join ? "radix_bits:" : "cache_kb:") + std::to_string(choice);
        if (out_choice) *out_choice = choice;
        if (out_ms) *out_ms = best_ms;
        return VEXQ_OK;
    } catch (const Status& s) {
        set_error(s.what());
        return s.code;
    } catch (const std::exception& e) {
        set_error(e.what());
        return VEXQ_EINVAL;
    }
}
