// shard.cpp — an aggregate or join split across row-group shards: each shard
// (a GPU, or a range of row groups on one GPU) runs the plan over its row
// groups and hands out its groups unfinished (a partial: per group its key,
// first-row order key and every accumulator); the partials travel as bytes
// and are merged in shard order into the finished result.
//
// This is ParallelHashAggregate's partial + merge (exec/parallel.go:124-210,
// mergePartialAgg :237-314) with shards in place of workers: counts and
// integer sums add (wrapping), MIN/MAX keep the extreme (the earlier shard's
// on a tie, so +0 against -0 resolves in shard order), float sums add in shard
// order with a compensation term (TwoSum), and a group's first-row key is the
// smallest, so groups come out in the serial path's first-occurrence order.
// Shard order is fixed, so the merged bits do not depend on which shard
// finished first. HAVING, ORDER BY and LIMIT run once, after the merge.
// Every shard must use the same plan shape over tables with the same
// dictionaries (each GPU holds the whole table and scans its row groups; a
// join's build side is the whole build table on every shard, the probe side
// is sharded). COUNT(DISTINCT) cannot be merged from counts and is refused, as
// the reference's planner refuses it in the parallel path
// (planner/parallel.go:218-228).
#include <cmath>
#include <cstring>
#include <unordered_map>

#include "plan.h"

namespace vq {
vexq_result_s* run_plan(Plan& p, int rg_start, int rg_end);
}  // namespace vq

using namespace vq;

struct vexq_partial_s {
    uint64_t shape = 0;
    Groups g;
    std::vector<char> bytes;  // serialised form, filled by vexq_partial_serialize
    double kernel_ms = 0;
};

namespace {

constexpr uint32_t kMagic = 0x31505156u;  // "VQP1"

// Shape of a plan's partials: path, banks and slot kinds; two plans whose
// partials could be merged have the same shape.
uint64_t plan_shape(const Plan& p) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) { h = (h ^ v) * 1099511628211ull; };
    mix((uint64_t)p.path);
    mix((uint64_t)p.ni);
    mix((uint64_t)p.nf);
    mix((uint64_t)p.domain);
    mix((uint64_t)p.keys.size());
    for (auto& k : p.keys) { mix((uint64_t)k.type); mix((uint64_t)k.bits); mix((uint64_t)k.shift); mix((uint64_t)k.vmin); }
    for (size_t s = 0; s < p.slots.size(); s++) { mix((uint64_t)p.slots[s].kind); mix((uint64_t)p.slot_pos[s]); }
    return h;
}

template <class F>
int32_t guard_p(F&& f) {
    try {
        set_error("");
        return f();
    } catch (const Status& s) {
        set_error(s.what());
        return s.code;
    } catch (const std::bad_alloc&) {
        set_error("host allocation failed");
        return VEXQ_ENOMEM;
    } catch (const std::exception& e) {
        set_error(e.what());
        return VEXQ_EINVAL;
    }
}

void vq_two_sum_host(double& hi, double& lo, double x) {
    const double s = hi + x;
    const double bb = s - hi;
    lo += (hi - (s - bb)) + (x - bb);
    hi = s;
}

// Float MIN/MAX of the register path's float bank (doubles) and of the group
// tables' int bank (order-preserving keys): the later shard replaces the
// earlier one only when strictly better.
struct Merger {
    const Plan& p;
    std::vector<int> ikind, fkind;  // per bank entry: 0 sum, 1 min, 2 max (int: 3 = float order key min, 4 = max)
    explicit Merger(const Plan& pp) : p(pp) {
        ikind.assign(p.ni, 0);
        fkind.assign(p.nf, 0);
        const bool regs = p.path == AggPath::Regs;
        for (size_t s = 0; s < p.slots.size(); s++) {
            const int pos = p.slot_pos[s];
            switch (p.slots[s].kind) {
                case S_IMIN: ikind[pos] = 1; break;
                case S_IMAX: ikind[pos] = 2; break;
                case S_FMIN: if (regs) fkind[pos] = 1; else ikind[pos] = 1; break;  // order keys compare as integers
                case S_FMAX: if (regs) fkind[pos] = 2; else ikind[pos] = 2; break;
                default: break;
            }
        }
        // on the group-table paths float MIN/MAX order keys are unsigned
        for (size_t s = 0; s < p.slots.size(); s++)
            if (!regs && (p.slots[s].kind == S_FMIN || p.slots[s].kind == S_FMAX)) ikind[p.slot_pos[s]] += 2;
    }
    void merge_int(int s, int64_t& d, int64_t v) const {
        switch (ikind[s]) {
            case 0: d = (int64_t)((uint64_t)d + (uint64_t)v); break;
            case 1: if (v < d) d = v; break;
            case 2: if (v > d) d = v; break;
            case 3: if ((uint64_t)v < (uint64_t)d) d = v; break;
            case 4: if ((uint64_t)v > (uint64_t)d) d = v; break;
        }
    }
    void merge_float(int s, double& d, double& comp, double v) const {
        switch (fkind[s]) {
            case 0:
                if (std::isfinite(d) && std::isfinite(v)) vq_two_sum_host(d, comp, v);
                else d = d + v;  // NaN / ±inf: IEEE addition, no compensation
                break;
            case 1: if (v < d) d = v; break;
            case 2: if (v > d) d = v; break;
        }
    }
};

}  // namespace

extern "C" {

int32_t vexq_plan_run_partial(vexq_plan_t plan, int32_t rg_start, int32_t rg_end, vexq_partial_t* out) {
    return guard_p([&]() -> int32_t {
        if (!plan || !out) fail(VEXQ_EINVAL, "null argument");
        *out = nullptr;
        Plan& p = *plan->p;
        if (p.ndist > 0) fail(VEXQ_ENOTSUP, "COUNT(DISTINCT) cannot be merged from shard partials");
        std::unique_ptr<vexq_partial_s> part(new vexq_partial_s);
        part->shape = plan_shape(p);
        std::lock_guard<std::mutex> lk(plan_mutex(&p));
        p.partial_out = &part->g;
        std::unique_ptr<vexq_result_s> r;
        try {
            r.reset(run_plan(p, rg_start, rg_end));
        } catch (...) {
            p.partial_out = nullptr;
            throw;
        }
        p.partial_out = nullptr;
        part->kernel_ms = r ? r->kernel_ms : 0;
        if (part->g.ival.size() != (size_t)p.ni) part->g.ival.resize(p.ni);
        if (part->g.fval.size() != (size_t)p.nf) part->g.fval.resize(p.nf);
        *out = part.release();
        return VEXQ_OK;
    });
}

int32_t vexq_partial_info(vexq_partial_t part, int64_t* groups, double* kernel_ms) {
    return guard_p([&]() -> int32_t {
        if (!part) fail(VEXQ_EINVAL, "null argument");
        if (groups) *groups = (int64_t)part->g.n();
        if (kernel_ms) *kernel_ms = part->kernel_ms;
        return VEXQ_OK;
    });
}

int32_t vexq_partial_serialize(vexq_partial_t part, const void** data, int64_t* len) {
    return guard_p([&]() -> int32_t {
        if (!part || !data || !len) fail(VEXQ_EINVAL, "null argument");
        const Groups& g = part->g;
        const uint64_t n = g.n();
        const uint32_t ni = (uint32_t)g.ival.size(), nf = (uint32_t)g.fval.size();
        std::vector<char>& b = part->bytes;
        b.assign(4 + 4 + 4 + 8 + 8 + n * 8 * (2 + ni + nf), 0);
        char* w = b.data();
        auto put = [&](const void* src, size_t k) { std::memcpy(w, src, k); w += k; };
        put(&kMagic, 4);
        put(&ni, 4);
        put(&nf, 4);
        put(&part->shape, 8);
        put(&n, 8);
        put(g.key.data(), n * 8);
        put(g.first.data(), n * 8);
        for (uint32_t s = 0; s < ni; s++) put(g.ival[s].data(), n * 8);
        for (uint32_t s = 0; s < nf; s++) put(g.fval[s].data(), n * 8);
        *data = b.data();
        *len = (int64_t)b.size();
        return VEXQ_OK;
    });
}

int32_t vexq_partial_deserialize(vexq_plan_t plan, const void* data, int64_t len, vexq_partial_t* out) {
    return guard_p([&]() -> int32_t {
        if (!plan || !out || (!data && len > 0)) fail(VEXQ_EINVAL, "null argument");
        *out = nullptr;
        const Plan& p = *plan->p;
        const char* r = (const char*)data;
        const char* end = r + len;
        auto get = [&](void* dst, size_t k) {
            if ((size_t)(end - r) < k) fail(VEXQ_EINVAL, "partial bytes are truncated");
            std::memcpy(dst, r, k);
            r += k;
        };
        uint32_t magic = 0, ni = 0, nf = 0;
        uint64_t shape = 0, n = 0;
        get(&magic, 4);
        if (magic != kMagic) fail(VEXQ_EINVAL, "not a partial (bad magic)");
        get(&ni, 4);
        get(&nf, 4);
        get(&shape, 8);
        get(&n, 8);
        if (shape != plan_shape(p) || ni != (uint32_t)p.ni || nf != (uint32_t)p.nf)
            fail(VEXQ_EINVAL, "partial comes from a plan of another shape");
        if (n > (uint64_t)(end - r) / 8) fail(VEXQ_EINVAL, "partial bytes are truncated");
        std::unique_ptr<vexq_partial_s> part(new vexq_partial_s);
        part->shape = shape;
        Groups& g = part->g;
        g.key.resize(n);
        g.first.resize(n);
        g.ival.assign(ni, std::vector<int64_t>(n));
        g.fval.assign(nf, std::vector<double>(n));
        get(g.key.data(), n * 8);
        get(g.first.data(), n * 8);
        for (uint32_t s = 0; s < ni; s++) get(g.ival[s].data(), n * 8);
        for (uint32_t s = 0; s < nf; s++) get(g.fval[s].data(), n * 8);
        if (r != end) fail(VEXQ_EINVAL, "partial bytes have trailing data");
        *out = part.release();
        return VEXQ_OK;
    });
}

int32_t vexq_partial_merge(vexq_plan_t plan, const vexq_partial_t* parts, int32_t n, vexq_result_t* out) {
    return guard_p([&]() -> int32_t {
        if (!plan || !out || n < 0 || (n > 0 && !parts)) fail(VEXQ_EINVAL, "null argument");
        *out = nullptr;
        Plan& p = *plan->p;
        const uint64_t shape = plan_shape(p);
        Merger m(p);
        Groups g;
        g.ival.assign(p.ni, {});
        g.fval.assign(p.nf, {});
        std::vector<std::vector<double>> comp(p.nf);
        std::unordered_map<uint64_t, size_t> at;
        for (int k = 0; k < n; k++) {
            if (!parts[k]) fail(VEXQ_EINVAL, "null partial");
            const Groups& s = parts[k]->g;
            if (parts[k]->shape != shape) fail(VEXQ_EINVAL, "partial comes from a plan of another shape");
            for (size_t i = 0; i < s.n(); i++) {
                auto it = at.find(s.key[i]);
                if (it == at.end()) {
                    at.emplace(s.key[i], g.key.size());
                    g.key.push_back(s.key[i]);
                    g.first.push_back(s.first[i]);
                    for (int b = 0; b < p.ni; b++) g.ival[b].push_back(s.ival[b][i]);
                    for (int b = 0; b < p.nf; b++) {
                        g.fval[b].push_back(s.fval[b][i]);
                        comp[b].push_back(0.0);
                    }
                    continue;
                }
                const size_t j = it->second;
                g.first[j] = std::min(g.first[j], s.first[i]);
                for (int b = 0; b < p.ni; b++) m.merge_int(b, g.ival[b][j], s.ival[b][i]);
                for (int b = 0; b < p.nf; b++) m.merge_float(b, g.fval[b][j], comp[b][j], s.fval[b][i]);
            }
        }
        for (int b = 0; b < p.nf; b++)
            if (m.fkind[b] == 0)
                for (size_t j = 0; j < g.n(); j++)
                    if (std::isfinite(g.fval[b][j])) g.fval[b][j] += comp[b][j];
        std::lock_guard<std::mutex> lk(plan_mutex(&p));
        *out = build_result(p, g);
        return VEXQ_OK;
    });
}

int32_t vexq_partial_free(vexq_partial_t part) {
    delete part;
    return VEXQ_OK;
}

}  // extern "C"
