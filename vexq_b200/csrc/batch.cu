// batch.cu — many aggregate plans in one batched execution.
//
// The plans are split by path: register-path plans (≤16 groups, per-block
// partials) and group-table plans (dense or hash tables, exact fixed-point
// sums). Each class runs as ONE persistent launch of a generated kernel that
// holds a body per distinct plan shape: blocks take (plan, chunk range) units
// from an atomic ticket, largest units first, so uneven plans share the GPU
// without one launch each. Table init, the class launches (on two forked
// streams), the partial merge and the table finalize are captured once in a
// CUDA graph and replayed by each execution, followed by one copy of every
// output back to pinned host memory. The autotuner picks the shared-memory group
// cache size (the shared-versus-global table cutover), the unit size and the
// block shape of each class by timing graph replays, and keeps its choice in a
// JSON file keyed by the batch's shape. A join whose build key range allows a
// direct-mapped table is batched too: its build runs as units of a third,
// build-class persistent launch ahead of the other two, its probe as units of
// the register or group-table class; the build's counts and error word come
// back with the outputs, and a build that failed (a repeated key) or was empty
// sends the join to a plain run. Other joins run after the graph, one after
// another, as vexq_plan_run would run them.
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <thread>

#include "internal.h"
#include "plan.h"

namespace vq {
__global__ void k_init_batch(const VQTableDesc* d, int n, long long total);
__global__ void k_finalize_batch(const VQTableDesc* d, int n, long long total);
__global__ void k_merge_batch(const VQMergeDesc* d, int n);

namespace {

constexpr int kBlockRegs = 128;   // register-path bodies: many accumulators per thread
constexpr int kBlockTable = 256;  // group-table bodies

size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

struct Item {
    Plan* p = nullptr;
    int cls = 2;  // 0 register path, 1 group table, 2 not batched
    std::vector<long long> seg;
    long long nchunks = 0, rows = 0;
    int64_t bytes = 0;
    int body = -1;
    long long units = 0;
    // register path
    int G = 0, nf = 0, ni = 0, nfb = 1;
    size_t a_part_f = 0, a_part_i = 0, a_kinds = 0, o_out_f = 0, o_out_i = 0;
    // group table
    long long cap = 0, nslots = 0, cap_out = 0;
    bool hash = false;
    int cache_n = 0;
    size_t a_keys = 0, a_first = 0, a_acc_i = 0, a_acc_fx = 0, a_special = 0, a_init = 0, a_lsb = 0, a_ngroups = 0;
    size_t o_nout = 0, o_err = 0, o_key = 0, o_first = 0, o_i = 0, o_f = 0;
    size_t a_seg = 0;
    // join (direct-mapped build): the build side's row ranges, its work units
    // in the build class, its parameter block (bparams[bix]), the key table,
    // the number → key array (GROUP BY the join key) and the build's counts
    // and error word, copied back with the outputs
    bool join = false, gid = false;
    int bix = -1, bbody = -1;
    std::vector<long long> bseg;
    long long bnchunks = 0, brows = 0, bunits = 0;
    long long dmin = 0;
    unsigned long long drange = 0;
    size_t a_bseg = 0, a_dmap = 0, a_jgkey = 0, o_jscal = 0;
};

struct ClassKernel {
    std::vector<int> items;  // indices into Batch::items
    std::string k_src;
    JitKernel k;
    int block = 256, smem_extra = 0, nbodies = 0, grid = 0;
    size_t a_units = 0;
    long long nunits = 0;
};

}  // namespace

struct Batch {
    std::vector<vexq_plan_s*> handles;
    std::vector<Item> items;
    ClassKernel ck[3];  // register path, group tables, join builds (run before both)
    int cache_kb = 96, unit_div = 4;
    DevBuf dev, out;
    PinnedBuf h_out;
    size_t out_bytes = 0, a_params = 0, a_bparams = 0, a_tdesc = 0, a_mdesc = 0, a_ticket = 0, o_aerr = 0;
    int njoins = 0;
    int n_tdesc = 0, n_mdesc = 0, merge_entries = 0;
    long long table_slots = 0;
    cudaStream_t s = nullptr, s2 = nullptr;
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};  // [4]: kernels done (before the copy back)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    double device_ms = 0, kernel_ms = 0;
    bool capturing = false;
    void chk(cudaStream_t st, const char* what) const { if (!capturing) launch_check(st, what); }
    int64_t bytes = 0, rows = 0;
    std::string explain;

    ~Batch() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (s2) cudaStreamDestroy(s2);
        if (s) cudaStreamDestroy(s);
    }

    void drop_graph() {
        if (gexec) cudaGraphExecDestroy(gexec);
        if (graph) cudaGraphDestroy(graph);
        gexec = nullptr;
        graph = nullptr;
    }

    // Sizes every buffer for the current tuning, fills and uploads the
    // parameter blocks, unit lists and descriptors.
    void layout() {
        drop_graph();
        // units: about unit_div units per resident block of each class, at
        // least 16 chunks (2,048 rows) each
        for (int c = 0; c < 3; c++) {
            long long chunks = 0;
            for (int i : ck[c].items) chunks += c == 2 ? items[i].bnchunks : items[i].nchunks;
            long long target = std::max<long long>(1, (long long)ck[c].grid * unit_div);
            long long U = std::max<long long>(16, (chunks + target - 1) / target);
            ck[c].nunits = 0;
            for (int i : ck[c].items) {
                Item& it = items[i];
                long long& u = c == 2 ? it.bunits : it.units;
                u = ((c == 2 ? it.bnchunks : it.nchunks) + U - 1) / U;
                ck[c].nunits += u;
            }
        }
        size_t off = 0, oo = 0;
        auto take = [&](size_t b) { size_t o = off; off += al(std::max<size_t>(b, 8)); return o; };
        auto otake = [&](size_t b) { size_t o = oo; oo += al(std::max<size_t>(b, 8)); return o; };
        a_params = take(items.size() * sizeof(VQParams));
        a_bparams = take((size_t)std::max(njoins, 1) * sizeof(VQParams));
        for (int c = 0; c < 3; c++) ck[c].a_units = take((size_t)ck[c].nunits * sizeof(VQUnit));
        n_tdesc = (int)ck[1].items.size();
        n_mdesc = (int)ck[0].items.size();
        a_tdesc = take(n_tdesc * sizeof(VQTableDesc));
        a_mdesc = take(n_mdesc * sizeof(VQMergeDesc));
        a_ticket = take(16);
        o_aerr = otake(8);
        table_slots = 0;
        merge_entries = 0;
        // uploaded pieces first, then device scratch (partials, tables)
        for (Item& it : items) {
            if (it.cls == 2) continue;
            it.a_seg = take(it.seg.size() * 8);
            if (it.join) it.a_bseg = take(it.bseg.size() * 8);
            if (it.cls == 0) {
                it.a_kinds = take((size_t)(it.nfb + it.ni + 1) * 4);
            } else {
                it.a_init = take((size_t)it.ni * 8);
                it.a_lsb = take((size_t)std::max(it.nf, 1) * 4);
            }
        }
        const size_t upload = off;
        for (Item& it : items) {
            if (it.cls == 2) continue;
            if (it.join) {
                it.a_dmap = take((size_t)it.drange * 8);
                it.a_jgkey = take((size_t)std::max<long long>(it.brows, 1) * 8);
                it.o_jscal = otake(32);
            }
            if (it.cls == 0) {
                it.a_part_f = take((size_t)it.units * it.G * it.nfb * 8);
                it.a_part_i = take((size_t)it.units * it.G * (it.ni + 1) * 8);
                it.o_out_f = otake((size_t)it.G * it.nfb * 8);
                it.o_out_i = otake((size_t)it.G * (it.ni + 1) * 8);
                merge_entries += it.G * it.nf + it.G * (it.ni + 1);
            } else {
                const long long ns = it.nslots;
                it.cache_n = it.hash || it.join ? 0 : dense_cache_groups(*it.p, cache_kb);
                it.a_keys = it.hash ? take(ns * 8) : 0;
                it.a_first = take(ns * 8);
                it.a_acc_i = take((size_t)it.ni * ns * 8);
                it.a_acc_fx = take((size_t)it.nf * ns * 32);
                it.a_special = take((size_t)it.nf * ns * 4);
                it.a_ngroups = take(8);
                it.o_nout = otake(8);
                it.o_err = otake(8);
                it.o_key = otake(it.cap_out * 8);
                it.o_first = otake(it.cap_out * 8);
                it.o_i = otake((size_t)it.ni * it.cap_out * 8);
                it.o_f = otake((size_t)it.nf * it.cap_out * 8);
                table_slots += ns;
            }
        }
        dev.ensure(off);
        out.ensure(oo);
        out_bytes = oo;
        h_out.ensure(oo);
        char* D = (char*)dev.p;
        char* O = (char*)out.p;
        // host images of the uploaded part
        std::vector<VQParams> params(items.size()), bparams((size_t)std::max(njoins, 1));
        std::vector<VQUnit> units[3];
        std::vector<VQTableDesc> td;
        std::vector<VQMergeDesc> md;
        std::vector<char> blob(upload, 0);
        auto put = [&](size_t at, const void* src, size_t n) { if (n) std::memcpy(blob.data() + at, src, n); };
        int e0 = 0;
        long long slot0 = 0;
        for (size_t ix = 0; ix < items.size(); ix++) {
            Item& it = items[ix];
            if (it.cls == 2) continue;
            Plan& p = *it.p;
            VQParams& P = params[ix];
            std::memset(&P, 0, sizeof P);
            set_plan_constants(p, P);
            set_columns(P, *p.t, false);
            P.seg = (const long long*)(D + it.a_seg);
            P.nseg = (int)it.seg.size() / 3;
            P.nchunks = it.nchunks;
            P.rg_rows = p.t->rg_rows;
            P.n_rg = p.t->n_rg;
            P.present = p.d_present.as<unsigned char>();
            for (size_t i = 0, o = 0; i < p.sets.size(); i++) { P.sets[i] = p.d_sets.as<unsigned>() + o; o += p.sets[i].size(); }
            put(it.a_seg, it.seg.data(), it.seg.size() * 8);
            if (it.join) {
                // probe: build-side columns read through build rows, the
                // direct-mapped key table
                set_columns(P, *p.bt, true);
                P.dmap = (unsigned long long*)(D + it.a_dmap);
                P.dmin = it.dmin;
                P.drange = it.drange;
                // build: its own parameter block over the build table (mode 3)
                VQParams& B = bparams[it.bix];
                std::memset(&B, 0, sizeof B);
                set_plan_constants(p, B);
                set_columns(B, *p.bt, false);
                B.seg = (const long long*)(D + it.a_bseg);
                B.nseg = (int)it.bseg.size() / 3;
                B.nchunks = it.bnchunks;
                B.rg_rows = p.bt->rg_rows;
                B.n_rg = p.bt->n_rg;
                B.present = p.d_bpresent.as<unsigned char>();
                for (size_t i = 0, o = 0; i < p.sets.size(); i++) { B.sets[i] = p.d_sets.as<unsigned>() + o; o += p.sets[i].size(); }
                B.mode = 3;
                B.dmap = P.dmap;
                B.dmin = it.dmin;
                B.drange = it.drange;
                B.jgkey = (unsigned long long*)(D + it.a_jgkey);
                B.jgid = it.gid ? (int*)B.jgkey : nullptr;  // a non-null flag: group numbers are handed out
                B.jgoff = p.gid_koff;
                B.jnkeys = (unsigned long long*)(O + it.o_jscal);
                B.error = (int*)(O + it.o_jscal + 8);
                B.jtotal = (unsigned long long*)(O + it.o_jscal + 16);
                put(it.a_bseg, it.bseg.data(), it.bseg.size() * 8);
            }
            if (it.cls == 0) {
                P.part_f = (double*)(D + it.a_part_f);
                P.part_i = (long long*)(D + it.a_part_i);
                P.error = (int*)(O + o_aerr);
                std::vector<int> kinds(it.nfb + it.ni + 1, 0);
                for (size_t i = 0; i < p.slots.size(); i++) {
                    int kd = p.slots[i].kind;
                    int code = (kd == S_IMIN || kd == S_FMIN) ? 1 : (kd == S_IMAX || kd == S_FMAX) ? 2 : 0;
                    kinds[p.slots[i].is_float() ? p.slot_pos[i] : it.nfb + p.slot_pos[i]] = code;
                }
                kinds[it.nfb + it.ni] = 1;
                put(it.a_kinds, kinds.data(), kinds.size() * 4);
                VQMergeDesc m;
                m.part_f = P.part_f;
                m.part_i = P.part_i;
                m.nblocks = (int)it.units;
                m.G = it.G;
                m.nf = it.nf;
                m.ni = it.ni;
                m.fkind = (const int*)(D + it.a_kinds);
                m.ikind = m.fkind + it.nfb;
                m.out_f = (double*)(O + it.o_out_f);
                m.out_i = (long long*)(O + it.o_out_i);
                m.e0 = e0;
                e0 += it.G * it.nf + it.G * (it.ni + 1);
                md.push_back(m);
            } else {
                P.keys = it.hash ? (unsigned long long*)(D + it.a_keys) : nullptr;
                P.first = (long long*)(D + it.a_first);
                P.acc_i = (long long*)(D + it.a_acc_i);
                P.acc_fx = (long long*)(D + it.a_acc_fx);
                P.special = (unsigned*)(D + it.a_special);
                P.ngroups = (unsigned long long*)(D + it.a_ngroups);
                P.error = (int*)(O + it.o_err);
                P.cap = (unsigned long long)it.cap;
                P.cap_mask = it.hash ? (unsigned long long)(it.cap - 1) : 0;
                P.cache_n = it.cache_n;
                std::vector<long long> iv = init_values(p);
                put(it.a_init, iv.data(), (size_t)it.ni * 8);
                put(it.a_lsb, p.fx_lsb.data(), (size_t)it.nf * 4);
                VQTableDesc t;
                std::memset(&t, 0, sizeof t);
                t.keys = P.keys;
                t.first = P.first;
                t.acc_i = P.acc_i;
                t.acc_fx = P.acc_fx;
                t.special = P.special;
                t.init_i = (const long long*)(D + it.a_init);
                t.fx_lsb = (const int*)(D + it.a_lsb);
                t.nslots = it.nslots;
                t.ni = it.ni;
                t.nf = it.nf;
                t.hash = it.hash ? 1 : 0;
                if (it.gid) {  // keys come from the build's number → key array
                    t.keys = (unsigned long long*)(D + it.a_jgkey);
                    t.hash = 1;
                    t.gid = 1;
                }
                t.n_out = (unsigned long long*)(O + it.o_nout);
                t.ngroups = P.ngroups;
                t.error = P.error;
                t.o_key = (unsigned long long*)(O + it.o_key);
                t.o_first = (long long*)(O + it.o_first);
                t.o_i = (long long*)(O + it.o_i);
                t.o_f = (double*)(O + it.o_f);
                t.cap_out = it.cap_out;
                t.slot0 = slot0;
                slot0 += it.nslots;
                td.push_back(t);
            }
        }
        for (int c = 0; c < 3; c++) {
            for (int i : ck[c].items) {
                const Item& it = items[i];
                const long long nu = c == 2 ? it.bunits : it.units, nc = c == 2 ? it.bnchunks : it.nchunks;
                if (!nu) continue;
                const long long u = (nc + nu - 1) / nu;
                for (long long k = 0; k < nu; k++) {
                    VQUnit w;
                    w.plan = c == 2 ? it.bix : i;  // build units index the build parameter blocks
                    w.body = c == 2 ? it.bbody : it.body;
                    w.cbeg = k * u;
                    w.cend = std::min(nc, (k + 1) * u);
                    w.pslot = k;
                    units[c].push_back(w);
                }
            }
            std::stable_sort(units[c].begin(), units[c].end(),
                             [](const VQUnit& a, const VQUnit& b) { return a.cend - a.cbeg > b.cend - b.cbeg; });
            put(ck[c].a_units, units[c].data(), units[c].size() * sizeof(VQUnit));
        }
        put(a_params, params.data(), params.size() * sizeof(VQParams));
        put(a_bparams, bparams.data(), (size_t)njoins * sizeof(VQParams));
        put(a_tdesc, td.data(), td.size() * sizeof(VQTableDesc));
        put(a_mdesc, md.data(), md.size() * sizeof(VQMergeDesc));
        h2d(dev.p, blob.data(), upload, s);
        std::ostringstream ex;
        ex << "batch plans=" << items.size() << " regs_plans=" << ck[0].items.size() << " regs_bodies=" << ck[0].nbodies
           << " regs_units=" << ck[0].nunits << " table_plans=" << ck[1].items.size() << " table_bodies=" << ck[1].nbodies
           << " table_units=" << ck[1].nunits << " joins=" << njoins << " build_units=" << ck[2].nunits << " cache_kb=" << cache_kb
           << " unit_div=" << unit_div;
        explain = ex.str();
    }

    int table_smem() const {
        int m = 0;
        for (int i : ck[1].items) {
            const Item& it = items[i];
            if (!it.hash) m = std::max(m, dense_cache_groups(*it.p, cache_kb) * cache_group_bytes(*it.p));
        }
        return m;
    }

    // Issues one execution on s (group tables, copy back) and s2 (register
    // path), forked and joined with events; captured once or launched directly.
    void enqueue() {
        char* D = (char*)dev.p;
        VQ_CUDA(cudaMemsetAsync(D + a_ticket, 0, 16, s));
        VQ_CUDA(cudaMemsetAsync((char*)out.p + o_aerr, 0, 8, s));
        for (const Item& it : items) {
            if (!it.join || it.cls == 2) continue;
            VQ_CUDA(cudaMemsetAsync(D + it.a_dmap, 0, (size_t)it.drange * 8, s));
            VQ_CUDA(cudaMemsetAsync((char*)out.p + it.o_jscal, 0, 32, s));
        }
        if (table_slots > 0) {
            int g = (int)std::min<long long>((table_slots + 255) / 256, (long long)sm_count() * 16);
            k_init_batch<<<g, 256, 0, s>>>((const VQTableDesc*)(D + a_tdesc), n_tdesc, table_slots);
            VQ_CUDA(cudaGetLastError());
            chk(s, "k_init_batch");
        }
        // the joins' builds: one persistent launch of build units, before
        // every probe (both classes below wait for it)
        if (ck[2].nunits > 0) {
            VQBatchArgs A{(const VQParams*)(D + a_bparams), (const VQUnit*)(D + ck[2].a_units), (unsigned*)(D + a_ticket) + 2,
                          (int)ck[2].nunits};
            jit_launch(ck[2].k, ck[2].grid, &A, sizeof A, s);
            chk(s, "vq_batch (join builds)");
        }
        VQ_CUDA(cudaEventRecord(ev[2], s));
        VQ_CUDA(cudaStreamWaitEvent(s2, ev[2], 0));
        if (ck[0].nunits > 0 || merge_entries > 0) {
            if (ck[0].nunits > 0) {
                VQBatchArgs A{(const VQParams*)(D + a_params), (const VQUnit*)(D + ck[0].a_units), (unsigned*)(D + a_ticket),
                              (int)ck[0].nunits};
                jit_launch(ck[0].k, ck[0].grid, &A, sizeof A, s2);
                chk(s2, "vq_batch (register path)");
            }
            if (merge_entries > 0) {
                k_merge_batch<<<(merge_entries + 7) / 8, 256, 0, s2>>>((const VQMergeDesc*)(D + a_mdesc), n_mdesc);
                VQ_CUDA(cudaGetLastError());
                chk(s2, "k_merge_batch");
            }
        }
        if (ck[1].nunits > 0) {
            VQBatchArgs A{(const VQParams*)(D + a_params), (const VQUnit*)(D + ck[1].a_units), (unsigned*)(D + a_ticket) + 1,
                          (int)ck[1].nunits};
            jit_launch(ck[1].k, ck[1].grid, &A, sizeof A, s);
            chk(s, "vq_batch (group tables)");
        }
        if (table_slots > 0) {
            int g = (int)std::min<long long>((table_slots + 255) / 256, (long long)sm_count() * 16);
            k_finalize_batch<<<g, 256, 0, s>>>((const VQTableDesc*)(D + a_tdesc), n_tdesc, table_slots);
            VQ_CUDA(cudaGetLastError());
            chk(s, "k_finalize_batch");
        }
        VQ_CUDA(cudaEventRecord(ev[3], s2));
        VQ_CUDA(cudaStreamWaitEvent(s, ev[3], 0));
    }

    void capture() {
        drop_graph();
        VQ_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        capturing = true;
        try {
            enqueue();
        } catch (...) {
            capturing = false;
            cudaGraph_t g = nullptr;
            cudaStreamEndCapture(s, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        capturing = false;
        VQ_CUDA(cudaStreamEndCapture(s, &graph));
        VQ_CUDA(cudaGraphInstantiate(&gexec, graph, 0));
    }

    // kernels done → copy every output back → done (events outside any graph)
    float finish_timing() {
        VQ_CUDA(cudaEventRecord(ev[4], s));
        VQ_CUDA(cudaMemcpyAsync(h_out.p, out.p, out_bytes, cudaMemcpyDeviceToHost, s));
        VQ_CUDA(cudaEventRecord(ev[1], s));
        VQ_CUDA(cudaStreamSynchronize(s));
        float ms = 0, km = 0;
        VQ_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        VQ_CUDA(cudaEventElapsedTime(&km, ev[0], ev[4]));
        kernel_ms = km;
        device_ms = ms;
        return ms;
    }

    float replay() {
        for (const Item& it : items) check_ranges(*it.p);
        if (!gexec) capture();
        VQ_CUDA(cudaEventRecord(ev[0], s));
        VQ_CUDA(cudaGraphLaunch(gexec, s));
        return finish_timing();
    }

    // One execution launched directly, for plan sets that run once.
    float run_direct() {
        for (const Item& it : items) check_ranges(*it.p);
        VQ_CUDA(cudaEventRecord(ev[0], s));
        enqueue();
        return finish_timing();
    }

    // Source of class c for its current block size (bodies are generated
    // per block size and cached per plan).
    void gen_class(int c) {
        ck[c].k_src.clear();
        ck[c].smem_extra = 0;
        ck[c].nbodies = 0;
        std::vector<Plan*> ps;
        for (int i : ck[c].items) ps.push_back(items[i].p);
        if (ps.empty()) return;
        std::vector<int> body_of;
        int smem = 0, nb = 0;
        ck[c].k_src = gen_batch_source(ps, ck[c].block, body_of, smem, nb, c == 2);
        ck[c].smem_extra = smem;
        ck[c].nbodies = nb;
        for (size_t j = 0; j < ps.size(); j++) (c == 2 ? items[ck[c].items[j]].bbody : items[ck[c].items[j]].body) = body_of[j];
    }

    // The batch's shape for the tuning cache: per class, the plans, distinct
    // bodies and chunks (log2), and the group-table slots (log2).
    std::string shape_key() const {
        std::ostringstream k;
        for (int c = 0; c < 2; c++) {
            long long chunks = 0, slots = 0;
            for (int i : ck[c].items) {
                chunks += items[i].nchunks;
                slots += items[i].nslots;
            }
            auto lg = [](long long v) { int l = 0; while (v > 1) { v >>= 1; l++; } return l; };
            k << (c ? "|t" : "r") << ck[c].items.size() << "b" << ck[c].nbodies << "c" << lg(chunks) << "s" << lg(slots);
        }
        return k.str();
    }

    // grid of each class at the current shared-memory size
    void size_grids() {
        for (int c = 0; c < 3; c++) {
            if (ck[c].items.empty()) continue;
            int smem = c == 1 ? table_smem() : ck[c].smem_extra;
            ck[c].k = jit_get(ck[c].k_src, "vq_batch", ck[c].block, smem);
            ck[c].grid = sm_count() * std::max(1, ck[c].k.max_blocks_per_sm);
        }
    }

    struct Tuning {
        int cache_kb, unit_div, block_regs, block_table;
    };
    Tuning tuning() const { return {cache_kb, unit_div, ck[0].block, ck[1].block}; }
    void apply(const Tuning& t) {
        cache_kb = t.cache_kb;
        unit_div = t.unit_div;
        for (int c = 0; c < 2; c++) {
            const int b = c ? t.block_table : t.block_regs;
            if (b != ck[c].block) {
                ck[c].block = b;
                gen_class(c);
            }
        }
        size_grids();
        for (int c = 0; c < 2; c++)
            if (!ck[c].items.empty() && ck[c].k.fn && ck[c].k.max_blocks_per_sm < 1)
                fail(VEXQ_ENOTSUP, "batch class kernel does not fit an SM at block " + std::to_string(ck[c].block));
        layout();
    }
    float time_replays() {
        replay();  // warm-up, graph capture
        float t = 1e30f;
        for (int r = 0; r < 3; r++) t = std::min(t, replay());
        return t;
    }

    // Times graph replays over cache sizes (0 = every group in the global
    // table) and unit sizes, then over block shapes at the best of those,
    // and keeps the fastest. The choice is kept in a JSON file beside the
    // kernel cache, keyed by the batch's shape, so a batch of the same shape
    // takes it without timing (flags & VEXQ_BATCH_RETUNE times again).
    void autotune(bool retune) {
        const std::string key = shape_key();
        Tuning t;
        if (!retune && tuning_cache_get(key, t)) {
            apply(t);
            explain += " autotuned(cached " + key + ")";
            return;
        }
        std::vector<Tuning> cands;
        std::vector<int> caches = ck[1].items.empty() ? std::vector<int>{cache_kb} : std::vector<int>{0, 48, 96, 160};
        const Tuning base = tuning();
        for (int c : caches)
            for (int u : {2, 4, 8}) cands.push_back({c, u, base.block_regs, base.block_table});
        Tuning best = base;
        float best_ms = 1e30f;
        int tried = 0;
        for (const Tuning& c : cands) {
            apply(c);
            const float ms = time_replays();
            tried++;
            if (ms < best_ms) { best_ms = ms; best = c; }
        }
        // block shapes at the best cache and unit sizes
        std::vector<Tuning> shapes;
        for (int br : {128, 256})
            for (int bt : {128, 256, 512}) {
                if (ck[0].items.empty() && br != base.block_regs) continue;
                if (ck[1].items.empty() && bt != base.block_table) continue;
                if (br == best.block_regs && bt == best.block_table) continue;
                shapes.push_back({best.cache_kb, best.unit_div, br, bt});
            }
        for (const Tuning& c : shapes) {
            float ms;
            try {
                apply(c);
                ms = time_replays();
            } catch (const Status&) {
                continue;  // a shape the kernels cannot launch (registers or shared memory)
            }
            tried++;
            if (ms < best_ms) { best_ms = ms; best = c; }
        }
        apply(best);
        tuning_cache_put(key, best, best_ms);
        explain += " autotuned(" + std::to_string(tried) + " candidates, best " + std::to_string(best_ms) + " ms, block " +
                   std::to_string(best.block_regs) + "/" + std::to_string(best.block_table) + ")";
    }

    // ---- the tuning cache: <kernel cache dir>/batch_tuning.json, one entry a
    // line: "key": {"cache_kb": C, "unit_div": U, "block_regs": R, "block_table": T, "ms": M}
    static std::mutex& tuning_mu() {
        static std::mutex m;
        return m;
    }
    static std::string tuning_path() { return jit_cache_dir() + "/batch_tuning.json"; }
    static bool tuning_cache_get(const std::string& key, Tuning& t) {
        std::lock_guard<std::mutex> lk(tuning_mu());
        std::ifstream f(tuning_path());
        std::string line;
        const std::string want = "\"" + key + "\":";
        while (std::getline(f, line)) {
            if (line.find(want) == std::string::npos) continue;
            auto num = [&](const char* name, int& v) {
                const size_t at = line.find(std::string("\"") + name + "\":");
                if (at == std::string::npos) return false;
                v = std::atoi(line.c_str() + at + std::strlen(name) + 3);
                return true;
            };
            return num("cache_kb", t.cache_kb) && num("unit_div", t.unit_div) && num("block_regs", t.block_regs) &&
                   num("block_table", t.block_table) && t.unit_div > 0 &&
                   (t.block_regs == 128 || t.block_regs == 256) &&
                   (t.block_table == 128 || t.block_table == 256 || t.block_table == 512);
        }
        return false;
    }
    static void tuning_cache_put(const std::string& key, const Tuning& t, float ms) {
        std::lock_guard<std::mutex> lk(tuning_mu());
        std::vector<std::string> keep;
        {
            std::ifstream f(tuning_path());
            std::string line;
            const std::string want = "\"" + key + "\":";
            while (std::getline(f, line))
                if (line.size() > 2 && line[0] == ' ' && line.find(want) == std::string::npos) {
                    if (line.back() == ',') line.pop_back();
                    keep.push_back(line);
                }
        }
        std::ostringstream e;
        e << "  \"" << key << "\": {\"cache_kb\": " << t.cache_kb << ", \"unit_div\": " << t.unit_div
          << ", \"block_regs\": " << t.block_regs << ", \"block_table\": " << t.block_table << ", \"ms\": " << ms << "}";
        keep.push_back(e.str());
        const std::string tmp = tuning_path() + ".tmp" + std::to_string(getpid());
        {
            std::ofstream f(tmp);
            f << "{\n";
            for (size_t i = 0; i < keep.size(); i++) f << keep[i] << (i + 1 < keep.size() ? ",\n" : "\n");
            f << "}\n";
        }
        std::rename(tmp.c_str(), tuning_path().c_str());
    }
};

// (Re)builds a batch over a plan set: ranges, classes, generated source,
// grids and layout. Device buffers only grow, so a reused batch allocates
// nothing once it has seen its largest plan set.
// A join joins the batch when its build can be direct-mapped (the build key
// column's range at most a few times its rows, keys not seen repeating): its
// build runs as units of the build class and its probe as units of the
// register or group-table class. Other joins run on their own afterwards.
static bool setup_join(Plan& p, Item& it) {
    if (p.radix_bits > 0 || !p.dmap_on || p.dmap_failed || p.staged) return false;
    // GROUP BY the join key with a LIMIT over more than 2^20 build rows: the
    // plain run keeps its device top-k (a batch copies every group back)
    if (p.join_gid && p.order.limit >= 0 && p.bt->nrows > (1 << 20)) return false;
    Table& bt = *p.bt;
    const Column& bkc = bt.cols[p.build_key];
    if (!bkc.has_range || bkc.imax < bkc.imin) return false;
    const __int128 r = (__int128)bkc.imax - (__int128)bkc.imin + 1;
    if (r > ((__int128)1 << 31) || r > 4 * (__int128)std::max<int64_t>(bt.nrows, 1) + 65536) return false;
    std::vector<uint8_t> bm = prune_mask(p, bt, p.zn_bpred, 0, bt.n_rg);
    ScanSegs bs = make_segments(bt, bm, 0, bt.n_rg, 128);
    if (bs.nchunks == 0) return false;  // an empty build emits nothing: the plain run says so
    it.join = true;
    it.gid = p.join_gid;
    it.dmin = bkc.imin;
    it.drange = (unsigned long long)r;
    it.bseg = bs.seg;
    it.bnchunks = bs.nchunks;
    it.brows = bs.rows;
    it.bytes += scanned_bytes(p, bt, bs.rows, true);
    return true;
}

void build_batch(Batch* b, vexq_plan_s* const* handles, int n) {
    b->drop_graph();
    b->handles.assign(handles, handles + n);
    b->items.clear();
    b->bytes = b->rows = 0;
    b->njoins = 0;
    for (int c = 0; c < 3; c++) {
        b->ck[c].items.clear();
        b->ck[c].k_src.clear();
        b->ck[c].nunits = 0;
        b->ck[c].nbodies = 0;
        b->ck[c].smem_extra = 0;
    }
    for (int i = 0; i < n; i++) {
        Item it;
        Plan* p = handles[i]->p;
        it.p = p;
        // COUNT(DISTINCT) and joins without a direct-mapped build run on their own after the graph
        if (p->ndist > 0 || (p->is_join && !setup_join(*p, it))) {
            it.join = false;
            b->items.push_back(std::move(it));
            continue;
        }
        if (it.join) it.bix = b->njoins++;
        Table& t = *p->t;
        std::vector<uint8_t> m = prune_mask(*p, t, p->zn_pred, 0, t.n_rg);
        ScanSegs ss = make_segments(t, m, 0, t.n_rg, 128);
        it.seg = ss.seg;
        it.nchunks = ss.nchunks;
        it.rows = ss.rows;
        it.bytes += scanned_bytes(*p, t, ss.rows, false);
        it.nf = p->nf;
        it.ni = p->ni;
        it.nfb = std::max(p->nf, 1);
        if (p->path == AggPath::Regs) {
            it.cls = 0;
            it.G = (int)p->domain;
        } else {
            it.cls = 1;
            it.hash = p->path == AggPath::Hash && !it.gid;
            if (it.gid) {
                it.cap = std::max<long long>(it.brows, 1);  // group numbers never exceed the build rows
            } else if (it.hash) {
                long long est = estimate_groups(*p, ss.rows, it.join ? it.brows : 0), cap = 16;
                while (cap < 2 * std::max<long long>(est, 8)) cap <<= 1;
                it.cap = cap;
            } else {
                it.cap = p->domain;
            }
            it.nslots = it.cap + 1;
            it.cap_out = it.nslots;
        }
        b->bytes += it.bytes;
        b->rows += it.rows;
        b->items.push_back(std::move(it));
    }
    b->ck[0].block = kBlockRegs;
    b->ck[1].block = kBlockTable;
    b->ck[2].block = 256;
    for (int c = 0; c < 2; c++)
        for (size_t i = 0; i < b->items.size(); i++)
            if (b->items[i].cls == c) b->ck[c].items.push_back((int)i);
    for (size_t i = 0; i < b->items.size(); i++)
        if (b->items[i].join && b->items[i].cls != 2) b->ck[2].items.push_back((int)i);
    for (int c = 0; c < 3; c++) b->gen_class(c);
    b->size_grids();
    b->layout();
}

Batch* new_batch() {
    std::unique_ptr<Batch> b(new Batch);
    VQ_CUDA(cudaStreamCreateWithFlags(&b->s, cudaStreamNonBlocking));
    VQ_CUDA(cudaStreamCreateWithFlags(&b->s2, cudaStreamNonBlocking));
    for (auto& e : b->ev) VQ_CUDA(cudaEventCreate(&e));
    return b.release();
}

Batch* create_batch(vexq_plan_s* const* handles, int n, uint32_t flags) {
    std::unique_ptr<Batch> b(new_batch());
    build_batch(b.get(), handles, n);
    if (flags & (VEXQ_BATCH_AUTOTUNE | VEXQ_BATCH_RETUNE)) b->autotune((flags & VEXQ_BATCH_RETUNE) != 0);
    return b.release();
}

// Results of the last execution, one per plan in plan order; plans that did
// not run in the batch (joins, hash-table overflow) run on their own here.
static void collect(Batch& b, vexq_result_s** out) {
    const size_t n = b.items.size();
    for (size_t i = 0; i < n; i++) out[i] = nullptr;
    const char* H = (const char*)b.h_out.p;
    std::vector<char> plain(n, 0);
    std::vector<std::string> errs(n);
    std::vector<int32_t> codes(n, 0);
    std::atomic<size_t> next{0};
    // the register class shares one error word: any flag sends its plans to plain runs
    const int rerr = *(const int*)(H + b.o_aerr);
    auto work = [&]() {
        for (size_t i = next++; i < n; i = next++) {
            Item& it = b.items[i];
            if (it.cls == 2) { plain[i] = 1; continue; }
            if (it.cls == 0 && rerr) { plain[i] = 1; continue; }
            if (it.join) {
                // the build's outcome: a repeated or out-of-range key (the hash
                // build from then on), no key, or uneven counts: a plain run
                const unsigned long long nk = *(const unsigned long long*)(H + it.o_jscal);
                const int berr = *(const int*)(H + it.o_jscal + 8);
                const unsigned long long ntot = *(const unsigned long long*)(H + it.o_jscal + 16);
                if (berr & (16 | 32)) it.p->dmap_failed = true;
                if (berr || nk == 0 || nk != ntot) { plain[i] = 1; continue; }
                if (it.cls == 1 && (*(const int*)(H + it.o_err) & 256)) { plain[i] = 1; continue; }
            }
            try {
                Plan& p = *it.p;
                Groups g;
                g.ival.assign(it.ni, {});
                g.fval.assign(it.nf, {});
                if (it.cls == 0) {
                    const double* hf = (const double*)(H + it.o_out_f);
                    const long long* hi = (const long long*)(H + it.o_out_i);
                    for (int gi = 0; gi < it.G; gi++) {
                        const long long* row = hi + (size_t)gi * (it.ni + 1);
                        if (row[p.slot_pos[0]] == 0) continue;
                        g.key.push_back((uint64_t)gi);
                        g.first.push_back(row[it.ni]);
                        for (int s = 0; s < it.ni; s++) g.ival[s].push_back(row[s]);
                        for (int s = 0; s < it.nf; s++) g.fval[s].push_back(hf[(size_t)gi * it.nf + s]);
                    }
                } else {
                    const int err = *(const int*)(H + it.o_err);
                    if (err & 1) { plain[i] = 1; continue; }  // hash table overflow: rerun with growth
                    if (err & 2) fail(VEXQ_ENOTSUP, "float sum exceeded its exact accumulation window");
                    const unsigned long long nout = *(const unsigned long long*)(H + it.o_nout);
                    const long long m = (long long)std::min<unsigned long long>(nout, (unsigned long long)it.cap_out);
                    const unsigned long long* ok = (const unsigned long long*)(H + it.o_key);
                    const long long* of = (const long long*)(H + it.o_first);
                    const long long* oi = (const long long*)(H + it.o_i);
                    const double* odf = (const double*)(H + it.o_f);
                    g.key.assign(ok, ok + m);
                    g.first.assign(of, of + m);
                    for (int s = 0; s < it.ni; s++) g.ival[s].assign(oi + (size_t)s * it.cap_out, oi + (size_t)s * it.cap_out + m);
                    for (int s = 0; s < it.nf; s++) g.fval[s].assign(odf + (size_t)s * it.cap_out, odf + (size_t)s * it.cap_out + m);
                }
                if (it.cls == 1) note_hot_groups(p, g);
                vexq_result_s* r = build_result(p, g);
                r->kernel_ms = b.kernel_ms;
                r->scan_ms = b.kernel_ms;
                r->launches = 0;
                r->rows_scanned = it.rows + it.brows;
                r->bytes_scanned = it.bytes;
                out[i] = r;
            } catch (const Status& e) {
                codes[i] = e.code;
                errs[i] = e.what();
            } catch (const std::exception& e) {
                codes[i] = VEXQ_EINVAL;
                errs[i] = e.what();
            }
        }
    };
    // host threads only pay off when there are many groups to order
    size_t groups = 0;
    for (const Item& it : b.items) groups += it.cls == 1 ? (size_t)it.cap_out : (size_t)it.G;
    const int nt = groups < 200000 ? 1
                   : (int)std::max<size_t>(1, std::min<size_t>({n, (size_t)16, (size_t)std::max(1u, std::thread::hardware_concurrency())}));
    std::vector<std::thread> th;
    for (int t = 1; t < nt; t++) th.emplace_back(work);
    work();
    for (auto& t : th) t.join();
    auto release = [&]() {
        for (size_t i = 0; i < n; i++) {
            delete out[i];
            out[i] = nullptr;
        }
    };
    for (size_t i = 0; i < n; i++)
        if (codes[i]) { release(); fail(codes[i], errs[i]); }
    try {
        for (size_t i = 0; i < n; i++)
            if (plain[i]) {
                std::lock_guard<std::mutex> lk(plan_mutex(b.items[i].p));
                out[i] = run_plan(*b.items[i].p, 0, -1);
            }
    } catch (...) {
        release();
        throw;
    }
}

void exec_batch(Batch& b, vexq_result_s** out) {
    b.replay();
    collect(b, out);
}

void run_batch_direct(Batch& b, vexq_plan_s* const* handles, int n, vexq_result_s** out) {
    build_batch(&b, handles, n);
    b.run_direct();
    collect(b, out);
}

double batch_kernel_ms(const Batch& b) { return b.kernel_ms; }

void destroy_batch(Batch* b) { delete b; }

}  // namespace vq

using namespace vq;

struct vexq_batch_s {
    Batch* b;
};

namespace {
template <class F>
int32_t guard_b(F&& f) {
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
}  // namespace

extern "C" {

int32_t vexq_batch_create(vexq_plan_t* plans, int32_t n, uint32_t flags, vexq_batch_t* out) {
    return guard_b([&]() -> int32_t {
        if (!out || n < 0 || (n > 0 && !plans)) fail(VEXQ_EINVAL, "null argument");
        for (int i = 0; i < n; i++)
            if (!plans[i]) fail(VEXQ_EINVAL, "null plan in batch");
        *out = new vexq_batch_s{create_batch(plans, n, flags)};
        return VEXQ_OK;
    });
}

int32_t vexq_batch_exec(vexq_batch_t b, vexq_result_t* out_results) {
    return guard_b([&]() -> int32_t {
        if (!b || (!b->b->items.empty() && !out_results)) fail(VEXQ_EINVAL, "null argument");
        exec_batch(*b->b, out_results);
        return VEXQ_OK;
    });
}

int32_t vexq_batch_stats(vexq_batch_t b, double* device_ms, double* kernel_ms, int64_t* bytes_scanned,
                         int64_t* rows_scanned) {
    return guard_b([&]() -> int32_t {
        if (!b) fail(VEXQ_EINVAL, "null argument");
        if (device_ms) *device_ms = b->b->device_ms;
        if (kernel_ms) *kernel_ms = b->b->kernel_ms;
        if (bytes_scanned) *bytes_scanned = b->b->bytes;
        if (rows_scanned) *rows_scanned = b->b->rows;
        return VEXQ_OK;
    });
}

const char* vexq_batch_explain(vexq_batch_t b) { return b ? b->b->explain.c_str() : ""; }

int32_t vexq_batch_destroy(vexq_batch_t b) {
    if (b) {
        delete b->b;
        delete b;
    }
    return VEXQ_OK;
}

}  // extern "C"
