// noalloc.cu — the one aggregate entry point that allocates no memory.
//
// vexq_plan_run_global_noalloc runs a prepared aggregate without GROUP BY
// (one output row: the filtered SUM(price*disc) scan, a global COUNT/AVG/...)
// through the same runtime-compiled register-path kernel and the same
// per-block-partial merge kernel as vexq_plan_run, but the partials, the row
// ranges, the merge outputs and the error flag live in one file-scope device
// array instead of per-plan device buffers, and results go to caller memory
// instead of a result handle.
//
// Who needs it: a serving loop that keeps many queries in flight on one GPU
// cannot let a query call cudaMalloc or cudaFree, because both synchronise the
// whole device and stall every other query; and a caller admitted under a
// fixed HBM budget must not grow the library's footprint on each call.
//
// Set-up: the first call on a device (with that device current) looks up the
// scratch array's device address with cudaGetSymbolAddress and makes sure the
// merge kernel's module is loaded; both can load code onto the device, so the
// first call on each device should come before any stream capture. Later calls
// make no allocation of device, pinned or managed memory.
//
// The scratch is one array per device shared by every call: calls that
// overlap in time (from two threads, or on two streams) race on it and
// corrupt each other's partials. Each call synchronises its stream before it
// returns, so calls made one after another from any threads are safe.
#include <cstring>
#include <mutex>

#include "internal.h"
#include "plan.h"

// Scratch for every no-allocation call on a device. Only the error flag must
// start at zero; every call clears it. Partials, ranges and merged values are
// written in full before they are read.
static __device__ __align__(256) unsigned char vq_noalloc_scratch[VEXQ_NOALLOC_SCRATCH_BYTES];

namespace vq {

// Per-block partial merge of the register path (run.cu).
__global__ void k_merge_regs(const double* part_f, const long long* part_i, int nblocks, int G, int nf, int ni,
                             const int* fkind, const int* ikind, double* out_f, long long* out_i);

namespace {

constexpr int kMaxDevices = 64;
constexpr int kMaxSegments = 512;      // row ranges after zone-map pruning, kept on the host stack
constexpr size_t kHostStage = 4096;    // host stack bytes for the combiner kinds and the merged values

std::mutex g_setup_mu;
unsigned char* g_scratch[kMaxDevices];

unsigned char* scratch_on(int dev) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch[dev]) {
        unsigned char* ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress((void**)&ptr, vq_noalloc_scratch);
        if (e != cudaSuccess) fail(VEXQ_EDEVICE, std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e));
        cudaFuncAttributes fa;
        e = cudaFuncGetAttributes(&fa, k_merge_regs);
        if (e != cudaSuccess) fail(VEXQ_EDEVICE, std::string("loading the partial-merge kernel: ") + cudaGetErrorString(e));
        g_scratch[dev] = ptr;
    }
    return g_scratch[dev];
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

void run_global_noalloc(Plan& p, int rg_start, int rg_end, cudaStream_t s, int64_t* out_values, uint8_t* out_valid,
                        int32_t n_out) {
    if (p.is_join) fail(VEXQ_ENOTSUP, "the no-allocation run takes aggregate plans over one table, not joins");
    if (p.having_root >= 0) fail(VEXQ_ENOTSUP, "the no-allocation run takes aggregates without HAVING");
    if (p.ndist > 0) fail(VEXQ_ENOTSUP, "the no-allocation run takes no COUNT(DISTINCT): its sets need device memory");
    for (const AggOut& a : p.outs)
        if (a.rank_dict) fail(VEXQ_ENOTSUP, "the no-allocation run takes no MIN/MAX over strings");
    check_ranges(p);
    if (!p.keys.empty() || p.path != AggPath::Regs || p.domain != 1)
        fail(VEXQ_ENOTSUP, "the no-allocation run takes aggregates without GROUP BY");
    if (n_out != (int32_t)p.outs.size())
        fail(VEXQ_EINVAL, "n_out is " + std::to_string(n_out) + " but the plan has " + std::to_string(p.outs.size()) +
                              " output columns");
    if (p.cancel.load()) { p.cancel = false; fail(VEXQ_ECANCELED, "plan cancelled"); }
    settle_pending(p);  // a submitted run of this plan finishes reading its staging buffer first
    Table& t = *p.t;
    int dev = -1;
    VQ_CUDA(cudaGetDevice(&dev));
    if (dev != t.device) fail(VEXQ_EINVAL, "the table's device must be current for a no-allocation run");
    if (dev < 0 || dev >= kMaxDevices) fail(VEXQ_EINVAL, "device ordinal out of range");
    unsigned char* base = scratch_on(dev);

    const int nf = p.nf, ni = p.ni, nfb = std::max(nf, 1);
    const size_t merged = (size_t)nfb * 8 + (size_t)(ni + 1) * 8;
    if (merged + 16 > kHostStage || (size_t)(nfb + ni + 1) * 4 > kHostStage)
        fail(VEXQ_EINVAL, "too many aggregate accumulators for a no-allocation run (at most 509)");

    // row ranges of the row groups the zone maps keep, as (start, end, first chunk)
    const int rge = rg_end < 0 ? t.n_rg : std::min(rg_end, t.n_rg);
    const int rgs = std::max(0, rg_start);
    long long seg[3 * kMaxSegments];
    int nseg = 0;
    const long long chunks = walk_segments(
        t, [&](int rg) { return zone_eval(p, p.zn_pred, t, rg); }, rgs, rge, p.tile,
        [&](long long a, long long b, long long c0) {
            if (nseg == kMaxSegments)
                fail(VEXQ_EINVAL, "more than 512 row ranges remain after zone-map pruning; the no-allocation run keeps at most 512");
            seg[3 * nseg] = a;
            seg[3 * nseg + 1] = b;
            seg[3 * nseg + 2] = c0;
            nseg++;
        });

    // grid as the plain path sizes it, shrunk while the partials do not fit
    const JitKernel& k = p.k_main;
    int grid = grid_for(k, chunks, p.staged, p.grid_per_sm);
    const size_t fixed = round256(merged + 16) + round256((size_t)(nfb + ni + 1) * 4) + round256((size_t)std::max(nseg, 1) * 24);
    const size_t per_block = (size_t)nfb * 8 + (size_t)(ni + 1) * 8;
    auto need = [&](int g) { return fixed + round256((size_t)g * nfb * 8) + round256((size_t)g * (ni + 1) * 8); };
    while (grid > sm_count() && need(grid) > VEXQ_NOALLOC_SCRATCH_BYTES) grid = std::max(sm_count(), grid / 2);
    if (need(grid) > VEXQ_NOALLOC_SCRATCH_BYTES)
        fail(VEXQ_EINVAL, "this aggregate needs " + std::to_string(need(grid)) + " bytes of scratch (" +
                              std::to_string(per_block) + " per block); the no-allocation run has " +
                              std::to_string((long long)VEXQ_NOALLOC_SCRATCH_BYTES));

    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += round256(bytes); return base + o; };
    unsigned char* d_out = take(merged + 16);  // merged values, then the error flag
    int* d_kinds = (int*)take((size_t)(nfb + ni + 1) * 4);
    long long* d_seg = (long long*)take((size_t)std::max(nseg, 1) * 24);
    double* part_f = (double*)take((size_t)grid * nfb * 8);
    long long* part_i = (long long*)take((size_t)grid * (ni + 1) * 8);
    double* out_f = (double*)d_out;
    long long* out_i = (long long*)(d_out + (size_t)nfb * 8);
    int* d_err = (int*)(d_out + merged);

    alignas(16) unsigned char stage[kHostStage];
    long long cnt = 0;
    const double* hf = (const double*)stage;
    const long long* hi = (const long long*)(stage + (size_t)nfb * 8);
    if (chunks > 0) {
        // combiner kind per bank entry (0 sum, 1 min, 2 max); the last int entry is the first-row key
        int* kinds = (int*)stage;
        std::memset(kinds, 0, (size_t)(nfb + ni + 1) * 4);
        for (size_t i = 0; i < p.slots.size(); i++) {
            int kd = p.slots[i].kind;
            int code = (kd == S_IMIN || kd == S_FMIN) ? 1 : (kd == S_IMAX || kd == S_FMAX) ? 2 : 0;
            kinds[p.slots[i].is_float() ? p.slot_pos[i] : nfb + p.slot_pos[i]] = code;
        }
        kinds[nfb + ni] = 1;
        // pageable sources: each copy has read its source when the call returns
        VQ_CUDA(cudaMemcpyAsync(d_kinds, kinds, (size_t)(nfb + ni + 1) * 4, cudaMemcpyHostToDevice, s));
        VQ_CUDA(cudaMemcpyAsync(d_seg, seg, (size_t)nseg * 24, cudaMemcpyHostToDevice, s));
        VQ_CUDA(cudaMemsetAsync(d_err, 0, 4, s));

        VQParams P;
        std::memset(&P, 0, sizeof P);
        set_plan_constants(p, P);
        for (size_t c = 0; c < t.cols.size(); c++) {
            P.col[c] = t.cols[c].values.p;
            P.valid[c] = t.cols[c].nullable ? t.cols[c].validity.as<unsigned char>() : nullptr;
        }
        P.seg = d_seg;
        P.nseg = nseg;
        P.nchunks = chunks;
        P.rg_rows = t.rg_rows;
        P.n_rg = t.n_rg;
        P.present = p.d_present.as<unsigned char>();
        for (size_t i = 0, o = 0; i < p.sets.size(); i++) { P.sets[i] = p.d_sets.as<unsigned>() + o; o += p.sets[i].size(); }
        P.part_f = part_f;
        P.part_i = part_i;
        P.error = d_err;
        jit_launch(k, grid, &P, sizeof P, s);
        k_merge_regs<<<(nf + ni + 1 + 7) / 8, 256, 0, s>>>(part_f, part_i, grid, 1, nf, ni, d_kinds, d_kinds + nfb, out_f, out_i);
        VQ_CUDA(cudaGetLastError());
        VQ_CUDA(cudaMemcpyAsync(stage, d_out, merged + 4, cudaMemcpyDeviceToHost, s));
        VQ_CUDA(cudaStreamSynchronize(s));
        check_regs_flags(*(const int*)(stage + merged));
        cnt = hi[p.slot_pos[0]];
    }

    // one output row with the aggregate NULL rules of the plain path
    for (int i = 0; i < n_out; i++) {
        const AggOut& a = p.outs[i];
        out_values[i] = 0;
        out_valid[i] = 0;
        if (cnt == 0) {  // no input rows: COUNT is 0, every other aggregate NULL
            if (a.kind == VEXQ_AGG_COUNT) out_valid[i] = 1;
            continue;
        }
        const long long nn = hi[p.slot_pos[a.nn_slot]];
        const int pos = p.slot_pos[a.value_slot];
        if (a.kind == VEXQ_AGG_COUNT) { out_valid[i] = 1; out_values[i] = hi[pos]; continue; }
        if (nn == 0) continue;
        out_valid[i] = 1;
        if (a.kind == VEXQ_AGG_AVG) {
            const double v = hf[pos] / (double)nn;
            std::memcpy(&out_values[i], &v, 8);
        } else if (p.slots[a.value_slot].is_float()) {
            std::memcpy(&out_values[i], &hf[pos], 8);
        } else {
            int64_t v = hi[pos];
            if (a.out_type == VEXQ_TYPE_DATE) v = (int64_t)(int32_t)v;
            if (a.out_type == VEXQ_TYPE_BOOL) v = v != 0;
            out_values[i] = v;
        }
    }
}

}  // namespace
}  // namespace vq

extern "C" int32_t vexq_plan_run_global_noalloc(vexq_plan_t plan, int32_t rg_start, int32_t rg_end, void* stream,
                                                int64_t* out_values, uint8_t* out_valid, int32_t n_out) {
    try {
        vq::set_error("");
        if (!plan || !out_values || !out_valid) vq::fail(VEXQ_EINVAL, "null argument");
        vq::run_global_noalloc(*plan->p, rg_start, rg_end, (cudaStream_t)stream, out_values, out_valid, n_out);
        return VEXQ_OK;
    } catch (const vq::Status& s) {
        vq::set_error(s.what());
        return s.code;
    } catch (const std::exception& e) {
        vq::set_error(e.what());
        return VEXQ_EINVAL;
    }
}
