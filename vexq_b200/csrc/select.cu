// select.cu — Filter as a streaming operator, and Project materialised on the
// device.
//
// vexq_filter_open/next/close replace exec.NewFilter over a TableScan
// (exec/filter.go:40-78, exec/scan.go:199-236): the predicate runs once over
// every row group the zone maps keep (one launch, a selection bitmap), then
// every 1024-row block's selection vector is built on the device — per-block
// counts, an exclusive scan, and one warp a block writing its uint16 row
// indices in order — and all of them come back in one copy. next() hands out
// the blocks in row order with the scan's batch (the table's columns, read
// from a pinned host mirror of the HBM columns) and the block's SelVec,
// skipping blocks where no row survives, as Filter.Next does; the views stay
// valid until the next call.
//
// vexq_project_run replaces exec.NewProject over that filter
// (exec/project.go:64-128): the projected expressions are evaluated on the
// device for the kept rows only and written compacted in row order (what
// Project.materialize does with a SelVec), then served in 1024-row batches
// by vexq_result_next.
#include <algorithm>
#include <cstring>

#include "plan.h"

namespace vq {
cudaStream_t plan_stream(Plan& p);

namespace {

// 32 bits of the bitmap starting at row r (r need not be a multiple of 32; the
// word array carries padding words past the last row)
__device__ __forceinline__ unsigned bits_at(const unsigned* w, long long r) {
    const long long i = r >> 5;
    const int s = (int)(r & 31);
    return s ? (w[i] >> s) | (w[i + 1] << (32 - s)) : w[i];
}

__device__ __forceinline__ unsigned lane_bits(const unsigned* w, long long row0, int len, int lane) {
    const int lo = lane * 32;
    if (lo >= len) return 0u;
    const unsigned b = bits_at(w, row0 + lo);
    const int n = len - lo;
    return n >= 32 ? b : b & ((1u << n) - 1u);
}

// Kept rows of each block (one warp a block).
__global__ void k_block_count(const unsigned* words, const long long* row0, const int* len, int nb, long long* cnt) {
    const int warp = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= nb) return;
    int c = __popc(lane_bits(words, row0[warp], len[warp], lane));
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[warp] = c;
}

// Each block's SelVec at its offset: lane l writes the kept rows among the
// block's rows 32l..32l+31, after the kept rows of lanes below it.
__global__ void k_block_selvec(const unsigned* words, const long long* row0, const int* len, int nb, const long long* off,
                               unsigned short* sel) {
    const int warp = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (warp >= nb) return;
    unsigned b = lane_bits(words, row0[warp], len[warp], lane);
    const int c = __popc(b);
    int inc = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    unsigned short* out = sel + off[warp] + (inc - c);
    while (b) {
        const int i = __ffs(b) - 1;
        *out++ = (unsigned short)(lane * 32 + i);
        b &= b - 1u;
    }
}

// Kept rows of each 128-row chunk (four bitmap words).
__global__ void k_chunk_count(const unsigned* words, long long nck, long long* cnt) {
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < nck; c += (long long)gridDim.x * blockDim.x) {
        const uint4 w = reinterpret_cast<const uint4*>(words)[c];
        cnt[c] = __popc(w.x) + __popc(w.y) + __popc(w.z) + __popc(w.w);
    }
}

// Exclusive scan of n 64-bit counts in place, in three steps: each 1024-entry
// tile scanned by one block (tile totals out), the totals scanned by one
// block, the totals added back. out[n] receives the grand total.
__device__ __forceinline__ long long block_incl_scan(long long v, long long* sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) sh[warp] = v;
    __syncthreads();
    if (warp == 0) {
        long long s = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const long long t = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += t;
        }
        sh[lane] = s;
    }
    __syncthreads();
    const long long r = v + (warp ? sh[warp - 1] : 0);
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(1024) k_scan64_tiles(long long* a, long long n, long long* tiles) {
    __shared__ long long sh[32];
    const long long i = blockIdx.x * 1024LL + threadIdx.x;
    const long long v = i < n ? a[i] : 0;
    const long long inc = block_incl_scan(v, sh);
    if (i < n) a[i] = inc - v;
    if (threadIdx.x == 1023) tiles[blockIdx.x] = inc;
}

__global__ void __launch_bounds__(1024) k_scan64_totals(long long* tiles, long long nt, long long* total) {
    __shared__ long long sh[32];
    __shared__ long long last;
    long long carry = 0;  // sum of the earlier 1024-entry rounds
    for (long long b = 0; b < nt; b += 1024) {
        const long long i = b + threadIdx.x;
        const long long v = i < nt ? tiles[i] : 0;
        const long long inc = block_incl_scan(v, sh);
        if (i < nt) tiles[i] = carry + inc - v;
        if (threadIdx.x == 1023) last = inc;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
    if (threadIdx.x == 0) *total = carry;
}

__global__ void k_scan64_add(long long* a, long long n, const long long* tiles) {
    const long long i = blockIdx.x * 1024LL + threadIdx.x;
    if (i < n) a[i] += tiles[blockIdx.x];
}

// Exclusive scan of a[0..n) in place (a needs no padding); *total (device)
// gets the sum. tiles: ceil(n / 1024) entries of scratch.
void scan64(long long* a, long long n, long long* tiles, long long* total, cudaStream_t s) {
    const long long nt = std::max<long long>(1, (n + 1023) / 1024);
    k_scan64_tiles<<<(unsigned)nt, 1024, 0, s>>>(a, n, tiles);
    launch_check(s, "k_scan64_tiles");
    k_scan64_totals<<<1, 1024, 0, s>>>(tiles, nt, total);
    launch_check(s, "k_scan64_totals");
    k_scan64_add<<<(unsigned)nt, 1024, 0, s>>>(a, n, tiles);
    launch_check(s, "k_scan64_add");
    VQ_CUDA(cudaGetLastError());
}

int type_width(int t) { return (t == VEXQ_TYPE_INT64 || t == VEXQ_TYPE_FLOAT64) ? 8 : t == VEXQ_TYPE_BOOL ? 1 : 4; }

// The table's columns in pinned host memory, copied from HBM (the columns'
// authoritative copy) on first use and again after the table is re-filled.
struct HostMirror {
    std::vector<std::unique_ptr<PinnedBuf>> vals, valid;
    uint64_t version = ~0ull;
};
std::mutex g_mirror_mu;
std::map<const Table*, std::unique_ptr<HostMirror>> g_mirrors;

}  // namespace

void drop_host_mirror(const Table* t) {
    std::lock_guard<std::mutex> lk(g_mirror_mu);
    g_mirrors.erase(t);
}

namespace {

HostMirror& host_mirror(Table& t, cudaStream_t s) {
    std::lock_guard<std::mutex> lk(g_mirror_mu);
    auto& m = g_mirrors[&t];
    if (!m) m.reset(new HostMirror);
    if (m->version == t.zone_version) return *m;
    m->vals.clear();
    m->valid.clear();
    for (const Column& c : t.cols) {
        auto v = std::make_unique<PinnedBuf>();
        auto b = std::make_unique<PinnedBuf>();
        const size_t nb = (size_t)std::max<int64_t>(t.nrows, 1) * type_width(c.type);
        v->ensure(nb);
        if (t.nrows > 0) VQ_CUDA(cudaMemcpyAsync(v->p, c.values.p, (size_t)t.nrows * type_width(c.type), cudaMemcpyDeviceToHost, s));
        const size_t vb = (size_t)(t.nrows + 7) / 8 + 8;
        b->ensure(vb);
        if (c.nullable && t.nrows > 0) {
            VQ_CUDA(cudaMemcpyAsync(b->p, c.validity.p, (size_t)(t.nrows + 7) / 8, cudaMemcpyDeviceToHost, s));
        } else {
            std::memset(b->p, 0xFF, vb);
        }
        m->vals.push_back(std::move(v));
        m->valid.push_back(std::move(b));
    }
    VQ_CUDA(cudaStreamSynchronize(s));
    m->version = t.zone_version;
    return *m;
}

// Row ranges kept by the zone maps, as the scan's segment list.
ScanSegs kept_segments(const Plan& p, const Table& t, int rgs, int rge) {
    std::vector<uint8_t> m = p.zn_pred >= 0 ? prune_mask(p, t, p.zn_pred, rgs, rge) : std::vector<uint8_t>(t.n_rg, 0);
    if (p.zn_pred < 0)
        for (int rg = rgs; rg < rge; rg++) m[rg] = 1;
    return make_segments(t, m, rgs, rge, 128);
}

// Scan parameters of a select plan over its table.
VQParams select_params(Plan& p, const Table& t, const DevBuf& seg, const ScanSegs& ss) {
    VQParams P;
    std::memset(&P, 0, sizeof P);
    set_plan_constants(p, P);
    set_columns(P, t, false);
    P.seg = seg.as<long long>();
    P.nseg = (int)ss.seg.size() / 3;
    P.nchunks = ss.nchunks;
    P.rg_rows = t.rg_rows;
    P.n_rg = t.n_rg;
    P.present = p.d_present.as<unsigned char>();
    for (size_t i = 0, o = 0; i < p.sets.size(); i++) {
        P.sets[i] = p.d_sets.as<unsigned>() + o;
        o += p.sets[i].size();
    }
    return P;
}

void check_range_args(const Table& t, int& rgs, int& rge) {
    if (rge < 0 || rge > t.n_rg) rge = t.n_rg;
    if (rgs < 0 || rgs > rge) fail(VEXQ_EINVAL, "row-group range out of bounds");
}

}  // namespace
}  // namespace vq

using namespace vq;

struct vexq_filter_s {
    std::unique_ptr<Plan> plan;
    Table* t = nullptr;
    HostMirror* mirror = nullptr;
    std::vector<long long> row0;    // per block: first table row
    std::vector<int> len, rg;       // rows and row group
    std::vector<long long> cnt, off;
    PinnedBuf h_sel;                // every block's SelVec, compacted
    long long selected = 0;
    size_t next_block = 0;
    // views of the current batch
    std::vector<vexq_vector_view> views;
    std::vector<std::vector<uint8_t>> vbits;
    std::vector<std::vector<uint32_t>> doff;
    std::vector<std::string> dbytes;
    double kernel_ms = 0;
};

namespace {

template <class F>
int32_t guard_s(F&& f) {
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

float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    VQ_CUDA(cudaEventElapsedTime(&ms, a, b));
    return ms;
}

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    Events() {
        VQ_CUDA(cudaEventCreate(&a));
        VQ_CUDA(cudaEventCreate(&b));
    }
    ~Events() {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

// The bitmap of the kept rows of segments ss (vq_pmark); words is sized to
// (nrows + kPadRows) / 32 + 8 words and zeroed on stream s first.
void mark_rows(Plan& p, const Table& t, const ScanSegs& ss, DevBuf& words, DevBuf& seg, cudaStream_t s) {
    words.ensure(((size_t)(t.nrows + kPadRows) / 32 + 8) * 4);
    VQ_CUDA(cudaMemsetAsync(words.p, 0, words.n, s));
    seg.ensure(std::max<size_t>(ss.seg.size(), 3) * 8);
    h2d(seg.p, ss.seg.data(), ss.seg.size() * 8, s);
    if (ss.nchunks <= 0) return;
    VQParams P = select_params(p, t, seg, ss);
    P.acc_i = words.as<long long>();
    jit_launch(p.k_main, grid_for(p.k_main, ss.nchunks, false, 0), &P, sizeof P, s);
    launch_check(s, "vq_pmark");
}

}  // namespace

extern "C" {

int32_t vexq_filter_open(vexq_table_t table, const vexq_expr* nodes, int32_t nnodes, const int32_t* children,
                         int32_t nchildren, int32_t predicate, int32_t rg_start, int32_t rg_end, vexq_filter_t* out) {
    return guard_s([&]() -> int32_t {
        if (!table || !out || !nodes) fail(VEXQ_EINVAL, "null argument");
        *out = nullptr;
        Table& t = *table->t;
        int rgs = rg_start, rge = rg_end;
        check_range_args(t, rgs, rge);
        std::unique_ptr<vexq_filter_s> f(new vexq_filter_s);
        f->t = &t;
        f->plan.reset(compile_select(&t, nodes, nnodes, children, nchildren, predicate, nullptr, 0));
        Plan& p = *f->plan;
        cudaStream_t s = plan_stream(p);
        f->mirror = &host_mirror(t, s);
        const ScanSegs ss = kept_segments(p, t, rgs, rge);
        // 1024-row blocks of the kept row groups (a block never spans two)
        for (int rg = rgs; rg < rge; rg++) {
            bool kept = false;
            for (size_t i = 0; i + 2 < ss.seg.size(); i += 3)
                if (ss.seg[i] <= t.rg_start(rg) && t.rg_start(rg) < ss.seg[i + 1]) kept = true;
            if (!kept) continue;
            for (int64_t r = t.rg_start(rg); r < t.rg_end(rg); r += VEXQ_BLOCK_ROWS) {
                f->row0.push_back(r);
                f->len.push_back((int)std::min<int64_t>(VEXQ_BLOCK_ROWS, t.rg_end(rg) - r));
                f->rg.push_back(rg);
            }
        }
        const int nb = (int)f->row0.size();
        f->cnt.assign(nb, 0);
        f->off.assign(nb, 0);
        if (nb > 0) {
            Events e;
            DevBuf words, seg, d_row0(nb * 8), d_len(nb * 4), d_cnt((size_t)(nb + 1) * 8),
                d_tiles((size_t)((nb + 1023) / 1024 + 1) * 8), d_total(8), d_sel((size_t)t.nrows * 2 + 16);
            VQ_CUDA(cudaEventRecord(e.a, s));
            mark_rows(p, t, ss, words, seg, s);
            h2d(d_row0.p, f->row0.data(), nb * 8, s);
            h2d(d_len.p, f->len.data(), nb * 4, s);
            const int wb = 256, grid = (int)(((long long)nb * 32 + wb - 1) / wb);
            k_block_count<<<grid, wb, 0, s>>>(words.as<unsigned>(), d_row0.as<long long>(), d_len.as<int>(), nb,
                                              d_cnt.as<long long>());
            launch_check(s, "k_block_count");
            VQ_CUDA(cudaMemcpyAsync(f->cnt.data(), d_cnt.p, nb * 8, cudaMemcpyDeviceToHost, s));
            scan64(d_cnt.as<long long>(), nb, d_tiles.as<long long>(), d_total.as<long long>(), s);
            k_block_selvec<<<grid, wb, 0, s>>>(words.as<unsigned>(), d_row0.as<long long>(), d_len.as<int>(), nb,
                                               d_cnt.as<long long>(), d_sel.as<unsigned short>());
            launch_check(s, "k_block_selvec");
            VQ_CUDA(cudaGetLastError());
            VQ_CUDA(cudaMemcpyAsync(f->off.data(), d_cnt.p, nb * 8, cudaMemcpyDeviceToHost, s));
            VQ_CUDA(cudaMemcpyAsync(&f->selected, d_total.p, 8, cudaMemcpyDeviceToHost, s));
            VQ_CUDA(cudaStreamSynchronize(s));
            f->h_sel.ensure((size_t)std::max<long long>(f->selected, 1) * 2);
            if (f->selected > 0)
                VQ_CUDA(cudaMemcpyAsync(f->h_sel.p, d_sel.p, (size_t)f->selected * 2, cudaMemcpyDeviceToHost, s));
            VQ_CUDA(cudaEventRecord(e.b, s));
            VQ_CUDA(cudaStreamSynchronize(s));
            f->kernel_ms = ev_ms(e.a, e.b);
        }
        // each STRING column's global dictionary, flattened once for the views
        const size_t nc = t.cols.size();
        f->views.assign(nc, vexq_vector_view{});
        f->vbits.assign(nc, std::vector<uint8_t>(VEXQ_BLOCK_ROWS / 8 + 1, 0));
        f->doff.assign(nc, {});
        f->dbytes.assign(nc, {});
        for (size_t c = 0; c < nc; c++) {
            const Column& col = t.cols[c];
            vexq_vector_view& v = f->views[c];
            v.name = col.name.c_str();
            v.type = col.type;
            if (col.type == VEXQ_TYPE_STRING) {
                f->doff[c].push_back(0);
                for (const std::string& k : col.dict.keys) {
                    f->dbytes[c] += k;
                    f->doff[c].push_back((uint32_t)f->dbytes[c].size());
                }
                v.dict_str_off = f->doff[c].data();
                v.dict_bytes = f->dbytes[c].data();
                v.dict_len = (int32_t)col.dict.keys.size();
            }
        }
        *out = f.release();
        return VEXQ_OK;
    });
}

int32_t vexq_filter_next(vexq_filter_t f, vexq_filter_batch* out) {
    return guard_s([&]() -> int32_t {
        if (!f || !out) fail(VEXQ_EINVAL, "null argument");
        std::memset(out, 0, sizeof *out);
        while (f->next_block < f->row0.size() && f->cnt[f->next_block] == 0) f->next_block++;
        if (f->next_block >= f->row0.size()) return VEXQ_OK;  // EOF: length 0
        const size_t b = f->next_block++;
        const Table& t = *f->t;
        const long long r0 = f->row0[b];
        const int n = f->len[b];
        for (size_t c = 0; c < t.cols.size(); c++) {
            vexq_vector_view& v = f->views[c];
            v.values = (const char*)f->mirror->vals[c]->p + (size_t)r0 * type_width(t.cols[c].type);
            // the block's validity bits from bit 0 (the mirror's bitmap is
            // table-wide; a block need not start on a byte)
            const uint8_t* src = (const uint8_t*)f->mirror->valid[c]->p;
            std::vector<uint8_t>& dst = f->vbits[c];
            std::fill(dst.begin(), dst.end(), 0);
            const int sh = (int)(r0 & 7);
            const long long b0 = r0 >> 3;
            for (int i = 0; i < (n + 7) / 8; i++) {
                unsigned x = (unsigned)src[b0 + i] >> sh;
                if (sh) x |= (unsigned)src[b0 + i + 1] << (8 - sh);
                dst[i] = (uint8_t)x;
            }
            if (n & 7) dst[(n - 1) / 8] &= (uint8_t)((1u << (n & 7)) - 1u);
            v.validity = dst.data();
        }
        out->ncols = (int32_t)t.cols.size();
        out->length = (int32_t)f->cnt[b];
        out->physical = n;
        out->rg = f->rg[b];
        out->row0 = r0;
        out->sel = (const uint16_t*)f->h_sel.p + f->off[b];
        out->cols = f->views.data();
        return VEXQ_OK;
    });
}

int32_t vexq_filter_stats(vexq_filter_t f, int64_t* selected, int64_t* blocks, double* kernel_ms) {
    return guard_s([&]() -> int32_t {
        if (!f) fail(VEXQ_EINVAL, "null argument");
        if (selected) *selected = f->selected;
        if (blocks) *blocks = (int64_t)f->row0.size();
        if (kernel_ms) *kernel_ms = f->kernel_ms;
        return VEXQ_OK;
    });
}

int32_t vexq_filter_close(vexq_filter_t f) {
    delete f;
    return VEXQ_OK;
}

int32_t vexq_project_run(vexq_table_t table, const vexq_expr* nodes, int32_t nnodes, const int32_t* children,
                         int32_t nchildren, int32_t predicate, const int32_t* roots, const char* const* names,
                         int32_t nexprs, int32_t rg_start, int32_t rg_end, vexq_result_t* out) {
    return guard_s([&]() -> int32_t {
        if (!table || !out || !nodes || !roots || nexprs <= 0) fail(VEXQ_EINVAL, "null argument or no expressions");
        *out = nullptr;
        Table& t = *table->t;
        int rgs = rg_start, rge = rg_end;
        check_range_args(t, rgs, rge);
        std::unique_ptr<Plan> pp(compile_select(&t, nodes, nnodes, children, nchildren, predicate, roots, nexprs));
        Plan& p = *pp;
        cudaStream_t s = plan_stream(p);
        const ScanSegs ss = kept_segments(p, t, rgs, rge);
        std::unique_ptr<vexq_result_s> r(new vexq_result_s);
        r->cols.resize(nexprs);
        for (int j = 0; j < nexprs; j++) {
            const INode& n = p.ir[p.key_nodes[j]];
            OutColumn& oc = r->cols[j];
            oc.name = names && names[j] ? names[j] : ("col" + std::to_string(j));
            oc.type = n.type;
            if (n.type == VEXQ_TYPE_STRING) oc.dict = &t.cols[n.col].dict;
        }
        long long total = 0;
        Events e;
        VQ_CUDA(cudaEventRecord(e.a, s));
        int launches = 0;
        if (ss.nchunks > 0) {
            DevBuf words, seg;
            mark_rows(p, t, ss, words, seg, s);
            const long long nck = (t.nrows + 127) / 128 + 1;
            DevBuf d_off((size_t)(nck + 1) * 8), d_tiles((size_t)((nck + 1023) / 1024 + 1) * 8), d_total(8);
            const int cg = (int)std::min<long long>((nck + 255) / 256, (long long)sm_count() * 8);
            k_chunk_count<<<cg, 256, 0, s>>>(words.as<unsigned>(), nck, d_off.as<long long>());
            launch_check(s, "k_chunk_count");
            scan64(d_off.as<long long>(), nck, d_tiles.as<long long>(), d_total.as<long long>(), s);
            VQ_CUDA(cudaMemcpyAsync(&total, d_total.p, 8, cudaMemcpyDeviceToHost, s));
            VQ_CUDA(cudaStreamSynchronize(s));
            launches = 5;
            if (total > 0) {
                const int ng = (nexprs + 7) / 8;
                std::vector<DevBuf> dv, dm;
                for (int j = 0; j < std::min(nexprs, 8); j++) {
                    dv.emplace_back((size_t)total * 8);
                    dm.emplace_back((size_t)total);
                }
                for (auto& oc : r->cols) {
                    oc.v.resize(total);
                    oc.valid.resize(total);
                }
                VQParams P = select_params(p, t, seg, ss);
                P.acc_i = words.as<long long>();
                P.first = d_off.as<long long>();
                for (size_t j = 0; j < dv.size(); j++) {
                    P.qpay[j] = dv[j].as<unsigned long long>();
                    P.qpayv[j] = dm[j].as<unsigned char>();
                }
                for (int g = 0; g < ng; g++) {
                    P.mode = g;
                    jit_launch(p.k_build, grid_for(p.k_build, ss.nchunks, false, 0), &P, sizeof P, s);
                    launch_check(s, "vq_pwrite");
                    launches++;
                    for (int j = g * 8; j < std::min(nexprs, g * 8 + 8); j++) {
                        VQ_CUDA(cudaMemcpyAsync(r->cols[j].v.data(), dv[j % 8].p, (size_t)total * 8, cudaMemcpyDeviceToHost, s));
                        VQ_CUDA(cudaMemcpyAsync(r->cols[j].valid.data(), dm[j % 8].p, (size_t)total, cudaMemcpyDeviceToHost, s));
                    }
                    VQ_CUDA(cudaStreamSynchronize(s));
                }
            }
        }
        VQ_CUDA(cudaEventRecord(e.b, s));
        VQ_CUDA(cudaStreamSynchronize(s));
        r->nrows = total;
        own_dictionaries(r.get());
        r->kernel_ms = ev_ms(e.a, e.b);
        r->scan_ms = r->kernel_ms;
        r->launches = launches;
        r->rows_scanned = ss.rows;
        *out = r.release();
        return VEXQ_OK;
    });
}

}  // extern "C"
