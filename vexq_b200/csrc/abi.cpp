// abi.cpp — the extern "C" entry points of include/vexq_cuda.h. Every entry
// point converts exceptions into a status code plus a thread-local message.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <thread>

#include "plan.h"

namespace vq {
Table* upload_table(const vexq_column_desc* cols, int32_t ncols, int64_t nrows, int32_t rg_rows,
                    const int8_t* has_null = nullptr);
void destroy_table(Table* t);
const std::string& last_error();
vexq_result_s* run_plan(Plan& p, int rg_start, int rg_end);
vexq_result_s* run_plan_host(Plan& p, const vexq_column_desc* cols, int32_t ncols);
int32_t result_next(vexq_result_s* r, vexq_batch_view* out);
std::vector<uint8_t> prune_mask(const Plan& p, const Table& t, int root, int rgs, int rge);
cudaStream_t plan_stream(Plan& p);
}  // namespace vq

using namespace vq;

namespace {

template <class F>
int32_t guard(F&& f) {
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

int64_t plan_footprint(const Plan& p) {
    // group table slots × (key + first + int bank + fixed-point digits + flags)
    // (a join grouping by its key numbers the build's distinct keys: at most
    // one slot per build row)
    int64_t slots = p.join_gid ? std::max<int64_t>(p.bt->nrows, 16) + 1
                  : p.path == AggPath::Hash ? 2 * std::max<int64_t>(p.t->nrows, 16)
                  : p.path == AggPath::Dense ? p.domain : 64;
    int64_t per = 16 + 8 * p.ni + 36 * p.nf;
    int64_t f = slots * per;
    if (p.is_join) f += (int64_t)p.bt->nrows * 2 * 24;
    // COUNT(DISTINCT) sets: 20 bytes a slot, twice the table's rows
    if (p.ndist > 0 && p.t) f += (int64_t)p.ndist * 2 * std::max<int64_t>(p.t->nrows, 512) * 20;
    return f;
}

}  // namespace

extern "C" {

int32_t vexq_abi_version(void) { return VEXQ_ABI_VERSION; }

const char* vexq_last_error(void) { return last_error().c_str(); }

int32_t vexq_init(int32_t device, uint32_t flags) {
    (void)flags;
    return guard([&]() -> int32_t {
        int n = 0;
        VQ_CUDA(cudaGetDeviceCount(&n));
        if (device < 0 || device >= n) fail(VEXQ_EINVAL, "device index out of range");
        VQ_CUDA(cudaSetDevice(device));
        VQ_CUDA(cudaFree(nullptr));
        return VEXQ_OK;
    });
}

int32_t vexq_table_upload(const vexq_column_desc* cols, int32_t ncols, int64_t nrows, int32_t rg_rows, vexq_table_t* out) {
    return guard([&]() -> int32_t {
        if (!out) fail(VEXQ_EINVAL, "null output handle");
        Table* t = upload_table(cols, ncols, nrows, rg_rows);
        *out = new vexq_table_s{t};
        return VEXQ_OK;
    });
}

int32_t vexq_table_destroy(vexq_table_t t) {
    return guard([&]() -> int32_t {
        if (!t) return VEXQ_OK;
        drop_host_mirror(t->t);
        destroy_table(t->t);
        delete t;
        return VEXQ_OK;
    });
}

int32_t vexq_table_num_row_groups(vexq_table_t t, int32_t* out) {
    if (!t || !out) return VEXQ_EINVAL;
    *out = t->t->n_rg;
    return VEXQ_OK;
}

int32_t vexq_table_device_bytes(vexq_table_t t, int64_t* out) {
    if (!t || !out) return VEXQ_EINVAL;
    *out = t->t->device_bytes();
    return VEXQ_OK;
}

int32_t vexq_table_zone_map(vexq_table_t t, int32_t col, int32_t rg, vexq_zone_map* out) {
    return guard([&]() -> int32_t {
        if (!t || !out || col < 0 || col >= (int)t->t->cols.size() || rg < 0 || rg >= t->t->n_rg)
            fail(VEXQ_EINVAL, "zone map index out of range");
        *out = t->t->cols[col].zones[rg];
        return VEXQ_OK;
    });
}

int32_t vexq_table_dict_size(vexq_table_t t, int32_t col, int32_t* out) {
    return guard([&]() -> int32_t {
        if (!t || !out || col < 0 || col >= (int)t->t->cols.size()) fail(VEXQ_EINVAL, "column out of range");
        *out = (int32_t)t->t->cols[col].dict.keys.size();
        return VEXQ_OK;
    });
}

int32_t vexq_table_dict_entry(vexq_table_t t, int32_t col, int32_t code, const char** out, int32_t* len) {
    return guard([&]() -> int32_t {
        if (!t || !out || !len || col < 0 || col >= (int)t->t->cols.size()) fail(VEXQ_EINVAL, "column out of range");
        const auto& d = t->t->cols[col].dict;
        if (code < 0 || code >= (int)d.keys.size()) fail(VEXQ_EINVAL, "dictionary code out of range");
        *out = d.keys[code].data();
        *len = (int32_t)d.keys[code].size();
        return VEXQ_OK;
    });
}

int32_t vexq_agg_plan_create(vexq_table_t t, const vexq_agg_plan_desc* d, vexq_plan_t* out) {
    return guard([&]() -> int32_t {
        if (!t || !d || !out) fail(VEXQ_EINVAL, "null argument");
        Plan* p = compile_agg(t->t, d);
        *out = new vexq_plan_s{p, t, plan_footprint(*p)};
        return VEXQ_OK;
    });
}

int32_t vexq_join_plan_create(vexq_table_t build, vexq_table_t probe, const vexq_join_plan_desc* d, vexq_plan_t* out) {
    return guard([&]() -> int32_t {
        if (!build || !probe || !d || !out) fail(VEXQ_EINVAL, "null argument");
        Plan* p = compile_join(build->t, probe->t, d);
        *out = new vexq_plan_s{p, probe, plan_footprint(*p)};
        return VEXQ_OK;
    });
}

int32_t vexq_plan_destroy(vexq_plan_t p) {
    return guard([&]() -> int32_t {
        if (!p) return VEXQ_OK;
        settle_pending(*p->p);  // a submitted run's result stays readable without its plan
        // a submitted run freed unread may still be writing the plan's pinned
        // staging buffer: its end event is waited for before the buffer goes
        if (p->p->ev[3]) (void)cudaEventSynchronize(p->p->ev[3]);
        delete p->p;
        delete p;
        return VEXQ_OK;
    });
}

const char* vexq_plan_explain(vexq_plan_t p) { return p ? p->p->explain.c_str() : ""; }

int32_t vexq_plan_set_having(vexq_plan_t p, const vexq_expr* nodes, int32_t nnodes, const int32_t* children,
                             int32_t nchildren, int32_t predicate, int32_t visible) {
    return guard([&]() -> int32_t {
        if (!p) fail(VEXQ_EINVAL, "null plan");
        std::lock_guard<std::mutex> lk(plan_mutex(p->p));
        settle_pending(*p->p);  // a submitted run settles under the HAVING it ran with
        set_having(*p->p, nodes, nnodes, children, nchildren, predicate, visible);
        return VEXQ_OK;
    });
}

int32_t vexq_zone_prune(vexq_plan_t p, uint8_t* out_mask, int32_t n_rg) {
    return guard([&]() -> int32_t {
        if (!p || !out_mask) fail(VEXQ_EINVAL, "null argument");
        const Table& t = *p->p->t;
        std::vector<uint8_t> m = prune_mask(*p->p, t, p->p->zn_pred, 0, t.n_rg);
        for (int i = 0; i < n_rg && i < t.n_rg; i++) out_mask[i] = m[i];
        return VEXQ_OK;
    });
}

int32_t vexq_plan_run(vexq_plan_t p, int32_t rg_start, int32_t rg_end, vexq_result_t* out) {
    return guard([&]() -> int32_t {
        if (!p || !out) fail(VEXQ_EINVAL, "null argument");
        *out = run_plan(*p->p, rg_start, rg_end);
        return VEXQ_OK;
    });
}

int32_t vexq_plan_submit(vexq_plan_t p, int32_t rg_start, int32_t rg_end, vexq_result_t* out) {
    return guard([&]() -> int32_t {
        if (!p || !out) fail(VEXQ_EINVAL, "null argument");
        *out = run_plan_submit(*p->p, rg_start, rg_end);
        return VEXQ_OK;
    });
}

int32_t vexq_plan_run_host(vexq_plan_t p, const vexq_column_desc* cols, int32_t ncols, vexq_result_t* out) {
    return guard([&]() -> int32_t {
        if (!p || !out || !cols) fail(VEXQ_EINVAL, "null argument");
        *out = run_plan_host(*p->p, cols, ncols);
        return VEXQ_OK;
    });
}

// Every read of a result settles a submitted run first (vq::settle): it waits
// for the run's kernels and returns the run's status.
int32_t vexq_result_num_rows(vexq_result_t r, int64_t* out) {
    return guard([&]() -> int32_t {
        if (!r || !out) return VEXQ_EINVAL;
        settle(r);
        *out = r->nrows;
        return VEXQ_OK;
    });
}

int32_t vexq_result_num_cols(vexq_result_t r, int32_t* out) {
    return guard([&]() -> int32_t {
        if (!r || !out) return VEXQ_EINVAL;
        settle(r);
        *out = (int32_t)r->cols.size();
        return VEXQ_OK;
    });
}

int32_t vexq_result_next(vexq_result_t r, vexq_batch_view* out) {
    return guard([&]() -> int32_t {
        if (!r || !out) fail(VEXQ_EINVAL, "null argument");
        settle(r);
        return result_next(r, out);
    });
}

int32_t vexq_result_free(vexq_result_t r) {
    // a submitted run freed unread: its plan stops waiting for it (the kernels
    // finish on the stream before the plan's next run reuses the buffers)
    if (r && r->owner && r->owner->pending == r) r->owner->pending = nullptr;
    delete r;
    return VEXQ_OK;
}

int32_t vexq_result_stats(vexq_result_t r, double* kernel_ms, int32_t* launches, int64_t* rows_scanned,
                          int64_t* bytes_scanned) {
    return guard([&]() -> int32_t {
        if (!r) return VEXQ_EINVAL;
        settle(r);
        if (kernel_ms) *kernel_ms = r->kernel_ms;
        if (launches) *launches = r->launches;
        if (rows_scanned) *rows_scanned = r->rows_scanned;
        if (bytes_scanned) *bytes_scanned = r->bytes_scanned;
        return VEXQ_OK;
    });
}

int32_t vexq_result_scan_ms(vexq_result_t r, double* out) {
    return guard([&]() -> int32_t {
        if (!r || !out) return VEXQ_EINVAL;
        settle(r);
        *out = r->scan_ms;
        return VEXQ_OK;
    });
}

int32_t vexq_result_info(vexq_result_t r, vexq_result_summary* out) {
    return guard([&]() -> int32_t {
        if (!r || !out) return VEXQ_EINVAL;
        settle(r);
        out->nrows = r->nrows;
        out->ncols = (int32_t)r->cols.size();
        out->launches = r->launches;
        out->kernel_ms = r->kernel_ms;
        out->scan_ms = r->scan_ms;
        out->rows_scanned = r->rows_scanned;
        out->bytes_scanned = r->bytes_scanned;
        return VEXQ_OK;
    });
}

int32_t vexq_plan_set_stream(vexq_plan_t p, void* stream) {
    return guard([&]() -> int32_t {
        if (!p) return VEXQ_EINVAL;
        // runs on the old stream finish first: a later run on the new stream
        // reuses the plan's buffers
        settle_pending(*p->p);
        if (p->p->ev[3]) (void)cudaEventSynchronize(p->p->ev[3]);
        p->p->ext_stream = (cudaStream_t)stream;
        return VEXQ_OK;
    });
}

int32_t vexq_filter_run(vexq_table_t t, const vexq_expr* nodes, int32_t nnodes, const int32_t* children, int32_t nchildren,
                        int32_t predicate, int64_t row_start, int64_t row_end, uint8_t* out_bits, int64_t* count) {
    return guard([&]() -> int32_t {
        if (!t || !nodes || !out_bits || !count) fail(VEXQ_EINVAL, "null argument");
        Table& tb = *t->t;
        if (row_end < 0 || row_end > tb.nrows) row_end = tb.nrows;
        if (row_start < 0 || row_start > row_end) fail(VEXQ_EINVAL, "row range out of bounds");
        std::unique_ptr<Plan> p(compile_filter(&tb, nodes, nnodes, children, nchildren, predicate));
        // one segment [row_start, row_end)
        std::vector<long long> seg;
        long long chunks = 0;
        const long long U = p->tile;
        if (row_end > row_start) {
            seg = {row_start, row_end, 0};
            chunks = (row_end - (row_start & ~(U - 1)) + U - 1) / U;
        }
        size_t words = (size_t)(tb.nrows + kPadRows) / 32 + 8;
        DevBuf bits(words * 4), dseg(24), scal(32);
        VQParams P;
        std::memset(&P, 0, sizeof P);
        for (size_t c = 0; c < tb.cols.size(); c++) {
            P.col[c] = tb.cols[c].values.p;
            P.valid[c] = tb.cols[c].nullable ? tb.cols[c].validity.as<unsigned char>() : nullptr;
        }
        for (size_t i = 0, off = 0; i < p->sets.size(); i++) { P.sets[i] = p->d_sets.as<unsigned>() + off; off += p->sets[i].size(); }
        P.present = p->d_present.as<unsigned char>();
        P.rg_rows = tb.rg_rows;
        P.n_rg = tb.n_rg;
        P.acc_i = bits.as<long long>();
        P.ngroups = scal.as<unsigned long long>();
        P.error = (int*)(scal.as<char>() + 16);
        P.seg = dseg.as<long long>();
        P.nseg = seg.empty() ? 0 : 1;
        P.nchunks = chunks;
        cudaStream_t s = plan_stream(*p);
        VQ_CUDA(cudaMemsetAsync(bits.p, 0, bits.n, s));
        VQ_CUDA(cudaMemsetAsync(scal.p, 0, 32, s));
        if (!seg.empty()) VQ_CUDA(cudaMemcpyAsync(dseg.p, seg.data(), 24, cudaMemcpyHostToDevice, s));
        if (chunks > 0) {
            int per_sm = std::max(1, p->k_main.max_blocks_per_sm);
            long long want = p->staged ? chunks : (chunks + 7) / 8;
            int grid = (int)std::max<long long>(1, std::min<long long>((long long)sm_count() * per_sm, want));
            jit_launch(p->k_main, grid, &P, sizeof P, s);
        }
        std::vector<uint32_t> h(words);
        unsigned long long sc[4] = {0, 0, 0, 0};
        VQ_CUDA(cudaMemcpyAsync(h.data(), bits.p, words * 4, cudaMemcpyDeviceToHost, s));
        VQ_CUDA(cudaMemcpyAsync(sc, scal.p, 32, cudaMemcpyDeviceToHost, s));
        VQ_CUDA(cudaStreamSynchronize(s));
        unsigned long long cnt = sc[0];
        if ((int)(sc[2] & 0xFFFFFFFF) & 8) fail(VEXQ_ETIMEDOUT, "a staged tile copy did not complete within the kernel's wait limit");
        // the device words are LSB-first, so byte k of the (little-endian)
        // word array holds rows 8k..8k+7: shift bytes by row_start's bit offset
        int64_t n = row_end - row_start;
        const uint8_t* hb = (const uint8_t*)h.data();
        const int64_t b0 = row_start >> 3, nb = (n + 7) / 8;
        const int sh = (int)(row_start & 7);
        for (int64_t i = 0; i < nb; i++) {
            unsigned v = (unsigned)hb[b0 + i] >> sh;
            if (sh) v |= (unsigned)hb[b0 + i + 1] << (8 - sh);  // the word array has 8 words of padding
            out_bits[i] = (uint8_t)v;
        }
        if (n & 7) out_bits[nb - 1] &= (uint8_t)((1u << (n & 7)) - 1u);
        *count = (int64_t)cnt;
        return VEXQ_OK;
    });
}

int32_t vexq_selvec_from_bits(const uint8_t* bits, int64_t nrows, int64_t block, uint16_t* out_sel, int32_t* out_len) {
    if (!bits || !out_sel || !out_len || block < 0) return VEXQ_EINVAL;
    int64_t s = block * VEXQ_BLOCK_ROWS, e = std::min<int64_t>(nrows, s + VEXQ_BLOCK_ROWS);
    int32_t n = 0;
    for (int64_t r = s; r < e; r++)
        if ((bits[r >> 3] >> (r & 7)) & 1) out_sel[n++] = (uint16_t)(r - s);
    *out_len = n;
    return VEXQ_OK;
}

int32_t vexq_cancel(vexq_plan_t p) {
    if (!p) return VEXQ_EINVAL;
    p->p->cancel = true;
    return VEXQ_OK;
}

int32_t vexq_debug_fail_alloc(int32_t after) {
    if (after < -1) return VEXQ_EINVAL;
    vq::g_fail_alloc_after.store(after);
    return VEXQ_OK;
}

int32_t vexq_debug_live_device_bytes(int64_t* out) {
    if (!out) return VEXQ_EINVAL;
    *out = (int64_t)vq::g_live_device_bytes.load();
    return VEXQ_OK;
}

int32_t vexq_debug_join_spec(vexq_plan_t p, int64_t keys_seen) {
    return guard([&]() -> int32_t {
        if (!p || !p->p->is_join || keys_seen < 1) fail(VEXQ_EINVAL, "a join plan and a positive key count");
        vq::Plan& pl = *p->p;
        std::lock_guard<std::mutex> lk(vq::plan_mutex(&pl));
        vq::force_join_spec(pl, keys_seen);
        return VEXQ_OK;
    });
}

}  // extern "C"
