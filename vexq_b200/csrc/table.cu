// table.cu — HBM-resident tables: column upload, per-row-group dictionary
// remap to one global dictionary per column (done once on the device, the
// remap exec/agg_intkey.go:118-134 performs per row group), and zone maps
// with the writer's rules (storage/writer.go:205-372).
#include <algorithm>
#include <cmath>
#include <cstring>

#include "internal.h"
#include "device_common.cuh"

namespace vq {

namespace {
thread_local std::string t_err;
int g_sm_count = 0;
}  // namespace

void set_error(const std::string& m) { t_err = m; }
const std::string& last_error() { return t_err; }
[[noreturn]] void fail(int32_t code, const std::string& msg) { throw Status(code, msg); }

// allocations left before an injected failure (-1: no injection)
std::atomic<int> g_fail_alloc_after{-1};
std::atomic<long long> g_live_device_bytes{0};

void DevBuf::alloc(size_t bytes) {
    n = bytes;
    if (bytes == 0) { p = nullptr; return; }
    int left = g_fail_alloc_after.load();
    while (left >= 0 && !g_fail_alloc_after.compare_exchange_weak(left, left - 1)) {}
    if (left == 0) {
        p = nullptr;
        n = 0;
        fail(VEXQ_ENOMEM, "cudaMalloc(" + std::to_string(bytes) + "): out of memory (injected)");
    }
    cudaError_t e = cudaMalloc(&p, bytes);
    if (e != cudaSuccess) {
        p = nullptr;
        n = 0;
        cudaGetLastError();
        fail(VEXQ_ENOMEM, "cudaMalloc(" + std::to_string(bytes) + "): " + cudaGetErrorString(e));
    }
    g_live_device_bytes += (long long)bytes;
}
void DevBuf::release() {
    if (p) {
        cudaFree(p);
        g_live_device_bytes -= (long long)n;
    }
    p = nullptr;
    n = 0;
}

PinnedBuf::~PinnedBuf() { if (p) cudaFreeHost(p); }
void PinnedBuf::ensure(size_t bytes) {
    if (bytes <= n) return;
    if (p) cudaFreeHost(p);
    p = nullptr;
    VQ_CUDA(cudaMallocHost(&p, bytes));
    n = bytes;
}

uint32_t GlobalDict::add(const std::string& s) {
    auto it = index.find(s);
    if (it != index.end()) return it->second;
    uint32_t c = (uint32_t)keys.size();
    index.emplace(s, c);
    keys.push_back(s);
    return c;
}

int sm_count() {
    if (!g_sm_count) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_sm_count, cudaDevAttrMultiProcessorCount, dev);
        if (g_sm_count <= 0) g_sm_count = 148;
    }
    return g_sm_count;
}

int64_t Table::device_bytes() const {
    int64_t b = 0;
    for (auto& c : cols) b += (int64_t)c.values.n + (int64_t)c.validity.n;
    return b;
}

static int type_width(int t) {
    switch (t) {
        case VEXQ_TYPE_INT64:
        case VEXQ_TYPE_FLOAT64: return 8;
        case VEXQ_TYPE_DATE:
        case VEXQ_TYPE_STRING: return 4;
        case VEXQ_TYPE_BOOL: return 1;
    }
    return 0;
}

// ---- kernels ------------------------------------------------------------------------

// local per-row-group dictionary code → global code; NULL rows read code 0.
__global__ void k_remap(unsigned* codes, const unsigned char* valid, long long nrows, long long rg_rows,
                        const unsigned* remap, const unsigned* rg_off, const unsigned* rg_len, int* err) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nrows; i += (long long)gridDim.x * blockDim.x) {
        bool ok = valid ? vq_bit(valid, i) : true;
        unsigned c = 0;
        if (ok) {
            const int rg = (int)(i / rg_rows);
            const unsigned l = codes[i];
            if (l < rg_len[rg]) c = remap[rg_off[rg] + l];
            else atomicOr(err, 1);
        }
        codes[i] = c;
    }
}

// Per (row group, column) min / max / null count / sum. A row group is split
// into slices, one block each, so every SM works on the upload (one block per
// row group left most of the GPU idle); the slices' partials are then combined
// in slice order by one thread per row group, so the float sum does not depend
// on scheduling.
struct ZoneAcc {
    long long nulls;
    long long isum;
    double fsum;
    long long imin, imax;
    double fmin, fmax;
    int has;
};

__device__ __forceinline__ void zone_comb(ZoneAcc& a, const ZoneAcc& b) {
    a.nulls += b.nulls;
    a.isum = (long long)((unsigned long long)a.isum + (unsigned long long)b.isum);
    a.imin = min(a.imin, b.imin);
    a.imax = max(a.imax, b.imax);
    a.fsum += b.fsum;
    a.fmin = fmin(a.fmin, b.fmin);
    a.fmax = fmax(a.fmax, b.fmax);
    a.has |= b.has;
}

__device__ __forceinline__ ZoneAcc zone_shfl(const ZoneAcc& a, int o) {
    ZoneAcc b;
    b.nulls = __shfl_down_sync(0xffffffffu, a.nulls, o);
    b.isum = __shfl_down_sync(0xffffffffu, a.isum, o);
    b.fsum = __shfl_down_sync(0xffffffffu, a.fsum, o);
    b.imin = __shfl_down_sync(0xffffffffu, a.imin, o);
    b.imax = __shfl_down_sync(0xffffffffu, a.imax, o);
    b.fmin = __shfl_down_sync(0xffffffffu, a.fmin, o);
    b.fmax = __shfl_down_sync(0xffffffffu, a.fmax, o);
    b.has = __shfl_down_sync(0xffffffffu, a.has, o);
    return b;
}

// Fixed-order block reduction (warp shuffle tree, then warps in order).
__device__ void zone_block_reduce(ZoneAcc a, ZoneAcc* out) {
    for (int o = 16; o > 0; o >>= 1) {
        ZoneAcc b = zone_shfl(a, o);
        zone_comb(a, b);
    }
    __shared__ ZoneAcc w[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) w[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        ZoneAcc z = w[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) zone_comb(z, w[k]);
        *out = z;
    }
}

template <class T>
__device__ void zone_part(const T* v, const unsigned char* valid, long long s, long long e, int type, ZoneAcc* out) {
    ZoneAcc a{0, 0, 0.0, 0x7FFFFFFFFFFFFFFFLL, (-0x7FFFFFFFFFFFFFFFLL - 1), 0.0, 0.0, 0};
    double fmn = __longlong_as_double(0x7FF0000000000000LL), fmx = -fmn;
    for (long long r = s + threadIdx.x; r < e; r += blockDim.x) {
        if (valid && !vq_bit(valid, r)) { a.nulls++; continue; }
        a.has = 1;
        if (type == VEXQ_TYPE_FLOAT64) {
            double d = (double)v[r];
            a.fsum += d;
            if (d < fmn) fmn = d;  // NaN never replaces a bound
            if (d > fmx) fmx = d;
        } else if (type != VEXQ_TYPE_STRING && type != VEXQ_TYPE_BOOL) {
            long long x = (long long)v[r];
            a.isum = (long long)((unsigned long long)a.isum + (unsigned long long)x);
            a.imin = min(a.imin, x);
            a.imax = max(a.imax, x);
        }
    }
    a.fmin = fmn;
    a.fmax = fmx;
    zone_block_reduce(a, out);
}

// Block (row group, slice): the slice's partial into part[rg * gridDim.y + slice].
__global__ void k_zones_part(const void* values, const unsigned char* valid, int type, long long nrows, long long rg_rows,
                             ZoneAcc* part) {
    const int rg = blockIdx.x, sl = blockIdx.y, ns = gridDim.y;
    const long long s = (long long)rg * rg_rows, e = min(nrows, s + rg_rows);
    const long long len = (e - s + ns - 1) / ns;
    const long long a = min(e, s + (long long)sl * len), b = min(e, a + len);
    ZoneAcc* out = part + (long long)rg * ns + sl;
    switch (type) {
        case VEXQ_TYPE_INT64: zone_part((const long long*)values, valid, a, b, type, out); break;
        case VEXQ_TYPE_FLOAT64: zone_part((const double*)values, valid, a, b, type, out); break;
        case VEXQ_TYPE_DATE: zone_part((const int*)values, valid, a, b, type, out); break;
        default: zone_part((const unsigned char*)values, valid, a, b, type, out); break;  // STRING / BOOL: null count
    }
}

// One warp per (column, row group): lane l folds slices l, l+32 in order, a
// fixed shuffle tree combines the lanes → the zone map, with the writer's
// rules for each type. All columns in one launch.
__global__ void k_zones_fin(const ZoneAcc* part, int ns, int n_rg, int ncols, const int* types, vexq_zone_map* out) {
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= (long long)n_rg * ncols) return;  // whole warps leave together
    const int c = (int)(w / n_rg), rg = (int)(w % n_rg), type = types[c];
    const ZoneAcc* pp = part + ((long long)c * n_rg + rg) * ns;
    ZoneAcc a{0, 0, 0.0, 0x7FFFFFFFFFFFFFFFLL, (-0x7FFFFFFFFFFFFFFFLL - 1), __longlong_as_double(0x7FF0000000000000LL),
              -__longlong_as_double(0x7FF0000000000000LL), 0};
    for (int k = lane; k < ns; k += 32) zone_comb(a, pp[k]);
    for (int o = 16; o > 0; o >>= 1) {
        ZoneAcc b = zone_shfl(a, o);
        zone_comb(a, b);
    }
    if (lane != 0) return;
    vexq_zone_map z{};
    z.null_count = a.nulls;
    if (type == VEXQ_TYPE_STRING || type == VEXQ_TYPE_BOOL) {  // null count only
        out[w] = z;
        return;
    }
    z.has_min_max = a.has;
    if (type == VEXQ_TYPE_FLOAT64) {
        z.sum = __double_as_longlong(a.fsum);
        if (z.has_min_max) {
            z.min = (unsigned long long)__double_as_longlong(a.fmin);
            z.max = (unsigned long long)__double_as_longlong(a.fmax);
        }
    } else if (type == VEXQ_TYPE_DATE) {  // zero-extended raw bits (writer.go:319)
        if (z.has_min_max) {
            z.min = (unsigned long long)(unsigned)(int)a.imin;
            z.max = (unsigned long long)(unsigned)(int)a.imax;
        }
    } else {
        z.sum = a.isum;
        if (z.has_min_max) { z.min = (unsigned long long)a.imin; z.max = (unsigned long long)a.imax; }
    }
    out[w] = z;
}

// ---- upload -------------------------------------------------------------------------

static bool any_null(const uint8_t* bm, int64_t nrows) {
    if (!bm) return false;
    int64_t full = nrows / 8;
    for (int64_t i = 0; i < full; i++) if (bm[i] != 0xFF) return true;
    for (int64_t r = full * 8; r < nrows; r++) if (!((bm[r >> 3] >> (r & 7)) & 1)) return true;
    return false;
}

static int64_t padded_rows(int64_t nrows) { return ((nrows + kPadRows - 1) / kPadRows + 1) * kPadRows; }

struct DictDev {
    DevBuf remap, off, len;
};
static std::map<const Column*, std::unique_ptr<DictDev>> g_dictdev;
static std::mutex g_dictdev_mu;

// Copies one column's host values (and bitmap) into its device buffers and
// remaps string codes. Used by upload and by the host-buffer run path.
void fill_column(Table& t, int ci, const vexq_column_desc& d, cudaStream_t s, DevBuf& err) {
    Column& c = t.cols[ci];
    int w = type_width(c.type);
    if (t.nrows > 0) VQ_CUDA(cudaMemcpyAsync(c.values.p, d.values, (size_t)w * t.nrows, cudaMemcpyDefault, s));
    if (c.nullable && t.nrows > 0) VQ_CUDA(cudaMemcpyAsync(c.validity.p, d.validity, (size_t)(t.nrows + 7) / 8, cudaMemcpyDefault, s));
    if (c.type == VEXQ_TYPE_STRING && c.per_rg_dicts && t.nrows > 0) {
        DictDev* dd;
        {
            std::lock_guard<std::mutex> lk(g_dictdev_mu);
            dd = g_dictdev[&c].get();
        }
        int grid = std::min<int64_t>((t.nrows + 255) / 256, 4L * sm_count() * 8);
        k_remap<<<grid, 256, 0, s>>>(c.values.as<unsigned>(), c.nullable ? c.validity.as<unsigned char>() : nullptr, t.nrows,
                                     t.rg_rows, dd->remap.as<unsigned>(), dd->off.as<unsigned>(), dd->len.as<unsigned>(),
                                     err.as<int>());
        VQ_CUDA(cudaGetLastError());
    }
}

void compute_zones(Table& t, cudaStream_t s) {
    t.zone_version++;
    if (t.n_rg == 0) return;
    DevBuf z(sizeof(vexq_zone_map) * t.n_rg * t.cols.size());
    // slices per row group: about eight blocks per SM over the table, each at
    // least 8,192 rows
    int ns = (int)std::max<long long>(1, std::min<long long>((long long)sm_count() * 8 / t.n_rg, ((long long)t.rg_rows + 8191) / 8192));
    ns = std::min(ns, 64);
    const int ncols = (int)t.cols.size();
    DevBuf part(sizeof(ZoneAcc) * (size_t)t.n_rg * ns * ncols + 4 * (size_t)ncols + 16);
    int* d_types = (int*)(part.as<char>() + sizeof(ZoneAcc) * (size_t)t.n_rg * ns * ncols);
    std::vector<int> types(ncols);
    for (int ci = 0; ci < ncols; ci++) {
        Column& c = t.cols[ci];
        types[ci] = c.type;
        k_zones_part<<<dim3(t.n_rg, ns), 256, 0, s>>>(c.values.p, c.nullable ? c.validity.as<unsigned char>() : nullptr, c.type,
                                                     t.nrows, t.rg_rows, part.as<ZoneAcc>() + (size_t)ci * t.n_rg * ns);
        VQ_CUDA(cudaGetLastError());
    }
    if (ncols > 0) {
        VQ_CUDA(cudaMemcpyAsync(d_types, types.data(), 4 * (size_t)ncols, cudaMemcpyHostToDevice, s));
        const long long warps = (long long)t.n_rg * ncols;
        k_zones_fin<<<(unsigned)((warps + 7) / 8), 256, 0, s>>>(part.as<ZoneAcc>(), ns, t.n_rg, ncols, d_types,
                                                               z.as<vexq_zone_map>());
        VQ_CUDA(cudaGetLastError());
    }
    std::vector<vexq_zone_map> h(t.n_rg * t.cols.size());
    VQ_CUDA(cudaMemcpyAsync(h.data(), z.p, z.n, cudaMemcpyDeviceToHost, s));
    VQ_CUDA(cudaStreamSynchronize(s));
    for (size_t ci = 0; ci < t.cols.size(); ci++) {
        Column& c = t.cols[ci];
        c.zones.assign(h.begin() + ci * t.n_rg, h.begin() + (ci + 1) * t.n_rg);
        if (c.type == VEXQ_TYPE_STRING) {  // writeStringBlocks: Min 0, Max dict size - 1 (writer.go:363-367)
            for (int rg = 0; rg < t.n_rg; rg++) {
                size_t n = c.per_rg_dicts ? 0 : c.dict.keys.size();
                if (c.per_rg_dicts) for (auto v : c.rg_present[rg]) n += v;
                c.zones[rg].has_min_max = n > 0;
                c.zones[rg].min = 0;
                c.zones[rg].max = n > 0 ? n - 1 : 0;
            }
        }
        // table-wide range for dense keys and exact-sum windows
        const bool had = c.has_range, was_finite = c.finite;
        const double ofmin = c.fmin, ofmax = c.fmax;
        const int64_t oimin = c.imin, oimax = c.imax;
        c.has_range = false;
        c.finite = true;
        for (int rg = 0; rg < t.n_rg; rg++) {
            const vexq_zone_map& zm = c.zones[rg];
            if (!zm.has_min_max || c.type == VEXQ_TYPE_STRING || c.type == VEXQ_TYPE_BOOL) continue;
            if (c.type == VEXQ_TYPE_FLOAT64) {
                double mn, mx;
                std::memcpy(&mn, &zm.min, 8);
                std::memcpy(&mx, &zm.max, 8);
                if (!c.has_range) { c.fmin = mn; c.fmax = mx; }
                else { c.fmin = std::min(c.fmin, mn); c.fmax = std::max(c.fmax, mx); }
                double zs;  // the zone sum is NaN/±inf when the row group holds NaN or ±inf
                std::memcpy(&zs, &zm.sum, 8);
                if (!std::isfinite(zs)) c.finite = false;
            } else {
                int64_t mn = c.type == VEXQ_TYPE_DATE ? (int64_t)(int32_t)(uint32_t)zm.min : (int64_t)zm.min;
                int64_t mx = c.type == VEXQ_TYPE_DATE ? (int64_t)(int32_t)(uint32_t)zm.max : (int64_t)zm.max;
                if (!c.has_range) { c.imin = mn; c.imax = mx; }
                else { c.imin = std::min(c.imin, mn); c.imax = std::max(c.imax, mx); }
            }
            c.has_range = true;
        }
        if (t.zones_ready) {
            bool wider = (was_finite && !c.finite);
            if (had && c.has_range)
                wider = wider || (c.type == VEXQ_TYPE_FLOAT64 ? (c.fmin < ofmin || c.fmax > ofmax)
                                                             : (c.imin < oimin || c.imax > oimax));
            if (wider) t.range_epoch++;
        }
    }
    t.zones_ready = true;
}

// has_null (optional, one flag per column) says which columns hold a NULL
// when the caller already knows; the values and bitmaps may then be device
// pointers (the copies infer their direction), as the .vxq loader hands over
// columns it decoded on the device. STRING columns with a table-wide
// dictionary are checked on the host and must be host buffers.
Table* upload_table(const vexq_column_desc* cols, int32_t ncols, int64_t nrows, int32_t rg_rows, const int8_t* has_null) {
    if (ncols < 0 || ncols > VQ_MAXCOLS) fail(VEXQ_EINVAL, "column count out of range (max 32)");
    if (nrows < 0 || nrows >= (int64_t(1) << 40)) fail(VEXQ_EINVAL, "row count out of range");
    if (ncols > 0 && !cols) fail(VEXQ_EINVAL, "null column array");
    std::unique_ptr<Table> t(new Table);
    cudaGetDevice(&t->device);
    t->nrows = nrows;
    t->rg_rows = rg_rows > 0 ? rg_rows : VEXQ_ROW_GROUP_ROWS;
    t->n_rg = (int32_t)((nrows + t->rg_rows - 1) / t->rg_rows);
    t->cols.resize(ncols);
    int64_t prow = padded_rows(nrows);
    cudaStream_t s;
    VQ_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct SG { cudaStream_t s; ~SG() { cudaStreamDestroy(s); } } sg{s};
    DevBuf err(sizeof(int));
    VQ_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    for (int ci = 0; ci < ncols; ci++) {
        const vexq_column_desc& d = cols[ci];
        Column& c = t->cols[ci];
        c.name = d.name ? d.name : "";
        c.type = d.type;
        int w = type_width(c.type);
        if (!w) fail(VEXQ_EINVAL, "column " + c.name + ": unknown type " + std::to_string(d.type));
        if (nrows > 0 && !d.values) fail(VEXQ_EINVAL, "column " + c.name + ": null values");
        c.nullable = has_null ? (has_null[ci] != 0 && d.validity != nullptr) : any_null(d.validity, nrows);
        c.values.alloc((size_t)w * prow);
        VQ_CUDA(cudaMemsetAsync(c.values.p, 0, c.values.n, s));
        if (c.nullable) {
            c.validity.alloc((size_t)prow / 8);
            VQ_CUDA(cudaMemsetAsync(c.validity.p, 0, c.validity.n, s));
        }
        if (c.type == VEXQ_TYPE_STRING) {
            if (!d.dict_str_off || !d.dict_bytes) fail(VEXQ_EINVAL, "column " + c.name + ": string column without dictionary");
            c.per_rg_dicts = d.dict_rg_first != nullptr;
            if (!c.per_rg_dicts) {
                for (int64_t e = 0; e < d.dict_entries; e++)
                    c.dict.add(std::string(d.dict_bytes + d.dict_str_off[e], d.dict_str_off[e + 1] - d.dict_str_off[e]));
                // validate codes on the host (cheap relative to the upload)
                const uint32_t* v = (const uint32_t*)d.values;
                for (int64_t r = 0; r < nrows; r++) {
                    bool ok = !c.nullable || ((d.validity[r >> 3] >> (r & 7)) & 1);
                    if (ok && v[r] >= c.dict.keys.size()) fail(VEXQ_EINVAL, "column " + c.name + ": dictionary code out of range");
                }
            } else {
                // getOrBuildRemap (agg_intkey.go:120-134), once per row group at upload
                std::vector<uint32_t> remap, off(t->n_rg), len(t->n_rg);
                c.rg_present.resize(t->n_rg);
                for (int rg = 0; rg < t->n_rg; rg++) {
                    uint32_t a = d.dict_rg_first[rg], b = d.dict_rg_first[rg + 1];
                    off[rg] = (uint32_t)remap.size();
                    len[rg] = b - a;
                    for (uint32_t e = a; e < b; e++)
                        remap.push_back(c.dict.add(std::string(d.dict_bytes + d.dict_str_off[e], d.dict_str_off[e + 1] - d.dict_str_off[e])));
                }
                for (int rg = 0; rg < t->n_rg; rg++) {
                    c.rg_present[rg].assign(c.dict.keys.size(), 0);
                    for (uint32_t k = 0; k < len[rg]; k++) c.rg_present[rg][remap[off[rg] + k]] = 1;
                }
                auto dd = std::make_unique<DictDev>();
                dd->remap.alloc(std::max<size_t>(remap.size(), 1) * 4);
                dd->off.alloc(std::max<size_t>(off.size(), 1) * 4);
                dd->len.alloc(std::max<size_t>(len.size(), 1) * 4);
                if (!remap.empty()) VQ_CUDA(cudaMemcpyAsync(dd->remap.p, remap.data(), remap.size() * 4, cudaMemcpyHostToDevice, s));
                if (!off.empty()) {
                    VQ_CUDA(cudaMemcpyAsync(dd->off.p, off.data(), off.size() * 4, cudaMemcpyHostToDevice, s));
                    VQ_CUDA(cudaMemcpyAsync(dd->len.p, len.data(), len.size() * 4, cudaMemcpyHostToDevice, s));
                }
                VQ_CUDA(cudaStreamSynchronize(s));  // host vectors go out of scope
                std::lock_guard<std::mutex> lk(g_dictdev_mu);
                g_dictdev[&c] = std::move(dd);
            }
        }
        fill_column(*t, ci, d, s, err);
    }
    int herr = 0;
    VQ_CUDA(cudaMemcpyAsync(&herr, err.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    VQ_CUDA(cudaStreamSynchronize(s));
    if (herr) fail(VEXQ_EINVAL, "dictionary code out of range for its row group's dictionary");
    compute_zones(*t, s);
    return t.release();
}

void destroy_table(Table* t) {
    if (!t) return;
    std::lock_guard<std::mutex> lk(g_dictdev_mu);
    for (auto& c : t->cols) g_dictdev.erase(&c);
    delete t;
}

// Re-fills every column from host buffers (end-to-end form): same schema and
// dictionaries as at upload; zone maps are recomputed on the device.
void refill_table(Table& t, const vexq_column_desc* cols, int32_t ncols, cudaStream_t s) {
    if (ncols != (int)t.cols.size()) fail(VEXQ_EINVAL, "column count differs from the uploaded table");
    DevBuf err(sizeof(int));
    VQ_CUDA(cudaMemsetAsync(err.p, 0, sizeof(int), s));
    for (int ci = 0; ci < ncols; ci++) {
        if (cols[ci].type != t.cols[ci].type) fail(VEXQ_EINVAL, "column type differs from the uploaded table");
        if (t.cols[ci].nullable != any_null(cols[ci].validity, t.nrows) && !t.cols[ci].nullable)
            fail(VEXQ_EINVAL, "NULLs in a column uploaded without NULLs");
        fill_column(t, ci, cols[ci], s, err);
    }
    compute_zones(t, s);
}

}  // namespace vq
