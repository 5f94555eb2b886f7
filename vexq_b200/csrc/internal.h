// internal.h — shared declarations of libvexqcuda (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/vexq_cuda.h"
#include "kparams.h"

namespace vq {

// ---- errors ---------------------------------------------------------------------
struct Status : std::runtime_error {
    int32_t code;
    Status(int32_t c, const std::string& m) : std::runtime_error(m), code(c) {}
};
[[noreturn]] void fail(int32_t code, const std::string& msg);
void set_error(const std::string& msg);
#define VQ_CUDA(x)                                                                      \
    do {                                                                                \
        cudaError_t _e = (x);                                                           \
        if (_e != cudaSuccess)                                                          \
            ::vq::fail(_e == cudaErrorMemoryAllocation ? VEXQ_ENOMEM : VEXQ_EDEVICE,    \
                       std::string(#x) + ": " + cudaGetErrorString(_e));                \
    } while (0)

// ---- device memory ------------------------------------------------------------------
// allocations left before an injected failure (-1: none; vexq_debug_fail_alloc)
extern std::atomic<int> g_fail_alloc_after;
// bytes held by live DevBufs (vexq_debug_live_device_bytes)
extern std::atomic<long long> g_live_device_bytes;

struct DevBuf {
    void* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t bytes) { alloc(bytes); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t bytes);
    void ensure(size_t bytes) { if (bytes > n) { release(); alloc(bytes); } }
    void release();
    template <class T> T* as() const { return (T*)p; }
};

// Host → device copy ordered on stream s: kernels launched on s afterwards see
// the bytes. (A plain cudaMemcpy from pageable memory may return before its
// DMA has landed, and the legacy stream it runs on does not order work on
// non-blocking streams, so a kernel launched next on such a stream could read
// the old contents.) The host buffer may be reused once this returns: pageable
// sources are staged before the call returns.
inline void h2d(void* dst, const void* src, size_t n, cudaStream_t s) {
    if (n) VQ_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, s));
}
// A one-time upload that has completed on the device when this returns (for
// buffers read later from any stream).
inline void h2d_now(void* dst, const void* src, size_t n) {
    if (!n) return;
    VQ_CUDA(cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, cudaStreamLegacy));
    VQ_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
}

struct PinnedBuf {
    void* p = nullptr;
    size_t n = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf();
    void ensure(size_t bytes);
};

// ---- tables ----------------------------------------------------------------------------
struct GlobalDict {
    std::vector<std::string> keys;
    std::unordered_map<std::string, uint32_t> index;
    uint32_t add(const std::string& s);
    int64_t find(const std::string& s) const {
        auto it = index.find(s);
        return it == index.end() ? -1 : (int64_t)it->second;
    }
};

struct Column {
    std::string name;
    int32_t type = 0;
    bool nullable = false;
    DevBuf values;      // padded to a multiple of kPadRows rows
    DevBuf validity;    // LSB-first bitmap (nullable columns only)
    // STRING
    GlobalDict dict;
    std::vector<std::vector<uint32_t>> rg_remap;   // per RG: local → global code
    std::vector<std::vector<uint8_t>> rg_present;  // per RG: global code present in the RG's dictionary
    bool per_rg_dicts = true;
    std::vector<vexq_zone_map> zones;              // per RG
    // table-wide min/max (numeric), for accumulator windows
    bool has_range = false;
    bool finite = true;             // FLOAT64: every row group's zone sum is finite (no NaN/±inf)
    double fmin = 0, fmax = 0;      // FLOAT64
    int64_t imin = 0, imax = 0;     // INT64 / DATE
};

struct Table {
    std::vector<Column> cols;
    int64_t nrows = 0;
    int32_t rg_rows = 65536;
    int32_t n_rg = 0;
    int device = 0;
    // bumped when re-filled values leave a column's earlier range (or bring in
    // NaN/±inf): plans compiled against the earlier ranges refuse to run
    uint64_t range_epoch = 0;
    bool zones_ready = false;
    uint64_t zone_version = 0;  // bumped every time the zone maps are recomputed
    int64_t rg_start(int rg) const { return (int64_t)rg * rg_rows; }
    int64_t rg_end(int rg) const { return std::min<int64_t>(nrows, (int64_t)(rg + 1) * rg_rows); }
    int64_t device_bytes() const;
};

constexpr int64_t kPadRows = 4096;  // device columns are padded so 128-bit tail loads stay in bounds

// ---- JIT ----------------------------------------------------------------------------------
struct JitModule;  // opaque: driver module + functions
struct JitKernel {
    std::shared_ptr<JitModule> mod;
    void* fn = nullptr;  // CUfunction
    int block = 256;
    int smem = 0;        // dynamic shared memory bytes
    int max_blocks_per_sm = 0;
    int regs = 0;        // registers a thread
};
JitKernel jit_get(const std::string& source, const std::string& entry, int block, int smem = 0);
void jit_launch(const JitKernel& k, int grid, const void* params, size_t params_size, cudaStream_t s);
std::string jit_cache_dir();

// ---- misc ----------------------------------------------------------------------------------
int sm_count();
const char* prelude_source();  // device helpers prepended to every generated kernel

}  // namespace vq
