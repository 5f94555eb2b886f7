// jit.cpp — compiles the generated scan kernels for sm_100a with NVRTC and
// loads them through driver entry points obtained from the runtime (so the
// library has no link-time dependency on libcuda and loads on hosts without
// a GPU). Compiled cubins are cached in memory and on disk, keyed by a hash
// of the source and options.
#include <cuda.h>
#include <dlfcn.h>
#include <cudaTypedefs.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <atomic>
#include <map>
#include <tuple>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "internal.h"

namespace vq {

struct JitModule {
    CUmodule mod = nullptr;
    std::mutex mu;
    std::map<std::string, int> smem_limit;  // per entry: dynamic shared memory opted in so far
    ~JitModule();
};

namespace {

struct Driver {
    PFN_cuModuleLoadData_v2000 load = nullptr;
    PFN_cuModuleUnload_v2000 unload = nullptr;
    PFN_cuModuleGetFunction_v2000 get = nullptr;
    PFN_cuLaunchKernel_v7000_ptsz launch = nullptr;
    PFN_cuOccupancyMaxActiveBlocksPerMultiprocessor_v6050 occ = nullptr;
    PFN_cuFuncSetAttribute_v9000 setattr = nullptr;
    PFN_cuFuncGetAttribute_v2020 getattr = nullptr;
    bool ok = false;
};

Driver& drv() {
    static Driver d;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q;
        auto get = [&](const char* name, void** fn) {
            return cudaGetDriverEntryPoint(name, fn, cudaEnableDefault, &q) == cudaSuccess && *fn;
        };
        d.ok = get("cuModuleLoadData", (void**)&d.load) && get("cuModuleUnload", (void**)&d.unload) &&
               get("cuModuleGetFunction", (void**)&d.get) && get("cuLaunchKernel", (void**)&d.launch) &&
               get("cuOccupancyMaxActiveBlocksPerMultiprocessor", (void**)&d.occ) &&
               get("cuFuncSetAttribute", (void**)&d.setattr) && get("cuFuncGetAttribute", (void**)&d.getattr);
    });
    if (!d.ok) fail(VEXQ_EDEVICE, "CUDA driver entry points unavailable");
    return d;
}

uint64_t fnv1a(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) { h ^= c; h *= 1099511628211ull; }
    return h;
}

std::mutex g_mu;
std::map<uint64_t, std::shared_ptr<std::mutex>> g_compiling;  // per source: compile and load once
std::map<uint64_t, std::vector<char>> g_cubins;
std::map<std::pair<uint64_t, int>, std::shared_ptr<JitModule>> g_modules;  // (hash, device)

const char* kOptions[] = {"--gpu-architecture=sm_100a", "--fmad=false", "--std=c++17", "-lineinfo",
                          "--device-as-default-execution-space", "-DVQ_JIT=1"};

std::vector<char> compile_cubin(const std::string& src, uint64_t h) {
    std::string dir = jit_cache_dir();
    char name[64];
    std::snprintf(name, sizeof name, "/%016llx.cubin", (unsigned long long)h);
    std::string path = dir + name;
    {
        std::ifstream f(path, std::ios::binary);
        if (f) {
            std::vector<char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
            if (!b.empty()) return b;
        }
    }
    nvrtcProgram prog;
    if (nvrtcCreateProgram(&prog, src.c_str(), "vexq_kernel.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
        fail(VEXQ_EJIT, "nvrtcCreateProgram failed");
    nvrtcResult r = nvrtcCompileProgram(prog, (int)(sizeof kOptions / sizeof kOptions[0]), kOptions);
    if (r != NVRTC_SUCCESS) {
        size_t n = 0;
        nvrtcGetProgramLogSize(prog, &n);
        std::string log(n, '\0');
        nvrtcGetProgramLog(prog, &log[0]);
        nvrtcDestroyProgram(&prog);
        // keep the failing source next to the cache for diagnosis
        std::ofstream(dir + "/failed.cu") << src;
        fail(VEXQ_EJIT, "kernel specialisation failed to compile: " + log.substr(0, 4000));
    }
    size_t n = 0;
    nvrtcGetCUBINSize(prog, &n);
    std::vector<char> cubin(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    // unique per writer: threads of one process compile the same source too
    static std::atomic<unsigned long long> seq{0};
    std::string tmp = path + ".tmp" + std::to_string(getpid()) + "." + std::to_string(seq++);
    {
        std::ofstream f(tmp, std::ios::binary);
        f.write(cubin.data(), (std::streamsize)cubin.size());
    }
    std::rename(tmp.c_str(), path.c_str());
    return cubin;
}

}  // namespace

JitModule::~JitModule() {
    if (mod) {
        Driver& d = drv();
        d.unload(mod);
    }
}

std::string jit_cache_dir() {
    const char* env = std::getenv("VEXQ_JIT_CACHE");
    std::string dir;
    if (env && *env) {
        dir = env;
    } else {
        // next to the shared library: <package>/_build/jitcache
        Dl_info info;
        std::string so = dladdr((void*)&jit_cache_dir, &info) && info.dli_fname ? info.dli_fname : "./libvexqcuda.so";
        size_t slash = so.rfind('/');
        dir = (slash == std::string::npos ? std::string(".") : so.substr(0, slash)) + "/_build/jitcache";
    }
    // mkdir -p
    std::string cur;
    std::stringstream ss(dir);
    std::string part;
    if (!dir.empty() && dir[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
    return dir;
}

// Compiles (or fetches) the cubin for `source`; loading on the device
// happens on first use in the calling thread's current device.
// Finished kernels by (source hash, device, entry, block, dynamic shared
// memory): a repeated request (a batch rebuilt for every served batch, a plan
// recompiled) returns without copying the cubin or querying the driver.
struct KernelKey {
    uint64_t h;
    int dev, block, smem;
    std::string entry;
    bool operator<(const KernelKey& o) const {
        return std::tie(h, dev, block, smem, entry) < std::tie(o.h, o.dev, o.block, o.smem, o.entry);
    }
};
static std::map<KernelKey, JitKernel> g_kernels;

JitKernel jit_get(const std::string& source, const std::string& entry, int block, int smem) {
    uint64_t h = fnv1a(source) ^ (fnv1a(entry) * 31);
    for (const char* o : kOptions) h = h * 1099511628211ull ^ fnv1a(o);
    int cur_dev = -1;
    if (cudaGetDevice(&cur_dev) != cudaSuccess) {
        (void)cudaGetLastError();
        cur_dev = -1;
    }
    const KernelKey kk{h, cur_dev, block, smem, entry};
    if (cur_dev >= 0) {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_kernels.find(kk);
        if (it != g_kernels.end()) return it->second;
    }
    // one compile and one module load per source: a thread that finds another
    // working on the same source waits for it
    std::shared_ptr<std::mutex> cm;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto& slot = g_compiling[h];
        if (!slot) slot = std::make_shared<std::mutex>();
        cm = slot;
    }
    std::lock_guard<std::mutex> same_source(*cm);
    std::vector<char> cubin;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_cubins.find(h);
        if (it != g_cubins.end()) cubin = it->second;
    }
    if (cubin.empty()) {
        cubin = compile_cubin(source, h);
        std::lock_guard<std::mutex> lk(g_mu);
        g_cubins[h] = cubin;
    }
    JitKernel k;
    k.block = block;
    k.smem = smem;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return k;  // no device: compile-only
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return k;
    std::shared_ptr<JitModule> m;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_modules.find({h, dev});
        if (it != g_modules.end()) m = it->second;
    }
    Driver& d = drv();
    if (!m) {
        VQ_CUDA(cudaFree(nullptr));  // make the primary context current
        m = std::make_shared<JitModule>();
        CUresult r = d.load(&m->mod, cubin.data());
        if (r != CUDA_SUCCESS) fail(VEXQ_EDEVICE, "cuModuleLoadData failed: " + std::to_string((int)r));
        std::lock_guard<std::mutex> lk(g_mu);
        g_modules[{h, dev}] = m;
    }
    CUfunction f;
    CUresult r = d.get(&f, m->mod, entry.c_str());
    if (r != CUDA_SUCCESS) fail(VEXQ_EDEVICE, "cuModuleGetFunction failed for " + entry);
    k.mod = m;
    k.fn = (void*)f;
    if (smem > 0) {  // static shared memory counts against the default 48 KB limit too
        // plans sharing a kernel may need different sizes: the limit only grows
        std::lock_guard<std::mutex> lk(m->mu);
        int& cur = m->smem_limit[entry];
        if (smem > cur) {
            CUresult ra = d.setattr(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, smem);
            if (ra != CUDA_SUCCESS) fail(VEXQ_EDEVICE, "cuFuncSetAttribute(max dynamic smem) failed: " + std::to_string((int)ra));
            cur = smem;
        }
    }
    int nb = 0;
    if (d.occ(&nb, f, block, (size_t)smem) == CUDA_SUCCESS) k.max_blocks_per_sm = nb;
    int regs = 0;
    if (d.getattr(&regs, CU_FUNC_ATTRIBUTE_NUM_REGS, f) == CUDA_SUCCESS) k.regs = regs;
    if (dev == cur_dev) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_kernels[kk] = k;
    }
    return k;
}

void jit_launch(const JitKernel& k, int grid, const void* params, size_t params_size, cudaStream_t s) {
    (void)params_size;
    if (!k.fn) fail(VEXQ_EDEVICE, "kernel not loaded (no CUDA device)");
    Driver& d = drv();
    void* args[] = {const_cast<void*>(params)};
    CUresult r = d.launch((CUfunction)k.fn, grid, 1, 1, k.block, 1, 1, (unsigned)k.smem, (CUstream)s, args, nullptr);
    if (r != CUDA_SUCCESS) fail(VEXQ_EDEVICE, "cuLaunchKernel failed: " + std::to_string((int)r));
}

}  // namespace vq
