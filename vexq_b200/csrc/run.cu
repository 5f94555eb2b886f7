// run.cu — plan execution: zone pruning → generated scan kernel → merge /
// finalize → group ordering → ORDER BY / LIMIT → host result batches.
//
// Reference behaviour reproduced here: group output in insertion order
// (exec/aggregate.go:209-216), SUM/MIN/MAX NULL when no non-NULL input, AVG =
// sum / float64(non-null count), COUNT never NULL (aggregate.go:780-876), a
// global aggregate over no rows emits one row (aggregate.go:961-982), and
// ExternalSort's comparison on raw int64 bits with NULLs first
// (exec/sort.go:130-163) followed by Limit (exec/limit.go:20-50).
#include <climits>
#include <cstdlib>
#include <algorithm>
#include <chrono>
#include <cstring>
#include <functional>
#include <numeric>
#include <set>

#include "plan.h"
#include "device_common.cuh"

namespace vq {

void refill_table(Table& t, const vexq_column_desc* cols, int32_t ncols, cudaStream_t s);

// ---- static kernels ----------------------------------------------------------------

// Entry of the calling warp: eight warps (256 threads) a block.
__device__ __forceinline__ int merge_warp() { return (int)blockIdx.x * 8 + ((int)threadIdx.x >> 5); }

__global__ void __launch_bounds__(256) k_merge_regs(const double* part_f, const long long* part_i, int nblocks, int G,
                                                    int nf, int ni, const int* fkind, const int* ikind, double* out_f,
                                                    long long* out_i) {
    merge_entry(merge_warp(), part_f, part_i, nblocks, G, nf, ni, fkind, ikind, out_f, out_i);
}

// The same merge launched as a programmatic dependent of the scan kernel: its
// blocks start while the scan drains and wait (griddepcontrol.wait) until the
// scan grid has finished and its writes are visible. Warp 0 also hands the
// scan's error word out with the results and clears it for the next run, so
// no memset precedes the scan.
__global__ void __launch_bounds__(256) k_merge_regs_dep(const double* part_f, const long long* part_i, int nblocks, int G,
                                                        int nf, int ni, const int* fkind, const int* ikind, double* out_f,
                                                        long long* out_i, int* err, int* err_out) {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    merge_entry(merge_warp(), part_f, part_i, nblocks, G, nf, ni, fkind, ikind, out_f, out_i);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *err_out = *err;
        *err = 0;
    }
}

// Batched merge: global warp w serves entry w - e0 of the plan whose range holds w.
__global__ void __launch_bounds__(256) k_merge_batch(const VQMergeDesc* d, int n) {
    const int w = merge_warp();
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d[mid].e0 <= w) lo = mid; else hi = mid - 1;
    }
    const VQMergeDesc m = d[lo];
    merge_entry(w - m.e0, m.part_f, m.part_i, m.nblocks, m.G, m.nf, m.ni, m.fkind, m.ikind, m.out_f, m.out_i);
}

// Atomic path: per-slot initial values (counts 0, MIN/MAX identities).
// Every slot at its identities in one pass (keys empty, first-row keys max,
// integer accumulators at their kind's identity, fixed-point digits and
// special flags 0), and the run's counters and error word cleared.
__global__ void k_init_table(unsigned long long* keys, long long* first, long long* acc_i, int ni, const long long* init_i,
                             long long* acc_fx, unsigned* special, int nf, long long nslots, int hash,
                             unsigned long long* ngroups, int* error, unsigned long long* n_out) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *ngroups = 0ull;
        *error = 0;
        *n_out = 0ull;
    }
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nslots; i += (long long)gridDim.x * blockDim.x) {
        if (hash) keys[i] = (i == nslots - 1) ? 0ull : VQ_EMPTY_KEY;
        first[i] = 0x7FFFFFFFFFFFFFFFLL;
        for (int s = 0; s < ni; s++) acc_i[(long long)s * nslots + i] = init_i[s];
        for (int f = 0; f < nf; f++) {
            long long* d = acc_fx + ((long long)f * nslots + i) * 4;  // 8-byte aligned only (odd slot counts)
            d[0] = 0;
            d[1] = 0;
            d[2] = 0;
            d[3] = 0;
            special[(long long)f * nslots + i] = 0u;
        }
    }
}

// Compacts occupied slots (count > 0) and turns exact fixed-point sums into
// correctly rounded doubles (NaN / ±inf flags applied IEEE-style). Output
// positions are taken one atomic per warp (per table within a warp).
__device__ __forceinline__ void finalize_write(long long i, unsigned long long pos, const unsigned long long* keys,
                                               const long long* first, const long long* acc_i, const long long* acc_fx,
                                               const unsigned* special, long long nslots, int ni, int nf,
                                               const int* fx_lsb, int hash, unsigned long long* o_key,
                                               long long* o_first, long long* o_i, double* o_f, long long cap_out) {
    if ((long long)pos >= cap_out) return;
    o_key[pos] = hash ? (i == nslots - 1 ? VQ_EMPTY_KEY : keys[i]) : (unsigned long long)i;
    o_first[pos] = first[i];
    for (int s = 0; s < ni; s++) o_i[(long long)s * cap_out + pos] = acc_i[(long long)s * nslots + i];
    for (int f = 0; f < nf; f++) {
        o_f[(long long)f * cap_out + pos] =
            vq_fx_result(acc_fx + ((long long)f * nslots + i) * 4, fx_lsb[f], special[(long long)f * nslots + i]);
    }
}

// Position of an occupied lane among the occupied lanes of its peer group
// (lanes of one table), with one atomicAdd on that table's counter per group.
__device__ __forceinline__ unsigned long long vq_claim(bool occ, unsigned peers, unsigned long long* n_out) {
    const int lane = threadIdx.x & 31;
    const unsigned b = __ballot_sync(0xffffffffu, occ) & peers;
    const int leader = __ffs(peers) - 1;
    unsigned long long base = 0;
    if (lane == leader && b) base = atomicAdd(n_out, (unsigned long long)__popc(b));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(b & ((1u << lane) - 1u));
}

// Output positions claimed per block: warp counts prefixed in shared memory,
// one atomic per block (a single counter taking an atomic per warp serialised
// large compactions). Every thread of the block calls it.
__device__ __forceinline__ unsigned long long vq_claim_block(bool occ, unsigned long long* n_out) {
    __shared__ unsigned wcnt[32];
    __shared__ unsigned long long base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    const unsigned b = __ballot_sync(0xffffffffu, occ);
    if (lane == 0) wcnt[warp] = __popc(b);
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned tot = 0;
        for (int w = 0; w < nw; w++) {
            const unsigned c = wcnt[w];
            wcnt[w] = tot;
            tot += c;
        }
        base = tot ? atomicAdd(n_out, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    const unsigned long long pos = base + wcnt[warp] + __popc(b & ((1u << lane) - 1u));
    __syncthreads();  // wcnt and base are rewritten by the next call
    return pos;
}

__global__ void k_finalize(const unsigned long long* keys, const long long* first, const long long* acc_i,
                           const long long* acc_fx, const unsigned* special, long long nslots, int ni, int nf,
                           const int* fx_lsb, int hash, unsigned long long* n_out, unsigned long long* o_key,
                           long long* o_first, long long* o_i, double* o_f, long long cap_out) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long b0 = (long long)blockIdx.x * blockDim.x; b0 < nslots; b0 += stride) {  // block-uniform trip count
        const long long i = b0 + threadIdx.x;
        const bool occ = i < nslots && acc_i[i] != 0;  // slot 0 of the int bank is the row count
        const unsigned long long pos = vq_claim_block(occ, n_out);
        if (occ) finalize_write(i, pos, keys, first, acc_i, acc_fx, special, nslots, ni, nf, fx_lsb, hash, o_key, o_first,
                                o_i, o_f, cap_out);
    }
}

// Batched group tables: global slot g belongs to the table whose slot0 is the
// largest not above g.
__device__ __forceinline__ int table_of(const VQTableDesc* d, int n, long long g) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (d[mid].slot0 <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_init_batch(const VQTableDesc* d, int n, long long total) {
    for (long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (long long)gridDim.x * blockDim.x) {
        const VQTableDesc& t = d[table_of(d, n, g)];
        const long long i = g - t.slot0;
        if (t.hash && !t.gid) t.keys[i] = (i == t.nslots - 1) ? 0ull : VQ_EMPTY_KEY;
        t.first[i] = 0x7FFFFFFFFFFFFFFFLL;
        for (int s = 0; s < t.ni; s++) t.acc_i[(long long)s * t.nslots + i] = t.init_i[s];
        for (int f = 0; f < t.nf; f++) {
            for (int k = 0; k < 4; k++) t.acc_fx[((long long)f * t.nslots + i) * 4 + k] = 0;
            t.special[(long long)f * t.nslots + i] = 0u;
        }
        if (i == 0) {
            *t.n_out = 0ull;
            *t.ngroups = 0ull;
            *t.error = 0;
        }
    }
}

__global__ void k_finalize_batch(const VQTableDesc* d, int n, long long total) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long b0 = (long long)blockIdx.x * blockDim.x; b0 < total; b0 += stride) {  // warp-uniform trip count
        const long long g = b0 + threadIdx.x;
        const int ti = g < total ? table_of(d, n, g) : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, ti);
        bool occ = false;
        if (ti >= 0) {
            const VQTableDesc& t = d[ti];
            occ = t.acc_i[g - t.slot0] != 0;
        }
        unsigned long long* cnt = ti >= 0 ? d[ti].n_out : nullptr;
        // every peer group claims from its own table's counter (a group without a table claims nothing)
        const unsigned long long pos = vq_claim(occ, peers, cnt ? cnt : (unsigned long long*)nullptr);
        if (occ) {
            const VQTableDesc& t = d[ti];
            finalize_write(g - t.slot0, pos, t.keys, t.first, t.acc_i, t.acc_fx, t.special, t.nslots, t.ni, t.nf,
                           t.fx_lsb, t.hash, t.o_key, t.o_first, t.o_i, t.o_f, t.cap_out);
        }
    }
}

// ---- exclusive scan (join build: slot counts → chain starts) ------------------------
__global__ void k_scan_blocks(const int* in, int* out, long long n, int* block_sums) {
    __shared__ int s[1024];
    long long base = (long long)blockIdx.x * 4096;
    int t = threadIdx.x;
    int v[4], sum = 0;
    for (int k = 0; k < 4; k++) {
        long long i = base + t * 4 + k;
        v[k] = i < n ? in[i] : 0;
        sum += v[k];
    }
    s[t] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        int x = t >= o ? s[t - o] : 0;
        __syncthreads();
        s[t] += x;
        __syncthreads();
    }
    int run = s[t] - sum;
    for (int k = 0; k < 4; k++) {
        long long i = base + t * 4 + k;
        if (i < n) out[i] = run;
        run += v[k];
    }
    if (t == 1023) block_sums[blockIdx.x] = s[1023];
}
__global__ void k_scan_sums(int* sums, int nb) {  // one block, sequential chunks
    __shared__ int s[1024];
    int carry = 0;
    for (int base = 0; base < nb; base += 1024) {
        int t = threadIdx.x;
        int v = base + t < nb ? sums[base + t] : 0;
        s[t] = v;
        __syncthreads();
        for (int o = 1; o < 1024; o <<= 1) {
            int x = t >= o ? s[t - o] : 0;
            __syncthreads();
            s[t] += x;
            __syncthreads();
        }
        if (base + t < nb) sums[base + t] = carry + s[t] - v;
        int tot = s[1023];
        __syncthreads();
        carry += tot;
    }
}
__global__ void k_scan_add(int* out, long long n, const int* sums) {
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += sums[i / 4096];
}
// Radix join: partition starts [np + 1] from the partition-major exclusive
// scan of the (partition, block) histogram.
__global__ void k_part_starts(const int* off, const int* hist, int np, int grid, long long* starts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < np) starts[i] = off[(long long)i * grid];
    if (i == np) {
        const long long n = (long long)np * grid;
        starts[np] = (long long)off[n - 1] + hist[n - 1];
    }
}

// Positions for m items a thread holds, claimed once per block: an exclusive
// scan of the threads' counts (warp shuffles, then the warps in order) and one
// atomic on the counter. Every thread of the block calls it.
__device__ __forceinline__ unsigned long long vq_claim_block_n(unsigned m, unsigned long long* ctr) {
    __shared__ unsigned wsum[32];
    __shared__ unsigned long long base;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
    unsigned incl = m;
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned tot = 0;
        for (int w = 0; w < nw; w++) {
            const unsigned c = wsum[w];
            wsum[w] = tot;
            tot += c;
        }
        base = tot ? atomicAdd(ctr, (unsigned long long)tot) : 0ull;
    }
    __syncthreads();
    const unsigned long long pos = base + wsum[warp] + (incl - m);
    __syncthreads();  // wsum and base are rewritten by the next call
    return pos;
}

// The probe's slots, four a thread at block-size stride (coalesced). For plans grouping by
// the join key (want_gid) each key also gets a group number (dense in
// 0..keys-1, claimed once per block) and gkey[number] = its key's code (key -
// koff); a one-row chain's count word is then ~number (negative), else -1, so
// the probe finds the row, and the group, in the slot.
__global__ void k_pack_slots(const unsigned long long* keys, const int* start, const int* count, const int* first,
                             int want_gid, int* gid, unsigned long long* gkey, unsigned long long* ngid, long long koff,
                             ulonglong2* slots, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x * 4;
    for (long long b0 = (long long)blockIdx.x * blockDim.x * 4; b0 < n; b0 += stride) {  // block-uniform trip count
        const long long i0 = b0 + threadIdx.x;
        int c[4];
        unsigned m = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const long long i = i0 + (long long)k * blockDim.x;
            c[k] = i < n ? count[i] : 0;
            m += c[k] > 0;
        }
        unsigned long long g = want_gid ? vq_claim_block_n(m, ngid) : 0ull;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const long long i = i0 + (long long)k * blockDim.x;
            if (i >= n) break;
            const int a = c[k] == 1 ? first[i] : start[i];  // start is computed only when some key repeats
            const int b = c[k] == 1 ? (want_gid ? ~(int)g : -1) : c[k];
            slots[i] = make_ulonglong2(keys[i], (unsigned long long)(unsigned)a | ((unsigned long long)(unsigned)b << 32));
            if (want_gid && c[k] > 0) {
                // the last slot holds the key equal to the empty sentinel (its key word is a used flag)
                const unsigned long long key = i == n - 1 ? VQ_EMPTY_KEY : keys[i];
                gid[i] = (int)g;
                gkey[g] = (unsigned long long)((long long)key - koff);
                g++;
            }
        }
    }
}

// Restores build-row order inside each key's chain (joinHashTable.insert keeps
// insertion order, exec/join_table.go:496-517): one thread per slot.
// Chains longer than kShortChain are listed (slot, length) for k_sort_long.
constexpr int kShortChain = 64;
__global__ void k_sort_chains(const int* start, const int* count, int* rows, long long nslots, int* unsorted,
                              int2* long_list, int* long_count, int long_cap) {
    for (long long sl = (long long)blockIdx.x * blockDim.x + threadIdx.x; sl < nslots; sl += (long long)gridDim.x * blockDim.x) {
        int c = count[sl];
        if (c < 2) continue;
        if (c > kShortChain) {
            const int at = atomicAdd(long_count, 1);
            if (at < long_cap) long_list[at] = make_int2((int)sl, c);
            else atomicOr(unsorted, 4);
            continue;
        }
        int* r = rows + start[sl];
        for (int i = 1; i < c; i++) {
            int x = r[i], j = i - 1;
            while (j >= 0 && r[j] > x) { r[j + 1] = r[j]; j--; }
            r[j + 1] = x;
        }
    }
}

// One block per long chain: bitonic sort of its row ids (padded to a power of
// two in scratch at soff[b]) back into build-row order.
__global__ void __launch_bounds__(1024) k_sort_long(const int2* list, const int* start, int* rows, int* scratch,
                                                    const long long* soff) {
    const int2 e = list[blockIdx.x];
    const int c = e.y;
    int M = 1;
    while (M < c) M <<= 1;
    int* w = scratch + soff[blockIdx.x];
    int* r = rows + start[e.x];
    for (int i = threadIdx.x; i < M; i += blockDim.x) w[i] = i < c ? r[i] : 0x7FFFFFFF;
    __syncthreads();
    for (int k = 2; k <= M; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < M; i += blockDim.x) {
                const int ij = i ^ j;
                if (ij > i) {
                    const int a = w[i], b = w[ij];
                    if ((a > b) == ((i & k) == 0)) { w[i] = b; w[ij] = a; }
                }
            }
            __syncthreads();
        }
    for (int i = threadIdx.x; i < c; i += blockDim.x) r[i] = w[i];
}

// Top-k support: order-preserving "better is larger" transform of a sort key.
__device__ __forceinline__ unsigned long long vq_rank(long long bits, bool isnull, int desc) {
    if (isnull) return 0xFFFFFFFFFFFFFFFFull;  // NULLs sort first (exec/sort.go:141-146)
    unsigned long long u = (unsigned long long)bits ^ 0x8000000000000000ull;  // signed order
    u = desc ? u : ~u;
    return u == 0xFFFFFFFFFFFFFFFFull ? u - 1 : u;
}
// The top-k kernels read the group count from the device (*np, written by
// the finalize or HAVING compaction), so they follow it without a copy back.
// One block samples S evenly spaced group ranks (S <= 16384) and finds the
// q-th largest of them (q < S) by radix select, most significant byte first: each round counts, in shared memory,
// the next byte of the samples that match the bytes chosen so far, and one
// warp walks the 256 counts from the top to the byte holding the q-th largest.
// The result is the selection threshold, so the host needs no copy of the
// samples.
__global__ void __launch_bounds__(1024) k_threshold(const unsigned long long* rank, int S, const unsigned long long* np, long long nmax,
                                                    int limit, unsigned long long* thr) {
    const long long n = (long long)min(*np, (unsigned long long)nmax);
    // few groups (at most 4·LIMIT + 4096): every group is a candidate
    if (n <= 4LL * limit + 4096) {
        if (threadIdx.x == 0) *thr = 0ull;
        return;
    }
    // expected (q+1)·n/S groups at or above the q-th largest sample: about
    // 4·LIMIT + 64 (n above 4·LIMIT + 4096 keeps q below S), and q at least 3:
    // the count above the q-th largest sample spreads like a Gamma(q+1)
    // variable, so with q = 0 about one run in 20 kept fewer than LIMIT groups
    // and fetched every group instead; from q = 3 (about 4·n/S candidates)
    // that is about one run in 10,000 at LIMIT 10
    const int q = max((int)ceil((4.0 * limit + 64.0) * S / (double)n) - 1, min(3, S - 1));
    __shared__ unsigned hist[256];
    __shared__ unsigned long long prefix;
    __shared__ unsigned need;
    // 16 samples a thread in registers (blockDim × 16 ≥ S), valid bits in a mask
    unsigned long long v[16];
    unsigned valid = 0u;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const int i = (int)threadIdx.x + k * (int)blockDim.x;
        v[k] = i < S ? rank[(long long)i * n / S] : 0ull;  // the sample: S evenly spaced groups
        if (i < S) valid |= 1u << k;
    }
    if (threadIdx.x == 0) { prefix = 0ull; need = (unsigned)q; }
    for (int shift = 56; shift >= 0; shift -= 8) {
        for (int i = threadIdx.x; i < 256; i += blockDim.x) hist[i] = 0u;
        __syncthreads();
        const unsigned long long hi_mask = shift == 56 ? 0ull : (~0ull << (shift + 8));
        const unsigned long long pre = prefix;
        const unsigned nd = need;  // both rewritten only after the next barrier
#pragma unroll
        for (int k = 0; k < 16; k++)
            if (((valid >> k) & 1u) && (v[k] & hi_mask) == pre) atomicAdd(&hist[(v[k] >> shift) & 255u], 1u);
        __syncthreads();
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            unsigned c[8], sum = 0u;
#pragma unroll
            for (int k = 0; k < 8; k++) { c[k] = hist[255 - (8 * lane + k)]; sum += c[k]; }
            unsigned incl = sum;
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned t = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += t;
            }
            const unsigned excl = incl - sum;
            if (excl <= nd && nd < incl) {  // exactly one lane holds the q-th largest
                unsigned acc = excl;
                for (int k = 0; k < 8; k++) {
                    if (nd < acc + c[k]) {
                        prefix = pre | ((unsigned long long)(255 - (8 * lane + k)) << shift);
                        need = nd - acc;
                        break;
                    }
                    acc += c[k];
                }
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *thr = q < S ? prefix : 0ull;
}
// The groups at or above the threshold, each gathered straight into its
// claimed row of the staging block (key, first-row key, integer bank, float
// bank as raw bits).
__global__ void k_select(const unsigned long long* rank, const unsigned long long* np, long long nmax, const unsigned long long* thrp,
                         unsigned long long* nsel, long long cap, const unsigned long long* key, const long long* first,
                         const long long* ival, const double* fval, long long cap_out, int ni, int nf, long long* out) {
    const long long n = (long long)min(*np, (unsigned long long)nmax);
    const unsigned long long thr = *thrp;
    const long long w = 2 + ni + nf;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (rank[i] >= thr) {
            const unsigned long long p = atomicAdd(nsel, 1ull);
            if ((long long)p >= cap) continue;
            long long* o = out + (long long)p * w;
            o[0] = (long long)key[i];
            o[1] = first[i];
            for (int s = 0; s < ni; s++) o[2 + s] = ival[(long long)s * cap_out + i];
            for (int f = 0; f < nf; f++) o[2 + ni + f] = __double_as_longlong(fval[(long long)f * cap_out + i]);
        }
    }
}
// Rank of one aggregate output per compacted group: its sort key's raw bits
// (NULL flag) mapped by vq_rank so that a larger rank sorts first.
__global__ void k_sortrank(const long long* o_i, const double* o_f, long long cap_out, const unsigned long long* np, int kind,
                           int vbank, int vpos, int nnpos, int fmin_key, int desc, unsigned long long* rank) {
    const long long n = (long long)min(*np, (unsigned long long)cap_out);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        long long nn = o_i[(long long)nnpos * cap_out + i];
        bool isnull = kind != VEXQ_AGG_COUNT && nn == 0;
        long long bits;
        if (vbank == 1) {  // float sum bank
            double v = o_f[(long long)vpos * cap_out + i];
            if (kind == VEXQ_AGG_AVG) v = v / (double)nn;
            bits = __double_as_longlong(v);
        } else {
            bits = o_i[(long long)vpos * cap_out + i];
            if (fmin_key) bits = __double_as_longlong(vq_fkey_inv((unsigned long long)bits));
        }
        rank[i] = vq_rank(bits, isnull, desc);
    }
}


}  // namespace vq

namespace vq {

double vq_fkey_inv_host(uint64_t k) {
    uint64_t b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    double d;
    std::memcpy(&d, &b, 8);
    return d;
}

// Grid of a scan kernel: every SM filled to its occupancy, never more blocks
// than loop units (staged kernels: one tile per block per iteration; chunk
// loops: one 128-row chunk per warp).
int grid_for(const JitKernel& k, long long units, bool staged, int cap_per_sm) {
    int per_sm = std::max(1, k.max_blocks_per_sm);
    if (cap_per_sm > 0) per_sm = std::min(per_sm, cap_per_sm);
    long long want = staged ? units : (units + (k.block / 32) - 1) / (k.block / 32);
    long long g = std::min<long long>((long long)sm_count() * per_sm, want);
    return (int)std::max<long long>(g, 1);
}

// COUNT(DISTINCT) sets of a plan for a scan over at most `rows` rows: twice
// that many slots (a power of two, at least 1,024), their states cleared on
// stream s before every launch (a hash-table rerun starts from empty sets).
void bind_distinct(Plan& p, VQParams& P, long long rows, cudaStream_t s) {
    if (p.ndist == 0) return;
    unsigned long long cap = 1024;
    while ((long long)cap < 2 * std::max<long long>(rows, 1)) cap <<= 1;
    for (int d = 0; d < p.ndist; d++) {
        p.dist_keys[d].ensure(cap * 16);
        p.dist_state[d].ensure(cap * 4);
        VQ_CUDA(cudaMemsetAsync(p.dist_state[d].p, 0, cap * 4, s));
        P.dkeys[d] = p.dist_keys[d].as<unsigned long long>();
        P.dstate[d] = p.dist_state[d].as<unsigned>();
    }
    P.dmask = cap - 1;
}

// A join probe that followed a direct-mapped build the host did not wait for
// raises the build's outcome in its own error word (64: the build met a
// repeated or out-of-range key, 128: it inserted no key, 256: it numbered more
// keys than the group table sized from the last build holds). The run is then
// repeated with the host waiting for the build.
struct SpecRetry {
    int bits;
};
static void check_spec_flags(int herr) {
    if (herr & (64 | 128 | 256)) throw SpecRetry{herr & (64 | 128 | 256)};
}

// Error bits of a COUNT(DISTINCT) set insert (vq_dset_insert).
static void check_distinct_flags(int herr) {
    if (herr & 16) fail(VEXQ_EDEVICE, "COUNT(DISTINCT) set reached its probe limit");
    if (herr & 32) fail(VEXQ_ETIMEDOUT, "COUNT(DISTINCT) set: a slot being written was not published within the wait limit");
}

void check_regs_flags(int herr) {
    check_spec_flags(herr);
    check_distinct_flags(herr);
    if (herr & 8) fail(VEXQ_ETIMEDOUT, "a staged tile copy did not complete within the kernel's wait limit");
    if (herr & 2) fail(VEXQ_ENOTSUP, "float sum exceeded its exact accumulation window");
    if (herr) fail(VEXQ_EDEVICE, "the scan kernel reported error flags " + std::to_string(herr));
}

void set_columns(VQParams& P, const Table& t, bool build_side) {
    for (size_t c = 0; c < t.cols.size(); c++) {
        const Column& col = t.cols[c];
        if (build_side) {
            P.bcol[c] = col.values.p;
            P.bvalid[c] = col.nullable ? col.validity.as<unsigned char>() : nullptr;
        } else {
            P.col[c] = col.values.p;
            P.valid[c] = col.nullable ? col.validity.as<unsigned char>() : nullptr;
        }
    }
}

int64_t slot_int(const Plan& p, const Groups& g, int slot, size_t i) { return g.ival[p.slot_pos[slot]][i]; }

double slot_float(const Plan& p, const Groups& g, int slot, size_t i) {
    if (p.path == AggPath::Regs || p.slots[slot].kind == S_FSUM) return g.fval[p.slot_pos[slot]][i];
    return vq_fkey_inv_host((uint64_t)g.ival[p.slot_pos[slot]][i]);
}

std::vector<long long> init_values(const Plan& p) {
    std::vector<long long> iv(std::max(p.ni, 1), 0);
    auto fkey = [](double d) {
        uint64_t b;
        std::memcpy(&b, &d, 8);
        return (long long)((b >> 63) ? ~b : (b | 0x8000000000000000ull));
    };
    for (size_t s = 0; s < p.slots.size(); s++) {
        if (p.slots[s].kind == S_FSUM) continue;
        long long v = 0;
        switch (p.slots[s].kind) {
            case S_IMIN: v = 0x7FFFFFFFFFFFFFFFLL; break;
            case S_IMAX: v = -0x7FFFFFFFFFFFFFFFLL - 1; break;
            case S_FMIN: v = fkey(1.7976931348623157e308); break;
            case S_FMAX: v = fkey(-1.7976931348623157e308); break;
            default: break;
        }
        iv[p.slot_pos[s]] = v;
    }
    return iv;
}

struct RunCtx {
    Plan& p;
    cudaStream_t s;
    float kernel_ms = 0;
    float scan_ms = 0;
    int launches = 0;
    const JitKernel* k = nullptr;  // main kernel other than p.k_main (partition join)
    int grid = 0;                  // and its grid
};

void ensure_events(Plan& p) {
    for (auto& e : p.ev)
        if (!e) VQ_CUDA(cudaEventCreate(&e));
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

// A register-path run whose launches are queued: what collecting it needs.
struct RegsPending {
    size_t nout_f = 0, nout_i = 0;
    bool mapped = false;
    int launches = 0;
    bool lazy = false;  // an event after the copy back marks the run's end (other runs may follow on the stream)
};

// Register path over prepared params: launch, merge, one copy back; the sync
// and the decode are regs_collect's.
static RegsPending regs_launch(RunCtx& rc, VQParams& P, long long nchunks, bool lazy) {
    Plan& p = rc.p;
    int G = (int)p.domain, nf = p.nf, ni = p.ni;
    int nfb = std::max(nf, 1);
    const JitKernel& K = rc.k ? *rc.k : p.k_main;
    int grid = rc.k ? rc.grid : grid_for(p.k_main, nchunks, p.staged, p.grid_per_sm);
    const bool fused = p.rfused && !rc.k;  // the scan merges its own partials
    if (!fused) {
        size_t pf = (size_t)grid * G * nfb, pi = (size_t)grid * G * (ni + 1);
        p.scratch_a.ensure(pf * 8);
        p.scratch_b.ensure(pi * 8);
        P.part_f = p.scratch_a.as<double>();
        P.part_i = p.scratch_b.as<long long>();
    }
    if (!p.d_kinds.p) {  // combiner kind per bank entry (0 sum, 1 min, 2 max), uploaded once
        std::vector<int> k(nfb + ni + 1, 0);
        for (size_t s = 0; s < p.slots.size(); s++) {
            int kd = p.slots[s].kind;
            int code = (kd == S_IMIN || kd == S_FMIN) ? 1 : (kd == S_IMAX || kd == S_FMAX) ? 2 : 0;
            k[p.slots[s].is_float() ? p.slot_pos[s] : nfb + p.slot_pos[s]] = code;
        }
        k[nfb + ni] = 1;  // first-occurrence key: min
        p.d_kinds.alloc(k.size() * 4);
        h2d(p.d_kinds.p, k.data(), k.size() * 4, rc.s);
    }
    const int* d_kinds = p.d_kinds.as<int>();
    size_t nout_f = (size_t)G * nfb * 8, nout_i = (size_t)G * (ni + 1) * 8;
    // layout: merged floats, merged ints, the error word handed out (copied
    // back with the results), then the error word the kernels raise
    const size_t before = p.scratch_c.n;
    p.scratch_c.ensure(nout_f + nout_i + 16);
    if (p.scratch_c.n != before) p.regs_err_clean = false;
    double* out_f = p.scratch_c.as<double>();
    long long* out_i = (long long*)((char*)p.scratch_c.p + nout_f);
    int* err_out = (int*)((char*)p.scratch_c.p + nout_f + nout_i);
    P.error = err_out + 2;
    p.h_stage.ensure(nout_f + nout_i + 16);
    // the merge writes the merged row and the handed-out error word straight
    // into the pinned staging buffer when the device can address it, so no
    // copy follows the merge (the kernels' own error word stays on the device)
    if (p.h_stage_mapped_for != p.h_stage.p) {  // looked up once per staging allocation
        p.h_stage_mapped = nullptr;
        if (cudaHostGetDevicePointer(&p.h_stage_mapped, p.h_stage.p, 0) != cudaSuccess) {
            (void)cudaGetLastError();
            p.h_stage_mapped = nullptr;
        }
        p.h_stage_mapped_for = p.h_stage.p;
    }
    void* mapped = p.h_stage_mapped;
    if (mapped) {
        out_f = (double*)mapped;
        out_i = (long long*)((char*)mapped + nout_f);
        err_out = (int*)((char*)mapped + nout_f + nout_i);
    }
    ensure_events(p);
    if (!p.regs_err_clean) VQ_CUDA(cudaMemsetAsync(P.error, 0, 4, rc.s));
    p.regs_err_clean = false;  // until the merge below has run
    if (fused) {
        // accumulators at their identities: fixed-point digits and flags 0,
        // integer entries by combiner kind, arrival count 0; the last block
        // of every run restores this state
        const size_t K = (size_t)std::max(1, p.rcopies);  // accumulator copies (block b adds into copy b % K)
        const size_t b_fx = K * G * nf * 32, b_i = K * G * (ni + 1) * 8, b_sp = (size_t)G * nf * 4;
        if (!p.racc.p) {
            std::vector<unsigned char> img(b_fx + b_i + b_sp + 16, 0);
            std::vector<long long> ident(ni + 1, 0);
            ident[ni] = LLONG_MAX;  // first-row key: min
            for (size_t s = 0; s < p.slots.size(); s++) {
                if (p.slots[s].is_float()) continue;
                const int kd = p.slots[s].kind;
                ident[p.slot_pos[s]] = kd == S_IMIN ? LLONG_MAX : kd == S_IMAX ? LLONG_MIN : 0;
            }
            long long* ii = (long long*)(img.data() + b_fx);
            for (size_t k = 0; k < K; k++)
                for (int gi = 0; gi < G; gi++)
                    for (int u = 0; u <= ni; u++) ii[(k * G + gi) * (ni + 1) + u] = ident[u];
            p.racc.alloc(img.size());
            h2d(p.racc.p, img.data(), img.size(), rc.s);
        }
        unsigned char* base = p.racc.as<unsigned char>();
        P.racc_fx = (long long*)base;
        P.racc_i = (long long*)(base + b_fx);
        P.racc_sp = (unsigned*)(base + b_fx + b_i);
        P.racc_done = (unsigned*)(base + b_fx + b_i + b_sp);
        P.rout_f = out_f;
        P.rout_i = out_i;
        P.rerr_out = err_out;
    }
    // the last block merges the partials inside the scan: no merge launch
    const bool last = !fused && p.merge_last;
    if (last) {
        if (!p.mdone.p) {
            p.mdone.alloc(16);
            VQ_CUDA(cudaMemsetAsync(p.mdone.p, 0, 16, rc.s));
        }
        P.mkinds = d_kinds;
        P.mout_f = out_f;
        P.mout_i = out_i;
        P.merr_out = err_out;
        P.mdone = p.mdone.as<unsigned>();
    }
    bind_distinct(p, P, nchunks * 128, rc.s);
    // the run's launches: start event, scan, merge, end event (events recorded
    // as external nodes when captured, so a replayed graph still times them;
    // plain records when launched directly, where the external flag is refused)
    auto launch_all = [&](bool checks) {
        if (checks) VQ_CUDA(cudaEventRecord(p.ev[0], rc.s));
        else VQ_CUDA(cudaEventRecordWithFlags(p.ev[0], rc.s, cudaEventRecordExternal));
        jit_launch(K, grid, &P, sizeof P, rc.s);
        if (checks) launch_check(rc.s, "p.k_main");
        // no event between the scan and its merge: an event record there stops the
        // merge's launch from overlapping the scan's drain (measured 5-6 us a run)
        if (!fused && !last) {
            const int tot = G * nf + G * (ni + 1);
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3((tot + 7) / 8);
            cfg.blockDim = dim3(256);
            cfg.stream = rc.s;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            at[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            VQ_CUDA(cudaLaunchKernelEx(&cfg, k_merge_regs_dep, (const double*)P.part_f, (const long long*)P.part_i, grid, G, nf,
                                       ni, d_kinds, d_kinds + nfb, out_f, out_i, P.error, err_out));
            if (checks) launch_check(rc.s, "k_merge_regs_dep");
        }
        if (checks) VQ_CUDA(cudaEventRecord(p.ev[2], rc.s));
        else VQ_CUDA(cudaEventRecordWithFlags(p.ev[2], rc.s, cudaEventRecordExternal));
    };
    // replayed as one CUDA graph while the parameter block and launch shape
    // are those it was captured with: one host call a run instead of four
    RegsGraphKey key;
    std::memset(&key, 0, sizeof key);
    key.P = P;
    key.fn = K.fn;
    key.s = rc.s;
    key.out_f = out_f;
    key.out_i = out_i;
    key.err_out = err_out;
    key.d_kinds = d_kinds;
    key.grid = grid;
    key.block = K.block;
    key.smem = K.smem;
    key.mode = fused ? 1 : last ? 2 : 0;
    if (p.graph_off || launch_checks_on()) {
        launch_all(true);
    } else if (p.rg_exec && std::memcmp(&key, &p.rg_key, sizeof key) == 0) {
        VQ_CUDA(cudaGraphLaunch(p.rg_exec, rc.s));
    } else {
        if (p.rg_exec) {
            cudaGraphExecDestroy(p.rg_exec);
            p.rg_exec = nullptr;
        }
        cudaGraph_t graph = nullptr;
        bool ok = cudaStreamBeginCapture(rc.s, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
        if (ok) {
            try {
                launch_all(false);
            } catch (const Status&) {
                ok = false;
            }
            const cudaError_t e = cudaStreamEndCapture(rc.s, &graph);
            ok = ok && e == cudaSuccess && graph;
        }
        if (ok) ok = cudaGraphInstantiate(&p.rg_exec, graph, 0) == cudaSuccess;
        if (graph) cudaGraphDestroy(graph);
        if (ok) {
            std::memcpy(&p.rg_key, &key, sizeof key);  // padding included: compared bytewise
            VQ_CUDA(cudaGraphLaunch(p.rg_exec, rc.s));
        } else {  // capture refused: direct launches from here on
            (void)cudaGetLastError();
            p.rg_exec = nullptr;
            p.graph_off = true;
            launch_all(true);
        }
    }
    if (!mapped) VQ_CUDA(cudaMemcpyAsync(p.h_stage.p, p.scratch_c.p, nout_f + nout_i + 4, cudaMemcpyDeviceToHost, rc.s));
    if (lazy) VQ_CUDA(cudaEventRecord(p.ev[3], rc.s));
    RegsPending q;
    q.nout_f = nout_f;
    q.nout_i = nout_i;
    q.mapped = mapped != nullptr;
    q.launches = fused || last ? 1 : 2;
    q.lazy = lazy;
    return q;
}

// Waits for a queued register-path run and decodes its merged row.
static Groups regs_collect(RunCtx& rc, const RegsPending& q) {
    Plan& p = rc.p;
    Groups g;
    const int G = (int)p.domain, nf = p.nf, ni = p.ni;
    const size_t nout_f = q.nout_f, nout_i = q.nout_i;
    if (q.lazy) VQ_CUDA(cudaEventSynchronize(p.ev[3]));
    else VQ_CUDA(cudaStreamSynchronize(rc.s));
    p.regs_err_clean = true;
    check_regs_flags(*(const int*)((const char*)p.h_stage.p + nout_f + nout_i));
    const float span = elapsed(p.ev[0], p.ev[2]);  // the scan and the merge (overlapping its drain, or inside it)
    rc.scan_ms += span;
    rc.kernel_ms += span;
    rc.launches += q.launches;
    const double* hf = (const double*)p.h_stage.p;
    const long long* hi = (const long long*)((const char*)p.h_stage.p + nout_f);
    g.ival.assign(ni, {});
    g.fval.assign(nf, {});
    for (int gi = 0; gi < G; gi++) {
        long long cnt = hi[(size_t)gi * (ni + 1) + p.slot_pos[0]];
        if (cnt == 0) continue;
        g.key.push_back((uint64_t)gi);
        g.first.push_back(hi[(size_t)gi * (ni + 1) + ni]);
        for (int s = 0; s < ni; s++) g.ival[s].push_back(hi[(size_t)gi * (ni + 1) + s]);
        for (int s = 0; s < nf; s++) g.fval[s].push_back(hf[(size_t)gi * nf + s]);
    }
    return g;
}

Groups run_regs(RunCtx& rc, VQParams& P, long long nchunks) {
    const RegsPending q = regs_launch(rc, P, nchunks, false);
    return regs_collect(rc, q);
}

// Atomic path: group table, main kernel (retried with a larger table when a
// probe limit is hit), finalize + compaction on the device.
struct Compacted {
    long long n = 0;           // groups (-1: not copied back yet; the device holds it in *n_dev)
    long long cap_out = 0;
    unsigned long long* key = nullptr;
    long long* first = nullptr;
    long long* ival = nullptr;
    double* fval = nullptr;
    const unsigned long long* n_dev = nullptr;  // the group count on the device
    const int* err_dev = nullptr;  // deferred run: the kernels' error word, read with the results
    bool hash = false;             // deferred run on a hash table: its group count sizes the next run
    long long rows = 0;
    bool having_done = false;  // only the groups HAVING keeps
};

// A deferred run (defer set) launches the table kernels and returns without
// waiting: the caller's top-k launches follow on the stream, and one copy back
// after them brings the group count and the error word with the results.
Compacted run_atomic(RunCtx& rc, VQParams& P, long long nchunks, long long estimate, long long rows, bool defer = false) {
    Plan& p = rc.p;
    // a join grouping by its key on the global table: one slot per build key
    // number, no key inserts; the keys come from the build's number→key array
    const bool gid = p.join_gid && !rc.k;
    bool hash = p.path == AggPath::Hash && !gid;
    long long cap, safe_cap = 16;
    if (gid) {
        cap = std::max<long long>(p.gid_groups, 1);
    } else if (hash) {
        while (safe_cap < 2 * std::max<long long>(estimate, 8)) safe_cap <<= 1;
        // a rerun sizes its table from the groups the last run found, scaled
        // up by the rows scanned (the row-count bound is usually far above the
        // distinct keys, and a table sized by rows leaves L2, sending every
        // atomic to DRAM); if that is too small, the probe limit is hit and
        // the rerun below takes the row-bounded size
        if (p.hash_groups_seen >= 0) {
            const double scale = std::max(1.0, (double)rows / (double)std::max<long long>(p.hash_rows_seen, 1));
            estimate = std::min<long long>(estimate, std::max<long long>((long long)(p.hash_groups_seen * scale), 1024));
        }
        cap = 16;
        while (cap < 2 * std::max<long long>(estimate, 8)) cap <<= 1;
    } else {
        cap = p.domain;
    }
    std::vector<long long> iv = init_values(p);
    ensure_events(p);
    for (int attempt = 0; attempt < 8; attempt++) {
        long long nslots = cap + 1;
        int ni = p.ni, nf = p.nf;
        size_t b_keys = hash ? nslots * 8 : 0, b_first = nslots * 8, b_i = (size_t)ni * nslots * 8,
               b_fx = (size_t)nf * nslots * 32, b_sp = (size_t)nf * nslots * 4;
        size_t tot = b_keys + b_first + b_i + b_fx + b_sp + 64 + iv.size() * 8 + 64;
        p.scratch_a.ensure(tot);
        char* base = (char*)p.scratch_a.p;
        P.keys = hash ? (unsigned long long*)base : nullptr;
        P.first = (long long*)(base + b_keys);
        P.acc_i = (long long*)(base + b_keys + b_first);
        P.acc_fx = (long long*)(base + b_keys + b_first + b_i);
        P.special = (unsigned*)(base + b_keys + b_first + b_i + b_fx);
        char* tail = base + b_keys + b_first + b_i + b_fx + b_sp;
        tail = (char*)(((uintptr_t)tail + 15) & ~(uintptr_t)15);
        P.ngroups = (unsigned long long*)tail;
        P.error = (int*)(tail + 8);
        long long* d_init = (long long*)(tail + 16);
        P.cap = (unsigned long long)cap;
        P.cap_mask = hash ? (unsigned long long)(cap - 1) : 0;
        for (int f = 0; f < nf && f < 16; f++) P.fx_lsb[f] = p.fx_lsb[f];
        // compacted output (upper bound: every slot occupied)
        long long cap_out = nslots;
        size_t o_bytes = 16 + cap_out * 16 + (size_t)ni * cap_out * 8 + (size_t)nf * cap_out * 8 + nf * 4 + 64;
        p.scratch_b.ensure(o_bytes);
        char* ob = (char*)p.scratch_b.p;
        Compacted c;
        c.cap_out = cap_out;
        unsigned long long* n_out = (unsigned long long*)ob;
        c.key = (unsigned long long*)(ob + 16);
        c.first = (long long*)(ob + 16 + cap_out * 8);
        c.ival = (long long*)(ob + 16 + cap_out * 16);
        c.fval = (double*)(ob + 16 + cap_out * 16 + (size_t)ni * cap_out * 8);
        (void)d_init;
        // the plan's constant identities and float-sum windows, uploaded once
        const size_t tinit = iv.size() * 8 + (size_t)std::max(nf, 1) * 4;
        if (p.d_tinit.n < tinit) {
            std::vector<char> img(tinit, 0);
            std::memcpy(img.data(), iv.data(), iv.size() * 8);
            if (nf) std::memcpy(img.data() + iv.size() * 8, p.fx_lsb.data(), (size_t)nf * 4);
            p.d_tinit.ensure(tinit);
            h2d(p.d_tinit.p, img.data(), tinit, rc.s);
        }
        const long long* d_iv = p.d_tinit.as<long long>();
        const int* d_lsb = (const int*)(p.d_tinit.as<char>() + iv.size() * 8);
        VQ_CUDA(cudaEventRecord(p.ev[0], rc.s));
        int ig = (int)std::min<long long>((nslots + 255) / 256, (long long)sm_count() * 16);
        k_init_table<<<ig, 256, 0, rc.s>>>(P.keys, P.first, P.acc_i, ni, d_iv, P.acc_fx, P.special, nf, nslots, hash, P.ngroups,
                                          P.error, n_out);
        launch_check(rc.s, "k_init_table");
        bind_distinct(p, P, nchunks * 128, rc.s);
        VQ_CUDA(cudaGetLastError());
        const JitKernel& K = rc.k ? *rc.k : p.k_main;
        int grid = rc.k ? rc.grid : grid_for(p.k_main, nchunks, p.staged);
        VQ_CUDA(cudaEventRecord(p.ev[1], rc.s));
        jit_launch(K, grid, &P, sizeof P, rc.s);
        launch_check(rc.s, "p.k_main");
        VQ_CUDA(cudaEventRecord(p.ev[2], rc.s));
        int fg = (int)std::min<long long>((nslots + 255) / 256, (long long)sm_count() * 16);
        k_finalize<<<fg, 256, 0, rc.s>>>(gid ? p.jt_gkey.as<unsigned long long>() : P.keys, P.first, P.acc_i, P.acc_fx, P.special,
                                         nslots, ni, nf, d_lsb, hash || gid, n_out, c.key, c.first, c.ival, c.fval, cap_out);
        launch_check(rc.s, "k_finalize");
        VQ_CUDA(cudaGetLastError());
        VQ_CUDA(cudaEventRecord(p.ev[3], rc.s));
        c.n_dev = n_out;
        if (defer) {
            c.n = -1;
            c.err_dev = P.error;
            c.hash = hash;
            c.rows = rows;
            rc.launches += 3;
            return c;
        }
        p.h_stage.ensure(32);
        VQ_CUDA(cudaMemcpyAsync(p.h_stage.p, n_out, 8, cudaMemcpyDeviceToHost, rc.s));
        VQ_CUDA(cudaMemcpyAsync((char*)p.h_stage.p + 8, P.error, 4, cudaMemcpyDeviceToHost, rc.s));
        VQ_CUDA(cudaStreamSynchronize(rc.s));
        rc.scan_ms += elapsed(p.ev[1], p.ev[2]);
        rc.kernel_ms += elapsed(p.ev[0], p.ev[3]);
        rc.launches += 3;
        unsigned long long nn = *(unsigned long long*)p.h_stage.p;
        int herr = *(int*)((char*)p.h_stage.p + 8);
        check_spec_flags(herr);
        check_distinct_flags(herr);
        if (herr & 8) fail(VEXQ_ETIMEDOUT, "a staged tile copy did not complete within the kernel's wait limit");
        if (herr & 2) fail(VEXQ_ENOTSUP, "float sum exceeded its exact accumulation window");
        if (herr & 1) {  // probe limit: grow the table and rerun
            if (!hash) fail(VEXQ_EDEVICE, "dense group table reported a probe failure");
            cap = std::max(cap << 1, safe_cap);
            continue;
        }
        c.n = (long long)std::min<unsigned long long>(nn, (unsigned long long)cap_out);
        if (hash) {
            p.hash_groups_seen = c.n;
            p.hash_rows_seen = rows;
        }
        return c;
    }
    fail(VEXQ_ENOMEM, "group table could not be sized");
}

Groups fetch_groups(RunCtx& rc, const Compacted& c) {
    Plan& p = rc.p;
    Groups g;
    const long long n = c.n;
    g.key.resize(n);
    g.first.resize(n);
    g.ival.assign(p.ni, std::vector<int64_t>(n));
    g.fval.assign(p.nf, std::vector<double>(n));
    if (n == 0) return g;
    VQ_CUDA(cudaMemcpyAsync(g.key.data(), c.key, n * 8, cudaMemcpyDeviceToHost, rc.s));
    VQ_CUDA(cudaMemcpyAsync(g.first.data(), c.first, n * 8, cudaMemcpyDeviceToHost, rc.s));
    for (int s = 0; s < p.ni; s++) VQ_CUDA(cudaMemcpyAsync(g.ival[s].data(), c.ival + (long long)s * c.cap_out, n * 8, cudaMemcpyDeviceToHost, rc.s));
    for (int s = 0; s < p.nf; s++) VQ_CUDA(cudaMemcpyAsync(g.fval[s].data(), c.fval + (long long)s * c.cap_out, n * 8, cudaMemcpyDeviceToHost, rc.s));
    VQ_CUDA(cudaStreamSynchronize(rc.s));
    return g;
}

// HAVING over the compacted groups on the device (vq_having): the groups it
// keeps, compacted again into scratch_f.
Compacted having_device(RunCtx& rc, const Compacted& c) {
    Plan& p = rc.p;
    Compacted o;
    o.having_done = true;
    o.cap_out = std::max<long long>(c.n, 1);
    p.scratch_f.ensure(64 + (size_t)o.cap_out * (16 + 8 * (size_t)(p.ni + p.nf)));
    char* b = (char*)p.scratch_f.p;
    unsigned long long* cnt = (unsigned long long*)b;
    o.key = (unsigned long long*)(b + 64);
    o.first = (long long*)(o.key + o.cap_out);
    o.ival = o.first + o.cap_out;
    o.fval = (double*)(o.ival + (size_t)p.ni * o.cap_out);
    VQ_CUDA(cudaEventRecord(p.ev[2], rc.s));
    VQ_CUDA(cudaMemsetAsync(cnt, 0, 8, rc.s));
    if (c.n > 0) {
        VQParams P;
        std::memset(&P, 0, sizeof P);
        P.keys = c.key;
        P.first = c.first;
        P.acc_i = c.ival;
        P.part_f = c.fval;
        P.cap = (unsigned long long)c.cap_out;
        P.nchunks = c.n;
        P.pkeys = o.key;
        P.part_i = o.first;
        P.racc_i = o.ival;
        P.rout_f = o.fval;
        P.jmask = (unsigned long long)o.cap_out;
        P.jtotal = cnt;
        const int grid = (int)std::min<long long>((c.n + 255) / 256, (long long)sm_count() * 8);
        jit_launch(p.k_having, grid, &P, sizeof P, rc.s);
        launch_check(rc.s, "vq_having");
        rc.launches++;
    }
    VQ_CUDA(cudaEventRecord(p.ev[3], rc.s));
    p.h_stage.ensure(16);
    VQ_CUDA(cudaMemcpyAsync(p.h_stage.p, cnt, 8, cudaMemcpyDeviceToHost, rc.s));
    VQ_CUDA(cudaStreamSynchronize(rc.s));
    rc.kernel_ms += elapsed(p.ev[2], p.ev[3]);
    o.n = (long long)std::min<unsigned long long>(*(const unsigned long long*)p.h_stage.p, (unsigned long long)o.cap_out);
    o.n_dev = cnt;
    return o;
}

// Device top-k candidates for ORDER BY <aggregate> LIMIT k: every group's sort
// rank (raw int64 bits in the ExternalSort order, NULLs first) is computed on
// the device; the q-th largest of a 4096-point sample, found on the device,
// is a threshold that keeps about 4·LIMIT + 64 groups (every group when there
// are at most 4·LIMIT + 4096); the groups at or above it (ties included) are
// gathered, and the host finishes the stable sort on them. The kernels read
// the group count on the device, so they follow a deferred table run without
// a copy back; one copy brings the count, the error word, the selected count
// and the first gathered rows. Returns 1 with g filled; 0 when the caller
// fetches every group instead (the plan has no such ORDER BY, the groups are
// few and already counted, or the sample was unlucky; c.n is set); -1 when a
// deferred run hit its table's probe limit and must run again.
bool topk_applies(const Plan& p, bool having_done) {
    const vexq_order_desc& o = p.order;
    // HAVING filters groups before the sort: every group comes back, unless
    // the device already kept only the groups HAVING passes
    return !((p.having_root >= 0 && !having_done) || o.sort_col < (int)p.keys.size() || o.limit < 0 || o.limit > 4096);
}

int topk_groups(RunCtx& rc, Compacted& c, Groups& g) {
    Plan& p = rc.p;
    const vexq_order_desc& o = p.order;
    const long long kCap = 65536;
    if (!topk_applies(p, c.having_done)) return 0;
    if (c.n >= 0 && c.n <= 4 * o.limit + 4096) return 0;
    const AggOut& a = p.outs[o.sort_col - (int)p.keys.size()];
    int vslot = a.value_slot;
    int vbank = (p.slots[vslot].kind == S_FSUM) ? 1 : 0;
    int fmin_key = (p.slots[vslot].kind == S_FMIN || p.slots[vslot].kind == S_FMAX) ? 1 : 0;
    if (a.kind == VEXQ_AGG_COUNT) vbank = 0;
    // 16,384 samples: with q at least 3 about 4·n/S ≈ 175 candidates for
    // Q3's ~700K groups (4,096 samples with q at least 7 kept ~1,400, whose
    // host sort cost more)
    const int S = 16384;
    const long long w = 2 + p.ni + p.nf;
    const long long nmax = c.n >= 0 ? c.n : c.cap_out;
    // rank | threshold, count | gathered rows
    size_t need = (size_t)nmax * 8 + 16 + (size_t)kCap * w * 8 + 64;
    p.scratch_d.ensure(need);
    unsigned long long* rank = p.scratch_d.as<unsigned long long>();
    unsigned long long* thr = rank + nmax;
    unsigned long long* nsel = thr + 1;
    long long* dout = (long long*)(nsel + 1);
    int gr = (int)std::min<long long>((nmax + 255) / 256, (long long)sm_count() * 8);
    k_sortrank<<<std::max(gr, 1), 256, 0, rc.s>>>(c.ival, c.fval, c.cap_out, c.n_dev, a.kind, vbank, p.slot_pos[vslot],
                                                  p.slot_pos[a.nn_slot], fmin_key, o.descending, rank);
    launch_check(rc.s, "k_sortrank");
    k_threshold<<<1, 1024, 0, rc.s>>>(rank, S, c.n_dev, nmax, (int)o.limit, thr);
    launch_check(rc.s, "k_threshold");
    VQ_CUDA(cudaMemsetAsync(nsel, 0, 8, rc.s));
    k_select<<<std::max(gr, 1), 256, 0, rc.s>>>(rank, c.n_dev, nmax, thr, nsel, kCap, c.key, c.first, c.ival, c.fval, c.cap_out,
                                                p.ni, p.nf, dout);
    launch_check(rc.s, "k_select");
    VQ_CUDA(cudaGetLastError());
    rc.launches += 3;
    // one copy back: group count, error word, selected count, and the first
    // R gathered rows (twice the last run's candidates and 256 more, at least
    // twice the expected 4·LIMIT + 64), rounded up to a power of two so the
    // pinned staging buffer grows only at doublings
    const long long want = std::max<long long>(2 * (4LL * o.limit + 64), p.topk_seen * 2 + 256);
    long long R = 1024;
    while (R < want) R <<= 1;
    R = std::min(R, kCap);
    p.h_stage.ensure(32 + (size_t)R * w * 8);
    char* hs = (char*)p.h_stage.p;
    std::memset(hs, 0, 32);
    VQ_CUDA(cudaMemcpyAsync(hs, c.n_dev, 8, cudaMemcpyDeviceToHost, rc.s));
    if (c.err_dev) VQ_CUDA(cudaMemcpyAsync(hs + 8, c.err_dev, 4, cudaMemcpyDeviceToHost, rc.s));
    VQ_CUDA(cudaMemcpyAsync(hs + 16, nsel, 8, cudaMemcpyDeviceToHost, rc.s));
    VQ_CUDA(cudaMemcpyAsync(hs + 32, dout, (size_t)R * w * 8, cudaMemcpyDeviceToHost, rc.s));
    if (c.n < 0) VQ_CUDA(cudaEventRecord(p.ev[3], rc.s));
    VQ_CUDA(cudaStreamSynchronize(rc.s));
    if (c.n < 0) {  // a deferred table run: its time, count and error word
        rc.scan_ms += elapsed(p.ev[1], p.ev[2]);
        rc.kernel_ms += elapsed(p.ev[0], p.ev[3]);
        c.n = (long long)std::min<unsigned long long>(*(const unsigned long long*)hs, (unsigned long long)c.cap_out);
        const int herr = *(const int*)(hs + 8);
        check_spec_flags(herr);
        check_distinct_flags(herr);
        if (herr & 8) fail(VEXQ_ETIMEDOUT, "a staged tile copy did not complete within the kernel's wait limit");
        if (herr & 2) fail(VEXQ_ENOTSUP, "float sum exceeded its exact accumulation window");
        if (herr & 1) {
            if (!c.hash) fail(VEXQ_EDEVICE, "dense group table reported a probe failure");
            return -1;
        }
        if (c.hash) {
            p.hash_groups_seen = c.n;
            p.hash_rows_seen = c.rows;
        }
    }
    const long long ns = (long long)*(const unsigned long long*)(hs + 16);
    p.topk_seen = std::min(ns, kCap);
    // few groups: all of them were selected; otherwise an unlucky sample (fewer
    // than LIMIT selected) or too many ties at the threshold: the caller
    // fetches every group
    if (c.n > 4 * o.limit + 4096 && (ns < o.limit || ns > kCap)) return 0;
    if (ns > kCap) return 0;
    g.having_done = c.having_done;
    std::vector<long long> rest;
    if (ns > R) {
        rest.resize((size_t)(ns - R) * w);
        VQ_CUDA(cudaMemcpyAsync(rest.data(), dout + R * w, rest.size() * 8, cudaMemcpyDeviceToHost, rc.s));
        VQ_CUDA(cudaStreamSynchronize(rc.s));
    }
    g.key.resize(ns);
    g.first.resize(ns);
    g.ival.assign(p.ni, std::vector<int64_t>(ns));
    g.fval.assign(p.nf, std::vector<double>(ns));
    const long long* head = (const long long*)(hs + 32);
    for (long long j = 0; j < ns; j++) {
        const long long* r = j < R ? head + j * w : rest.data() + (j - R) * w;
        g.key[j] = (uint64_t)r[0];
        g.first[j] = r[1];
        for (int s = 0; s < p.ni; s++) g.ival[s][j] = r[2 + s];
        for (int f = 0; f < p.nf; f++) std::memcpy(&g.fval[f][j], &r[2 + p.ni + f], 8);
    }
    return 1;
}

// Decodes group keys, computes aggregate outputs, orders groups, and applies
// ORDER BY / LIMIT.
// HAVING evaluation over one output row: the IR semantics of the scan
// kernels' expression code (validity and value per node: comparisons and
// arithmetic propagate NULL; AND/OR combine values and validity bitwise;
// NOT flips valid bits; float x/0 is NaN and integer x/0 is 0; IN tests the
// value set; CASE takes the first true branch), over the output columns.
struct HVal {
    bool ok = false, b = false;
    int64_t i = 0;
    double d = 0;
};

static HVal having_eval(const std::vector<INode>& ir, int idx, const std::vector<OutColumn>& cols, size_t row) {
    const INode& n = ir[idx];
    HVal v;
    auto E = [&](int k) { return having_eval(ir, n.ch[k], cols, row); };
    switch (n.k) {
        case NK::Col: {
            const OutColumn& c = cols[n.col];
            v.ok = c.valid[row] != 0;
            const int64_t raw = c.v[row];
            switch (n.type) {
                case VEXQ_TYPE_FLOAT64: std::memcpy(&v.d, &raw, 8); break;
                case VEXQ_TYPE_DATE: v.i = (int32_t)raw; break;
                case VEXQ_TYPE_BOOL: v.b = v.ok && raw != 0; break;
                case VEXQ_TYPE_STRING: v.i = (uint32_t)raw; break;
                default: v.i = raw; break;
            }
            return v;
        }
        case NK::Lit:
            v.ok = true;
            if (n.type == VEXQ_TYPE_FLOAT64) v.d = n.lf;
            else if (n.type == VEXQ_TYPE_DATE) v.i = n.ld;
            else if (n.type == VEXQ_TYPE_BOOL) v.b = n.lb;
            else if (n.type == VEXQ_TYPE_INT64) v.i = n.li;
            return v;
        case NK::Cmp: {
            const HVal a = E(0), b = E(1);
            v.ok = a.ok && b.ok;
            const bool fl = ir[n.ch[0]].type == VEXQ_TYPE_FLOAT64;
            bool c = false;
            switch (n.op) {
                case VEXQ_OP_EQ: c = fl ? a.d == b.d : a.i == b.i; break;
                case VEXQ_OP_NE: c = fl ? a.d != b.d : a.i != b.i; break;
                case VEXQ_OP_LT: c = fl ? a.d < b.d : a.i < b.i; break;
                case VEXQ_OP_LE: c = fl ? a.d <= b.d : a.i <= b.i; break;
                case VEXQ_OP_GT: c = fl ? a.d > b.d : a.i > b.i; break;
                case VEXQ_OP_GE: c = fl ? a.d >= b.d : a.i >= b.i; break;
            }
            v.b = v.ok && c;
            return v;
        }
        case NK::Arith: {
            const HVal a = E(0), b = E(1);
            v.ok = a.ok && b.ok;
            if (!v.ok) return v;
            if (n.type == VEXQ_TYPE_FLOAT64) {
                switch (n.op) {
                    case VEXQ_OP_ADD: v.d = a.d + b.d; break;
                    case VEXQ_OP_SUB: v.d = a.d - b.d; break;
                    case VEXQ_OP_MUL: v.d = a.d * b.d; break;
                    case VEXQ_OP_DIV: {  // applyArithFloat64: x/0 → math.NaN()
                        if (b.d == 0.0) { const int64_t nan = 0x7FF8000000000001LL; std::memcpy(&v.d, &nan, 8); }
                        else v.d = a.d / b.d;
                        break;
                    }
                }
            } else {
                const uint64_t x = (uint64_t)a.i, y = (uint64_t)b.i;
                switch (n.op) {
                    case VEXQ_OP_ADD: v.i = (int64_t)(x + y); break;
                    case VEXQ_OP_SUB: v.i = (int64_t)(x - y); break;
                    case VEXQ_OP_MUL: v.i = (int64_t)(x * y); break;
                    case VEXQ_OP_DIV: v.i = b.i == 0 ? 0 : b.i == -1 ? (int64_t)(0ull - x) : a.i / b.i; break;
                }
            }
            return v;
        }
        case NK::Cast: {
            const HVal a = E(0);
            v.ok = a.ok;
            v.d = (double)a.i;
            return v;
        }
        case NK::And:
        case NK::Or: {
            const bool isand = n.k == NK::And;
            for (size_t k = 0; k < n.ch.size(); k++) {
                const HVal a = E((int)k);
                if (k == 0) { v.b = a.b; v.ok = a.ok; }
                else if (isand) { v.b = v.b && a.b; v.ok = v.ok && a.ok; }
                else { v.b = v.b || a.b; v.ok = v.ok || a.ok; }
            }
            return v;
        }
        case NK::Not: {
            const HVal a = E(0);
            v.ok = a.ok;
            v.b = a.b != a.ok;
            return v;
        }
        case NK::IsNull:
        case NK::IsNotNull: {
            const HVal a = E(0);
            v.ok = true;
            v.b = n.k == NK::IsNull ? !a.ok : a.ok;
            return v;
        }
        case NK::InInt:
        case NK::InFloat: {
            const HVal a = E(0);
            v.ok = a.ok;
            bool in = false;
            if (n.k == NK::InInt) { for (auto x : n.seti) in = in || a.i == x; }
            else { for (auto x : n.setf) in = in || a.d == x; }
            v.b = a.ok && in;
            return v;
        }
        case NK::InFalse:
            v.ok = E(0).ok;
            return v;
        case NK::InCodes: {
            const HVal a = E(0);
            v.ok = a.ok;
            v.b = a.ok && (uint64_t)a.i < n.codes.size() && n.codes[(size_t)a.i];
            return v;
        }
        case NK::StrEq: {
            if (n.streq_code < 0) { v.ok = v.b = n.negate; return v; }  // literal in no dictionary
            const HVal a = E(0);
            v.ok = a.ok;
            v.b = a.ok && ((a.i == n.streq_code) != n.negate);
            return v;
        }
        case NK::Case: {
            const int nw = (int)(n.ch.size() - (n.has_else ? 1 : 0)) / 2;
            for (int w = 0; w < nw; w++) {
                const HVal c = E(2 * w);
                if (c.ok && c.b) return E(2 * w + 1);
            }
            if (n.has_else) return E((int)n.ch.size() - 1);
            return v;
        }
    }
    return v;
}

vexq_result_s* build_result(Plan& p, Groups& g) {
    auto* r = new vexq_result_s;
    size_t n = g.n();
    bool emptyGlobal = n == 0 && p.keys.empty();
    // insertion order: first-occurrence order key
    std::vector<size_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0);
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return g.first[a] < g.first[b]; });
    size_t rows = emptyGlobal ? 1 : n;
    r->nrows = (int64_t)rows;
    // group-by columns
    for (size_t ki = 0; ki < p.keys.size(); ki++) {
        const KeyCol& k = p.keys[ki];
        const Table* tt = k.build ? p.bt : p.t;
        const Column& col = tt->cols[k.col];
        OutColumn oc;
        oc.name = k.name.empty() ? col.name : k.name;
        oc.type = k.type;
        oc.v.assign(rows, 0);
        oc.valid.assign(rows, 0);
        if (k.type == VEXQ_TYPE_STRING) oc.dict = &col.dict;
        int64_t stride = 1;
        for (size_t kj = 0; kj < ki; kj++) stride *= p.keys[kj].domain > 0 ? p.keys[kj].domain : 1;
        for (size_t j = 0; j < n; j++) {
            uint64_t key = g.key[idx[j]];
            int64_t code;
            bool isnull = false;
            if (p.path != AggPath::Hash) {
                code = (int64_t)((key / (uint64_t)stride) % (uint64_t)k.domain);
                isnull = k.nullable && code == k.domain - 1;
            } else {
                uint64_t m = k.bits >= 64 ? ~0ull : ((1ull << k.bits) - 1);
                uint64_t raw = (key >> k.shift) & m;
                if (k.domain > 0) { code = (int64_t)raw; isnull = k.nullable && code == k.domain - 1; }
                else if (k.type == VEXQ_TYPE_DATE) { isnull = (raw >> 32) & 1; code = (int64_t)(int32_t)(uint32_t)raw; }
                else code = (int64_t)raw;
            }
            if (isnull) continue;
            oc.valid[j] = 1;
            if (k.domain > 0 && (k.type == VEXQ_TYPE_DATE || k.type == VEXQ_TYPE_INT64)) oc.v[j] = code + k.vmin;
            else oc.v[j] = code;
        }
        r->cols.push_back(std::move(oc));
    }
    // aggregates
    for (auto& a : p.outs) {
        OutColumn oc;
        oc.name = a.name;
        oc.type = a.out_type;
        oc.v.assign(rows, 0);
        oc.valid.assign(rows, 0);
        if (a.rank_dict) oc.dict = a.rank_dict;  // string MIN/MAX: codes of this dictionary
        if (emptyGlobal) {
            if (a.kind == VEXQ_AGG_COUNT) oc.valid[0] = 1;
            r->cols.push_back(std::move(oc));
            continue;
        }
        for (size_t j = 0; j < n; j++) {
            size_t i = idx[j];
            int64_t nn = slot_int(p, g, a.nn_slot, i);
            if (a.kind == VEXQ_AGG_COUNT) { oc.valid[j] = 1; oc.v[j] = slot_int(p, g, a.value_slot, i); continue; }
            if (nn == 0) continue;
            oc.valid[j] = 1;
            const Slot& sl = p.slots[a.value_slot];
            if (a.kind == VEXQ_AGG_AVG) {
                double v = slot_float(p, g, a.value_slot, i) / (double)nn;
                std::memcpy(&oc.v[j], &v, 8);
            } else if (sl.is_float()) {
                double v = slot_float(p, g, a.value_slot, i);
                std::memcpy(&oc.v[j], &v, 8);
            } else {
                int64_t v = slot_int(p, g, a.value_slot, i);
                if (a.rank_dict) {  // the winning rank back to its code
                    if (v < 0 || (size_t)v >= a.rank_code.size()) fail(VEXQ_EDEVICE, "string MIN/MAX rank out of range");
                    v = a.rank_code[(size_t)v];
                }
                if (a.out_type == VEXQ_TYPE_DATE) v = (int64_t)(int32_t)v;
                if (a.out_type == VEXQ_TYPE_BOOL) v = v != 0;
                oc.v[j] = v;
            }
        }
        r->cols.push_back(std::move(oc));
    }
    // HAVING: keep the rows whose predicate is true and valid, then drop the
    // hidden columns
    if (p.having_root >= 0 && !g.having_done) {
        std::vector<size_t> keep;
        for (size_t j = 0; j < rows; j++) {
            const HVal h = having_eval(p.having_ir, p.having_root, r->cols, j);
            if (h.ok && h.b) keep.push_back(j);
        }
        if (keep.size() != rows) {
            for (auto& c : r->cols) {
                for (size_t j = 0; j < keep.size(); j++) { c.v[j] = c.v[keep[j]]; c.valid[j] = c.valid[keep[j]]; }
                c.v.resize(keep.size());
                c.valid.resize(keep.size());
            }
            rows = keep.size();
            r->nrows = (int64_t)rows;
        }
    }
    if (p.having_root >= 0 && p.having_visible >= 0 && p.having_visible < (int)r->cols.size()) r->cols.resize(p.having_visible);
    // ORDER BY (stable, raw int64 bits, NULLs first) + LIMIT
    const vexq_order_desc& o = p.order;
    if (o.sort_col >= 0) {
        if (o.sort_col >= (int)r->cols.size()) fail(VEXQ_EINVAL, "ORDER BY column out of range");
        const OutColumn& k = r->cols[o.sort_col];
        std::vector<size_t> ord(rows);
        std::iota(ord.begin(), ord.end(), 0);
        std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
            bool an = !k.valid[a], bn = !k.valid[b];
            if (an && bn) return false;
            if (an) return true;
            if (bn) return false;
            if (k.type == VEXQ_TYPE_STRING) {
                const std::string &sa = k.dict->keys[k.v[a]], &sb = k.dict->keys[k.v[b]];
                if (sa == sb) return false;
                return o.descending ? sa > sb : sa < sb;
            }
            if (k.v[a] == k.v[b]) return false;
            return o.descending ? k.v[a] > k.v[b] : k.v[a] < k.v[b];
        });
        for (auto& c : r->cols) {
            std::vector<int64_t> v(rows);
            std::vector<uint8_t> va(rows);
            for (size_t j = 0; j < rows; j++) { v[j] = c.v[ord[j]]; va[j] = c.valid[ord[j]]; }
            c.v.swap(v);
            c.valid.swap(va);
        }
    }
    if (o.limit >= 0 && (size_t)o.limit < rows) {
        for (auto& c : r->cols) { c.v.resize(o.limit); c.valid.resize(o.limit); }
        r->nrows = o.limit;
    }
    own_dictionaries(r);
    return r;
}

void own_dictionaries(vexq_result_s* r) {
    for (OutColumn& oc : r->cols) {
        if (!oc.dict) continue;
        auto d = std::make_unique<GlobalDict>();
        std::unordered_map<int64_t, uint32_t> local;
        for (size_t j = 0; j < oc.v.size(); j++) {
            if (!oc.valid[j]) continue;
            const int64_t g = oc.v[j];
            if (g < 0 || (size_t)g >= oc.dict->keys.size()) fail(VEXQ_EDEVICE, "result string code outside its dictionary");
            auto it = local.find(g);
            if (it == local.end()) {
                it = local.emplace(g, (uint32_t)d->keys.size()).first;
                d->keys.push_back(oc.dict->keys[(size_t)g]);
            }
            oc.v[j] = it->second;
        }
        oc.dict = d.get();
        r->owned_dicts.push_back(std::move(d));
    }
}

long long estimate_groups(const Plan& p, long long rows, long long join_keys) {
    if (p.path != AggPath::Hash) return p.domain;
    long long est = rows;
    if (p.is_join) {
        // a group key containing the join key has at most (distinct build keys) × (other domains) groups
        long long other = 1;
        bool has_join_key = false;
        for (auto& k : p.keys) {
            bool jk = (k.build && k.col == p.build_key) || (!k.build && k.col == p.ir[p.probe_key].col);
            if (jk) has_join_key = true;
            else other *= k.domain > 0 ? k.domain : (1LL << 30);
            if (other > (1LL << 30)) other = 1LL << 30;
        }
        if (has_join_key) est = std::min<long long>(est, join_keys * other);
    }
    if (p.domain > 0) est = std::min<long long>(est, p.domain);
    return std::max<long long>(est, 1);
}

std::vector<uint8_t> prune_mask(const Plan& p, const Table& t, int root, int rgs, int rge) {
    std::vector<uint8_t> m(t.n_rg, 0);
    for (int rg = rgs; rg < rge; rg++) m[rg] = zone_eval(p, root, t, rg);
    return m;
}

// Runs the scan kernel over prepared params and returns host groups plus the
// compacted device arrays (atomic path) for top-k.
static vexq_result_s* finish_groups(RunCtx& rc, VQParams& P, long long nchunks, long long estimate, long long rows) {
    Plan& p = rc.p;
    Groups g;
    if (p.path == AggPath::Regs) {
        g = run_regs(rc, P, nchunks);
    } else {
        // ORDER BY an aggregate with a LIMIT and no HAVING: the top-k kernels
        // follow the table run without waiting for its count
        const bool defer = !p.partial_out && p.having_root < 0 && p.ndist == 0 && topk_applies(p, false);
        Compacted c = run_atomic(rc, P, nchunks, estimate, rows, defer);
        if (p.partial_out) {
            g = fetch_groups(rc, c);  // a shard's partial: every group, no HAVING, no LIMIT
        } else {
            if (p.k_having.fn) c = having_device(rc, c);
            int st = topk_groups(rc, c, g);
            if (st < 0) {  // the deferred run's hash table was too small: the sizing loop runs it again
                c = run_atomic(rc, P, nchunks, estimate, rows);
                st = topk_groups(rc, c, g);
            }
            if (st == 0) {
                g = fetch_groups(rc, c);
                g.having_done = c.having_done;
            }
        }
    }
    if (p.partial_out) {
        *p.partial_out = std::move(g);
        auto* r = new vexq_result_s;
        r->kernel_ms = rc.kernel_ms;
        r->scan_ms = rc.scan_ms;
        r->launches = rc.launches;
        return r;
    }
    note_hot_groups(p, g);
    vexq_result_s* r = build_result(p, g);
    r->kernel_ms = rc.kernel_ms;
    r->scan_ms = rc.scan_ms;
    r->launches = rc.launches;
    return r;
}

cudaStream_t plan_stream(Plan& p);

// A submitted register-path run: the launches are queued and the result
// settles on its first read (the sync, the merged row's decode and the
// result columns), so the host prepares the next run while this one runs.
static vexq_result_s* submit_regs(RunCtx& rc, VQParams& P, long long nchunks) {
    Plan& p = rc.p;
    const RegsPending q = regs_launch(rc, P, nchunks, true);
    auto* r = new vexq_result_s;
    Plan* pp = &p;
    const float k0 = rc.kernel_ms, s0 = rc.scan_ms;
    const int l0 = rc.launches;
    r->settle_fn = [pp, q, k0, s0, l0](vexq_result_s* res) {
        RunCtx rc2{*pp, plan_stream(*pp)};
        rc2.kernel_ms = k0;
        rc2.scan_ms = s0;
        rc2.launches = l0;
        Groups g = regs_collect(rc2, q);
        std::unique_ptr<vexq_result_s> full(build_result(*pp, g));
        const int64_t rows = res->rows_scanned, bytes = res->bytes_scanned;
        *res = std::move(*full);
        res->rows_scanned = rows;
        res->bytes_scanned = bytes;
        res->kernel_ms = rc2.kernel_ms;
        res->scan_ms = rc2.scan_ms;
        res->launches = rc2.launches;
    };
    r->owner = pp;
    p.pending = r;
    return r;
}

void settle(vexq_result_s* r) {
    if (!r) return;
    if (r->settle_code) fail(r->settle_code, r->settle_msg);
    if (!r->settle_fn) return;
    std::function<void(vexq_result_s*)> f = std::move(r->settle_fn);
    r->settle_fn = nullptr;
    if (r->owner && r->owner->pending == r) r->owner->pending = nullptr;
    r->owner = nullptr;
    try {
        f(r);
    } catch (const Status& e) {
        r->settle_code = e.code;
        r->settle_msg = e.what();
        throw;
    }
}

void settle_pending(Plan& p) {
    if (!p.pending) return;
    try {
        settle(p.pending);
    } catch (const Status&) {
        // kept in the pending result: its next read returns the status
    }
}

void note_hot_groups(Plan& p, const Groups& g) {
    if (p.hot_n <= 0 || p.path != AggPath::Dense || p.is_join || g.key.empty()) return;
    int cs = -1;
    for (size_t s = 0; s < p.slots.size(); s++)
        if (p.slots[s].kind == S_CNT) { cs = (int)s; break; }
    if (cs < 0) return;
    const std::vector<int64_t>& cnt = g.ival[p.slot_pos[cs]];
    std::vector<size_t> idx(g.key.size());
    std::iota(idx.begin(), idx.end(), 0);
    const size_t k = std::min<size_t>((size_t)p.hot_n, idx.size());
    std::partial_sort(idx.begin(), idx.begin() + k, idx.end(), [&](size_t a, size_t b) {
        return cnt[a] != cnt[b] ? cnt[a] > cnt[b] : g.key[a] < g.key[b];
    });
    std::vector<unsigned long long> hot;
    for (size_t i = 0; i < k; i++) hot.push_back((unsigned long long)g.key[idx[i]]);
    std::lock_guard<std::mutex> lk(p.hot_mu);
    p.hot_keys = hot;
}

int64_t scanned_bytes(const Plan& p, const Table& t, long long rows, bool build) {
    // algorithmic bytes: reference width of every column of `t` the scan reads × rows
    std::set<int> cols;
    std::function<void(int)> walk = [&](int i) {
        if (i < 0) return;
        const INode& n = p.ir[i];
        if (n.k == NK::Col && n.tab == &t && !n.build) cols.insert(n.col);
        for (int c : n.ch) walk(c);
    };
    if (build) {
        walk(p.bpred);
        cols.insert(p.build_key);
    } else {
        walk(p.pred);
        if (p.is_join) { walk(p.probe_key); walk(p.resid); }
        for (auto& k : p.keys) if (!k.build) cols.insert(k.col);
        for (auto& s : p.slots) walk(s.input);
    }
    int64_t w = 0;
    for (int c : cols) {
        int ty = t.cols[c].type;
        w += (ty == VEXQ_TYPE_INT64 || ty == VEXQ_TYPE_FLOAT64) ? 8 : (ty == VEXQ_TYPE_BOOL ? 1 : 4);
    }
    return w * rows;
}

std::mutex& plan_mutex(Plan* p) {
    static std::mutex m;
    static std::map<Plan*, std::unique_ptr<std::mutex>> mus;
    std::lock_guard<std::mutex> lk(m);
    auto& u = mus[p];
    if (!u) u.reset(new std::mutex);
    return *u;
}

bool launch_checks_on() {
    static const bool on = [] {
        const char* e = std::getenv("VEXQ_SYNC_CHECK");
        return e && *e && *e != '0';
    }();
    return on;
}

void launch_check(cudaStream_t s, const char* what) {
    if (!launch_checks_on()) return;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) fail(VEXQ_EDEVICE, std::string("after ") + what + ": " + cudaGetErrorString(e));
}

cudaStream_t plan_stream(Plan& p) {
    if (p.ext_stream) return p.ext_stream;
    if (!p.stream) VQ_CUDA(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
    return p.stream;
}

// Sets " name=value" in the plan's explain string (appended the first time).
static void explain_tag(Plan& p, const std::string& name, const std::string& value) {
    const std::string k = " " + name + "=";
    const size_t at = p.explain.find(k);
    if (at != std::string::npos) {
        const size_t end = p.explain.find(' ', at + 1);
        if (p.explain.compare(at + k.size(), (end == std::string::npos ? p.explain.size() : end) - at - k.size(), value) == 0) return;
        p.explain.erase(at, end == std::string::npos ? std::string::npos : end - at);
    }
    p.explain += k + value;
}

// One radix partition pass over a side (Q: its columns, row ranges, filter
// inputs): histogram, partition-major scan, starts, then — unless a
// partition exceeds the shared-memory capacity and *maxpart is asked for —
// the scatter of (key, row) into keys/rows. Returns the entries written.
static long long radix_pass(RunCtx& rc, const JitKernel& kp, VQParams Q, int pbits, long long* d_starts, DevBuf& keys,
                            DevBuf& rows, long long* maxpart, int cap) {
    Plan& p = rc.p;
    const int np = 1 << pbits;
    const int grid = grid_for(kp, Q.nchunks, false);
    const long long n = (long long)np * grid;
    p.rp_hist.ensure(n * 4);
    p.rp_off.ensure(n * 4);
    const int nbk = (int)((n + 4095) / 4096);
    p.rp_scalar.ensure((size_t)(nbk + 16) * 4);
    Q.nparts = np;
    Q.pbits = pbits;
    Q.mode = 0;
    Q.phist = p.rp_hist.as<int>();
    JitKernel k = kp;
    k.smem = np * 4;
    jit_launch(k, grid, &Q, sizeof Q, rc.s);
    launch_check(rc.s, "vq_part (histogram)");
    int* off = p.rp_off.as<int>();
    int* bsums = p.rp_scalar.as<int>();
    k_scan_blocks<<<nbk, 1024, 0, rc.s>>>(Q.phist, off, n, bsums);
    launch_check(rc.s, "k_scan_blocks");
    k_scan_sums<<<1, 1024, 0, rc.s>>>(bsums, nbk);
    launch_check(rc.s, "k_scan_sums");
    k_scan_add<<<(int)((n + 255) / 256), 256, 0, rc.s>>>(off, n, bsums);
    launch_check(rc.s, "k_scan_add");
    k_part_starts<<<(np + 1 + 255) / 256, 256, 0, rc.s>>>(off, Q.phist, np, grid, d_starts);
    launch_check(rc.s, "k_part_starts");
    std::vector<long long> hs(np + 1);
    VQ_CUDA(cudaMemcpyAsync(hs.data(), d_starts, (size_t)(np + 1) * 8, cudaMemcpyDeviceToHost, rc.s));
    VQ_CUDA(cudaStreamSynchronize(rc.s));
    rc.launches += 5;
    const long long total = hs[np];
    if (maxpart) {
        long long mx = 0;
        for (int i = 0; i < np; i++) mx = std::max(mx, hs[i + 1] - hs[i]);
        *maxpart = mx;
        if (mx > cap) return total;
    }
    keys.ensure((size_t)std::max<long long>(total, 1) * 8);
    rows.ensure((size_t)std::max<long long>(total, 1) * 4);
    Q.mode = 1;
    Q.phist = off;
    Q.pkeys = keys.as<unsigned long long>();
    Q.prows = rows.as<int>();
    jit_launch(k, grid, &Q, sizeof Q, rc.s);
    launch_check(rc.s, "vq_part (scatter)");
    rc.launches += 1;
    return total;
}

// The next run speculates (vexq_debug_join_spec): the state a direct-mapped
// build over the current build rows with keys_seen keys would have left.
void force_join_spec(Plan& p, long long keys_seen) {
    Table& bt = *p.bt;
    std::vector<uint8_t> bm = prune_mask(p, bt, p.zn_bpred, 0, bt.n_rg);
    const ScanSegs bs = make_segments(bt, bm, 0, bt.n_rg, p.btile);
    p.dmap_failed = false;
    p.dmap_used = true;
    p.join_rows_seen = bs.rows;
    p.join_keys_seen = keys_seen;
    p.gid_groups = keys_seen;
}

vexq_result_s* run_plan(Plan& p, int rg_start, int rg_end) {
    settle_pending(p);  // the last submitted run's output is still in the staging buffer
    if (p.cancel.load()) { p.cancel = false; fail(VEXQ_ECANCELED, "plan cancelled"); }
    check_ranges(p);
    RunCtx rc{p, plan_stream(p)};
    VQParams P;
    std::memset(&P, 0, sizeof P);
    set_plan_constants(p, P);
    Table& t = *p.t;
    int rge = rg_end < 0 ? t.n_rg : std::min(rg_end, t.n_rg);
    int rgs = std::max(0, rg_start);
    long long join_keys = 0;
    int64_t bytes = 0, rows_scanned = 0;
    bool use_radix = false;
    bool spec = false;  // the probe follows a direct-mapped build without the host waiting
    int pbits = 0;
    if (p.is_join) {
        Table& bt = *p.bt;
        // ---- build phase ----
        std::vector<uint8_t> bm = prune_mask(p, bt, p.zn_bpred, 0, bt.n_rg);
        ScanSegs bs = make_segments(bt, bm, 0, bt.n_rg, p.btile);
        // radix partitioning (RadixBitsFor, exec/parallel_join.go:72-89): none
        // below 65,536 build rows; partitions sized to fit shared memory
        // automatic choice: the global table until partitioning measures faster
        // (VEXQ_RADIX=1 partitions with automatic bits, for measurement)
        static const bool radix_env = std::getenv("VEXQ_RADIX") && std::getenv("VEXQ_RADIX")[0] == '1';
        use_radix = p.radix && !p.staged && p.btile == 128 && p.tile == 128 &&
                    (p.radix_bits > 0 || (p.radix_bits < 0 && radix_env && bs.rows >= 65536));
        if (use_radix) {
            VQParams B;
            std::memset(&B, 0, sizeof B);
            set_plan_constants(p, B);
            set_columns(B, bt, false);
            if (bs.seg != p.bseg_cache || !p.d_bseg.p) {
                p.d_bseg.ensure(std::max<size_t>(bs.seg.size(), 3) * 8);
                h2d(p.d_bseg.p, bs.seg.data(), bs.seg.size() * 8, rc.s);
                p.bseg_cache = bs.seg;
            }
            B.seg = p.d_bseg.as<long long>();
            B.nseg = (int)bs.seg.size() / 3;
            B.nchunks = bs.nchunks;
            B.rg_rows = bt.rg_rows;
            B.n_rg = bt.n_rg;
            B.present = p.d_bpresent.as<unsigned char>();
            for (size_t i = 0, off = 0; i < p.sets.size(); i++) { B.sets[i] = p.d_sets.as<unsigned>() + off; off += p.sets[i].size(); }
            if (p.radix_bits > 0) {
                pbits = std::min(p.radix_bits, VQ_RADIX_MAX_BITS);
            } else {
                pbits = 1;
                while (pbits < VQ_RADIX_MAX_BITS && (bs.rows >> pbits) > p.rcap / 2) pbits++;
            }
            p.rp_start.ensure((size_t)2 * ((1 << VQ_RADIX_MAX_BITS) + 1) * 8);
            long long* bstart = p.rp_start.as<long long>();
            ensure_events(p);
            VQ_CUDA(cudaEventRecord(p.ev[4], rc.s));
            long long total = 0;
            for (;;) {
                long long mx = 0;
                total = bs.nchunks > 0 ? radix_pass(rc, p.k_part_b, B, pbits, bstart, p.rp_bkeys, p.rp_brows, &mx, p.rcap) : 0;
                if (mx <= p.rcap) break;
                if (pbits >= VQ_RADIX_MAX_BITS) { use_radix = false; break; }  // one key's chain is too long: global table
                while (pbits < VQ_RADIX_MAX_BITS && mx > p.rcap) { pbits++; mx = (mx + 1) / 2; }
            }
            VQ_CUDA(cudaEventRecord(p.ev[5], rc.s));
            VQ_CUDA(cudaEventSynchronize(p.ev[5]));
            rc.kernel_ms += elapsed(p.ev[4], p.ev[5]);
            if (use_radix) {
                bytes += scanned_bytes(p, bt, bs.rows, true);
                rows_scanned += bs.rows;
                join_keys = total;  // at least the distinct build keys
                set_columns(P, bt, true);
                P.bstart = bstart;
                P.bkeys = p.rp_bkeys.as<unsigned long long>();
                P.brows = p.rp_brows.as<int>();
                P.nparts = 1 << pbits;
                P.pbits = pbits;
                if (total == 0 || bs.nchunks == 0) {  // empty build: the join emits nothing (parallel_join.go:790-795)
                    Groups g;
                    g.ival.assign(p.ni, {});
                    g.fval.assign(p.nf, {});
                    vexq_result_s* r = build_result(p, g);
                    r->kernel_ms = rc.kernel_ms;
                    r->launches = rc.launches;
                    r->rows_scanned = rows_scanned;
                    r->bytes_scanned = bytes;
                    return r;
                }
            }
        }
    }
    if (p.is_join && !use_radix) {
        Table& bt = *p.bt;
        ScanMemo& bmemo = p.build_memo;  // the build side's pruning, kept until its zone maps change
        if (bmemo.zone_version != bt.zone_version || bmemo.rgs != 0 || bmemo.rge != bt.n_rg) {
            std::vector<uint8_t> bm = prune_mask(p, bt, p.zn_bpred, 0, bt.n_rg);
            bmemo.ss = make_segments(bt, bm, 0, bt.n_rg, p.btile);
            bmemo.zone_version = bt.zone_version;
            bmemo.rgs = 0;
            bmemo.rge = bt.n_rg;
        }
        const ScanSegs& bs = bmemo.ss;
        // build table: twice the distinct keys the last build found (scaled by
        // the rows scanned), else twice the rows; a build that hits the probe
        // limit reruns at the row-bounded size (a table sized by rows leaves
        // most slots empty, and every per-slot pass pays for them)
        long long jsafe = 16;
        while (jsafe < 2 * std::max<long long>(bs.rows, 8)) jsafe <<= 1;
        long long jcap = jsafe;
        if (p.join_keys_seen >= 0) {
            const double scale = std::max(1.0, (double)bs.rows / (double)std::max<long long>(p.join_rows_seen, 1));
            const long long est = std::min<long long>(bs.rows, std::max<long long>((long long)(p.join_keys_seen * scale), 1024));
            jcap = 16;
            while (jcap < 2 * std::max<long long>(est, 8)) jcap <<= 1;
        }
        VQParams B;
        std::memset(&B, 0, sizeof B);
        set_plan_constants(p, B);
        set_columns(B, bt, false);
        if (bs.seg != p.bseg_cache || !p.d_bseg.p) {  // uploaded once per distinct pruning
            p.d_bseg.ensure(std::max<size_t>(bs.seg.size(), 3) * 8);
            h2d(p.d_bseg.p, bs.seg.data(), bs.seg.size() * 8, rc.s);
            p.bseg_cache = bs.seg;
        }
        B.seg = p.d_bseg.as<long long>();
        B.nseg = (int)bs.seg.size() / 3;
        B.nchunks = bs.nchunks;
        B.rg_rows = bt.rg_rows;
        B.n_rg = bt.n_rg;
        B.present = p.d_bpresent.as<unsigned char>();
        B.sets[0] = nullptr;
        for (size_t i = 0, off = 0; i < p.sets.size(); i++) { B.sets[i] = p.d_sets.as<unsigned>() + off; off += p.sets[i].size(); }
        // keys unique in the last build (the primary-key side of a join): one
        // pass straight into the probe's 16-byte slots
        bool fast_unique = p.fast_build && p.join_unique_seen && !p.join_fast_failed;
        // a build key column whose value range is at most a few times its rows
        // (dense primary keys): a word per key value, indexed by key - imin,
        // one CAS a build row and one load a probe row, no hashing or packing
        const Column& bkc = bt.cols[p.build_key];
        bool direct = false;
        long long dmin = 0;
        unsigned long long drange = 0;
        if (p.dmap_on && !p.dmap_failed && bkc.has_range && bkc.imax >= bkc.imin) {
            const __int128 r = (__int128)bkc.imax - (__int128)bkc.imin + 1;
            if (r <= ((__int128)1 << 31) && r <= 4 * (__int128)std::max<int64_t>(bt.nrows, 1) + 65536) {
                direct = true;
                dmin = bkc.imin;
                drange = (unsigned long long)r;
            }
        }
        // the last build was direct-mapped over the same rows: this one is
        // launched and the probe follows without the host waiting for it (the
        // group table sized from the last build's key count); the probe
        // raises a failed, empty or larger build in its error word
        spec = direct && p.dmap_used && p.join_rows_seen == bs.rows && p.join_keys_seen > 0 && p.spec_on;
        p.dmap_used = false;
        for (;;) {
        if (direct) {
            p.jt_scalar.ensure(64);
            p.jt_gid.ensure(8);  // a non-null flag: group numbers are handed out
            p.jt_gkey.ensure((size_t)std::max<long long>(bs.rows, 1) * 8);
            p.jt_dmap.ensure((size_t)drange * 8);
            B.jnkeys = p.jt_scalar.as<unsigned long long>();
            B.error = (int*)(p.jt_scalar.as<char>() + 8);
            B.jtotal = (unsigned long long*)(p.jt_scalar.as<char>() + 24);
            ensure_events(p);
            VQ_CUDA(cudaEventRecord(p.ev[4], rc.s));
            VQ_CUDA(cudaMemsetAsync(p.jt_scalar.p, 0, 40, rc.s));
            VQ_CUDA(cudaMemsetAsync(p.jt_dmap.p, 0, (size_t)drange * 8, rc.s));
            VQParams F = B;
            F.mode = 3;
            F.dmap = p.jt_dmap.as<unsigned long long>();
            F.dmin = dmin;
            F.drange = drange;
            F.jgid = p.join_gid ? p.jt_gid.as<int>() : nullptr;
            F.jgkey = p.jt_gkey.as<unsigned long long>();
            F.jgoff = p.gid_koff;
            if (bs.nchunks > 0) {
                jit_launch(p.k_build, grid_for(p.k_build, bs.nchunks, p.staged), &F, sizeof F, rc.s);
                launch_check(rc.s, "p.k_build (direct-mapped)");
            }
            rc.launches += 1;
            if (spec) {
                VQ_CUDA(cudaEventRecord(p.ev[5], rc.s));
                p.dmap_used = true;
                join_keys = p.join_keys_seen;
                break;
            }
            int herr = 0;
            unsigned long long nk = 0, ntot = 0;
            VQ_CUDA(cudaMemcpyAsync(&herr, B.error, 4, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaMemcpyAsync(&nk, B.jnkeys, 8, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaMemcpyAsync(&ntot, B.jtotal, 8, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaEventRecord(p.ev[5], rc.s));
            VQ_CUDA(cudaStreamSynchronize(rc.s));
            rc.kernel_ms += elapsed(p.ev[4], p.ev[5]);
            if (herr & 8) fail(VEXQ_ETIMEDOUT, "a staged tile copy did not complete within the kernel's wait limit");
            if (!(herr & (16 | 32)) && nk == ntot) {
                p.dmap_used = true;
                join_keys = (long long)nk;
                p.gid_groups = join_keys;
                p.join_keys_seen = join_keys;
                p.join_rows_seen = bs.rows;
                break;
            }
            // a repeated key (or a key outside the column's recorded range):
            // the hash table from here on
            p.dmap_failed = true;
            direct = false;
            continue;
        }
        long long nslots = jcap + 1;
        p.jt_keys.ensure(nslots * 8);
        p.jt_count.ensure(nslots * 4);
        p.jt_start.ensure(nslots * 4);
        p.jt_fill.ensure(nslots * 4);
        p.jt_rows.ensure(std::max<long long>(bs.rows, 1) * 4);
        p.jt_meta.ensure(nslots * 16);
        p.jt_first.ensure(nslots * 4);
        p.jt_gid.ensure(nslots * 4);
        p.jt_gkey.ensure(nslots * 8);
        p.jt_scalar.ensure(64 + ((nslots + 4095) / 4096 + 1) * 4);
        B.jkeys = p.jt_keys.as<unsigned long long>();
        B.jcount = p.jt_count.as<int>();
        B.jstart = p.jt_start.as<int>();
        B.jfill = p.jt_fill.as<int>();
        B.jrows = p.jt_rows.as<int>();
        B.jfirst = p.jt_first.as<int>();
        B.jnkeys = p.jt_scalar.as<unsigned long long>();
        B.error = (int*)(p.jt_scalar.as<char>() + 8);
        B.jtotal = (unsigned long long*)(p.jt_scalar.as<char>() + 24);
        B.jgid = p.jt_gid.as<int>();
        unsigned long long* d_ngid = (unsigned long long*)(p.jt_scalar.as<char>() + 32);
        int* bsums = (int*)(p.jt_scalar.as<char>() + 64);
        B.jmask = (unsigned long long)(jcap - 1);
        if (fast_unique) {
            // one CAS a row on the slot's key word, then the chain word (the
            // build row; with GROUP BY the join key, the key's group number,
            // claimed once per warp and chunk); no per-slot counts, chain
            // pass or packing pass. A repeated key (bit 16) or a full table
            // (bit 0) sends this build to the general path below.
            ensure_events(p);
            VQ_CUDA(cudaEventRecord(p.ev[4], rc.s));
            VQ_CUDA(cudaMemsetAsync(p.jt_scalar.p, 0, 40, rc.s));
            static_assert(VQ_EMPTY_KEY == ~0ull, "the empty-key fill is a byte memset");
            VQ_CUDA(cudaMemsetAsync(p.jt_meta.p, 0xFF, (size_t)jcap * 16, rc.s));
            VQ_CUDA(cudaMemsetAsync(p.jt_meta.as<char>() + (size_t)jcap * 16, 0, 16, rc.s));
            VQParams F = B;
            F.mode = 2;
            F.jslot = p.jt_meta.as<ulonglong2>();
            F.jgid = p.join_gid ? B.jgid : nullptr;
            F.jgkey = p.jt_gkey.as<unsigned long long>();
            F.jgoff = p.gid_koff;
            if (bs.nchunks > 0) {
                jit_launch(p.k_build, grid_for(p.k_build, bs.nchunks, p.staged), &F, sizeof F, rc.s);
                launch_check(rc.s, "p.k_build (unique keys)");
            }
            int herr = 0;
            unsigned long long nk = 0, ntot = 0;
            VQ_CUDA(cudaMemcpyAsync(&herr, B.error, 4, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaMemcpyAsync(&nk, B.jnkeys, 8, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaMemcpyAsync(&ntot, B.jtotal, 8, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaEventRecord(p.ev[5], rc.s));
            VQ_CUDA(cudaStreamSynchronize(rc.s));
            rc.kernel_ms += elapsed(p.ev[4], p.ev[5]);
            rc.launches += 1;
            if (herr & 8) fail(VEXQ_ETIMEDOUT, "a staged tile copy did not complete within the kernel's wait limit");
            if (!(herr & (1 | 16)) && nk == ntot) {
                p.join_unique_seen = true;
                join_keys = (long long)nk;
                p.gid_groups = join_keys;
                p.join_keys_seen = join_keys;
                p.join_rows_seen = bs.rows;
                break;
            }
            fast_unique = false;
            p.join_fast_failed = (herr & 16) != 0;  // keys repeat now: the general build from here on
            if (herr & 1) jcap = jsafe;
            continue;
        }
        {
            ensure_events(p);
            VQ_CUDA(cudaEventRecord(p.ev[4], rc.s));
            VQ_CUDA(cudaMemsetAsync(p.jt_scalar.p, 0, 40, rc.s));
            VQ_CUDA(cudaMemsetAsync(B.jcount, 0, nslots * 4, rc.s));
            VQ_CUDA(cudaMemsetAsync(B.jfill, 0, nslots * 4, rc.s));
            int ig = (int)std::min<long long>((nslots + 255) / 256, (long long)sm_count() * 16);
            static_assert(VQ_EMPTY_KEY == ~0ull, "the empty-key fill is a byte memset");
            VQ_CUDA(cudaMemsetAsync(B.jkeys, 0xFF, (size_t)jcap * 8, rc.s));
            VQ_CUDA(cudaMemsetAsync(B.jkeys + jcap, 0, 8, rc.s));
            B.mode = 0;
            int grid = grid_for(p.k_build, bs.nchunks, p.staged);
            if (bs.nchunks > 0) jit_launch(p.k_build, grid, &B, sizeof B, rc.s);
            if (bs.nchunks > 0) launch_check(rc.s, "p.k_build");
            // keys, inserted rows and errors of pass 0; a build whose keys never
            // repeat needs no row lists: every chain is its slot's first row
            int herr = 0, nlong = 0;
            unsigned long long nk = 0, ntot = 0;
            VQ_CUDA(cudaMemcpyAsync(&herr, B.error, 4, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaMemcpyAsync(&nk, B.jnkeys, 8, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaMemcpyAsync(&ntot, B.jtotal, 8, cudaMemcpyDeviceToHost, rc.s));
            VQ_CUDA(cudaStreamSynchronize(rc.s));
            const bool unique = nk == ntot && !(herr & 1);
            p.join_unique_seen = unique && nk > 0;
            if (!unique && !(herr & 1)) {
                int nb = (int)((nslots + 4095) / 4096);
                k_scan_blocks<<<nb, 1024, 0, rc.s>>>(B.jcount, B.jstart, nslots, bsums);
                launch_check(rc.s, "k_scan_blocks");
                k_scan_sums<<<1, 1024, 0, rc.s>>>(bsums, nb);
                launch_check(rc.s, "k_scan_sums");
                k_scan_add<<<(int)((nslots + 255) / 256), 256, 0, rc.s>>>(B.jstart, nslots, bsums);
                launch_check(rc.s, "k_scan_add");
                B.mode = 1;
                if (bs.nchunks > 0) jit_launch(p.k_build, grid, &B, sizeof B, rc.s);
                if (bs.nchunks > 0) launch_check(rc.s, "p.k_build");
                const int long_cap = (int)(bs.rows / (kShortChain + 1) + 2);
                p.jt_long.ensure((size_t)long_cap * 8);
                int* long_count = (int*)(p.jt_scalar.as<char>() + 16);
                k_sort_chains<<<ig, 256, 0, rc.s>>>(B.jstart, B.jcount, B.jrows, nslots, B.error, p.jt_long.as<int2>(),
                                                    long_count, long_cap);
                launch_check(rc.s, "k_sort_chains");
                VQ_CUDA(cudaMemcpyAsync(&herr, B.error, 4, cudaMemcpyDeviceToHost, rc.s));
                VQ_CUDA(cudaMemcpyAsync(&nlong, long_count, 4, cudaMemcpyDeviceToHost, rc.s));
                VQ_CUDA(cudaStreamSynchronize(rc.s));
                if (nlong > 0 && !(herr & 4)) {  // long chains: one block each, scratch for the power-of-two pad
                    std::vector<int2> lst(nlong);
                    VQ_CUDA(cudaMemcpyAsync(lst.data(), p.jt_long.p, (size_t)nlong * 8, cudaMemcpyDeviceToHost, rc.s));
                    VQ_CUDA(cudaStreamSynchronize(rc.s));
                    std::vector<long long> soff(nlong);
                    long long tot = 0;
                    for (int i = 0; i < nlong; i++) {
                        long long m = 1;
                        while (m < lst[i].y) m <<= 1;
                        soff[i] = tot;
                        tot += m;
                    }
                    p.jt_sort.ensure((size_t)tot * 4 + (size_t)nlong * 8);
                    long long* d_soff = (long long*)(p.jt_sort.as<char>() + (size_t)tot * 4);
                    VQ_CUDA(cudaMemcpyAsync(d_soff, soff.data(), (size_t)nlong * 8, cudaMemcpyHostToDevice, rc.s));
                    k_sort_long<<<nlong, 1024, 0, rc.s>>>(p.jt_long.as<int2>(), B.jstart, B.jrows, p.jt_sort.as<int>(), d_soff);
                    launch_check(rc.s, "k_sort_long");
                    rc.launches += 1;
                }
                rc.launches += 5;
            }
            k_pack_slots<<<(int)std::min<long long>((nslots + 1023) / 1024, (long long)sm_count() * 16), 256, 0, rc.s>>>(
                B.jkeys, B.jstart, B.jcount, B.jfirst, p.join_gid ? 1 : 0, B.jgid, p.jt_gkey.as<unsigned long long>(), d_ngid,
                p.gid_koff, p.jt_meta.as<ulonglong2>(), nslots);
            launch_check(rc.s, "k_pack_slots");
            VQ_CUDA(cudaGetLastError());
            VQ_CUDA(cudaEventRecord(p.ev[5], rc.s));
            VQ_CUDA(cudaEventSynchronize(p.ev[5]));
            rc.kernel_ms += elapsed(p.ev[4], p.ev[5]);
            rc.launches += 2;
            if (herr & 8) fail(VEXQ_ETIMEDOUT, "a staged tile copy did not complete within the kernel's wait limit");
            if (herr & 1) {
                if (jcap >= jsafe) fail(VEXQ_EDEVICE, "join build table probe limit reached");
                jcap = jsafe;  // the last build's key count was too small a guess
                continue;
            }
            if (herr & 4) fail(VEXQ_EDEVICE, "join build: more long chains than the sort list holds");
            join_keys = (long long)nk;
            p.gid_groups = join_keys;
            p.join_keys_seen = join_keys;
            p.join_rows_seen = bs.rows;
        }
        break;
        }
        explain_tag(p, "build", direct ? "direct" : "hash");
        bytes += scanned_bytes(p, bt, bs.rows, true);
        rows_scanned += bs.rows;
        // ---- probe phase parameters ----
        set_columns(P, bt, true);
        P.jkeys = B.jkeys;
        P.jcount = B.jcount;
        P.jstart = B.jstart;
        P.jrows = B.jrows;
        P.jslot = p.jt_meta.as<ulonglong2>();
        P.jgid = p.jt_gid.as<int>();
        P.jmask = B.jmask;
        P.dmap = direct ? p.jt_dmap.as<unsigned long long>() : nullptr;
        P.dmin = dmin;
        P.drange = drange;
        P.berr = spec ? (const int*)(p.jt_scalar.as<char>() + 8) : nullptr;
        P.bnk = spec ? p.jt_scalar.as<unsigned long long>() : nullptr;
        if (join_keys == 0) {  // empty build: the join emits nothing (parallel_join.go:790-795)
            Groups g;
            g.ival.assign(p.ni, {});
            g.fval.assign(p.nf, {});
            vexq_result_s* r = build_result(p, g);
            r->kernel_ms = rc.kernel_ms;
            r->launches = rc.launches;
            r->rows_scanned = rows_scanned;
            r->bytes_scanned = bytes;
            return r;
        }
    }
    ScanMemo& sm = p.scan_memo;
    if (sm.rgs != rgs || sm.rge != rge || sm.zone_version != t.zone_version) {
        std::vector<uint8_t> m = prune_mask(p, t, p.zn_pred, rgs, rge);
        sm.ss = make_segments(t, m, rgs, rge, p.tile);
        sm.bytes = scanned_bytes(p, t, sm.ss.rows, false);
        sm.rgs = rgs;
        sm.rge = rge;
        sm.zone_version = t.zone_version;
    }
    const ScanSegs& ss = sm.ss;
    set_columns(P, t, false);
    if (ss.seg != p.seg_cache || !p.d_seg.p) {  // segment list uploaded once per distinct pruning
        p.d_seg.ensure(std::max<size_t>(ss.seg.size(), 3) * 8);
        h2d(p.d_seg.p, ss.seg.data(), ss.seg.size() * 8, rc.s);
        p.seg_cache = ss.seg;
    }
    P.seg = p.d_seg.as<long long>();
    P.nseg = (int)ss.seg.size() / 3;
    P.nchunks = ss.nchunks;
    P.rg_rows = t.rg_rows;
    P.n_rg = t.n_rg;
    P.present = p.d_present.as<unsigned char>();
    for (size_t i = 0, off = 0; i < p.sets.size(); i++) { P.sets[i] = p.d_sets.as<unsigned>() + off; off += p.sets[i].size(); }

    bytes += sm.bytes;
    rows_scanned += ss.rows;
    if (use_radix && ss.nchunks > 0) {
        // probe side: the same partitions, then one block per partition joins
        ensure_events(p);
        VQ_CUDA(cudaEventRecord(p.ev[4], rc.s));
        long long* qstart = p.rp_start.as<long long>() + ((1 << VQ_RADIX_MAX_BITS) + 1);
        // payload columns: sized for every probe row of the scanned ranges
        VQParams Q = P;
        for (size_t j = 0; j < p.qpay_cols.size(); j++) {
            p.rp_qpay[j].ensure((size_t)std::max<long long>(ss.rows, 1) * 8);
            Q.qpay[j] = P.qpay[j] = p.rp_qpay[j].as<unsigned long long>();
            if (t.cols[p.qpay_cols[j]].nullable) {
                p.rp_qpayv[j].ensure((size_t)std::max<long long>(ss.rows, 1));
                Q.qpayv[j] = P.qpayv[j] = p.rp_qpayv[j].as<unsigned char>();
            }
        }
        radix_pass(rc, p.k_part_p, Q, pbits, qstart, p.rp_qkeys, p.rp_qrows, nullptr, p.rcap);
        VQ_CUDA(cudaEventRecord(p.ev[5], rc.s));
        VQ_CUDA(cudaEventSynchronize(p.ev[5]));
        rc.kernel_ms += elapsed(p.ev[4], p.ev[5]);
        P.qstart = qstart;
        P.qkeys = p.rp_qkeys.as<unsigned long long>();
        P.qrows = p.rp_qrows.as<int>();
        rc.k = &p.k_rjoin;
        rc.grid = (int)std::min<long long>(P.nparts, (long long)sm_count() * std::max(1, p.k_rjoin.max_blocks_per_sm));
    }
    vexq_result_s* r;
    if (ss.nchunks == 0) {
        Groups g;
        g.ival.assign(p.ni, {});
        g.fval.assign(p.nf, {});
        if (p.partial_out) {
            *p.partial_out = g;
            r = new vexq_result_s;
        } else {
            r = build_result(p, g);
        }
        r->kernel_ms = rc.kernel_ms;
        r->launches = rc.launches;
    } else {
        long long est = estimate_groups(p, ss.rows, join_keys);
        if (p.submit_lazy && p.path == AggPath::Regs && !p.is_join && !p.partial_out && !rc.k) {
            r = submit_regs(rc, P, ss.nchunks);
            r->rows_scanned = rows_scanned;
            r->bytes_scanned = bytes;
            return r;
        }
        try {
            r = finish_groups(rc, P, ss.nchunks, est, ss.rows);
        } catch (const SpecRetry& e) {
            // the build the probe did not wait for failed (a repeated key: the
            // hash table from here on), was empty or numbered more keys: run
            // again with the host reading the build's outcome first
            if (e.bits & 64) p.dmap_failed = true;
            p.dmap_used = false;
            return run_plan(p, rg_start, rg_end);
        }
        if (spec) r->kernel_ms += elapsed(p.ev[4], p.ev[5]);
    }
    r->rows_scanned = rows_scanned;
    r->bytes_scanned = bytes;
    return r;
}

vexq_result_s* run_plan_submit(Plan& p, int rg_start, int rg_end) {
    struct Lazy {
        Plan& p;
        explicit Lazy(Plan& q) : p(q) { p.submit_lazy = true; }
        ~Lazy() { p.submit_lazy = false; }
    } lazy(p);
    return run_plan(p, rg_start, rg_end);
}

vexq_result_s* run_plan_host(Plan& p, const vexq_column_desc* cols, int32_t ncols) {
    refill_table(*p.t, cols, ncols, plan_stream(p));
    return run_plan(p, 0, -1);
}

// ---- Next(): ≤ 1024-row batches (exec/aggregate.go:209-216) ----------------------------
int32_t result_next(vexq_result_s* r, vexq_batch_view* out) {
    int64_t n = std::min<int64_t>(VEXQ_BLOCK_ROWS, r->nrows - r->pos);
    if (n < 0) n = 0;
    size_t nc = r->cols.size();
    r->views.assign(nc, vexq_vector_view{});
    r->vbuf.assign(nc, {});
    r->bbuf.assign(nc, {});
    r->doff.assign(nc, {});
    r->dbytes.assign(nc, {});
    for (size_t c = 0; c < nc; c++) {
        OutColumn& oc = r->cols[c];
        vexq_vector_view& v = r->views[c];
        v.name = oc.name.c_str();
        v.type = oc.type;
        std::vector<uint8_t>& bm = r->bbuf[c];
        bm.assign((n + 7) / 8, 0);
        for (int64_t i = 0; i < n; i++) if (oc.valid[r->pos + i]) bm[i >> 3] |= (uint8_t)(1u << (i & 7));
        std::vector<char>& vb = r->vbuf[c];
        switch (oc.type) {
            case VEXQ_TYPE_INT64:
            case VEXQ_TYPE_FLOAT64:
                vb.resize(n * 8);
                std::memcpy(vb.data(), oc.v.data() + r->pos, n * 8);
                break;
            case VEXQ_TYPE_DATE: {
                vb.resize(n * 4);
                for (int64_t i = 0; i < n; i++) { int32_t x = (int32_t)oc.v[r->pos + i]; std::memcpy(vb.data() + i * 4, &x, 4); }
                break;
            }
            case VEXQ_TYPE_BOOL: {
                vb.resize(n);
                for (int64_t i = 0; i < n; i++) vb[i] = oc.v[r->pos + i] != 0;
                break;
            }
            case VEXQ_TYPE_STRING: {  // a fresh per-batch dictionary (exec.newStringVector)
                vb.resize(n * 4);
                std::unordered_map<int64_t, uint32_t> local;
                std::vector<uint32_t>& off = r->doff[c];
                std::string& bytes = r->dbytes[c];
                off.push_back(0);
                for (int64_t i = 0; i < n; i++) {
                    uint32_t code = 0;
                    if (oc.valid[r->pos + i]) {
                        auto it = local.find(oc.v[r->pos + i]);
                        if (it == local.end()) {
                            code = (uint32_t)local.size();
                            local.emplace(oc.v[r->pos + i], code);
                            bytes += oc.dict->keys[oc.v[r->pos + i]];
                            off.push_back((uint32_t)bytes.size());
                        } else {
                            code = it->second;
                        }
                    }
                    std::memcpy(vb.data() + i * 4, &code, 4);
                }
                v.dict_str_off = off.data();
                v.dict_bytes = bytes.data();
                v.dict_len = (int32_t)local.size();
                break;
            }
        }
        v.values = vb.data();
        v.validity = bm.data();
    }
    out->ncols = (int32_t)nc;
    out->length = (int32_t)n;
    out->cols = r->views.data();
    r->pos += n;
    return VEXQ_OK;
}

}  // namespace vq
