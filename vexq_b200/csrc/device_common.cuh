// device_common.cuh — device helpers shared by the runtime-specialised scan
// kernels (prepended to every generated source) and the static kernels.
#pragma once

typedef long long vq_i64;
typedef unsigned long long vq_u64;

__device__ __host__ inline double __longlong_as_double_portable(vq_i64 b) {
#ifdef __CUDA_ARCH__
    return __longlong_as_double(b);
#else
    double d;
    __builtin_memcpy(&d, &b, 8);
    return d;
#endif
}

#define VQ_EMPTY_KEY 0xFFFFFFFFFFFFFFFFull
#define VQ_MAX_PROBES 4096

// Validity bit of row r in an LSB-first bitmap (1 = valid), storage/codec.go:13-39.
__device__ __forceinline__ bool vq_bit(const unsigned char* bm, vq_i64 r) {
    return (bm[r >> 3] >> (r & 7)) & 1;
}
// Four validity bits of rows r0..r0+3 (r0 % 4 == 0).
__device__ __forceinline__ unsigned vq_bits4(const unsigned char* bm, vq_i64 r0) {
    return (__ldg(bm + (r0 >> 3)) >> (r0 & 7)) & 0xFu;
}

// 128-bit vectorised loads of four consecutive rows (r0 % 4 == 0) through the
// read-only path; columns are 256-byte aligned and padded past the last row.
// A kernel generated with VQ_STREAM_LOADS reads its columns as streaming
// (ld.global.cs: evict first), so a table the kernel keeps probing stays in L2
// while the columns pass through it once.
#ifdef VQ_STREAM_LOADS
#define VQ_LDC(p) __ldcs(p)
#else
#define VQ_LDC(p) __ldg(p)
#endif
__device__ __forceinline__ void vq_ld4_i64(const void* p, vq_i64 r0, vq_i64* v) {
    const longlong2* q = reinterpret_cast<const longlong2*>(static_cast<const vq_i64*>(p) + r0);
    longlong2 a = VQ_LDC(q), b = VQ_LDC(q + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void vq_ld4_f64(const void* p, vq_i64 r0, double* v) {
    const double2* q = reinterpret_cast<const double2*>(static_cast<const double*>(p) + r0);
    double2 a = VQ_LDC(q), b = VQ_LDC(q + 1);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void vq_ld4_i32(const void* p, vq_i64 r0, int* v) {
    int4 a = VQ_LDC(reinterpret_cast<const int4*>(static_cast<const int*>(p) + r0));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void vq_ld4_u32(const void* p, vq_i64 r0, unsigned* v) {
    uint4 a = VQ_LDC(reinterpret_cast<const uint4*>(static_cast<const unsigned*>(p) + r0));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void vq_ld4_u8(const void* p, vq_i64 r0, unsigned* v) {
    unsigned w = VQ_LDC(reinterpret_cast<const unsigned*>(static_cast<const unsigned char*>(p) + r0));
    v[0] = w & 0xFF; v[1] = (w >> 8) & 0xFF; v[2] = (w >> 16) & 0xFF; v[3] = w >> 24;
}

// radixHash (exec/parallel_join.go:91-99): the murmur3 64-bit finalizer.
__device__ __forceinline__ vq_u64 vq_hash(vq_u64 x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return x;
}

// Order-preserving map of doubles onto unsigned 64-bit keys (NaN excluded by callers).
__device__ __forceinline__ vq_u64 vq_fkey(double d) {
    vq_u64 b = (vq_u64)__double_as_longlong(d);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double vq_fkey_inv(vq_u64 k) {
    vq_u64 b = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFull) : ~k;
    return __longlong_as_double((vq_i64)b);
}

// A 64-bit shared-memory counter updated with 32-bit atomics (64-bit ones on
// shared memory measured 6x slower, 50x under contention): a (low, high) word
// pair; the low word takes the digit's low 32 bits, and the
// high word its high 32 bits plus the carry out of that addition, read from
// the returned old value — the pair still sums every digit exactly.
__device__ __forceinline__ void vq_add64_as32(vq_i64* c, vq_i64 d) {
    if (!d) return;
    unsigned* w = reinterpret_cast<unsigned*>(c);  // little-endian: w[0] low, w[1] high
    const unsigned lo = (unsigned)(unsigned long long)d, hi = (unsigned)((unsigned long long)d >> 32);
    const unsigned old = atomicAdd(w, lo);
    const unsigned carry = (unsigned)(old + lo < old);
    if (hi + carry) atomicAdd(w + 1, hi + carry);
}
// Exact float summation: x is added, as an integer multiple of 2^lsb, into
// four signed 64-bit counters holding 32-bit digits (c[k] weighs 2^(32k+lsb)).
// Integer addition is associative, so the sum is the same whatever order the
// atomics land in. Bits of x below 2^lsb are truncated (the window is chosen
// so that only values below 2^-45 of the largest possible |x| lose bits).
// Non-finite values set flags instead. stride is the distance between digits.
template <bool kAtomic, bool kPair32 = false>
__device__ __forceinline__ void vq_fx_add(vq_i64* c, double x, int lsb, unsigned* special, int* err) {
    vq_u64 b = (vq_u64)__double_as_longlong(x);
    int e = (int)((b >> 52) & 0x7FF);
    if (e == 0x7FF) {  // inf / nan
        unsigned f = (b & 0xFFFFFFFFFFFFFull) ? 1u : ((b >> 63) ? 4u : 2u);
        if (kAtomic) atomicOr(special, f); else *special |= f;
        return;
    }
    vq_u64 m = b & 0xFFFFFFFFFFFFFull;
    if (e == 0) { if (m == 0) return; e = 1; } else m |= 1ull << 52;
    int sh = e - 1075 - lsb;  // position of m's bit 0 above the window's LSB
    if (sh < 0) {
        if (sh <= -53) return;
        m >>= -sh;
        sh = 0;
        if (m == 0) return;
    }
    int d = sh >> 5, off = sh & 31;
    vq_u64 lo = m << off;
    unsigned hi = off ? (unsigned)(m >> (64 - off)) : 0u;
    vq_i64 dg[3] = {(vq_i64)(lo & 0xFFFFFFFFull), (vq_i64)(lo >> 32), (vq_i64)hi};
    bool neg = b >> 63;
#pragma unroll
    for (int k = 0; k < 3; k++) {
        if (dg[k] == 0) continue;
        int idx = d + k;
        if (idx >= VQ_FX_DIGITS) { atomicOr(reinterpret_cast<unsigned*>(err), 2u); continue; }
        vq_i64 v = neg ? -dg[k] : dg[k];
        if (kAtomic && kPair32) vq_add64_as32(c + idx, v);  // shared memory
        else if (kAtomic) atomicAdd(reinterpret_cast<unsigned long long*>(c + idx), (unsigned long long)v);
        else c[idx] += v;
    }
}

// The same fixed-point image as a 128-bit two's-complement integer in four
// 32-bit words (w[0] least significant), for folding the values of several
// lanes before one accumulator update. Magnitudes above 2^121 (impossible
// inside the window's bounds) raise err bit 1 so a 32-value fold cannot wrap.
__device__ __forceinline__ void vq_fx_words(double x, int lsb, unsigned* w, unsigned& special, int* err) {
    w[0] = w[1] = w[2] = w[3] = 0u;
    special = 0u;
    vq_u64 b = (vq_u64)__double_as_longlong(x);
    int e = (int)((b >> 52) & 0x7FF);
    if (e == 0x7FF) {
        special = (b & 0xFFFFFFFFFFFFFull) ? 1u : ((b >> 63) ? 4u : 2u);
        return;
    }
    vq_u64 m = b & 0xFFFFFFFFFFFFFull;
    if (e == 0) { if (m == 0) return; e = 1; } else m |= 1ull << 52;
    int sh = e - 1075 - lsb;
    if (sh < 0) {
        if (sh <= -53) return;
        m >>= -sh;
        sh = 0;
    }
    if (sh > 69) { atomicOr(reinterpret_cast<unsigned*>(err), 2u); return; }
    vq_u64 lo = sh < 64 ? m << sh : 0ull;
    vq_u64 hi = sh == 0 ? 0ull : (sh < 64 ? m >> (64 - sh) : m << (sh - 64));
    if (b >> 63) { lo = ~lo + 1ull; hi = ~hi + (lo == 0ull ? 1ull : 0ull); }
    w[0] = (unsigned)lo; w[1] = (unsigned)(lo >> 32); w[2] = (unsigned)hi; w[3] = (unsigned)(hi >> 32);
}

// Adds carry-save digits (d[k] weighs 2^(32k+lsb)) to the four counters.
template <bool kAtomic>
__device__ __forceinline__ void vq_fx_add_digits(vq_i64* c, vq_i64 d0, vq_i64 d1, vq_i64 d2, vq_i64 d3) {
    if (kAtomic) {
        if (d0) atomicAdd(reinterpret_cast<unsigned long long*>(c + 0), (unsigned long long)d0);
        if (d1) atomicAdd(reinterpret_cast<unsigned long long*>(c + 1), (unsigned long long)d1);
        if (d2) atomicAdd(reinterpret_cast<unsigned long long*>(c + 2), (unsigned long long)d2);
        if (d3) atomicAdd(reinterpret_cast<unsigned long long*>(c + 3), (unsigned long long)d3);
    } else {
        c[0] += d0; c[1] += d1; c[2] += d2; c[3] += d3;
    }
}

// The same with the four counters `stride` words apart: the shared-memory
// group cache keeps digit d of every group contiguous, so the lanes of a warp
// updating different groups spread over the banks.
__device__ __forceinline__ void vq_fx_add_digits_s(vq_i64* c, long long stride, vq_i64 d0, vq_i64 d1, vq_i64 d2, vq_i64 d3) {
    if (d0) atomicAdd(reinterpret_cast<unsigned long long*>(c), (unsigned long long)d0);
    if (d1) atomicAdd(reinterpret_cast<unsigned long long*>(c + stride), (unsigned long long)d1);
    if (d2) atomicAdd(reinterpret_cast<unsigned long long*>(c + 2 * stride), (unsigned long long)d2);
    if (d3) atomicAdd(reinterpret_cast<unsigned long long*>(c + 3 * stride), (unsigned long long)d3);
}

// The four digits with 32-bit shared-memory atomics (vq_add64_as32).
__device__ __forceinline__ void vq_fx_add_digits_s32(vq_i64* c, long long stride, vq_i64 d0, vq_i64 d1, vq_i64 d2, vq_i64 d3) {
    vq_add64_as32(c, d0);
    vq_add64_as32(c + stride, d1);
    vq_add64_as32(c + 2 * stride, d2);
    vq_add64_as32(c + 3 * stride, d3);
}

// The shared-memory group cache in limb form: a float sum's 128-bit fixed-point
// image as eight 16-bit limbs of its magnitude, each added with a plain 32-bit
// atomic (no returned value, no carry) into its own counter, positive and
// negative values in separate sets of eight (L[j * C], L[(8 + j) * C]). A
// counter takes at most 0xFFFF a row, so 32,768 rows of a group between two
// normalisations (vq_limbs_norm) keep every counter below 2^31. d0..d3 are
// the canonical 32-bit words of the two's-complement image (d3 signed).
__device__ __forceinline__ void vq_limbs_add(unsigned* L, long long C, long long d0, long long d1, long long d2, long long d3) {
    unsigned m0 = (unsigned)d0, m1 = (unsigned)d1, m2 = (unsigned)d2, m3 = (unsigned)d3;
    if (d3 < 0) {  // magnitude of a negative image: ~x + 1 over 128 bits
        m0 = ~m0; m1 = ~m1; m2 = ~m2; m3 = ~m3;
        m0 += 1u;
        const unsigned c0 = m0 == 0u;
        m1 += c0;
        const unsigned c1 = c0 & (m1 == 0u);
        m2 += c1;
        m3 += c1 & (m2 == 0u);
        L += 8 * C;
    }
    const unsigned m[4] = {m0, m1, m2, m3};
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const unsigned limb = (m[j >> 1] >> (16 * (j & 1))) & 0xFFFFu;
        if (limb) atomicAdd(L + j * C, limb);
    }
}
// Moves every counter's bits above 16 into the next limb up (both sets; the
// top limb keeps its high bits): atomic, so adds landing meanwhile are kept.
__device__ __forceinline__ void vq_limbs_norm(unsigned* L, long long C) {
#pragma unroll
    for (int s = 0; s < 2; s++)
#pragma unroll
        for (int j = 0; j < 7; j++) {
            const unsigned old = atomicAnd(L + (8 * s + j) * C, 0xFFFFu);
            if (old >> 16) atomicAdd(L + (8 * s + j + 1) * C, old >> 16);
        }
}
// The block's limbs as the global table's carry-save digit d (weight 2^(32d)).
__device__ __forceinline__ long long vq_limbs_digit(const unsigned* L, long long C, int d) {
    return (long long)L[(2 * d) * C] + ((long long)L[(2 * d + 1) * C] << 16) - (long long)L[(8 + 2 * d) * C] -
           ((long long)L[(8 + 2 * d + 1) * C] << 16);
}

// ---- warp reductions over a peer mask (redux.sync; every lane named in the
// mask executes the same call with the same mask) ----
__device__ __forceinline__ unsigned vq_redux_add(unsigned mask, unsigned v) {
    unsigned r;
    asm volatile("redux.sync.add.u32 %0, %1, %2;" : "=r"(r) : "r"(v), "r"(mask));
    return r;
}
__device__ __forceinline__ unsigned vq_redux_min(unsigned mask, unsigned v) {
    unsigned r;
    asm volatile("redux.sync.min.u32 %0, %1, %2;" : "=r"(r) : "r"(v), "r"(mask));
    return r;
}
__device__ __forceinline__ unsigned vq_redux_max(unsigned mask, unsigned v) {
    unsigned r;
    asm volatile("redux.sync.max.u32 %0, %1, %2;" : "=r"(r) : "r"(v), "r"(mask));
    return r;
}
__device__ __forceinline__ unsigned vq_redux_or(unsigned mask, unsigned v) {
    unsigned r;
    asm volatile("redux.sync.or.b32 %0, %1, %2;" : "=r"(r) : "r"(v), "r"(mask));
    return r;
}
// Sum of one 32-bit word over the peers, exact in 64 bits (two 16-bit halves).
__device__ __forceinline__ vq_i64 vq_wsum32(unsigned mask, unsigned v) {
    return (vq_i64)vq_redux_add(mask, v & 0xFFFFu) + ((vq_i64)vq_redux_add(mask, v >> 16) << 16);
}
// Wrapping 64-bit sum over the peers (four 16-bit quarters).
__device__ __forceinline__ vq_u64 vq_wsum64(unsigned mask, vq_u64 v) {
    vq_u64 r = 0;
#pragma unroll
    for (int q = 0; q < 4; q++) r += (vq_u64)vq_redux_add(mask, (unsigned)(v >> (16 * q)) & 0xFFFFu) << (16 * q);
    return r;
}
// Unsigned 64-bit min / max over the peers: the high words first, then the
// low words among the lanes holding the extreme high word.
__device__ __forceinline__ vq_u64 vq_wmin64(unsigned mask, vq_u64 v) {
    const unsigned h = (unsigned)(v >> 32);
    const unsigned mh = vq_redux_min(mask, h);
    const unsigned m2 = __ballot_sync(mask, h == mh);
    unsigned ml = 0u;
    if (h == mh) ml = vq_redux_min(m2, (unsigned)v);
    ml = __shfl_sync(mask, ml, __ffs(m2) - 1);
    return ((vq_u64)mh << 32) | ml;
}
__device__ __forceinline__ vq_u64 vq_wmax64(unsigned mask, vq_u64 v) {
    const unsigned h = (unsigned)(v >> 32);
    const unsigned mh = vq_redux_max(mask, h);
    const unsigned m2 = __ballot_sync(mask, h == mh);
    unsigned ml = 0u;
    if (h == mh) ml = vq_redux_max(m2, (unsigned)v);
    ml = __shfl_sync(mask, ml, __ffs(m2) - 1);
    return ((vq_u64)mh << 32) | ml;
}

__device__ __host__ inline int vq_clz64(vq_u64 x) {
#ifdef __CUDA_ARCH__
    return __clzll((long long)x);
#else
    return __builtin_clzll(x);
#endif
}

// mant · 2^e2 for a 53-bit mantissa (bit 52 set), built from the bits so no
// math library is needed; results below the normal range flush through a
// scaled multiply (sums that small do not occur in the workloads).
__device__ __host__ inline double vq_make_double(vq_u64 mant, int e2) {
    int eb = e2 + 52 + 1023;
    if (eb >= 2047) return __longlong_as_double_portable(0x7FF0000000000000ll);
    if (eb > 0) return __longlong_as_double_portable((vq_i64)(((vq_u64)eb << 52) | (mant & 0xFFFFFFFFFFFFFull)));
    double m = (double)mant;
    int e = e2;
    while (e < -1000) { m *= 0x1p-1000; e += 1000; }
    double scale = __longlong_as_double_portable((vq_i64)((vq_u64)(e + 1023) << 52));
    return m * scale;
}

// Correctly rounded (nearest, ties to even) double of sum_k c[k]·2^(32k+lsb).
__device__ __host__ inline double vq_fx_value(const vq_i64* c, int lsb) {
    // exact 256-bit two's-complement sum of the four counters (c[k] << 32k)
    vq_u64 w[4] = {0, 0, 0, 0};
    for (int k = 0; k < VQ_FX_DIGITS; k++) {
        const vq_i64 v = c[k];
        const vq_u64 ext = v < 0 ? ~0ull : 0ull;
        const int q = (32 * k) >> 6, r = (32 * k) & 63;
        vq_u64 part[4];
        // part = v sign-extended to 256 bits, shifted left by 32k
        for (int i = 0; i < 4; i++) {
            const int s = i - q;
            const vq_u64 lo_word = s == 0 ? (vq_u64)v : (s >= 1 ? ext : 0);
            const vq_u64 below = s == 1 ? (vq_u64)v : (s >= 2 ? ext : 0);
            part[i] = s < 0 ? 0 : (r ? ((lo_word << r) | (below >> (64 - r))) : lo_word);
        }
        vq_u64 carry = 0;
        for (int i = 0; i < 4; i++) {
            const vq_u64 t = w[i] + part[i];
            const vq_u64 c1 = t < w[i];
            const vq_u64 t2 = t + carry;
            const vq_u64 c2 = t2 < t;
            w[i] = t2;
            carry = c1 | c2;
        }
    }
    const bool neg = (w[3] >> 63) & 1;
    if (neg) {  // magnitude = -w
        vq_u64 carry = 1;
        for (int i = 0; i < 4; i++) {
            w[i] = ~w[i];
            const vq_u64 t = w[i] + carry;
            carry = t < w[i] ? 1 : 0;
            w[i] = t;
        }
    }
    int top = -1;
    for (int i = 3; i >= 0; i--)
        if (w[i]) { top = i * 64 + 63 - vq_clz64(w[i]); break; }
    if (top < 0) return 0.0;
    // 64-bit window ending at `top`: bits [top-63, top]
    const int lo_bit = top - 63;
    auto word_at = [&](int pos) -> vq_u64 {  // 64 bits starting at bit pos (pos may be < 0)
        if (pos <= -64) return 0;
        if (pos < 0) return w[0] << (-pos);
        const int q = pos >> 6, r = pos & 63;
        const vq_u64 a = q < 4 ? w[q] : 0, b = q + 1 < 4 ? w[q + 1] : 0;
        return r ? (a >> r) | (b << (64 - r)) : a;
    };
    const vq_u64 top64 = word_at(lo_bit);  // bit 63 is the leading one
    vq_u64 mant = top64 >> 11;             // 53 bits
    const vq_u64 rest = top64 & 0x7FFull;  // 11 bits below the mantissa
    bool sticky = (rest & 0x3FFull) != 0;
    if (!sticky && lo_bit > 0) {           // any set bit below the 64-bit window
        for (int i = 0; i < 4 && !sticky; i++) {
            const int base = i * 64;
            if (base >= lo_bit) break;
            const vq_u64 m = (lo_bit - base >= 64) ? ~0ull : ((1ull << (lo_bit - base)) - 1);
            if (w[i] & m) sticky = true;
        }
    }
    const bool guard = (rest >> 10) & 1;
    int exp2 = lo_bit + 11 + lsb;
    if (guard && (sticky || (mant & 1))) {
        mant++;
        if (mant >> 53) { mant >>= 1; exp2++; }
    }
    const double r = vq_make_double(mant, exp2);
    return neg ? -r : r;
}

// The value of an exact float sum: NaN when a NaN or both infinities were
// added, else the infinity that was added, else the fixed-point total.
__device__ __forceinline__ double vq_fx_result(const vq_i64* c, int lsb, unsigned sp) {
    if ((sp & 1u) || (sp & 6u) == 6u) return __longlong_as_double(0x7FF8000000000001LL);
    if (sp & 2u) return __longlong_as_double(0x7FF0000000000000LL);
    if (sp & 4u) return __longlong_as_double((long long)0xFFF0000000000000ULL);
    return vq_fx_value(c, lsb);
}

// COUNT(DISTINCT) set insert: open addressing over (group key k0, value
// image k1) pairs. A slot's state goes 0 → 1 (claimed, being written) → 2
// (published); a thread that finds a slot being written waits for it. Returns
// true for the one insert that adds a pair, so summing the results per group
// counts its distinct values whatever order rows arrive in. Both waits are
// bounded: error bit 16 when the probe limit is reached (the table is sized
// for twice the rows scanned, so only a broken size reaches it), bit 32 when
// a claimed slot is not published in time.
__device__ __forceinline__ bool vq_dset_insert(unsigned long long* keys, unsigned* state, unsigned long long mask,
                                               unsigned long long k0, unsigned long long k1, int* error) {
    const unsigned long long h = vq_hash(k0 * 0x9E3779B97F4A7C15ull ^ vq_hash(k1 + 0x632BE59BD9B4E019ull));
    const int limit = mask < 4095ull ? (int)mask + 1 : 4096;
    for (int probe = 0; probe < limit; probe++) {
        const unsigned long long i = (h + (unsigned long long)probe) & mask;
        unsigned s = *(volatile unsigned*)(state + i);
        if (s == 0u) {
            s = atomicCAS(state + i, 0u, 1u);
            if (s == 0u) {
                keys[2 * i] = k0;
                keys[2 * i + 1] = k1;
                __threadfence();
                atomicExch(state + i, 2u);
                return true;
            }
        }
        for (int spin = 0; s == 1u; spin++) {
            if (spin > (1 << 22)) {
                atomicOr(error, 32);
                return false;
            }
            s = *(volatile unsigned*)(state + i);
        }
        __threadfence();
        const unsigned long long a = *(volatile unsigned long long*)(keys + 2 * i);
        const unsigned long long b = *(volatile unsigned long long*)(keys + 2 * i + 1);
        if (a == k0 && b == k1) return false;
    }
    atomicOr(error, 16);
    return false;
}

#define VQ_NOSLOT 0xFFFFFFFFFFFFFFFFull

// Open-addressing insert (linear probing, atomicCAS on the key). The key equal
// to the empty sentinel lives in the extra slot `cap`, whose key word is a
// used-flag. Returns VQ_NOSLOT and raises err bit 0 when the probe limit is
// reached, so a full table ends the kernel's work instead of spinning. New
// keys are counted in *nkeys when it is not null (a block-local counter: one
// global word taking an atomic per key serialises the whole insert).
__device__ __forceinline__ vq_u64 vq_insert(vq_u64* keys, vq_u64 mask, vq_u64 cap, vq_u64 key,
                                            vq_u64* nkeys, int* err) {
    if (key == VQ_EMPTY_KEY) {
        if (atomicCAS(keys + cap, 0ull, 1ull) == 0ull && nkeys) atomicAdd(nkeys, 1ull);
        return cap;
    }
    vq_u64 i = vq_hash(key) & mask;
    const vq_u64 limit = mask < (vq_u64)VQ_MAX_PROBES ? mask + 1 : (vq_u64)VQ_MAX_PROBES;
    for (vq_u64 n = 0; n < limit; n++) {
        // one round trip: claim the slot or learn its key
        vq_u64 old = atomicCAS(keys + i, VQ_EMPTY_KEY, key);
        if (old == VQ_EMPTY_KEY) {
            if (nkeys) atomicAdd(nkeys, 1ull);  // callers count in shared memory, not one global word
            return i;
        }
        if (old == key) return i;
        i = (i + 1) & mask;
    }
    atomicOr(err, 1);
    return VQ_NOSLOT;
}

// Insert that also reports whether this call claimed the key's slot.
__device__ __forceinline__ vq_u64 vq_insert_fresh(vq_u64* keys, vq_u64 mask, vq_u64 cap, vq_u64 key, bool& fresh, int* err) {
    fresh = false;
    if (key == VQ_EMPTY_KEY) {
        fresh = atomicCAS(keys + cap, 0ull, 1ull) == 0ull;
        return cap;
    }
    vq_u64 i = vq_hash(key) & mask;
    const vq_u64 limit = mask < (vq_u64)VQ_MAX_PROBES ? mask + 1 : (vq_u64)VQ_MAX_PROBES;
    for (vq_u64 n = 0; n < limit; n++) {
        const vq_u64 old = atomicCAS(keys + i, VQ_EMPTY_KEY, key);
        if (old == VQ_EMPTY_KEY) { fresh = true; return i; }
        if (old == key) return i;
        i = (i + 1) & mask;
    }
    atomicOr(err, 1);
    return VQ_NOSLOT;
}

// A kernel generated with VQ_KEEP_TABLES reads the join's slot table with an
// L2 evict-last policy, so the table stays in L2 while the probe columns
// stream past it.
__device__ __forceinline__ ulonglong2 vq_ld_slot(const ulonglong2* p) {
#ifdef VQ_KEEP_TABLES
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    ulonglong2 v;
    asm volatile("ld.global.nc.L2::cache_hint.v2.u64 {%0, %1}, [%2], %3;" : "=l"(v.x), "=l"(v.y) : "l"(p), "l"(pol));
    return v;
#else
    return __ldg(p);
#endif
}

// The same for one word of the direct-mapped build table.
__device__ __forceinline__ unsigned long long vq_ld_dword(const unsigned long long* p) {
#ifdef VQ_KEEP_TABLES
    unsigned long long pol, v;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    asm volatile("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
    return v;
#else
    return __ldg(p);
#endif
}

// Probe of the packed build table (key + chain in one 16-byte slot). Returns
// whether the key is present and its chain word.
__device__ __forceinline__ bool vq_find_slot(const ulonglong2* slots, vq_u64 mask, vq_u64 key, vq_u64& chain, vq_u64& at) {
    if (key == VQ_EMPTY_KEY) {
        const ulonglong2 s = vq_ld_slot(slots + mask + 1);
        chain = s.y;
        at = mask + 1;
        return s.x != 0ull;
    }
    vq_u64 i = vq_hash(key) & mask;
    for (vq_u64 n = 0; n <= mask; n++) {
        const ulonglong2 s = vq_ld_slot(slots + i);
        if (s.x == key) { chain = s.y; at = i; return true; }
        if (s.x == VQ_EMPTY_KEY) return false;
        i = (i + 1) & mask;
    }
    return false;
}

// The same probe continued from its first slot, loaded ahead (the probe
// kernel issues the first loads of a lane's four rows together): i0 is the
// key's home slot (mask + 1 for the sentinel key) and s its contents.
__device__ __forceinline__ bool vq_find_slot_from(const ulonglong2* slots, vq_u64 mask, vq_u64 key, vq_u64 i0, ulonglong2 s,
                                                  vq_u64& chain, vq_u64& at) {
    if (key == VQ_EMPTY_KEY) {
        chain = s.y;
        at = mask + 1;
        return s.x != 0ull;
    }
    vq_u64 i = i0;
    for (vq_u64 n = 0; n <= mask; n++) {
        if (s.x == key) { chain = s.y; at = i; return true; }
        if (s.x == VQ_EMPTY_KEY) return false;
        i = (i + 1) & mask;
        s = vq_ld_slot(slots + i);
    }
    return false;
}

// Read-only lookup in a table no kernel is writing any more.
__device__ __forceinline__ vq_u64 vq_find(const vq_u64* keys, vq_u64 mask, vq_u64 cap, vq_u64 key) {
    if (key == VQ_EMPTY_KEY) return __ldg(keys + cap) ? cap : VQ_NOSLOT;
    vq_u64 i = vq_hash(key) & mask;
    for (vq_u64 n = 0; n <= mask; n++) {
        vq_u64 k = __ldg(keys + i);
        if (k == key) return i;
        if (k == VQ_EMPTY_KEY) return VQ_NOSLOT;
        i = (i + 1) & mask;
    }
    return VQ_NOSLOT;
}

// Combiners of partial accumulators (kind 0 sum, 1 min, 2 max), following
// mergePartialAgg (exec/parallel.go:262-297): a float MIN/MAX partial only
// replaces the running value when strictly smaller/larger.
__device__ __forceinline__ double vq_fminr(double a, double b) { return b < a ? b : a; }
__device__ __forceinline__ double vq_fmaxr(double a, double b) { return b > a ? b : a; }
__device__ __forceinline__ double vq_fcomb(int kind, double a, double b) {
    return kind == 1 ? vq_fminr(a, b) : kind == 2 ? vq_fmaxr(a, b) : a + b;
}
// Register path with the merge folded into the scan: one block partial into
// its global accumulator (kind 0 wrapping sum, 1 min, 2 max). A partial equal
// to the kind's identity changes nothing and takes no atomic.
__device__ __forceinline__ vq_i64 vq_racc_identity(int kind) {
    return kind == 1 ? (vq_i64)0x7FFFFFFFFFFFFFFFLL : kind == 2 ? (vq_i64)(-0x7FFFFFFFFFFFFFFFLL - 1) : (vq_i64)0;
}
__device__ __forceinline__ void vq_racc_add(vq_i64* a, int kind, vq_i64 v) {
    if (v == vq_racc_identity(kind)) return;
    if (kind == 1) atomicMin(reinterpret_cast<long long*>(a), (long long)v);
    else if (kind == 2) atomicMax(reinterpret_cast<long long*>(a), (long long)v);
    else atomicAdd(reinterpret_cast<unsigned long long*>(a), (unsigned long long)v);
}
__device__ __forceinline__ vq_i64 vq_icomb(int kind, vq_i64 a, vq_i64 b) {
    return kind == 1 ? (b < a ? b : a) : kind == 2 ? (b > a ? b : a) : (vq_i64)((vq_u64)a + (vq_u64)b);
}

// Compensated addition (Knuth's TwoSum): hi + lo carries the running sum, lo
// the rounding error of each step.
__device__ __forceinline__ void vq_two_sum(double& hi, double& lo, double x) {
    double s = hi + x;
    double bb = s - hi;
    lo += (hi - (s - bb)) + (x - bb);
    hi = s;
}

// One merged output entry of the register path, computed by one warp: lane l
// folds partials l, l+32, l+64, ... in that order (a compensated TwoSum pair
// for float sums, min/max/wrapping sum otherwise), then a fixed shuffle tree
// combines the lanes, so the result does not depend on scheduling. Loads are
// issued eight at a time ahead of their folds.
static __device__ __noinline__ void merge_entry(int e, const double* part_f, const long long* part_i, int nblocks, int G, int nf, int ni,
                            const int* fkind, const int* ikind, double* out_f, long long* out_i) {
    const int lane = threadIdx.x & 31;
    const int totf = G * nf, toti = G * (ni + 1);
    if (e < totf) {
        const int kind = fkind[e % nf];
        double hi = kind == 1 ? 1.7976931348623157e308 : kind == 2 ? -1.7976931348623157e308 : 0.0, lo = 0.0;
        for (int b0 = lane; b0 < nblocks; b0 += 32 * 8) {
            double x[8];
#pragma unroll
            for (int j = 0; j < 8; j++) x[j] = b0 + 32 * j < nblocks ? part_f[(long long)(b0 + 32 * j) * totf + e] : 0.0;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                if (b0 + 32 * j >= nblocks) break;
                if (kind == 0) vq_two_sum(hi, lo, x[j]);
                else hi = vq_fcomb(kind, hi, x[j]);
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double h2 = __shfl_down_sync(0xffffffffu, hi, o), l2 = __shfl_down_sync(0xffffffffu, lo, o);
            if (kind == 0) {
                double h = hi, l = lo + l2;
                vq_two_sum(h, l, h2);
                hi = h;
                lo = l;
            } else {
                hi = vq_fcomb(kind, hi, h2);
            }
        }
        if (lane == 0) out_f[e] = kind == 0 ? hi + lo : hi;
    } else if (e < totf + toti) {
        const int u = e - totf;
        const int kind = ikind[u % (ni + 1)];
        long long v = kind == 1 ? 0x7FFFFFFFFFFFFFFFLL : kind == 2 ? (-0x7FFFFFFFFFFFFFFFLL - 1) : 0LL;
        for (int b0 = lane; b0 < nblocks; b0 += 32 * 8) {
            long long x[8];
#pragma unroll
            for (int j = 0; j < 8; j++) x[j] = b0 + 32 * j < nblocks ? part_i[(long long)(b0 + 32 * j) * toti + u] : 0LL;
#pragma unroll
            for (int j = 0; j < 8; j++) {
                if (b0 + 32 * j >= nblocks) break;
                v = vq_icomb(kind, v, x[j]);
            }
        }
        for (int o = 16; o > 0; o >>= 1) v = vq_icomb(kind, v, (long long)__shfl_down_sync(0xffffffffu, v, o));
        if (lane == 0) out_i[u] = v;
    }
}

// ---- bulk asynchronous copies (TMA, untiled) into a shared-memory ring ----
// One thread issues cp.async.bulk copies of a tile's column slices into a
// stage and arms the stage's mbarrier with the byte count; consumers wait on
// the barrier's phase. Addresses and sizes are multiples of 16 bytes (tiles
// start on 512-row boundaries of 256-byte aligned columns). No multicast.
__device__ __forceinline__ unsigned vq_smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void vq_mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(vq_smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void vq_fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void vq_fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void vq_mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(vq_smem_addr(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void vq_bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(vq_smem_addr(dst)), "l"(src), "r"(bytes), "r"(vq_smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool vq_mbar_try_wait(unsigned long long* bar, unsigned phase) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(vq_smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `limit` polls and reports false (the caller
// raises the kernel's error flag and leaves the tile loop).
__device__ __forceinline__ bool vq_mbar_wait(unsigned long long* bar, unsigned phase, int limit) {
    for (int n = 0; n < limit; n++)
        if (vq_mbar_try_wait(bar, phase)) return true;
    return false;
}
// Four consecutive rows from a staged shared-memory slice (row offset o % 4 == 0).
__device__ __forceinline__ void vq_sld4_i64(const unsigned char* s, int o, vq_i64* v) {
    const longlong2* q = reinterpret_cast<const longlong2*>(s) + (o >> 1);
    longlong2 a = q[0], b = q[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void vq_sld4_f64(const unsigned char* s, int o, double* v) {
    const double2* q = reinterpret_cast<const double2*>(s) + (o >> 1);
    double2 a = q[0], b = q[1];
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
__device__ __forceinline__ void vq_sld4_i32(const unsigned char* s, int o, int* v) {
    int4 a = reinterpret_cast<const int4*>(s)[o >> 2];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void vq_sld4_u32(const unsigned char* s, int o, unsigned* v) {
    uint4 a = reinterpret_cast<const uint4*>(s)[o >> 2];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
// Validity of rows lane, lane+32, lane+64, lane+96 of a staged 128-row chunk
// (LSB-first bitmap: word k holds rows 32k..32k+31), as bits 0..3.
__device__ __forceinline__ unsigned vq_sbits4_strided(const unsigned char* s, int lane) {
    const uint4 w = *reinterpret_cast<const uint4*>(s);
    return ((w.x >> lane) & 1u) | (((w.y >> lane) & 1u) << 1) | (((w.z >> lane) & 1u) << 2) | (((w.w >> lane) & 1u) << 3);
}
__device__ __forceinline__ void vq_sld4_u8(const unsigned char* s, int o, unsigned* v) {
    unsigned w = reinterpret_cast<const unsigned*>(s)[o >> 2];
    v[0] = w & 0xFF; v[1] = (w >> 8) & 0xFF; v[2] = (w >> 16) & 0xFF; v[3] = w >> 24;
}
// Per-warp asynchronous copies (cp.async, 16 bytes, L2 only) into shared memory.
__device__ __forceinline__ void vq_cp16(void* sdst, const void* gsrc) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(vq_smem_addr(sdst)), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void vq_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void vq_cp_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

__device__ __forceinline__ unsigned vq_sbits4(const unsigned char* s, int o) {
    return (s[o >> 3] >> (o & 7)) & 0xFu;
}
