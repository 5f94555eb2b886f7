// kparams.h — the parameter block of every generated scan kernel. Shared
// verbatim by the host (nvcc/g++) and by the runtime-compiled kernels
// (NVRTC), so it uses only fixed-width scalar fields and raw pointers.
#pragma once

#define VQ_MAXCOLS 32
#define VQ_MAXSETS 16
#define VQ_FX_DIGITS 4  // 32-bit digits of the exact fixed-point float sums
#define VQ_MAXLITS 32   // numeric literals passed at launch (raw 8-byte images)
#define VQ_MAXHOT 4     // dense path: hottest groups accumulated in registers
#define VQ_RADIX_CAP 4096      // radix join: build entries of one partition held in shared memory
#define VQ_RADIX_MAX_BITS 12   // radix join: at most 4,096 partitions
#define VQ_MAXDIST 4    // COUNT(DISTINCT) aggregates of one plan

struct VQParams {
    // ---- scanned table (aggregate: the table; join: probe or build side) ----
    const void* col[VQ_MAXCOLS];
    const unsigned char* valid[VQ_MAXCOLS];
    // ---- build-side columns read through build row ids (join probe) ----
    const void* bcol[VQ_MAXCOLS];
    const unsigned char* bvalid[VQ_MAXCOLS];
    // ---- code sets for IN / LIKE over large dictionaries ----
    const unsigned* sets[VQ_MAXSETS];
    // ---- row ranges: seg[3*i+0..2] = start row, end row, first chunk ----
    const long long* seg;
    // ---- StringEqExpr per-row-group dictionary presence, [npresent][n_rg] ----
    const unsigned char* present;
    // ---- register path: per-block partials ----
    double* part_f;            // [grid][G][NF]
    long long* part_i;         // [grid][G][NI]
    long long* part_first;     // [grid][G]
    // ---- atomic path: group table ----
    unsigned long long* keys;  // [cap + 1]; slot cap holds the sentinel key
    long long* first;          // [cap + 1] first-occurrence order key
    long long* acc_i;          // [NI][cap + 1]
    long long* acc_fx;         // [NF][cap + 1][4]
    unsigned* special;         // [NF][cap + 1]: bit0 NaN, bit1 +inf, bit2 -inf
    unsigned long long* ngroups;  // occupied slots
    int* error;                // [0] overflow / probe-limit flag
    // ---- join build table ----
    unsigned long long* jkeys; // [jcap + 1]
    int* jcount;               // [jcap + 1]
    int* jstart;               // [jcap + 1]
    int* jfill;                // [jcap + 1]
    int* jrows;                // build row ids, grouped by slot in row order
    // [jcap + 1] probe view of the build table, one 16-byte load a probe step:
    // .x the slot's key (slot jcap: used flag of the empty-sentinel key), .y the
    // chain: low 32 bits the first row position and high 32 bits the row count,
    // or, for a key with one build row, the build row id and -1
    int* jfirst;               // [jcap + 1] build row of the slot's first insert (pass 0)
    int* jgid;                 // [jcap + 1] group number of the slot's key (GROUP BY the join key)
    unsigned long long* jtotal;    // build rows inserted (pass 0)
    const ulonglong2* jslot;
    unsigned long long* jnkeys;
    unsigned long long* jgkey;     // join build, mode 2 with group numbers: each number's key code
    long long jgoff;               //   the key's code offset
    // direct-mapped build table (mode 3; keys unique and inside a dense range):
    // [drange] chain words indexed by key - dmin, 0 where no build row has
    // the key; a word is the one build row and ~group number, as in .y of jslot
    unsigned long long* dmap;
    long long dmin;
    unsigned long long drange;
    // probe after a direct-mapped build that the host did not wait for: the
    // build's error word and key count, checked by the probe's first thread
    // (error bit 64: the build failed, 128: it inserted no key)
    const int* berr;
    const unsigned long long* bnk;
    // ---- radix-partitioned join ----
    unsigned long long* pkeys;     // partition pass: keys written per partition
    int* prows;                    //                 their row ids
    int* phist;                    // [nparts][grid] row counts (histogram) / offsets (scatter)
    const long long* bstart;       // join: [nparts + 1] build partition starts in bkeys/brows
    const unsigned long long* bkeys;
    const int* brows;
    const long long* qstart;       // join: [nparts + 1] probe partition starts in qkeys/qrows
    const unsigned long long* qkeys;
    const int* qrows;
    unsigned long long* qpay[8];   // probe columns used above the join, per probe entry (raw 8-byte words)
    unsigned char* qpayv[8];       // their validity (nullable columns)
    // ---- register path with the merge folded into the scan (racc_i set):
    //      every block adds its partials into these accumulators and the
    //      last block to arrive writes the merged row and resets them ----
    long long* racc_fx;            // [G][NF][4] fixed-point digits of the float sums
    unsigned* racc_sp;             // [G][NF] non-finite flags (bit0 NaN, bit1 +inf, bit2 -inf)
    long long* racc_i;             // [G][NI + 1] integer accumulators, first-row key last
    unsigned* racc_done;           // blocks that have added their partials
    double* rout_f;                // [G][NF] merged float entries
    long long* rout_i;             // [G][NI + 1] merged integer entries
    int* rerr_out;                 // the error word handed out with the merged row
    // ---- register path, partials merged by the last block (mdone set): every
    //      block writes its partial row, the last to arrive merges all of them
    //      in block order (the merge kernel's fold) and resets mdone ----
    const int* mkinds;             // combiner kind per bank entry: float bank, then int bank
    double* mout_f;                // [G][NF] merged float entries
    long long* mout_i;             // [G][NI + 1] merged integer entries
    int* merr_out;                 // the error word handed out with the merged row
    unsigned* mdone;               // blocks that have written their partials
    // ---- COUNT(DISTINCT) sets, one per distinct aggregate: [cap][2] (group
    //      key, value image) and a state word per slot (0 empty, 1 being
    //      written, 2 published); cap = dmask + 1 ----
    unsigned long long* dkeys[VQ_MAXDIST];
    unsigned* dstate[VQ_MAXDIST];
    unsigned long long dmask;
    // ---- numeric literals of the plan's expressions (int64, date, float64 bits):
    //      plans that differ only in constants share one compiled kernel ----
    long long lit[VQ_MAXLITS];
    // ---- 8-byte scalars ----
    long long nchunks;
    long long rg_rows;
    unsigned long long cap_mask;   // atomic path: capacity - 1 (hash) or unused (dense)
    unsigned long long cap;        // slots (hash: power of two; dense: domain)
    unsigned long long jmask;      // join table capacity - 1
    unsigned long long hot[VQ_MAXHOT];  // dense path: groups a thread accumulates in registers (~0 = none)
    // ---- 4-byte scalars ----
    int nseg;
    int n_rg;
    int mode;                  // join build: 0 = insert/count, 1 = fill, 2 = unique keys into jslot, 3 = unique keys into dmap
    int cache_n;               // dense path: groups held in the block's shared-memory cache
    int nparts;                // radix join: partitions (a power of two)
    int pbits;                 // radix join: partition = top pbits bits of the key hash
    int fx_lsb[16];            // per float-sum slot: exponent of the window's LSB
};

// One unit of a batched launch: chunks [cbeg, cend) of one plan, run by one
// block; pslot is the unit's partial row within its plan (register path).
struct VQUnit {
    int plan;
    int body;
    long long cbeg, cend;
    long long pslot;
};

// Parameters of a batched launch: blocks take units from *ticket in order.
struct VQBatchArgs {
    const VQParams* params;
    const VQUnit* units;
    unsigned* ticket;
    int nunits;
};
