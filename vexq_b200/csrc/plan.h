// plan.h — compiled plans: typed expression IR, accumulator slots, and the
// generated scan kernels.
#pragma once

#include <functional>

#include "internal.h"

namespace vq {

enum class NK {
    Col, Lit, Cmp, Arith, Cast, And, Or, Not, IsNull, IsNotNull,
    InInt, InFloat, InCodes, InFalse, StrEq, Case,
    StrRank  // a STRING column's code → its place in the dictionary's byte order (MIN/MAX)
};

struct INode {
    NK k = NK::Lit;
    int type = 0;          // VEXQ_TYPE_*
    int op = 0;
    int col = -1;          // Col / StrEq / InCodes: column (in its side's table)
    bool build = false;    // column read through the build row (join above-scope)
    const Table* tab = nullptr;  // table the column belongs to
    int64_t li = 0;
    double lf = 0;
    int32_t ld = 0;
    bool lb = false;
    std::vector<int> ch;
    std::vector<int64_t> seti;
    std::vector<double> setf;
    std::vector<uint8_t> codes;   // InCodes: membership per global code
    int set_idx = -1;             // InCodes with a large dictionary: device set index
    int64_t streq_code = -1;      // StrEq: global code of the literal (-1 absent)
    bool negate = false;
    int present_idx = -1;         // StrEq: row of the presence table (-1: constant)
    bool has_else = false;
    bool nullable = false;
    // |value| bound from zone maps by interval arithmetic (exact-sum windows)
    bool bounded = false;
    double lo = 0, hi = 0;
    // a valid value is never NaN or ±inf (non-float types always; floats from
    // zone sums and bounded interval arithmetic)
    bool finite = false;
    bool is_literal_raw = false;  // literal before coercion (SQL level)
    int lit_kind = 0;
    int lit_slot = -1;            // numeric literal passed at launch: index into VQParams::lit
    std::vector<uint32_t> rank;   // StrRank: rank of each global code (device table at set_idx)
};

// Accumulator slot kinds.
enum SlotKind { S_CNT = 0, S_NN, S_ISUM, S_IMIN, S_IMAX, S_FSUM, S_FMIN, S_FMAX };

struct Slot {
    SlotKind kind;
    int input = -1;  // IR node (value), -1 for CNT
    // COUNT(DISTINCT): an S_NN slot whose row condition is "the (group,
    // value) pair entered distinct set `dset` for the first time"
    int dset = -1;
    bool is_float() const { return kind == S_FSUM || kind == S_FMIN || kind == S_FMAX; }
};

struct AggOut {
    int kind;         // VEXQ_AGG_*
    int value_slot;   // slot index (-1 for COUNT(*))
    int nn_slot;      // slot giving the non-null count (CNT when the input is never NULL)
    int out_type;     // result vector type
    std::string name;
    // MIN/MAX over a STRING column: the slot holds the rank of the string in
    // the dictionary's byte order; rank_code maps it back to the code
    std::vector<uint32_t> rank_code;
    const GlobalDict* rank_dict = nullptr;
};

struct KeyCol {
    std::string name; // output column name
    int col;          // column index in its side's table
    bool build;       // join: build-side column
    int type;
    bool nullable;
    // dense encoding: code in [0, domain): dict code / (value - vmin); NULL → domain-1
    int64_t vmin = 0;
    int64_t domain = 0;
    int bits = 0;     // packed-key width
    int shift = 0;
};

enum class AggPath { Regs, Dense, Hash };

struct ScanSegs {
    std::vector<long long> seg;  // start, end, chunk0 triples
    long long nchunks = 0;
    long long rows = 0;
};

// Zone-map pruning and segment list of one row-group range of a table, kept
// by a plan while the table's zone maps are unchanged.
struct ScanMemo {
    int rgs = -1, rge = -1;
    uint64_t zone_version = ~0ull;
    ScanSegs ss;
    int64_t bytes = 0;  // algorithmic bytes the scan of those segments reads
};

// What a captured register-path run depends on: the parameter block, the
// scan kernel and its shape, the merge's outputs and the stream.
struct RegsGraphKey {
    VQParams P;
    void* fn;
    cudaStream_t s;
    void* out_f;
    void* out_i;
    void* err_out;
    const void* d_kinds;
    int grid, block, smem, mode;
};

struct Plan {
    bool is_join = false;
    Table* t = nullptr;        // aggregate table or probe table
    Table* bt = nullptr;       // build table
    std::vector<INode> ir;
    int pred = -1;             // scan predicate (probe predicate for joins)
    int bpred = -1;            // join build predicate
    int resid = -1;            // join residual
    int build_key = -1, probe_key = -1;
    int bkey_node = -1;        // join: the build key's IR node (scoped to the build table)
    // SQL-level predicate trees kept for zone maps
    std::vector<vexq_expr> zn_nodes;
    std::vector<int32_t> zn_children;
    int zn_pred = -1, zn_bpred = -1;
    std::vector<KeyCol> keys;
    bool intkey_order = false;     // reference int-key path ordering rules apply
    int ndist = 0;                 // COUNT(DISTINCT) aggregates (device sets)
    struct Groups* partial_out = nullptr;  // set: a run hands its groups here unfinished (a shard's partial)
    DevBuf dist_keys[VQ_MAXDIST], dist_state[VQ_MAXDIST];
    int intkey_width = 32;
    std::vector<Slot> slots;
    std::vector<AggOut> outs;
    std::vector<int> gb_types;
    vexq_order_desc order{-1, 0, -1};
    AggPath path = AggPath::Hash;
    int64_t domain = 1;            // dense key domain
    int nf = 0, ni = 0;            // float / int slots (path-specific layout)
    std::vector<int> slot_pos;     // slot → index within its float/int bank
    std::vector<int> fx_lsb;       // per float-sum slot
    std::vector<long long> lits;   // launch-time literal table (VQParams::lit)
    std::vector<int> key_nodes;    // IR roots of the GROUP BY keys
    std::mutex body_mu;            // batch body text per block size, generated once
    std::map<int, std::string> batch_body;
    std::vector<std::vector<uint32_t>> sets;  // large InCodes sets (bitsets)
    std::vector<std::pair<int, int64_t>> presence;   // (column, code) rows: scanned / probe table
    std::vector<std::pair<int, int64_t>> bpresence;  // rows for the join build table
    DevBuf d_sets, d_present, d_bpresent;
    // generated kernels
    std::string src_main, src_build;
    JitKernel k_main, k_build;
    std::string explain;
    int radix_bits = 0;
    // tunables of the generated scan kernel (chosen at compile time)
    int block = 256;
    bool block_claim = true;   // direct join build: group numbers claimed once per block and chunk step
    bool pipeline = true;
    bool staged = true;        // TMA bulk-copy staging of row tiles into shared memory
    bool regs_pred = true;     // register path: branch-free predicated updates
    bool warp_agg = true;      // atomic path: fold lanes of one group before updating
    int smem_groups = 0;       // dense path: groups cached in block-private shared memory
    int stage_budget = 0;      // bytes of the stage ring per block (0: default)
    int tile = 128, smem = 0;  // main kernel: rows per loop unit, dynamic shared memory
    int async_stages = 0;      // >1: per-warp cp.async pipeline of that many 128-row chunks
    int min_blocks = 0;        // >0: __launch_bounds__ minimum resident blocks per SM
    int grid_per_sm = 0;       // >0: register path grid of at most this many blocks per SM
    bool merge_last = false;   // register path: the last block merges the partials (no merge launch)
    DevBuf mdone;              //   its arrival counter (0 between runs)
    bool stream_loads = false; // columns read evict-first (ld.global.cs): tables the kernel probes stay in L2
    bool keep_tables = false;  // join slot table read with an L2 evict-last policy
    // join build straight into the probe's 16-byte slots when the last build's
    // keys were unique (measured slower than count + pack at 1.5M keys: the
    // slot table is twice the key table the CAS walks), so off by default
    bool fast_build = false;
    // register-path accumulator forms, per slot (aggregate scans only):
    //  rdx    integer-valued sum (COUNT, integer SUM, float SUM of an integer
    //         input) kept as a double, exact while |sum| <= 2^53
    //  ralias slot whose accumulator this slot shares (-1: its own)
    //  rfma   float SUM of a never-NaN/inf value, updated as fma(v, hit, acc)
    std::vector<char> rdx, rfma;
    std::vector<int> ralias;
    // register path, merge folded into the scan: blocks add their partials
    // into global accumulators (float sums as exact fixed-point digits) and
    // the last block writes the merged row; racc holds those accumulators
    // (kept at their identities between runs) and the arrival counter
    bool rfused = false;
    int rcopies = 0;  // copies of those accumulators (block b adds into copy b % rcopies); 0: chosen with the fold
    DevBuf racc;
    // HAVING over the merged output (exec.Filter above the aggregate,
    // planner/build.go:59-75): predicate IR over the output columns (group-by
    // columns, then aggregates) typed by a host-only schema table, and the
    // number of leading output columns kept (buildHavingProjection,
    // planner/build.go:617-637); -1: none
    std::vector<INode> having_ir;
    int having_root = -1;
    int having_visible = -1;
    std::unique_ptr<Table> having_schema;
    // HAVING on the device over the compacted group table (empty: host)
    std::string src_having;
    JitKernel k_having;
    // value-range epochs of the tables the plan was compiled against
    uint64_t range_epoch = 0, brange_epoch = 0;
    int btile = 128, bsmem = 0;  // join build kernel
    // per-run caches (host-side overhead of a run)
    std::vector<long long> seg_cache;      // last uploaded segment list
    DevBuf d_seg;
    std::vector<long long> bseg_cache;     // join build side: last uploaded segment list
    DevBuf d_bseg;
    DevBuf d_kinds;                        // register-path combiner kinds
    DevBuf d_tinit;                        // group tables: identities of the int bank, float-sum windows
    PinnedBuf h_stage;                     // pinned staging for small results
    void* h_stage_mapped = nullptr;        // its device address (null: not addressable, copy back)
    void* h_stage_mapped_for = nullptr;    // the staging allocation that address belongs to
    bool regs_err_clean = false;           // register path: the error word is zero (the merge clears it)
    // a submitted register-path run whose result has not been read: its
    // output is in h_stage until the result settles (the next run of the
    // plan, or its destruction, settles it first)
    vexq_result_s* pending = nullptr;
    bool submit_lazy = false;              // set for the duration of a vexq_plan_submit call
    ScanMemo scan_memo;                    // main-table pruning of the last run's row-group range
    ScanMemo build_memo;                   // join build side's pruning (whole table), until its zone maps change
    long long hash_groups_seen = -1;       // hash path: groups the last run found (sizes the next table)
    // dense path: the kernel accumulates hot_n groups per thread in registers;
    // which groups is a launch value, the largest-count groups of the last run
    int hot_n = 0;
    // dense path, shared-memory cache: counts added as 32-bit atomics on the
    // counter's low word; fixed-point digits as 32-bit atomics with the carry
    // (from the returned old value) added to the high word
    bool cache_cnt32 = false, cache_fx32 = false;
    bool cache_limbs = false;      // cached float sums as 16-bit limbs (plain adds, normalised every 32,768 rows)
    std::vector<unsigned long long> hot_keys;
    mutable std::mutex hot_mu;
    long long hash_rows_seen = 0;          //   and the rows that run scanned
    // GROUP BY exactly the (non-NULL int64) join key on a group-table path:
    // the global join numbers the build's distinct keys (0..nk-1) and the
    // group table is indexed by that number (gid_koff: the key's code offset)
    bool join_gid = false;
    long long gid_koff = 0;
    long long gid_groups = 0;              // group numbers the last build handed out
    long long join_keys_seen = -1;         // join build: distinct keys the last build inserted
    long long join_rows_seen = 0;          //   from this many build rows
    bool join_fast_failed = false;         // a one-pass (unique-key) build met a repeated key
    bool join_unique_seen = false;         // the last build inserted every key once
    // direct-mapped build table: a word per value of the build key column's
    // range [imin, imax] (keys unique and the range at most a few times the
    // build rows); a build that meets a repeated key takes the hash table
    bool dmap_on = true;                   // allowed (VEXQ_TUNE dmap=0 turns it off)
    bool dmap_failed = false;              // a direct-mapped build met a repeated key
    bool dmap_used = false;                // the last build was direct-mapped
    bool spec_on = true;                   // a repeated direct-mapped build goes without a host wait (VEXQ_TUNE spec=0: off)
    DevBuf jt_dmap;
    cudaEvent_t ev[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // [4], [5]: join build phase
    // the register path's launches captured as a graph, replayed while
    // rg_key matches (graph_off: capture was refused, direct launches)
    cudaGraphExec_t rg_exec = nullptr;
    RegsGraphKey rg_key{};
    bool graph_off = false;
    long long topk_seen = 0;       // top-k candidates the last run gathered (sizes the next copy back)
    std::atomic<bool> cancel{false};
    cudaStream_t stream = nullptr;       // the plan's own stream (created lazily)
    cudaStream_t ext_stream = nullptr;   // caller-owned stream, when set
    // scratch reused across runs
    DevBuf scratch_a, scratch_b, scratch_c, scratch_d, scratch_e, scratch_f, scratch_g;
    DevBuf jt_keys, jt_count, jt_start, jt_fill, jt_rows, jt_scalar, jt_meta, jt_long, jt_sort, jt_first, jt_gid, jt_gkey;
    // radix-partitioned join: kernels and buffers
    bool radix = false;
    std::string src_part_b, src_part_p, src_rjoin;
    JitKernel k_part_b, k_part_p, k_rjoin;
    DevBuf rp_bkeys, rp_brows, rp_qkeys, rp_qrows, rp_hist, rp_off, rp_start, rp_scalar;
    std::vector<int> qpay_cols;    // probe columns carried in the partition payload (≤ 8)
    bool rlocal = false;           // GROUP BY the join key: groups aggregated per partition in shared memory
    int rcap = VQ_RADIX_CAP;       // build entries a partition may hold
    DevBuf rp_qpay[8], rp_qpayv[8];
    ~Plan();
};

// Host result columns (group-insertion order, after ORDER BY / LIMIT).
struct OutColumn {
    std::string name;
    int type;
    std::vector<int64_t> v;      // raw bits (int64 / float64 / date / bool / string code)
    std::vector<uint8_t> valid;
    const GlobalDict* dict = nullptr;
};

Plan* compile_agg(Table* t, const vexq_agg_plan_desc* d);
Plan* compile_join(Table* bt, Table* pt, const vexq_join_plan_desc* d);
Plan* compile_filter(Table* t, const vexq_expr* nodes, int nnodes, const int32_t* children, int nchildren, int pred);
// Filter (pred >= 0, else every row) → Project (nroots expressions, 0: none)
// over one table: k_main = vq_pmark (selection bitmap), k_build = vq_pwrite
// (kept rows' projected values in row order); key_nodes = the expressions' IR.
Plan* compile_select(Table* t, const vexq_expr* nodes, int nnodes, const int32_t* children, int nchildren, int pred,
                     const int32_t* roots, int nroots);
void set_having(Plan& p, const vexq_expr* nodes, int nnodes, const int32_t* children, int nchildren, int root, int visible);
bool zone_eval(const Plan& p, int root, const Table& t, int rg);
// Copies the plan's launch-time constants (literals, float-sum windows, cache size) into P.
void set_plan_constants(const Plan& p, VQParams& P);
// Fails when a table the plan reads was re-filled with values outside the
// ranges (or finiteness) the plan's kernels were generated for.
void check_ranges(const Plan& p);
// Source of one batched launch over aggregate plans of one class: a body per
// distinct plan shape (body_of[i] for plans[i]) and the vq_batch dispatcher;
// smem = dynamic shared memory the bodies need beyond the dense caches.
std::string gen_batch_source(const std::vector<Plan*>& plans, int block, std::vector<int>& body_of, int& smem,
                             int& nbodies, bool build_role = false);
// Groups a dense plan caches in shared memory within cache_kb KB (0: not dense).
int dense_cache_groups(const Plan& p, int cache_kb);
int cache_group_bytes(const Plan& p);  // shared-memory cache bytes a group
int cache_bytes(const Plan& p);

// ---- runtime pieces shared by the plain and batched paths (run.cu) ----
// Host-side group rows collected from either path.
struct Groups {
    std::vector<uint64_t> key;
    std::vector<int64_t> first;
    std::vector<std::vector<int64_t>> ival;   // per int-bank slot
    std::vector<std::vector<double>> fval;    // per float-bank slot
    bool having_done = false;                 // HAVING already applied on the device
    size_t n() const { return key.size(); }
};
std::vector<long long> init_values(const Plan& p);
vexq_result_s* build_result(Plan& p, Groups& g);
// Gives the result's STRING columns dictionaries of their own (the strings
// they use, codes renumbered), so the result outlives the tables it read.
void own_dictionaries(vexq_result_s* r);
// Dense path: the groups with the largest counts of a finished run become the
// groups the next run accumulates in registers.
void note_hot_groups(Plan& p, const Groups& g);
int64_t scanned_bytes(const Plan& p, const Table& t, long long rows, bool build);
long long estimate_groups(const Plan& p, long long rows, long long join_keys);
void set_columns(VQParams& P, const Table& t, bool build_side);
vexq_result_s* run_plan(Plan& p, int rg_start, int rg_end);
// The same run, returning as soon as its launches are queued when the plan
// takes the register path (no join, no shard partial): the result settles
// on its first read. Any other plan returns a finished result.
vexq_result_s* run_plan_submit(Plan& p, int rg_start, int rg_end);
// Waits for a submitted run and fills its result (nothing for a finished
// one); throws the run's status, which the result keeps.
void settle(vexq_result_s* r);
// Settles the plan's pending result before its buffers are used again; a
// failure stays with that result (its next read returns it).
void settle_pending(Plan& p);
// One plain run of a plan at a time: its group/join tables are per plan.
std::mutex& plan_mutex(Plan* p);
// VEXQ_SYNC_CHECK=1: synchronise after every launch and name the kernel on
// an error (diagnostics; off by default).
void launch_check(cudaStream_t s, const char* what);
bool launch_checks_on();  // VEXQ_SYNC_CHECK: a synchronize after every launch
void force_join_spec(Plan& p, long long keys_seen);
std::vector<uint8_t> prune_mask(const Plan& p, const Table& t, int root, int rgs, int rge);

// Batched execution of many plans (batch.cu).
struct Batch;
Batch* create_batch(vexq_plan_s* const* handles, int n, uint32_t flags);
void exec_batch(Batch& b, vexq_result_s** out);
void destroy_batch(Batch* b);
// A reusable batch workspace (streams, events, grow-only buffers) and one
// direct, uncaptured execution of a plan set on it (the serving loop's launch).
Batch* new_batch();
void run_batch_direct(Batch& b, vexq_plan_s* const* handles, int n, vexq_result_s** out);
double batch_kernel_ms(const Batch& b);

// Descriptors of batched launches (device arrays).
struct VQTableDesc {           // one group table
    unsigned long long* keys;
    long long* first;
    long long* acc_i;
    long long* acc_fx;
    unsigned* special;
    const long long* init_i;
    const int* fx_lsb;
    long long nslots;
    int ni, nf, hash;
    int gid;                   // a join's build-key-numbered table: keys[] is the number → key array, not initialised
    unsigned long long* n_out;
    unsigned long long* ngroups;
    int* error;
    unsigned long long* o_key;
    long long* o_first;
    long long* o_i;
    double* o_f;
    long long cap_out;
    long long slot0;           // first global slot of this table
};
struct VQMergeDesc {           // one register-path plan's partials
    const double* part_f;
    const long long* part_i;
    int nblocks, G, nf, ni;
    const int* fkind;
    const int* ikind;
    double* out_f;
    long long* out_i;
    int e0;                    // first global merge entry of this plan
};
ScanSegs make_segments(const Table& t, const std::vector<uint8_t>& rg_mask, int rg_start, int rg_end, int unit);
// The row ranges a scan covers: each maximal run of kept row groups in
// [rg_start, rg_end) becomes one (start row, end row, first chunk) triple,
// handed to emit(a, b, chunk0); a range of rows [a, b) takes the chunks of
// `unit` rows from a rounded down to a multiple of unit. Returns the chunks.
// The one place the chunk arithmetic the kernels' segment lookup relies on is
// written (make_segments and the no-allocation run both use it).
template <class Keep, class Emit>
long long walk_segments(const Table& t, Keep&& keep, int rg_start, int rg_end, int unit, Emit&& emit) {
    const long long U = unit;
    long long chunks = 0;
    int rg = rg_start;
    while (rg < rg_end) {
        if (!keep(rg)) { rg++; continue; }
        int e = rg + 1;
        while (e < rg_end && keep(e)) e++;
        const long long a = t.rg_start(rg), b = t.rg_end(e - 1);
        if (b > a) {
            emit(a, b, chunks);
            chunks += (b - (a & ~(U - 1)) + U - 1) / U;
        }
        rg = e;
    }
    return chunks;
}
// Grid of a scan kernel: every SM filled to its occupancy (at most cap_per_sm
// blocks an SM when > 0), never more blocks than loop units.
int grid_for(const JitKernel& k, long long units, bool staged, int cap_per_sm = 0);
// Status of a register-path scan from its error word: bit 8 a staged copy
// timed out, bit 2 a float sum left its exact window; any other bit is a
// device error. Returns normally when the word is 0.
void check_regs_flags(int herr);
bool parse_date(const char* s, int64_t* days);
// Frees the pinned host copy of a table's columns the filter operator reads
// (select.cu); called when the table is destroyed.
void drop_host_mirror(const Table* t);

}  // namespace vq

struct vexq_result_s {
    // a submitted run not yet waited for (vexq_plan_submit): the first read
    // waits for its kernels and fills the fields below; owner is the plan
    // whose staging buffer holds its output until then. A run that failed
    // keeps its status, returned by every later read.
    std::function<void(vexq_result_s*)> settle_fn;
    vq::Plan* owner = nullptr;
    int32_t settle_code = 0;
    std::string settle_msg;
    std::vector<vq::OutColumn> cols;
    int64_t nrows = 0;
    int64_t pos = 0;
    double kernel_ms = 0;
    double scan_ms = 0;
    int32_t launches = 0;
    int64_t rows_scanned = 0, bytes_scanned = 0;
    // current batch views and their storage
    std::vector<vexq_vector_view> views;
    std::vector<std::vector<char>> vbuf;
    std::vector<std::vector<uint8_t>> bbuf;
    std::vector<std::vector<uint32_t>> doff;
    std::vector<std::string> dbytes;
    // the strings of the result's STRING columns, copied out of the tables'
    // dictionaries: a result stays readable after its plan and tables are gone
    std::vector<std::unique_ptr<vq::GlobalDict>> owned_dicts;
};

// Opaque handles of the C ABI.
struct vexq_table_s {
    vq::Table* t;
};
struct vexq_plan_s {
    vq::Plan* p;
    vexq_table_s* table;
    int64_t footprint;  // bytes of group/join tables a run allocates (admission)
};
