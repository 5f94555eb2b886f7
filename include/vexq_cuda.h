/*
 * vexq_cuda.h — C ABI of libvexqcuda, the B200 (sm_100a) execution path for
 * vexq's Filter → Project → HashAggregate / ParallelHashAggregate /
 * ParallelHashJoinAggregate operators.
 *
 * The ABI is shaped for one cgo crossing per query phase (upload, plan, run,
 * fetch), never one per 1024-row batch. Every entry point takes plain
 * pointers and sizes, returns an int32 status (0 = ok, negative = error) and
 * records a message retrievable with vexq_last_error() on the calling thread.
 *
 * Reference interfaces each group of entry points stands in for (paths are
 * within the vexq repository):
 *   tables    storage.Open / Reader.OpenColumn / ColumnReader.NextBlock +
 *             Dictionary()            storage/reader.go:186,203; storage/rowgroup.go:101-193
 *   zone maps planner.buildZonePredicate / zonePredEval / zoneRangePred
 *                                     planner/physical.go:624-750
 *   agg plan  exec.NewFilter / exec.NewHashAggregate /
 *             exec.NewParallelHashAggregate
 *                                     exec/filter.go:40; exec/aggregate.go:131;
 *                                     exec/parallel.go:78
 *   join plan exec.NewParallelHashJoinAggregate
 *                                     exec/parallel_join.go:718
 *   results   Operator.Next / Schema / Close
 *                                     exec/operator.go:28-32
 *   filter    Filter.Next + BoolToSelVecInto
 *                                     exec/filter.go:49-78; exec/expr.go:1545-1564
 */
#ifndef VEXQ_CUDA_H
#define VEXQ_CUDA_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VEXQ_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------ */
enum {
    VEXQ_OK         = 0,
    VEXQ_EINVAL     = -22,   /* bad argument / unsupported plan shape        */
    VEXQ_ENOMEM     = -12,   /* device or host allocation failed             */
    VEXQ_EADMIT     = -11,   /* admission rejected: HBM footprint too large  */
    VEXQ_ETIMEDOUT  = -110,  /* a bounded device wait ran out                */
    VEXQ_EDEVICE    = -5,    /* CUDA runtime / driver error                  */
    VEXQ_ECANCELED  = -125,  /* cancelled through vexq_cancel                */
    VEXQ_ENOTSUP    = -95,   /* feature outside the supported subset         */
    VEXQ_ECORRUPT   = -74,   /* a .vxq file fails a checksum or does not parse
                                (storage.ErrChecksum / ErrCorruptFooter /
                                ErrBadMagic, storage/errors.go:9-17)         */
    VEXQ_EJIT       = -201   /* kernel specialisation failed to compile      */
};

/* ---- column types: the numeric values of storage.DataType
 *      (storage/format.go:30-36) ----------------------------------------- */
enum {
    VEXQ_TYPE_INT64   = 1,
    VEXQ_TYPE_FLOAT64 = 2,
    VEXQ_TYPE_BOOL    = 3,
    VEXQ_TYPE_STRING  = 4,   /* dictionary coded, uint32 codes             */
    VEXQ_TYPE_DATE    = 5    /* int32 days since 1970-01-01                */
};

/* BlockRows (storage/format.go:8): rows per batch handed out by Next. */
#define VEXQ_BLOCK_ROWS 1024
/* RowGroupRows (storage/format.go:10): default row-group size. */
#define VEXQ_ROW_GROUP_ROWS 65536

/* ---- library ------------------------------------------------------------ */

/* Binds the calling thread's CUDA device and creates the library state.
 * Replaces nothing in the reference (the Go engine has no device). */
int32_t vexq_init(int32_t device, uint32_t flags);
/* Message of the last failing call on this thread ("" if none). */
const char* vexq_last_error(void);
/* ABI version compiled into the library. */
int32_t vexq_abi_version(void);

/* ---- tables --------------------------------------------------------------
 * One host column as the reference's storage layer hands it to TableScan:
 * fixed-width little-endian values plus an LSB-first validity bitmap
 * (1 = valid, storage/codec.go:13-39). STRING columns carry per-row-group
 * dictionaries whose codes are in first-occurrence order
 * (storage/writer.go:374-420); the upload remaps them to one global
 * dictionary per column, the remap accumulateIntKey performs per row group
 * (exec/agg_intkey.go:118-134), done once. */
typedef struct {
    const char*     name;
    int32_t         type;          /* VEXQ_TYPE_*                                  */
    const void*     values;        /* nrows × {int64, double, uint8, uint32, int32} */
    const uint8_t*  validity;      /* (nrows+7)/8 bytes, NULL = no NULLs           */
    /* STRING only ---------------------------------------------------------- */
    const uint32_t* dict_rg_first; /* n_rg+1 entry indices: RG r owns
                                      [dict_rg_first[r], dict_rg_first[r+1]).
                                      NULL: one table-wide dictionary of
                                      dict_entries entries, codes are global    */
    const uint32_t* dict_str_off;  /* total_entries+1 byte offsets into bytes     */
    const char*     dict_bytes;
    int64_t         dict_entries;  /* entries when dict_rg_first is NULL          */
} vexq_column_desc;

typedef struct vexq_table_s*  vexq_table_t;
typedef struct vexq_plan_s*   vexq_plan_t;
typedef struct vexq_result_s* vexq_result_t;

/* Copies the columns to HBM (synchronous: the host buffers may be freed on
 * return, as cgo requires) and computes per-row-group zone maps with the
 * writer's rules (storage/writer.go:205-372). rg_rows = 0 selects 65,536. */
int32_t vexq_table_upload(const vexq_column_desc* cols, int32_t ncols,
                          int64_t nrows, int32_t rg_rows, vexq_table_t* out);
int32_t vexq_table_destroy(vexq_table_t t);
int32_t vexq_table_num_row_groups(vexq_table_t t, int32_t* out);
/* Device bytes held by the table (columns, bitmaps, dictionaries). */
int32_t vexq_table_device_bytes(vexq_table_t t, int64_t* out);
/* ---- .vxq files ------------------------------------------------------------
 * Replaces storage.Open + ColumnReader.NextBlock / Dictionary + TableScan's
 * block decode (storage/reader.go:175-190, 295-408; storage/rowgroup.go:101-
 * 195; exec/scan.go:199-409) for a table that is then scanned on the GPU:
 * the file's footer CRC and every block and dictionary CRC of the selected
 * columns are checked (CRC-32/IEEE, internal/encoding/crc.go), the columns
 * decoded on the host cores and uploaded as vexq_table_upload uploads them,
 * the file's row groups becoming the table's (every row group but the last
 * must hold the same number of rows, else VEXQ_ENOTSUP). `columns` names the
 * columns to load, in the table's order; NULL loads every column. Corrupt
 * files fail with VEXQ_ECORRUPT and a message naming the row group, column
 * and file offset. */
int32_t vexq_table_load_vxq(const char* path, const char* const* columns, int32_t ncolumns,
                            vexq_table_t* out);
/* Host-only check of a whole file (no device): footer, every block and
 * dictionary CRC, RLE and dictionary structure, dictionary codes in range.
 * The block checks `vexq fsck` makes (runFsck, cmd/vexq/main.go:241-330). */
typedef struct {
    int64_t nrows;
    int32_t ncols;
    int32_t n_rg;
    int32_t rg_rows;        /* rows of every row group but the last */
    int32_t null_columns;   /* columns holding at least one NULL     */
    int64_t bytes_checked;  /* column section bytes read and verified */
} vexq_vxq_summary;
int32_t vexq_vxq_verify(const char* path, vexq_vxq_summary* out);

/* Zone map of (column, row group): storage.ZoneMap (storage/schema.go:26-35). */
typedef struct {
    int64_t  null_count;
    int64_t  sum;          /* raw bits, as the writer stores them */
    uint64_t min, max;     /* raw bits                             */
    int32_t  has_min_max;
} vexq_zone_map;
int32_t vexq_table_zone_map(vexq_table_t t, int32_t col, int32_t rg, vexq_zone_map* out);
/* Global dictionary of a STRING column: number of entries and entry i. */
int32_t vexq_table_dict_size(vexq_table_t t, int32_t col, int32_t* out);
int32_t vexq_table_dict_entry(vexq_table_t t, int32_t col, int32_t code,
                              const char** out, int32_t* len);

/* ---- expressions -----------------------------------------------------------
 * SQL-level expression nodes (sql/ast.go) over a table's columns. The library
 * performs the planner's translation to executable form itself: literal
 * coercion (planner/physical.go:773-818), StringEqExpr selection (:548-566),
 * int→float casts (:575-588), BETWEEN→AND(GE,LE) (exec/expr.go:1328-1339),
 * and derives the zone-map predicate from the same tree (:624-750).
 * Children of node n are children[n.child0 .. n.child0+n.nchildren-1]:
 *   BINARY  [left, right]             AND/OR [a, b, ...]     NOT/NEG [x]
 *   IS_NULL / IS_NOT_NULL [x]         BETWEEN [x, lo, hi]    (op=1: NOT)
 *   IN [x, lit...] (op=1: NOT IN)     LIKE [x, pattern] (op=1: NOT LIKE)
 *   CASE [cond0, res0, cond1, res1, ..., else?]  (op=1: has ELSE)        */
enum {
    VEXQ_E_COLUMN = 1, VEXQ_E_LITERAL, VEXQ_E_BINARY, VEXQ_E_AND, VEXQ_E_OR,
    VEXQ_E_NOT, VEXQ_E_NEG, VEXQ_E_IS_NULL, VEXQ_E_IS_NOT_NULL, VEXQ_E_BETWEEN,
    VEXQ_E_IN, VEXQ_E_LIKE, VEXQ_E_CASE
};
enum {
    VEXQ_OP_EQ = 1, VEXQ_OP_NE, VEXQ_OP_LT, VEXQ_OP_LE, VEXQ_OP_GT, VEXQ_OP_GE,
    VEXQ_OP_ADD, VEXQ_OP_SUB, VEXQ_OP_MUL, VEXQ_OP_DIV
};
enum { VEXQ_LIT_INT = 1, VEXQ_LIT_FLOAT, VEXQ_LIT_STRING, VEXQ_LIT_BOOL };

typedef struct {
    int32_t     kind;       /* VEXQ_E_*                                        */
    int32_t     op;         /* BINARY: VEXQ_OP_*; BETWEEN/IN/LIKE: 1 = negated;
                               CASE: 1 = has ELSE                              */
    int32_t     column;     /* COLUMN: column index in the node's scope        */
    int32_t     lit_kind;   /* LITERAL: VEXQ_LIT_*                             */
    int64_t     lit_int;    /* INT and BOOL literals                           */
    double      lit_float;
    const char* lit_str;    /* STRING literal, NUL terminated                  */
    int32_t     child0;
    int32_t     nchildren;
} vexq_expr;

/* AggKind values of exec/aggregate.go:15-21 (COUNT DISTINCT is not offered:
 * the reference's planner runs it serially, planner/parallel.go:224-228). */
enum { VEXQ_AGG_COUNT = 0, VEXQ_AGG_SUM = 1, VEXQ_AGG_AVG = 2,
       VEXQ_AGG_MIN = 3, VEXQ_AGG_MAX = 4,
       /* COUNT(DISTINCT col): the number of distinct non-NULL values per group
        * (exec/aggregate.go:117-124, 474-493, 810-823); never NULL. Strings
        * compare by value, every other type by its raw 64-bit image. */
       VEXQ_AGG_COUNT_DISTINCT = 5 };

typedef struct {
    int32_t     kind;       /* VEXQ_AGG_*                                      */
    int32_t     input;      /* expression root; -1 = COUNT(*)                  */
    const char* out_name;
} vexq_agg_desc;

/* ORDER BY <output column> [DESC] LIMIT n applied to the merged aggregate,
 * as planner.Parallel wraps ExternalSort + Limit (planner/parallel.go:241-266).
 * sort_col = -1: no sort; limit = -1: no limit. */
typedef struct {
    int32_t sort_col;
    int32_t descending;
    int64_t limit;
} vexq_order_desc;

/* Filter → (Project) → HashAggregate over one table. */
typedef struct {
    const vexq_expr*     nodes;     int32_t nnodes;
    const int32_t*       children;  int32_t nchildren;
    int32_t              predicate; /* root of WHERE, -1 = none            */
    const int32_t*       group_by;  int32_t ngroup_by;  /* column indices   */
    const vexq_agg_desc* aggs;      int32_t naggs;
    vexq_order_desc      order;
} vexq_agg_plan_desc;

/* Filter(build) ⋈ Filter(probe) → (residual Filter) → HashAggregate.
 * Node COLUMN indices are scoped: build_predicate over the build table,
 * probe_predicate over the probe table, and residual / group_by / aggs over
 * the joined schema (build columns, then probe columns), as HashJoin lays out
 * its output (exec/join.go:59-61). */
typedef struct {
    const vexq_expr*     nodes;     int32_t nnodes;
    const int32_t*       children;  int32_t nchildren;
    int32_t              build_key;        /* build-table column (INT64/DATE) */
    int32_t              probe_key;        /* probe-table column              */
    int32_t              build_predicate;  /* -1 = none                       */
    int32_t              probe_predicate;
    int32_t              residual;         /* over the joined schema          */
    const int32_t*       group_by;  int32_t ngroup_by;
    const vexq_agg_desc* aggs;      int32_t naggs;
    vexq_order_desc      order;
    int32_t              radix_bits;       /* -1 = autotuned                  */
} vexq_join_plan_desc;

/* Compiles a plan against a table: resolves types, coerces literals, builds
 * the zone predicate, chooses the aggregation strategy and generates the
 * specialised sm_100a kernel (cached per plan signature). */
int32_t vexq_agg_plan_create(vexq_table_t t, const vexq_agg_plan_desc* d, vexq_plan_t* out);
int32_t vexq_join_plan_create(vexq_table_t build, vexq_table_t probe,
                              const vexq_join_plan_desc* d, vexq_plan_t* out);
int32_t vexq_plan_destroy(vexq_plan_t p);
/* HAVING over the merged aggregate: the Filter the planner puts above the
 * aggregate (planner/build.go:59-75), evaluated with the WHERE expression
 * rules (exec/filter.go:49-78) over the plan's output columns — group-by
 * columns, then aggregates, in order — before ORDER BY / LIMIT. Node COLUMN
 * indices are output column indices. Then only the first `visible` output
 * columns are kept (-1: all), dropping the hidden aggregates the planner
 * appends for a HAVING aggregate missing from the SELECT list
 * (rewriteHavingAggs / buildHavingProjection, planner/build.go:512-637).
 * predicate = -1 removes the HAVING. Plans with HAVING return every group
 * to the host before the sort (no device top-k). */
int32_t vexq_plan_set_having(vexq_plan_t p, const vexq_expr* nodes, int32_t nnodes,
                             const int32_t* children, int32_t nchildren, int32_t predicate,
                             int32_t visible);
/* Short description of the chosen strategy (for logs and tests). */
const char* vexq_plan_explain(vexq_plan_t p);

/* Zone-map pruning on the host: out_mask[rg] = 1 where the row group may
 * hold a matching row (TableScan's skip, exec/scan.go:212-215). */
int32_t vexq_zone_prune(vexq_plan_t p, uint8_t* out_mask, int32_t n_rg);

/* Runs the plan over row groups [rg_start, rg_end) (rg_end = -1: all) and
 * returns the merged result on the host. Synchronous on the plan's stream. */
int32_t vexq_plan_run(vexq_plan_t p, int32_t rg_start, int32_t rg_end, vexq_result_t* out);

/* Submits the same run and returns once its launches are queued, when the
 * plan takes the register path (no join); any other plan returns a finished
 * result as vexq_plan_run does. The first read of the result
 * (vexq_result_info, _num_rows, _num_cols, _next, _stats, _scan_ms) waits
 * for the run and returns its status, as the reference's aggregate does its
 * work and reports its error in the first Next
 * (ParallelHashAggregate.Next, exec/parallel.go:109-120). The plan's next
 * run, vexq_plan_set_having and vexq_plan_destroy settle a pending result
 * first; freeing it unread drops it. Runs of different plans submitted on
 * one stream execute back to back while the host reads the earlier ones.
 * A table is refilled (vexq_plan_run_host) only while no run over it is
 * pending on another stream. */
int32_t vexq_plan_submit(vexq_plan_t p, int32_t rg_start, int32_t rg_end, vexq_result_t* out);

/* Same as vexq_plan_run, but the plan's table columns are first re-filled
 * from the given HOST buffers (same layout as at upload) inside the call:
 * the end-to-end form used when the caller owns the data in host memory. */
int32_t vexq_plan_run_host(vexq_plan_t p, const vexq_column_desc* cols, int32_t ncols,
                           vexq_result_t* out);

/* ---- results: the Next/Schema contract --------------------------------- */
typedef struct {
    const char*     name;
    int32_t         type;      /* VEXQ_TYPE_*                                */
    const void*     values;    /* length × {int64, double, int32, uint32 code} */
    const uint8_t*  validity;  /* LSB-first, 1 = valid                        */
    /* STRING: codes index this batch's dictionary (exec.newStringVector) */
    const uint32_t* dict_str_off;  /* dict_len+1 offsets */
    const char*     dict_bytes;
    int32_t         dict_len;
} vexq_vector_view;

typedef struct {
    int32_t                 ncols;
    int32_t                 length;   /* 0 at EOF                         */
    const vexq_vector_view* cols;     /* valid until the next call        */
} vexq_batch_view;

int32_t vexq_result_num_rows(vexq_result_t r, int64_t* out);
int32_t vexq_result_num_cols(vexq_result_t r, int32_t* out);
/* Next(): ≤ VEXQ_BLOCK_ROWS rows in group-insertion order (first occurrence
 * in row order, the serial HashAggregate's order, exec/aggregate.go:209-216);
 * length 0 = EOF. A global aggregate over no rows yields one row
 * (exec/aggregate.go:961-982). */
int32_t vexq_result_next(vexq_result_t r, vexq_batch_view* out);
int32_t vexq_result_free(vexq_result_t r);
/* Device timing of the last run: kernel milliseconds and launches. */
int32_t vexq_result_stats(vexq_result_t r, double* kernel_ms, int32_t* launches,
                          int64_t* rows_scanned, int64_t* bytes_scanned);
/* Duration of the run's scan kernel launches (CUDA events on the plan's
 * stream), in milliseconds. On the register path a scan and the partial merge
 * launched as its programmatic dependent overlap, and the pair is timed as
 * one span; the atomic paths time the scan alone. */
int32_t vexq_result_scan_ms(vexq_result_t r, double* out);
/* Everything above in one call (rows, columns, kernel and scan milliseconds,
 * launches, rows and bytes scanned); any pointer may be NULL. No reference
 * counterpart: it saves a binding one crossing per accessor. */
typedef struct {
    int64_t nrows;
    int32_t ncols;
    int32_t launches;
    double  kernel_ms;
    double  scan_ms;
    int64_t rows_scanned;
    int64_t bytes_scanned;
} vexq_result_summary;
int32_t vexq_result_info(vexq_result_t r, vexq_result_summary* out);

/* Runs a plan on a caller-owned CUDA stream (a cudaStream_t, e.g. the stream
 * the caller times with events); NULL restores the plan's own stream. A
 * submitted run still pending settles first, and one freed unread is waited
 * for. No reference counterpart: the Go engine has no streams. */
int32_t vexq_plan_set_stream(vexq_plan_t p, void* stream);

/* ---- standalone filter: Filter.Next + BoolToSelVecInto ----------------- */
/* Evaluates a predicate over rows [row_start, row_end) and writes a
 * selection bitmap (bit i = row row_start+i passes; LSB-first) into out_bits
 * (host, (n+7)/8 bytes) and the number of selected rows into *count. */
int32_t vexq_filter_run(vexq_table_t t, const vexq_expr* nodes, int32_t nnodes,
                        const int32_t* children, int32_t nchildren, int32_t predicate,
                        int64_t row_start, int64_t row_end,
                        uint8_t* out_bits, int64_t* count);
/* Selection vectors of one 1024-row block from a selection bitmap: the
 * []uint16 SelVec of exec/batch.go:10 (physical indices within the block). */
int32_t vexq_selvec_from_bits(const uint8_t* bits, int64_t nrows, int64_t block,
                              uint16_t* out_sel, int32_t* out_len);

/* ---- Filter as a streaming operator: exec.Filter over exec.TableScan ----
 * Replaces exec.NewFilter(TableScan, predicate) and its Next
 * (exec/filter.go:40-78, exec/scan.go:199-236). Open evaluates the predicate
 * once over the row groups [rg_start, rg_end) (rg_end < 0: to the end) that
 * the zone maps keep, and builds every 1024-row block's selection vector on
 * the device. Next hands out one block per call, in row order, as the scan's
 * batch with its SelVec installed: the table's columns for the block's rows
 * (from a pinned host copy of the HBM columns, made on first use), `length`
 * = len(SelVec) kept rows among `physical` rows. Blocks where no row
 * survives are skipped, as Filter.Next skips them; length 0 is EOF. A batch
 * never spans two row groups. The views and the SelVec stay valid until the
 * next call on this filter (exec/filter.go:10-28's ownership contract).
 * STRING vectors carry codes of the column's table-wide dictionary, which the
 * view's dictionary fields hold. The table must outlive the filter;
 * re-filling it invalidates open filters. Results (vexq_result_t) own the
 * strings they show and stay readable after their plan and tables are gone. */
typedef struct vexq_filter_s* vexq_filter_t;
typedef struct {
    int32_t                 ncols;
    int32_t                 length;    /* len(SelVec); 0 at EOF              */
    int32_t                 physical;  /* rows in the vectors (<= 1024)      */
    int32_t                 rg;        /* row group of the block             */
    int64_t                 row0;      /* table row of the vectors' first row */
    const uint16_t*         sel;       /* ascending indices into [0, physical) */
    const vexq_vector_view* cols;      /* every column of the table          */
} vexq_filter_batch;
int32_t vexq_filter_open(vexq_table_t t, const vexq_expr* nodes, int32_t nnodes,
                         const int32_t* children, int32_t nchildren, int32_t predicate,
                         int32_t rg_start, int32_t rg_end, vexq_filter_t* out);
int32_t vexq_filter_next(vexq_filter_t f, vexq_filter_batch* out);
/* Rows kept, blocks scanned, and the device milliseconds of open. */
int32_t vexq_filter_stats(vexq_filter_t f, int64_t* selected, int64_t* blocks, double* kernel_ms);
int32_t vexq_filter_close(vexq_filter_t f);

/* ---- Project over a filtered scan: exec.Project -------------------------
 * Replaces exec.NewProject(Filter(TableScan), exprs) (exec/project.go:64-128):
 * each of the nexprs expressions (roots into nodes; names may be NULL) is
 * evaluated on the device for the rows the predicate keeps (predicate < 0:
 * every row of the kept row groups), and the kept rows are written compacted
 * in row order, as Project.materialize writes them under a SelVec. The result
 * has no SelVec (rows are materialised) and is read with vexq_result_next in
 * 1024-row batches. A STRING expression must be a column reference. */
int32_t vexq_project_run(vexq_table_t t, const vexq_expr* nodes, int32_t nnodes,
                         const int32_t* children, int32_t nchildren, int32_t predicate,
                         const int32_t* roots, const char* const* names, int32_t nexprs,
                         int32_t rg_start, int32_t rg_end, vexq_result_t* out);

/* ---- batching: many aggregates in one persistent launch ----------------
 * No reference counterpart: the Go engine runs one operator tree per query.
 * A batch holds n prepared plans (each over its own table). Aggregate plans
 * are split by path (register accumulators / group tables); each class runs
 * as ONE persistent launch of a generated kernel with a body per distinct
 * plan shape, whose blocks take (plan, row-chunk range) units from an atomic
 * ticket, largest first. Table init, both launches (on forked streams), the
 * partial merge and the table finalize are captured in a CUDA graph on the
 * first vexq_batch_exec and replayed by every later one, each followed by one
 * copy of all outputs to pinned host memory. A join whose build key column
 * allows a direct-mapped table runs inside the batch: its build as units of a
 * third persistent launch ahead of the other two, its probe as units of the
 * register or group-table class; a join whose build turns out to repeat a key
 * or be empty, and every other join, runs on its own after the graph, one
 * after another. Results match vexq_plan_run's: keys, counts, integer
 * aggregates and group-table float sums bit for bit; register-path float sums
 * may differ in the last bits (a different row partition), both within their
 * stated tolerance. Repeated execs give identical bits.
 * flags: VEXQ_BATCH_AUTOTUNE times graph replays over the shared-memory
 * group-cache size (the shared-versus-global table cutover), the unit size
 * and each class's block shape, and keeps the fastest; the choice is stored
 * in batch_tuning.json beside the kernel cache, keyed by the batch's shape,
 * and a later batch of that shape takes it without timing.
 * VEXQ_BATCH_RETUNE times again and replaces the stored choice. */
#define VEXQ_BATCH_AUTOTUNE 1u
#define VEXQ_BATCH_RETUNE 2u
typedef struct vexq_batch_s* vexq_batch_t;
int32_t vexq_batch_create(vexq_plan_t* plans, int32_t n, uint32_t flags, vexq_batch_t* out);
/* One result per plan, in plan order (each freed with vexq_result_free). */
int32_t vexq_batch_exec(vexq_batch_t b, vexq_result_t* out_results);
/* Last exec: device time of the whole graph replay and of its kernels alone
 * (before the copy back), CUDA events; algorithmic bytes and rows scanned. */
int32_t vexq_batch_stats(vexq_batch_t b, double* device_ms, double* kernel_ms, int64_t* bytes_scanned,
                         int64_t* rows_scanned);
const char* vexq_batch_explain(vexq_batch_t b);
int32_t vexq_batch_destroy(vexq_batch_t b);
/* create + exec + destroy in one call. */
int32_t vexq_batch_run(vexq_plan_t* plans, int32_t n, vexq_result_t* out_results);

/* ---- serving loop ------------------------------------------------------
 * No reference counterpart (the Go engine serves no request loop).
 * Tables and plans stay resident; queries are submitted as prepared plans.
 * Admission: the head of the FIFO queue starts when a query slot is free
 * (max_inflight) and its group/join-table footprint fits hbm_budget_bytes
 * beside the queries in flight. Continuous batching: a free worker takes
 * the queued aggregate queries that fit at that moment (up to
 * max_inflight / nworkers) into ONE batched execution, or one join, so queries
 * arriving while others are on the GPU join the next launch, and the
 * launches of different workers (nworkers, each on its own streams) overlap
 * on the device. flags: VEXQ_SERVE_NO_BATCH runs one query per launch
 * through the plain per-query path. Results match vexq_plan_run's, as the
 * batched execution's do. */
typedef struct vexq_server_s* vexq_server_t;
#define VEXQ_SERVE_NO_BATCH 1u
int32_t vexq_server_start(int64_t hbm_budget_bytes, int32_t max_inflight, int32_t nworkers, uint32_t flags,
                          vexq_server_t* out);
/* Launches so far, queries they carried, the largest launch and the most
 * launches that were running at once. */
int32_t vexq_server_stats(vexq_server_t s, int64_t* launches, int64_t* queries, int32_t* max_batch,
                          int32_t* max_concurrent);
/* Queues plan p; returns a ticket. A plan may be submitted many times. */
int32_t vexq_server_submit(vexq_server_t s, vexq_plan_t p, int64_t* ticket);
/* Non-blocking poll: *done = 1 and *out set when the ticket has finished. */
int32_t vexq_server_poll(vexq_server_t s, int64_t ticket, int32_t* done, vexq_result_t* out);
/* Blocking wait with a timeout in milliseconds (VEXQ_ETIMEDOUT after it). */
int32_t vexq_server_wait(vexq_server_t s, int64_t ticket, int64_t timeout_ms, vexq_result_t* out);
/* Latency (submit → result ready) of a finished ticket, in milliseconds. */
int32_t vexq_server_latency(vexq_server_t s, int64_t ticket, double* ms);
int32_t vexq_server_stop(vexq_server_t s);

/* ---- per-plan tuning ------------------------------------------------------
 * Times the plan's own runs over its launch-time choices and keeps the
 * fastest: a join's build table (0 = the global table, else radix
 * partitioning at 6, 8, 10 or 12 bits — the reference fixes the bits from the
 * build size, RadixBitsFor, exec/parallel_join.go:72-81); a dense group
 * table's shared-memory group cache (0, 48, 96 or 160 KB). Other paths have
 * nothing to choose (*out_choice = -1). The choice is stored in
 * plan_tuning.json beside the kernel cache, keyed by the plan's shape and
 * sizes; a later plan of that shape takes it without timing unless flags has
 * VEXQ_PLAN_RETUNE. *out_ms: the best time measured (0 when stored). */
#define VEXQ_PLAN_RETUNE 1u
int32_t vexq_plan_autotune(vexq_plan_t p, uint32_t flags, int32_t* out_choice, double* out_ms);

/* Host-set cancellation flag polled between launches of a running plan. */
int32_t vexq_cancel(vexq_plan_t p);

/* ---- shards: partials merged in shard order ------------------------------
 * Replaces ParallelHashAggregate's per-worker partial aggregates and
 * mergePartialAgg (exec/parallel.go:124-210, 237-314) with shards of row
 * groups: each shard (one per GPU, each GPU holding the whole table, or a
 * row-group range on one GPU) runs the plan over [rg_start, rg_end) and gets a
 * partial — every group unfinished: key, first-row order key, accumulators.
 * Partials travel as bytes (serialize / deserialize, e.g. over
 * torch.distributed) and vexq_partial_merge folds them in array order — counts
 * and integer sums add, MIN/MAX keep the extreme (the earlier partial's on a
 * tie), float sums add with a compensation term — then applies HAVING, ORDER BY
 * and LIMIT once and returns the result. A join's probe side is sharded; its
 * build side is the whole build table on every shard. COUNT(DISTINCT) returns
 * VEXQ_ENOTSUP (planner/parallel.go:218-228). */
typedef struct vexq_partial_s* vexq_partial_t;
int32_t vexq_plan_run_partial(vexq_plan_t p, int32_t rg_start, int32_t rg_end, vexq_partial_t* out);
/* Groups in the partial and device milliseconds of its run. */
int32_t vexq_partial_info(vexq_partial_t part, int64_t* groups, double* kernel_ms);
/* Bytes of the partial, valid until the next call on it or its free. */
int32_t vexq_partial_serialize(vexq_partial_t part, const void** data, int64_t* len);
/* A partial from bytes made by a plan of the same shape (VEXQ_EINVAL otherwise). */
int32_t vexq_partial_deserialize(vexq_plan_t p, const void* data, int64_t len, vexq_partial_t* out);
int32_t vexq_partial_merge(vexq_plan_t p, const vexq_partial_t* parts, int32_t n, vexq_result_t* out);
int32_t vexq_partial_free(vexq_partial_t part);

/* Fault injection on the host, for tests of the error paths (the reference's
 * counterpart is the failing-operator tests of exec/parallel_join.go:430-476:
 * the first error wins and the query returns it). After `after` more device
 * allocations succeed, the next one fails as cudaMalloc does when memory is
 * exhausted, and the call that made it returns VEXQ_ENOMEM; the injection then
 * switches itself off. -1 switches it off at once. No device fault is made. */
int32_t vexq_debug_fail_alloc(int32_t after);
/* Bytes of device memory the library holds right now (tables, plan buffers,
 * batch workspaces), all devices together: a leak check for the tests. */
int32_t vexq_debug_live_device_bytes(int64_t* out);
/* Makes the join plan's next run take the speculative direct-mapped build (the
 * probe launched without the host reading the build's outcome) as if the last
 * build had been direct-mapped over the same rows with `keys_seen` keys, so a
 * test can reach the probe-raised retries on the host: a build that repeats a
 * key, an empty build, or more keys than the group table sized from
 * `keys_seen` holds. VEXQ_EINVAL for aggregate plans; no device fault is made. */
int32_t vexq_debug_join_spec(vexq_plan_t p, int64_t keys_seen);

/* ---- global aggregate without allocation --------------------------------
 * No counterpart in the reference: its operators work on the Go heap.
 * Runs an aggregate plan without GROUP BY (one result row) through the same
 * scan kernel as vexq_plan_run but allocates no device, pinned or managed
 * memory. The per-block partials are always merged by the separate merge
 * kernel (a fixed-order TwoSum merge); where vexq_plan_run folds the merge
 * into the scan (float sums merged exactly in fixed point), float SUM/AVG
 * may differ from its result by rounding in the last bits. Otherwise the
 * results are equal. Memory: the per-block partials, row ranges, merge outputs and error flag
 * live in one static device array of VEXQ_NOALLOC_SCRATCH_BYTES per device,
 * and the row is written to caller memory. Meant for callers that must not
 * allocate: a serving loop with other queries in flight (cudaMalloc and
 * cudaFree synchronise the whole device) or a caller held to a fixed HBM
 * budget.
 *   stream      cudaStream_t to run on (NULL: the legacy default stream); the
 *               call synchronises it before returning.
 *   out_values  n_out 8-byte cells, one per output column in plan order:
 *               int64 values, float64 bit patterns, dates sign-extended,
 *               bools 0/1.
 *   out_valid   n_out bytes, 0 where the cell is NULL.
 * The first call on a device does set-up (looks up the scratch address and
 * loads the merge kernel's module); make it before any stream capture.
 * Calls that overlap in time race on the shared scratch: issue them one at a
 * time per device. Errors: VEXQ_ENOTSUP for joins and plans with GROUP BY;
 * VEXQ_EINVAL when n_out differs from the plan's output columns, when more
 * than 512 row ranges remain after zone-map pruning, or when the partials do
 * not fit in the scratch even at one block per SM. */
#define VEXQ_NOALLOC_SCRATCH_BYTES (1 << 20)
int32_t vexq_plan_run_global_noalloc(vexq_plan_t plan, int32_t rg_start, int32_t rg_end, void* stream,
                                     int64_t* out_values, uint8_t* out_valid, int32_t n_out);

#ifdef __cplusplus
}
#endif
#endif /* VEXQ_CUDA_H */
