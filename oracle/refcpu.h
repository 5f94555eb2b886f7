/*
 * refcpu.h — TEST INFRASTRUCTURE ONLY. CPU oracle for the vexq hot path.
 *
 * A C++ restatement of vexq's Go execution path (no Go toolchain exists in
 * this environment, so the reference cannot be run): Filter → Project →
 * HashAggregate (serial, planner.Physical) and the morsel-parallel
 * ParallelHashAggregate / ParallelHashJoinAggregate, over the same plan
 * descriptors the GPU library accepts (include/vexq_cuda.h). It is linked
 * only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
 * as the checker or as the timed CPU baseline — never by the product path.
 *
 * Parity is pinned by the reference's own known-answer tests (tests/golden/)
 * and, for the filter selection, by the reference's own C++ AVX2 filter
 * kernel compiled from its sources into oracle/_ref/.
 */
#ifndef VEXQ_REFCPU_H
#define VEXQ_REFCPU_H

#include <stdint.h>
#include "../include/vexq_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ref_table_s*  ref_table_t;
typedef struct ref_result_s* ref_result_t;

/* Same column layout as vexq_table_upload; the oracle copies the data. */
int32_t ref_table_new(const vexq_column_desc* cols, int32_t ncols, int64_t nrows,
                      int32_t rg_rows, ref_table_t* out);
void    ref_table_free(ref_table_t t);
/* RadixBitsFor / radixPart (exec/parallel_join.go:72-109). */
int32_t ref_radix_bits_for(int64_t est_rows);
int32_t ref_radix_part(int64_t key, uint64_t mask);
int32_t ref_table_zone_map(ref_table_t t, int32_t col, int32_t rg, vexq_zone_map* out);

/* workers = 0: serial planner.Physical path (strict row-order fold, the
 * deterministic float reference). workers >= 1: ParallelHashAggregate with
 * that many threads, one row group per morsel, partials merged in worker-id
 * order (one admissible order of the reference's channel-arrival merge). */
int32_t ref_agg_run(ref_table_t t, const vexq_agg_plan_desc* d, int32_t rg_start,
                    int32_t rg_end, int32_t workers, ref_result_t* out);
int32_t ref_join_run(ref_table_t build, ref_table_t probe, const vexq_join_plan_desc* d,
                     int32_t workers, ref_result_t* out);
/* Zone-map pruning mask (planner.buildZonePredicate). */
int32_t ref_zone_prune(ref_table_t t, const vexq_agg_plan_desc* d, uint8_t* mask, int32_t n_rg);
/* Filter selection over the whole table: bit i = row i selected. */
int32_t ref_filter_run(ref_table_t t, const vexq_expr* nodes, int32_t nnodes,
                       const int32_t* children, int32_t nchildren, int32_t predicate,
                       uint8_t* out_bits, int64_t* count);

int64_t     ref_result_rows(ref_result_t r);
int32_t     ref_result_cols(ref_result_t r);
int32_t     ref_result_col_type(ref_result_t r, int32_t col);
const char* ref_result_col_name(ref_result_t r, int32_t col);
/* Raw 64-bit value (int64 / float64 bits / date / bool), validity, and for
 * STRING columns the string. */
int32_t ref_result_get(ref_result_t r, int64_t row, int32_t col, int64_t* bits,
                       int32_t* valid, const char** str, int32_t* len);
/* Exact sum (correctly rounded, Shewchuk) of the float aggregate inputs per
 * output row, for SUM/AVG columns; NaN for others. Serial results only. */
int32_t ref_result_exact(ref_result_t r, int64_t row, int32_t col, double* out);
/* Filter (predicate < 0: none) → Project of nroots expressions over row
 * groups [rg_start, rg_end) with zone-map pruning; rows in row order. */
int32_t ref_project_run(ref_table_t t, const vexq_expr* nodes, int32_t nnodes,
                        const int32_t* children, int32_t nchildren, int32_t predicate,
                        const int32_t* roots, int32_t nroots, int32_t rg_start, int32_t rg_end,
                        ref_result_t* out);
/* HAVING over a result, then the column cut and ORDER BY / LIMIT. */
int32_t ref_result_having(ref_result_t r, const vexq_expr* nodes, int32_t nnodes,
                          const int32_t* children, int32_t nchildren, int32_t predicate,
                          int32_t visible, const vexq_order_desc* order);
void    ref_result_free(ref_result_t r);
const char* ref_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
