/*
 * mettle_oracle.h — CPU oracle for the offloaded SQL subset (TEST INFRASTRUCTURE).
 *
 * This library is the parity checker and the timed CPU baseline. It is NOT
 * part of the product: only tests/, __graft_entry__.smoke() and bench.py's
 * CPU legs load it. It restates, on the host, the semantics that the
 * reference's GPU path approximates and that DuckDB (the reference's own
 * correctness oracle, DuckDB v1.5.1 pinned in Cargo.lock:513-515) defines:
 *
 *   - predicate compare ops follow the op codes of
 *     src/metal/shaders/kernels.metal:70-173 (0 '=', 1 '<', 2 '<=', 3 '>', 4 '>=');
 *   - selection vectors are row ids in ascending order (the reference's
 *     filter_to_indices, kernels.metal:684, is unordered; order is a choice
 *     of this build and the product matches it);
 *   - INTEGER/BIGINT arithmetic is exact with DuckDB's overflow error;
 *     FLOAT arithmetic is IEEE binary32;
 *   - SUM(BIGINT) is a 128-bit integer (DuckDB HUGEINT), AVG(BIGINT) is
 *     (long double)sum / (long double)count rounded to double (DuckDB's
 *     IntegerAverageOperationHugeint), SUM/AVG(FLOAT) accumulate in
 *     extended precision (the "FP64 sum" the tolerance is stated against);
 *   - DECIMAL(15,2) is a scaled int64; price*(1-discount) is the scale-4
 *     product price_cents*(100-discount_cents), summed in 128 bits;
 *   - grouped top-K ties are ordered by the full ORDER BY, then by the
 *     remaining group keys ascending (kernels.metal:1102-1118 orders ties by
 *     sum DESC, secondary ASC, row id ASC).
 *
 * Parallel loops use OpenMP; thread count follows OMP_NUM_THREADS.
 */
#ifndef METTLE_ORACLE_H
#define METTLE_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Column physical types understood by orc_filter. */
#define ORC_I32 1
#define ORC_I64 2
#define ORC_F32 3
#define ORC_F64 4

/* Conjunctive filter: rows where every predicate holds, ascending row ids.
 * ilits hold integer literals, flits float literals (compared in the column's
 * own type, i.e. (float)flit for ORC_F32). Returns the number of rows. */
int64_t orc_filter(int32_t n_pred, const void *const *cols, const int32_t *types,
                   const int32_t *ops, const int64_t *ilits, const double *flits,
                   int64_t n, int64_t *out_rows);

/* Gathers/projections over a selection vector. Return 0, or 1 on overflow. */
int32_t orc_gather_i32(const int32_t *col, const int64_t *rows, int64_t s, int32_t *out);
int32_t orc_gather_i64(const int64_t *col, const int64_t *rows, int64_t s, int64_t *out);
int32_t orc_gather_f32(const float *col, const int64_t *rows, int64_t s, float *out);
int32_t orc_gather_i32_mul(const int32_t *col, const int64_t *rows, int64_t s, int32_t k, int32_t *out);
int32_t orc_gather_i32_add(const int32_t *col, const int64_t *rows, int64_t s, int32_t k, int32_t *out);
int32_t orc_gather_i64_add(const int64_t *col, const int64_t *rows, int64_t s, int64_t k, int64_t *out);
int32_t orc_gather_i64_mul(const int64_t *col, const int64_t *rows, int64_t s, int64_t k, int64_t *out);
int32_t orc_gather_f32_mul(const float *col, const int64_t *rows, int64_t s, float k, float *out);

/* Stable ORDER BY on a 32-bit or 64-bit signed key over a selection vector
 * (ties keep ascending row order). desc != 0 sorts descending. */
void orc_sort_rows_i32(const int32_t *key, int64_t *rows, int64_t s, int32_t desc);
void orc_sort_rows_i64(const int64_t *key, int64_t *rows, int64_t s, int32_t desc);

/* C3: SELECT k, SUM(v), COUNT(*), MIN(v), MAX(v), AVG(v), SUM(f), MIN(f),
 * MAX(f), AVG(f) FROM t GROUP BY k ORDER BY SUM(v) DESC, k LIMIT limit.
 * When limit < 0 every group is returned, ordered by k ascending.
 * Output arrays must hold min(limit, groups) (or all groups) entries; sums
 * are 128-bit as (lo, hi) pairs. Returns the number of groups written, and
 * the total number of groups in *n_groups. */
int64_t orc_groupby_c3(const int64_t *k, const int64_t *v, const float *f, int64_t n,
                       int64_t limit, int64_t *n_groups,
                       int64_t *o_key, uint64_t *o_sumv_lo, int64_t *o_sumv_hi,
                       int64_t *o_count, int64_t *o_minv, int64_t *o_maxv, double *o_avgv,
                       double *o_sumf, float *o_minf, float *o_maxf, double *o_avgf);

/* AVG of a BIGINT column as DuckDB computes it: 128-bit sum, then
 * (long double)sum / (long double)count rounded to double. */
double orc_avg_i128(uint64_t sum_lo, int64_t sum_hi, int64_t count);

/* C4 (TPC-H Q3 shape), all DECIMAL(15,2) values as int64 cents:
 *   SELECT l_orderkey, SUM(l_extendedprice*(1-l_discount)) AS revenue,
 *          o_orderdate, o_shippriority
 *   FROM customer, orders, lineitem
 *   WHERE c_mktsegment = seg AND c_custkey = o_custkey
 *     AND l_orderkey = o_orderkey AND o_orderdate < d AND l_shipdate > d
 *   GROUP BY l_orderkey, o_orderdate, o_shippriority
 *   ORDER BY revenue DESC, o_orderdate [, l_orderkey] LIMIT limit
 * revenue is at scale 4 as a 128-bit (lo, hi) pair. Keys need not be dense
 * or unique on the fact side; the build keys c_custkey and o_orderkey must
 * be unique (primary keys), as in the reference's PK-FK join
 * (kernels.metal:175-209). Returns rows written; *n_groups gets the group
 * count. limit < 0 returns every group in that order. */
int64_t orc_q3(const int32_t *c_custkey, const int32_t *c_segment, int64_t n_cust,
               const int32_t *o_orderkey, const int32_t *o_custkey, const int32_t *o_orderdate,
               const int32_t *o_shippriority, int64_t n_ord,
               const int32_t *l_orderkey, const int64_t *l_price, const int64_t *l_discount,
               const int32_t *l_shipdate, int64_t n_li,
               int32_t segment, int32_t date, int64_t limit, int64_t *n_groups,
               int32_t *o_key, uint64_t *o_rev_lo, int64_t *o_rev_hi, int32_t *o_date,
               int32_t *o_prio);

/* Date helpers (civil date <-> days since 1970-01-01), the same civil
 * algorithm as src/plan/parser.rs:426-449. */
int32_t orc_days_from_civil(int32_t y, int32_t m, int32_t d);
void orc_civil_from_days(int32_t days, int32_t *y, int32_t *m, int32_t *d);

/* Number of OpenMP threads the oracle uses. */
int32_t orc_threads(void);

#ifdef __cplusplus
}
#endif
#endif
