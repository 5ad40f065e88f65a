/*
 * bolt_oracle.h — CPU restatement of the reference's relational hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is the checker the parity tests compare
 * the CUDA library against, and the timed CPU baseline of bench.py. It is
 * never linked into, loaded by or called from the product library.
 *
 * Every function restates a named function of the reference (Craton Bolt,
 * Rust) with its semantics: row order of sequential folds, overflow checks,
 * key packing, NULL handling, float canonicalisation and output order.
 * Pointers here are HOST pointers.
 */
#ifndef BOLT_ORACLE_H
#define BOLT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_I32 = 0, ORC_I64 = 1, ORC_F32 = 2, ORC_F64 = 3, ORC_DEC128 = 4, ORC_U32 = 5 };
enum { ORC_OK = 0, ORC_DECLINE = 1, ORC_OVERFLOW = 3, ORC_CAPACITY = 4, ORC_INVALID = 7 };
enum { ORC_SUM = 0, ORC_COUNT_STAR = 1, ORC_COUNT = 2, ORC_MIN = 3, ORC_MAX = 4, ORC_AVG = 5 };
enum { ORC_LT = 0, ORC_LE = 1, ORC_GT = 2, ORC_GE = 3, ORC_EQ = 4, ORC_NE = 5 };

typedef struct {
    const void* data;
    const uint8_t* validity; /* Arrow LSB bitmap or NULL */
    int32_t dtype;
    int32_t scale;
} orc_col;

typedef struct { int32_t col; int32_t cmp; int64_t lit_i; double lit_f; } orc_pred;
typedef struct { int32_t op; int32_t input_col; } orc_agg;

/* GROUP BY (groupby.rs:295-833 semantics).
 * Outputs (caller-allocated, cap rows each):
 *   out_keys[g]         packed key of group g (sorted ascending as i64);
 *   out_key_null[g]     1 for the NULL-key group (emitted last);
 *   out_vals[a]         per aggregate: int64_t (SUM int, COUNT, MIN/MAX int
 *                       widened), double (SUM/AVG f64, MIN/MAX float widened),
 *                       or 16-byte i128 (SUM DEC128) per group;
 *   out_valid[a][g]     0 when the aggregate is NULL;
 *   out_accurate[a]     optional (may be NULL entries): for f64 SUM/AVG a
 *                       compensated (Neumaier) sum / count, for diagnostics.
 * Returns ORC_OK, ORC_OVERFLOW (message in err), ORC_DECLINE or ORC_CAPACITY. */
int orc_groupby(uint64_t n, const orc_col* cols, int32_t n_cols,
                const int32_t* key_cols, int32_t n_keys,
                const orc_pred* preds, int32_t n_preds,
                const orc_agg* aggs, int32_t n_aggs,
                int64_t* out_keys, uint8_t* out_key_null,
                void** out_vals, uint8_t** out_valid, double** out_accurate,
                uint64_t cap, uint64_t* n_groups, char* err, int32_t err_cap);

/* orc_groupby on `threads` host threads (range partitions of the packed key,
 * each folded in row order by one thread): identical outputs and status. */
int orc_groupby_par(uint64_t n, const orc_col* cols, int32_t n_cols,
                    const int32_t* key_cols, int32_t n_keys,
                    const orc_pred* preds, int32_t n_preds,
                    const orc_agg* aggs, int32_t n_aggs,
                    int64_t* out_keys, uint8_t* out_key_null,
                    void** out_vals, uint8_t** out_valid, double** out_accurate,
                    uint64_t cap, uint64_t* n_groups, char* err, int32_t err_cap, int32_t threads);

/* Packs one row's key exactly as pack_keys (groupby_common.rs:352). */
int64_t orc_pack_key(const orc_col* cols, const int32_t* key_cols, int32_t n_keys, uint64_t row);

/* WHERE conjunction for one row (NULL -> false). */
int orc_row_passes(const orc_col* cols, const orc_pred* preds, int32_t n_preds, uint64_t row);

/* INNER hash join (join.rs:843-858 build_hash_map + probe): pairs
 * (probe_row, build_row) in probe-row order. Duplicate build keys ->
 * ORC_DECLINE (the GPU path's unique-key gate, join.rs:1354-1391). */
int orc_hash_join(uint64_t n_build, const orc_col* build_key,
                  uint64_t n_probe, const orc_col* probe_key,
                  uint32_t* out_probe, uint32_t* out_build, uint64_t cap, uint64_t* n_out);

/* GROUP BY over two integer key columns that do not pack into 64 bits: the
 * reference's host wide-key reduction (src/exec/groupby_wide.rs:85-262): a
 * row with a NULL key is dropped; per group and aggregate, in row order,
 * SUM over integers wraps in i64 (groupby_wide.rs:695-705), SUM / AVG over
 * floats add in f64, MIN / MAX keep the first valid value and replace it
 * only when `x < v` / `x > v` (a NaN never replaces a value), COUNT(col)
 * counts valid inputs; groups ordered by (key0, key1) as signed integers
 * (cmp_tuple, groupby_wide.rs:410). An aggregate with no valid input in its
 * group is reported NULL (valid = 0). Per aggregate a: integer results in
 * out_i[a * cap + g], float results in out_f[a * cap + g]. */
int orc_groupby_wide(uint64_t n, const orc_col* key0, const orc_col* key1, int32_t n_aggs, const int32_t* ops,
                     const orc_col* inputs, int64_t* out_k0, int64_t* out_k1, int64_t* out_i, double* out_f,
                     uint8_t* out_valid, uint64_t cap, uint64_t* n_groups);

/* INNER hash join with any build keys, duplicates included: the reference's
 * host join (join.rs:843-855 build_hash_map keeps each key's build rows in
 * ascending order; join.rs:407-425 probes in row order and emits one pair per
 * matching build row). Pairs ordered by probe row, then build row. */
int orc_hash_join_multi(uint64_t n_build, const orc_col* build_key,
                        uint64_t n_probe, const orc_col* probe_key,
                        uint32_t* out_probe, uint32_t* out_build, uint64_t cap, uint64_t* n_out);

/* Join then GROUP BY build payload: SUM(value) (i128, checked add in probe
 * order, aggregate.rs:1220 message) and COUNT(*), sorted by group. */
int orc_join_groupby(uint64_t n_build, const orc_col* build_key, const int32_t* build_payload,
                     uint64_t n_probe, const orc_col* probe_key, const orc_col* value,
                     int32_t* out_group, int64_t* out_sum_lo, int64_t* out_sum_hi,
                     int64_t* out_count, uint64_t cap, uint64_t* n_groups,
                     char* err, int32_t err_cap);

/* Radix sort keys of gpu_sort.rs:1089-1163 (ASC; DESC = bitwise NOT). */
uint64_t orc_sort_key(const orc_col* key, uint64_t row, int32_t descending);

/* Stable ORDER BY permutation; NULL rows last (or first), in input order. */
int orc_sort_perm(uint64_t n, const orc_col* key, int32_t descending, int32_t nulls_first,
                  uint32_t* perm);
int orc_sort_perm_multi(uint64_t n, const orc_col* keys, int32_t n_keys,
                        const int32_t* descending, const int32_t* nulls_first, uint32_t* perm);

/* Order-preserving filter (compact.rs:61-146): selected row indices. */
int orc_compact(uint64_t n, const orc_col* cols, const orc_pred* preds, int32_t n_preds,
                uint32_t* out_rows, uint64_t* n_out);

/* Fixture generators restated from the reference's tests/common/mod.rs:46-111. */
void orc_xorshift64star_fill(uint64_t seed, uint64_t* out, uint64_t n);
void orc_shuffle_deterministic_u32(uint32_t* xs, uint64_t n, uint64_t seed);

/* Threads used by the batch helpers below (1 = the reference's scalar path). */
void orc_set_threads(int32_t n);

#ifdef __cplusplus
}
#endif

#endif
