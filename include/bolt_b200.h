/*
 * bolt_b200.h — C ABI of the B200-native relational hot path.
 *
 * This is the drop-in boundary for the GPU operators of the Craton Bolt
 * engine: hash GROUP BY (shared-memory tier + global hash tier, with an
 * optional fused WHERE), hash-join build/probe (plus the fused
 * join -> GROUP BY build-attribute aggregate), LSD radix sort producing an
 * ORDER BY permutation, prefix-scan filter compaction, and the batched /
 * served filter + GROUP BY forms.
 *
 * Contract (mirrors the reference's borrow-checked launch contract,
 * src/exec/launch.rs:162-368 and src/cuda/smart_ptrs.rs:36-367):
 *   - every `data` / `validity` pointer in a bolt_col_view / bolt_col_mut is
 *     a DEVICE pointer owned by the caller (the reference's GpuVec owns the
 *     allocation, GpuView / GpuViewMut are non-owning borrows);
 *   - inputs are read-only; outputs are written exclusively by the call;
 *   - all work is ordered on the caller's CUDA stream (`bolt_stream` is a
 *     cudaStream_t passed as an opaque pointer; NULL = legacy default stream);
 *   - a call returns after its results (and the row count) are on the host
 *     unless BOLT_FLAG_ASYNC is set, like the reference's synchronising
 *     launch (launch.rs:308-368);
 *   - one bolt_ctx per host thread / stream at a time (the reference's
 *     Engine is !Sync, launch.rs:84-100); different contexts may run
 *     concurrently;
 *   - errors are status codes, never device traps. A device-side bounded
 *     wait or probe limit records a status the host reads back.
 *
 * Validity bitmaps use the Arrow layout: bit (i & 7) of byte (i >> 3) is 1
 * when row i is valid. A NULL validity pointer means "no NULLs".
 */
#ifndef BOLT_B200_H
#define BOLT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes — the reference's BoltResult / BoltError taxonomy           */
/* (src/error.rs:21-100) plus the executor's Option "decline"               */
/* (src/exec/groupby_shmem_exec.rs:53, src/exec/groupby_tier2_exec.rs:30).  */
/* ------------------------------------------------------------------------ */
typedef enum {
    BOLT_OK = 0,
    BOLT_DECLINE = 1,        /* shape not handled: caller takes its next path (== None)  */
    BOLT_ERR_SPILL = 2,      /* soft miss (== "partition_reduce spill:" prefix)           */
    BOLT_ERR_OVERFLOW = 3,   /* SUM(integer) / SUM(Decimal128) overflow (== BoltError::Type) */
    BOLT_ERR_CAPACITY = 4,   /* output / scratch too small (== BoltError::GpuCapacity)    */
    BOLT_ERR_TIMEOUT = 5,    /* a bounded device wait gave up                              */
    BOLT_ERR_CUDA = 6,       /* CUDA runtime error (== BoltError::Cuda / CudaWithCode)     */
    BOLT_ERR_INVALID = 7     /* bad argument (== BoltError::Plan / Other)                  */
} bolt_status;

typedef enum {
    BOLT_I32 = 0,
    BOLT_I64 = 1,
    BOLT_F32 = 2,
    BOLT_F64 = 3,
    BOLT_DEC128 = 4,         /* 16-byte little-endian two's-complement unscaled value */
    BOLT_U32 = 5             /* row indices / permutations                            */
} bolt_dtype;

/* Read-only column borrow (== GpuView<'a, T>, smart_ptrs.rs:268). */
typedef struct {
    const void* data;
    const uint8_t* validity;   /* Arrow LSB bitmap or NULL */
    uint64_t len;
    int32_t dtype;             /* bolt_dtype */
    int32_t scale;             /* Decimal128 scale, else 0 */
} bolt_col_view;

/* Exclusive output column borrow (== GpuViewMut<'a, T>, smart_ptrs.rs:367). */
typedef struct {
    void* data;
    uint8_t* validity;         /* written when the column can hold NULLs; may be NULL */
    uint64_t cap;              /* capacity in rows */
    int32_t dtype;
    int32_t scale;
} bolt_col_mut;

typedef void* bolt_stream;     /* cudaStream_t */
typedef struct bolt_ctx bolt_ctx;

/* Call flags. */
#define BOLT_FLAG_ASYNC        0x1u  /* do not synchronise; counts land in device memory */
#define BOLT_FLAG_PROFILE      0x2u  /* record device time of the call (bolt_ctx_last_device_ms) */
#define BOLT_FLAG_FORCE_GLOBAL 0x4u  /* GROUP BY: skip the shared-memory tier (testing) */
#define BOLT_FLAG_FORCE_SHMEM  0x8u  /* GROUP BY: shared-memory tier only; spill -> BOLT_ERR_SPILL */
#define BOLT_FLAG_NO_TUNE      0x10u /* GROUP BY: ignore the context's autotuned choices */
#define BOLT_FLAG_KERNEL_REGS  0x20u /* GROUP BY: aggregate with the register-tile kernel; compaction: per-element
                                       copies instead of bulk-staged tiles (testing) */
#define BOLT_FLAG_KERNEL_STAGED 0x40u /* GROUP BY: aggregate with the generic staged kernel where it applies, not
                                        the streaming kernel compiled for the query's layout (testing) */
#define BOLT_FLAG_NO_PART      0x80u /* GROUP BY: never use the hash-partitioned tier (global hash table instead) */
#define BOLT_FLAG_FORCE_PART   0x100u /* GROUP BY: use the hash-partitioned tier wherever it applies, whatever the
                                        groups hint (testing) */
#define BOLT_FLAG_KERNEL_TIMES 0x200u /* record only the dominant kernel's device time (bolt_ctx_kernel_times), not
                                        the whole call's: two events per call instead of four */

/* ------------------------------------------------------------------------ */
/* Context: device, scratch arena, tuning cache, status word, last error.   */
/* Replaces the reference's per-Engine device pool + stream pool            */
/* (src/cuda/mem_pool.rs:1144, src/exec/launch.rs:84).                       */
/* ------------------------------------------------------------------------ */
/* scratch_bytes = 0 picks 1/4 of the device's free memory. */
bolt_status bolt_ctx_create(int device, uint64_t scratch_bytes, bolt_ctx** out);
void        bolt_ctx_destroy(bolt_ctx* ctx);
/* Human-readable message of the last failing call on this context
 * (the Display text of the matching BoltError). */
const char* bolt_ctx_last_error(const bolt_ctx* ctx);
const char* bolt_status_str(bolt_status s);
/* Device milliseconds of the last call made with BOLT_FLAG_PROFILE. */
double      bolt_ctx_last_device_ms(const bolt_ctx* ctx);
/* Number of kernels the last call launched (all are this library's). */
uint32_t    bolt_ctx_last_launches(const bolt_ctx* ctx);
/* Which GROUP BY tier served the last bolt_groupby on this context: 1 = the
 * shared-memory tier over a global hash table, 2 = the hash-partitioned tier
 * (the reference's Tier-1 / Tier-2 executors), 3 = the sort-based wide-key
 * path (groupby_wide.rs); 0 before any GROUP BY. */
int32_t     bolt_ctx_last_groupby_tier(const bolt_ctx* ctx);
/* Device milliseconds of the dominant kernel of every call made with
 * BOLT_FLAG_PROFILE or BOLT_FLAG_KERNEL_TIMES since the previous read (up to 256 calls, oldest first).
 * Waits for those kernels; returns how many times were written to `ms`. */
uint32_t    bolt_ctx_kernel_times(bolt_ctx* ctx, double* ms, uint32_t max);
/* Waits for the stream and returns the device-recorded status of every
 * BOLT_FLAG_ASYNC call issued since the previous check. */
bolt_status bolt_ctx_sync_status(bolt_ctx* ctx, bolt_stream stream);
/* Bytes of scratch arena the context owns. */
uint64_t    bolt_ctx_scratch_bytes(const bolt_ctx* ctx);
/* Library build identification ("bolt-b200 <version> sm_100a"). */
const char* bolt_version(void);

/* ------------------------------------------------------------------------ */
/* GROUP BY                                                                  */
/* Replaces groupby::execute_groupby (src/exec/groupby.rs:295-833), the      */
/* Tier-1 shared-memory executors (groupby_shmem_exec.rs:53), the Tier-2     */
/* hash-partitioned executors (groupby_tier2_exec.rs:30,                     */
/* groupby_tier2_orchestrator.rs:214) and the WHERE + GROUP BY executor      */
/* (groupby_with_pre.rs:222).                                                 */
/*                                                                            */
/* Semantics follow the reference:                                           */
/*   keys: 1 column (I32/I64/F32/F64) or 2 columns of 32-bit types, packed   */
/*         exactly as pack_keys (groupby_common.rs:352): I32 sign-extended,  */
/*         (I32,I32) -> (a << 32) | (u32)b, floats by bit pattern after      */
/*         -0.0 -> +0.0 and NaN -> one canonical NaN;                         */
/*   wide keys: 2 integer columns with at least one I64 (no 64-bit packing)  */
/*         follow the reference's host wide reduction (groupby_wide.rs:85):  */
/*         synchronous calls without WHERE only; rows with a NULL in either  */
/*         key are dropped; groups sorted by (key0, key1) as signed integers; */
/*         each aggregate is a row-order fold (integer SUM wraps in i64, SUM/ */
/*         AVG over F64 add in order, MIN/MAX keep the first valid value and */
/*         replace it on < / >, so a NaN replaces nothing); SUM/AVG over     */
/*         I32/I64/F64 and MIN/MAX over I32/I64/F32/F64, else BOLT_DECLINE;  */
/*   output rows sorted by the packed key as a signed 64-bit integer,        */
/*         ascending (groupby.rs:789-800); rows with a NULL key (single-key   */
/*         only) form one group emitted last with a NULL key;                 */
/*   SUM(I32) -> I64, SUM(I64) -> I64 with overflow -> BOLT_ERR_OVERFLOW,     */
/*   SUM(F64) -> F64, SUM(DEC128(p,s)) -> DEC128(38,s),                       */
/*   COUNT(*) / COUNT(col) -> I64, MIN/MAX keep the input type (float NaN is */
/*   the largest value), AVG -> F64 = SUM / COUNT(col). SUM/MIN/MAX/AVG of a  */
/*   group whose inputs are all NULL are NULL.                                */
/* ------------------------------------------------------------------------ */
typedef enum {
    BOLT_AGG_SUM = 0,
    BOLT_AGG_COUNT_STAR = 1,
    BOLT_AGG_COUNT = 2,
    BOLT_AGG_MIN = 3,
    BOLT_AGG_MAX = 4,
    BOLT_AGG_AVG = 5
} bolt_agg_op;

typedef struct {
    int32_t op;                /* bolt_agg_op */
    int32_t input_col;         /* index into the table columns; -1 for COUNT(*) */
} bolt_agg_spec;

typedef enum {
    BOLT_CMP_LT = 0, BOLT_CMP_LE = 1, BOLT_CMP_GT = 2,
    BOLT_CMP_GE = 3, BOLT_CMP_EQ = 4, BOLT_CMP_NE = 5
} bolt_cmp;

/* One conjunct of a fused WHERE: cols[col] <cmp> literal. A NULL input
 * makes the conjunct false (SQL three-valued WHERE). Integer columns use
 * lit_i, float columns lit_f. Replaces the `pre` predicate kernel
 * (src/jit/scan_kernel.rs:265) for this path. */
typedef struct {
    int32_t col;
    int32_t cmp;               /* bolt_cmp */
    int64_t lit_i;
    double  lit_f;
} bolt_pred;

typedef struct {
    const bolt_col_view* cols; /* the table's columns */
    int32_t n_cols;
    const int32_t* key_cols;   /* 1 or 2 indices into cols */
    int32_t n_keys;
    const bolt_pred* preds;    /* conjunction; may be NULL */
    int32_t n_preds;
    const bolt_agg_spec* aggs;
    int32_t n_aggs;
    uint64_t groups_hint;      /* expected distinct groups; 0 = unknown */
} bolt_groupby_desc;

typedef struct {
    bolt_col_mut* keys;        /* n_keys columns (input key dtypes); validity marks the NULL group */
    bolt_col_mut* aggs;        /* n_aggs columns of the output dtypes above */
    uint64_t n_groups;         /* set on return (host) */
    uint64_t* n_groups_dev;    /* with BOLT_FLAG_ASYNC: device word that receives the count */
} bolt_groupby_out;

bolt_status bolt_groupby(bolt_ctx* ctx, const bolt_groupby_desc* desc,
                         bolt_groupby_out* out, uint32_t flags, bolt_stream stream);

/* GROUP BY over HOST-resident columns: every data / validity pointer of
 * desc->cols is host memory (pinned memory lets the copies overlap); the
 * outputs are device columns, exactly as for bolt_groupby. Replaces the
 * reference's host RecordBatch path, which uploads each column before its
 * kernels (src/exec/groupby.rs:295-833; the uploads are ~78 % of the h2o q1
 * time, groupby.rs:270-272). Here the rows stream to the device in chunks on
 * a second stream while the aggregation folds the chunks already there, so
 * transfer and aggregation overlap and no column is resident in full.
 * Always synchronises (BOLT_FLAG_ASYNC -> BOLT_ERR_INVALID). A query whose
 * SUM(Int64) needs the row-order overflow check returns BOLT_DECLINE: run it
 * on device columns through bolt_groupby. Keys wider than 64 bits (the wide
 * form above) sort every row at once: their columns are uploaded whole, not
 * streamed. */
bolt_status bolt_groupby_host(bolt_ctx* ctx, const bolt_groupby_desc* desc,
                              bolt_groupby_out* out, uint32_t flags, bolt_stream stream);

/* GROUP BY that allocates no device memory. No counterpart in the
 * reference. For callers that may not call cudaMalloc / cudaFree at all (an
 * engine whose own pool owns all of HBM, or a latency-critical loop where an
 * allocation would synchronise the device) and so cannot hold a bolt_ctx.
 * Same semantics and outputs as bolt_groupby (device columns in, device
 * columns out), for at most 6144 groups: the table starts at the size the
 * groups hint asks for and grows, up to 8192 slots, when the groups outnumber
 * the hint. Its scratch is one fixed 2 MiB device array inside this library,
 * held by every GPU that loads it until the process exits. The first call on
 * each device (with that device current) resolves the array's address with
 * cudaGetSymbolAddress: make that first call before any stream capture
 * begins. Calls share the array and clear it on entry, so calls that overlap
 * on the GPU race: serialise them. Every call waits for its own work on
 * `stream` before it returns (it reads the group count and status back).
 * Returns: more than 6144 groups, or out_cap below the group count ->
 * BOLT_ERR_CAPACITY; a SUM(Int64) whose inputs are large enough to need the
 * row-order overflow check (bolt_groupby runs it with scratch it allocates)
 * -> BOLT_DECLINE. `err` (nullable, err_cap bytes) receives the message of a
 * failure. */
bolt_status bolt_groupby_noalloc(const bolt_groupby_desc* desc, bolt_groupby_out* out,
                                 bolt_stream stream, char* err, int32_t err_cap);

/* Autotuner (replaces the reference's fixed dispatch thresholds,
 * groupby_shmem_dispatch.rs:126-131, groupby_tier2_dispatch.rs:171-225):
 * times the GROUP BY of `desc` on the device under candidate launch choices
 * (thread-block size, shared-memory table size, warp pre-aggregation,
 * hash-table load factor) and keeps the fastest for this query shape in the
 * context; later calls of the same shape use it. `out` receives a valid
 * result; best_ms (nullable) the winner's device time. */
bolt_status bolt_groupby_autotune(bolt_ctx* ctx, const bolt_groupby_desc* desc,
                                  bolt_groupby_out* out, bolt_stream stream, double* best_ms);
/* Saves / loads the context's tuning cache (text, one shape per line). */
bolt_status bolt_ctx_tuning_save(const bolt_ctx* ctx, const char* path);
bolt_status bolt_ctx_tuning_load(bolt_ctx* ctx, const char* path);

/* ------------------------------------------------------------------------ */
/* Hash join (INNER, single equi-key, I32/I64 keys, unique build keys).      */
/* Replaces gpu_join::hash_join_indices_on_gpu{,_aos}                        */
/* (src/exec/gpu_join.rs:1295,1403) behind join::try_gpu_inner_join          */
/* (src/exec/join.rs:1336). NULL keys never match. The table lives in the    */
/* context's scratch arena until bolt_hash_join_release or the next build.   */
/* ------------------------------------------------------------------------ */
typedef struct bolt_join_table bolt_join_table;

/* Build. Duplicate build keys (the reference's collision-list path,
 * src/jit/hash_join_kernel.rs:1183,1368) make a multi-match table: the
 * probe then pairs each probe row with every build row of its key, in
 * ascending build-row order (the reference's host join, src/exec/join.rs:
 * 407-425, 843-855). With BOLT_FLAG_ASYNC the duplicate is only reported
 * (BOLT_DECLINE at the status check) instead of rebuilt. `payload`
 * (nullable) is an I32 build column carried in the table for
 * bolt_join_groupby, which declines on a multi-match table. */
bolt_status bolt_hash_join_build(bolt_ctx* ctx, const bolt_col_view* build_key,
                                 const bolt_col_view* payload, uint32_t flags,
                                 bolt_stream stream, bolt_join_table** table_out);

/* Probe: emits (probe_row, build_row) u32 pairs ordered by probe row.
 * n_out receives the pair count; pairs beyond the capacity of the two
 * output columns give BOLT_ERR_CAPACITY (n_out still reports the count). */
bolt_status bolt_hash_join_probe(bolt_ctx* ctx, const bolt_join_table* table,
                                 const bolt_col_view* probe_key,
                                 bolt_col_mut* probe_idx, bolt_col_mut* build_idx,
                                 uint64_t* n_out, uint32_t flags, bolt_stream stream);

void bolt_hash_join_release(bolt_ctx* ctx, bolt_join_table* table);

/* Fused probe -> GROUP BY <build payload>: for
 *   SELECT b.g, SUM(p.amount), COUNT(*) FROM p JOIN b ON p.fk = b.k GROUP BY b.g
 * The joined rows are never materialised (the reference composes JOIN ->
 * arrow take -> GROUP BY, src/exec/join.rs:843-858 + groupby.rs:1168).
 * `value` is I32/I64/DEC128; SUM(DEC128(p,s)) -> DEC128(38,s) with
 * overflow -> BOLT_ERR_OVERFLOW. Output sorted by g ascending. */
bolt_status bolt_join_groupby(bolt_ctx* ctx, const bolt_join_table* table,
                              const bolt_col_view* probe_key, const bolt_col_view* value,
                              bolt_col_mut* out_group, bolt_col_mut* out_sum,
                              bolt_col_mut* out_count, uint64_t* n_groups,
                              uint32_t flags, bolt_stream stream);

/* ------------------------------------------------------------------------ */
/* ORDER BY: stable LSD radix sort -> u32 row permutation.                   */
/* Replaces gpu_sort::sort_indices_on_gpu_radix_multi                         */
/* (src/exec/gpu_sort.rs:995-1058) and the host lexsort_to_indices default    */
/* (src/exec/sort.rs:191-229). Key transforms follow gpu_sort.rs:1089-1163:   */
/* integers flip the sign bit, floats canonicalise NaN (sorted last for ASC)  */
/* and -0.0 == +0.0; DESC is the bitwise NOT of the ASC key. NULL rows go     */
/* last (nulls_first = 0) or first, in input order.                           */
/* ------------------------------------------------------------------------ */
bolt_status bolt_radix_sort_perm(bolt_ctx* ctx, const bolt_col_view* key,
                                 int32_t descending, int32_t nulls_first,
                                 bolt_col_mut* perm, uint32_t flags, bolt_stream stream);

/* Multi-key ORDER BY: LSD over the keys from last to first
 * (gpu_sort.rs:995-1058). desc / nulls_first have n_keys entries. */
bolt_status bolt_radix_sort_perm_multi(bolt_ctx* ctx, const bolt_col_view* keys,
                                       int32_t n_keys, const int32_t* descending,
                                       const int32_t* nulls_first, bolt_col_mut* perm,
                                       uint32_t flags, bolt_stream stream);

/* ------------------------------------------------------------------------ */
/* Filter compaction: out[rank(i)] = col[i] for rows passing the WHERE       */
/* conjunction, input order preserved.                                        */
/* Replaces gpu_compact::compact_columns_on_gpu (src/exec/gpu_compact.rs:1005)*/
/* with prefix_scan_mask (gpu_compact.rs:415) and the predicate kernel        */
/* (scan_kernel.rs:265) fused: one decoupled look-back pass, or for inputs of */
/* 4M rows and more a count pass over the WHERE columns, a scan of the tile  */
/* counts and a scatter pass that stages whole tiles with bulk copies.        */
/* `out[c]` receives column c (validity carried); `row_ids` (nullable, U32)   */
/* receives the selected row indices.                                          */
/* ------------------------------------------------------------------------ */
bolt_status bolt_compact(bolt_ctx* ctx, const bolt_col_view* cols, int32_t n_cols,
                         const bolt_pred* preds, int32_t n_preds,
                         bolt_col_mut* out, bolt_col_mut* row_ids, uint64_t* n_out,
                         uint32_t flags, bolt_stream stream);

/* Mask-driven variant: keep rows whose byte mask[i] != 0
 * (the reference's u8 mask contract, gpu_compact.rs:415). */
bolt_status bolt_compact_mask(bolt_ctx* ctx, const bolt_col_view* cols, int32_t n_cols,
                              const uint8_t* mask, bolt_col_mut* out, bolt_col_mut* row_ids,
                              uint64_t* n_out, uint32_t flags, bolt_stream stream);

/* ------------------------------------------------------------------------ */
/* Batched filter + GROUP BY: many queries in one persistent launch.         */
/* No counterpart in the reference (one query at a time per Engine,          */
/* launch.rs:308-368); each query's result equals bolt_groupby's.             */
/* ------------------------------------------------------------------------ */
typedef struct {
    bolt_groupby_desc desc;
    bolt_groupby_out out;
    uint64_t row_begin;        /* the query reads rows [row_begin, row_end) of its columns */
    uint64_t row_end;
    bolt_status status;        /* per-query result */
} bolt_query;

bolt_status bolt_batch_groupby(bolt_ctx* ctx, bolt_query* queries, int32_t n_queries,
                               uint32_t flags, bolt_stream stream);

/* Scratch bytes bolt_groupby would use for a query (the serving admission
 * footprint). */
uint64_t bolt_groupby_footprint(const bolt_groupby_desc* desc, uint64_t n_rows);

/* A batch of queries captured once as a CUDA graph and replayed: the graph
 * owns a private scratch arena and descriptor copies, so replays are
 * independent of other calls. Every replay re-reads the queries' columns
 * (so they may be updated in place between replays) and rewrites their
 * outputs. Tables must be large enough for the data (no growth retries
 * inside a graph): a query that would need one reports BOLT_ERR_SPILL in
 * bolt_graph_sync_status. */
typedef struct bolt_graph bolt_graph;
bolt_status bolt_batch_graph_create(int device, bolt_query* queries, int32_t n_queries, bolt_graph** out);
bolt_status bolt_graph_launch(bolt_graph* g, bolt_stream stream);
/* Waits for the stream; fills per-query statuses and group counts (each
 * array nullable, n_queries entries). Returns the first failing status. */
bolt_status bolt_graph_sync_status(bolt_graph* g, bolt_stream stream, int32_t* statuses, uint64_t* n_groups);
void        bolt_graph_destroy(bolt_graph* g);

/* ------------------------------------------------------------------------ */
/* Serving: a request loop that keeps columns resident, admits queries by    */
/* their HBM footprint and runs them in continuously formed batches on       */
/* overlapping streams. No counterpart in the reference.                      */
/* ------------------------------------------------------------------------ */
typedef struct bolt_server bolt_server;

typedef struct {
    int32_t device;
    uint64_t scratch_bytes;    /* HBM budget for in-flight queries */
    int32_t max_batch;         /* queries per batch launch */
    int32_t n_lanes;           /* concurrent batches (streams) */
} bolt_server_config;

bolt_status bolt_server_create(const bolt_server_config* cfg, bolt_server** out);
/* Submits a query; `q` and every buffer it names must stay alive until
 * bolt_server_wait returns for the ticket. */
bolt_status bolt_server_submit(bolt_server* srv, bolt_query* q, uint64_t* ticket);
/* Submits n queries at once (no counterpart in the reference, which runs one
 * query at a time): tickets[i] receives query i's ticket. The burst is
 * enqueued under one lock and announced once, so the lanes form full batches
 * from it. All or none: BOLT_ERR_CAPACITY when any query's footprint exceeds
 * a lane's share of HBM. Same lifetime rule as bolt_server_submit. */
bolt_status bolt_server_submit_batch(bolt_server* srv, bolt_query* qs, int32_t n, uint64_t* tickets);
/* Blocks until the ticket completes; latency_us receives submit -> done. */
bolt_status bolt_server_wait(bolt_server* srv, uint64_t ticket, double* latency_us);
void        bolt_server_destroy(bolt_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* BOLT_B200_H */
