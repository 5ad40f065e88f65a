// groupby.cuh — hash GROUP BY plan, kernels and host entry shared with the
// batched / served forms.
#pragma once

#include "ctx.cuh"

namespace bolt {

// Per-group state kinds (8-byte words inside a hash slot). Every state's
// identity is all-zero words, so a table is initialised with one memset.
enum StKind : int32_t {
    K_COUNT = 0,      // 1 word: count of valid inputs (or rows)
    K_SUM_I32 = 1,    // 1 word: i64 sum of i32 inputs
    K_SUM_I64 = 2,    // 2 words: sum of low 32 bits (u64), sum of high 32 bits (i64)
    K_SUM_FX = 3,     // i128 fixed-point sum. Global table, 3 words updated without returning
                      // adds: sums of bits 0-31, of bits 32-63 and of the signed high word
                      // of the contributions. Shared table, 2 words: lo with carry, hi.
    K_SUM_FATOM = 4,  // 1 word: f64 atomicAdd (fallback for non-finite / huge values)
    K_MAX_ORD = 5,    // 1 word: max of an order-preserving u64 image
    K_MIN_ORD = 6,    // 1 word: max of the bitwise NOT of that image
    K_SUM_D64 = 7,    // 2 words: like K_SUM_I64 over Decimal128 values that fit in i64
    K_SUM_D128 = 8,   // 3 words: low word with carry, low half of the high words + carries,
                      // signed high half of the high words (exact 192-bit sum)
};

constexpr int GB_MAX_STATES = 8;
constexpr int GB_MAX_PREDS = 4;
constexpr int GB_MAX_AGGS = 16;
constexpr int GB_MAX_SC = 2 + GB_MAX_PREDS + GB_MAX_STATES;  // staged columns

struct StateDesc {
    const void* col;
    const uint8_t* valid;
    int32_t kind;
    int32_t dtype;
    int32_t word;    // offset of the state's first word inside a global-table slot (key is word 0)
    int32_t nwords;
    int32_t sword;   // the same inside a shared-table slot (K_SUM_FX is one word shorter there)
    int32_t pad;
};

struct PredDesc {
    const void* col;
    const uint8_t* valid;
    int32_t dtype;
    int32_t cmp;
    ll lit_i;
    double lit_f;
};

struct AggOut {
    int32_t op;
    int32_t in_dtype;
    int32_t out_dtype;
    int32_t sum_state;   // index into states or -1
    int32_t cnt_state;   // state deciding NULL-ness / COUNT value, or -1
    int32_t mm_state;    // MIN/MAX state or -1
    int32_t nullable;    // output can be NULL (input column has validity)
    int32_t pad;
    void* out;
    uint8_t* out_valid;
};

// Both descriptors are copied into shared memory as 16-byte words, so their
// sizes are multiples of 16 (alignas).
struct alignas(16) GbParams {
    const void* kcol[2];
    const uint8_t* kvalid[2];
    int32_t kdtype[2];
    int32_t n_keys;
    int32_t n_pred;
    PredDesc pred[GB_MAX_PREDS];
    StateDesc st[GB_MAX_STATES];
    int32_t n_st;
    int32_t slot_words;  // words per global-table slot
    int32_t sslot_words; // words per shared-table slot
    int32_t pad_s;
    uint64_t row_begin;
    uint64_t n_rows;
    ull* gtab;           // (cap + 2) * slot_words words; slot cap = key -1, cap + 1 = NULL key
    int32_t log2cap;
    uint32_t max_probe;
    int32_t smem_log2;   // 0 disables the shared-memory tier
    int32_t fx_e;
    int32_t warp_agg;
    uint32_t smem_fill;  // keys the shared tier admits before it only serves lookups
    int32_t spec;        // compiled row-loop layout (gb_spec_of), 0 = generic
    int32_t cnt32;       // COUNT fits 32 bits per shared table (see merge_words_smem)
    int32_t pad1;
    uint32_t* status;
    ull* occupancy;
    ull grow_limit;
    // Largest bit length of |v| over int64 SUM inputs (nullptr when the
    // query has no int64 SUM).
    uint32_t* i64_bits;
    // Join source: when jslots is set the group key of a row is the payload
    // of the build slot its probe key matches (rows without a match are
    // skipped) instead of its packed key columns.
    const ull* jslots;
    int32_t jlog2cap;
    int32_t jkdt;
    const void* jkey;
    const uint8_t* jkvalid;
    // Staged kernel: the distinct input columns (element width, byte offset
    // inside one stage) and the staged column each key / predicate / state
    // reads (-1: none).
    int32_t n_sc;
    uint32_t stage_bytes;   // one stage: tile_rows x the staged row width
    uint32_t tile_rows;
    int32_t n_stages;
    int32_t chunks;         // 32-row chunks per consumer warp per tile
    int32_t pad2;
    const void* sc_col[GB_MAX_SC];
    int32_t sc_w[GB_MAX_SC];
    uint32_t sc_off[GB_MAX_SC];
    int8_t k_sc[2];
    int8_t pr_sc[GB_MAX_PREDS];
    int8_t st_sc[GB_MAX_STATES];
};

struct alignas(16) GbFinal {
    ull* gtab;
    int32_t slot_words;
    int32_t log2cap;
    int32_t n_keys;
    int32_t kdtype[2];
    int32_t n_aggs;
    int32_t fx_e;
    StateDesc st[GB_MAX_STATES];
    AggOut agg[GB_MAX_AGGS];
    void* out_key[2];
    uint8_t* out_key_valid[2];
    uint64_t out_cap;
    ull* order_keys;     // compacted order keys (large path)
    uint32_t* slots;     // compacted slots
    uint32_t* sorted;    // sorted slots
    ull* n_nonnull;      // device: groups excluding the NULL group
    ull* n_groups;       // device: groups written (incl. NULL group)
    ull* n_groups_user;  // optional user device word
    uint32_t* status;
    // Most sort entries (order_keys / slots) the aggregation can have
    // written: cap + 1 for the global table, cap for the partitioned tier's
    // compact array (its group counter may run past it when the array must
    // grow; entries beyond were never written).
    ull n_max;
};

// A fully planned GROUP BY (one query).
struct GbPlan {
    GbParams prm;
    GbFinal fin;
    uint64_t cap = 0;
    int32_t smem_entries = 0;
    int32_t block = 512;
    int32_t grid = 0;
    int32_t u = 4;
    int32_t n_aggs = 0;
    bool small_final = false;
    int32_t mode = 0;
    uint32_t flags = 0;
    ull* words = nullptr;  // device: [0] occupancy, [1] non-NULL groups, [2] groups, [3] status
    uint64_t shape = 0;    // autotuning key of the query shape
    bolt_ctx::GbTune tune{512, 1, 0, 1, 4, 0, 0.0};
    uint64_t groups_hint = 0;  // expected groups (the caller's hint, at most the rows)
    // Hash-partitioned tier (groupby_part.cu): shared-table size of its
    // streaming kernel (log2; 0 = default), 32-row chunks per consumer warp
    // per tile, the partition count used (log2), and whether the finalize
    // finds the groups already compacted with their sort keys.
    int32_t part_hot_log2 = 0;
    int32_t part_chunks = 2;
    int32_t part_pbits = 0;
    bool precompacted = false;
};

// Key of a query shape for the autotuning cache: key / predicate / state
// layout plus the row and group counts rounded to powers of two.
uint64_t gb_shape_key(const GbParams& p, uint64_t n_rows, uint64_t groups_hint);
// Compiled row-loop layout serving these canonically ordered states (0 = generic).
int gb_spec_of(const StateDesc* st, int n);

// Plan modes selected after a flagged first attempt.
constexpr int GB_MODE_F64_ATOMIC = 1;  // f64 SUM with plain atomics (non-finite / huge inputs)
constexpr int GB_MODE_WIDE_DEC = 2;    // Decimal128 SUM with the exact 192-bit state

// Builds the plan for `desc` over rows [row_begin, row_end) (no device work).
// `force_tune` (nullable) overrides the context's tuning cache.
bolt_status gb_plan(bolt_ctx* ctx, const bolt_groupby_desc* desc, const bolt_groupby_out* out,
                    uint64_t row_begin, uint64_t row_end, uint32_t flags, int mode,
                    uint64_t cap_override, GbPlan* plan, const bolt_ctx::GbTune* force_tune = nullptr);

// Bytes of scratch the plan needs (table + finalize buffers).
uint64_t gb_plan_scratch(const GbPlan& plan);

// Launch shape of the staged aggregation kernel for one plan.
struct GbStagedLaunch {
    int block;
    uint32_t tile_rows;
    int n_stages;
    uint32_t stage_bytes;
    int smem_log2;
    size_t smem;
};
// GROUP BY over two integer key columns at least one of which is Int64 (keys
// that do not pack into 64 bits), without WHERE: sort-based, synchronous.
bool gb_wide_applies(const bolt_groupby_desc* d);
bolt_status gb_wide(bolt_ctx* ctx, const bolt_groupby_desc* d, bolt_groupby_out* out, uint32_t flags,
                    cudaStream_t s);

bool gb_staged_layout(const bolt_ctx* ctx, const GbPlan& plan, GbStagedLaunch* out);

// Allocates scratch and enqueues table init, aggregation and finalize of
// `nq` planned queries (one persistent aggregation launch when nq > 1).
// query_status: every query reports through its own status word (batches),
// even when nq == 1; otherwise a single query reports through the context's.
bolt_status gb_run(bolt_ctx* ctx, GbPlan** plans, int nq, cudaStream_t s, uint32_t flags, bool query_status = false);

}  // namespace bolt
