// groupby_part.cuh — the hash-partitioned tier of GROUP BY (groupby_part.cu).
#pragma once

#include "groupby.cuh"

namespace bolt {

// Compiled key layouts of the partitioned tier's streaming kernel.
constexpr int GB_KP_I32X2 = 0;  // two Int32 key columns, packed (a << 32) | b
constexpr int GB_KP_I32 = 1;    // one Int32 key column (sign-extended)
constexpr int GB_KP_I64 = 2;    // one Int64 key column

constexpr int GB_PART_MAX_FIELDS = 3;                // distinct value columns a spilled row carries
constexpr uint64_t GB_PART_MIN_GROUPS = 1ull << 15;  // expected groups from which the tier is used
constexpr uint64_t GB_LEAN_MIN_ROWS = 1ull << 18;    // rows from which the streaming kernel serves a query
constexpr uint64_t GB_STAGED_MIN_ROWS = 1ull << 22;  // rows from which the generic staged kernel is used untuned
constexpr uint64_t GB_PART_RED_GROUPS = 512;         // expected groups per partition
constexpr int GB_PART_MAX_PBITS = 13;                // at most 8192 partitions

// Device-side description of one partitioned run (all pointers device).
struct alignas(16) GbPart {
    int32_t pbits;        // partitions = 1 << pbits (multiplicative hash of the stored key)
    int32_t n_fields;     // value words per spilled row
    int8_t field_of_state[GB_MAX_STATES];    // field feeding each state (-1: COUNT(*))
    int8_t field_sc[GB_PART_MAX_FIELDS];     // staged column of each field
    int8_t field_w[GB_PART_MAX_FIELDS];      // its width in bytes (4 or 8)
    int8_t field_float[GB_PART_MAX_FIELDS];  // 1 for float32 / float64
    int8_t state_float[GB_MAX_STATES];       // MIN / MAX over a float column
    int8_t pad0[7];
    // The WHERE conjunct on an Int32 column as a range test: a row passes when
    // (pred_lo <= v && v <= pred_hi) != pred_neg. has_pred = 0: every row.
    int32_t has_pred;
    int32_t pred_lo, pred_hi, pred_neg;
    int32_t grid_a;       // pass-A CTAs = spill segments
    int32_t hot_cap;      // slots of a pass-A shared table = partial records per segment
    int32_t red_log2;     // slots of a pass-C table (log2)
    uint32_t red_fill;    // keys a pass-C table admits before the partition spills
    uint64_t seg_stride;  // rows one spill segment holds
    ull* skey;            // [grid_a * seg_stride] spilled rows: complemented packed key
    ull* sfield[GB_PART_MAX_FIELDS];  // ... and the raw 64-bit value images
    uint32_t* n_spill;    // [grid_a] rows in each segment
    ull* ppart;           // [grid_a * hot_cap] partial records (shared-table slot layout)
    uint32_t* n_part;     // [grid_a] partial records of each segment
    uint32_t* cnt_raw;    // [grid_a][P] rows per (segment, partition)
    uint32_t* cnt_par;    // [grid_a][P] partial records per (segment, partition)
    uint32_t* rel_raw;    // [grid_a][P] exclusive prefix over segments
    uint32_t* rel_par;
    uint32_t* base_raw;   // [P + 1] first row of each partition
    uint32_t* base_par;   // [P + 1]
    uint32_t* done;       // CTAs of the scan that finished
    ull* drec;            // spilled rows in partition order: 32-byte records {key, field 0, 1, 2}
    ull* dpar;            // partial records in partition order
};

// Whether the streaming kernel (compiled key / predicate / state layouts over
// dense, 16-byte aligned columns of 4M+ rows) serves this planned query.
bool gb_lean_applies(const GbPlan& pl, uint32_t flags);

// Whether the partitioned tier serves this planned query.
bool gb_part_applies(const bolt_ctx* ctx, const GbPlan& pl, uint32_t flags);

// The global-table tier's aggregation through the streaming kernel (misses
// go to the global hash table, set up in prm). Returns false when the
// streaming kernel does not serve the query (the caller launches the staged
// or register kernel); otherwise *st is the launch status.
bool gb_lean_global(bolt_ctx* ctx, GbPlan* pl, cudaStream_t s, uint32_t flags, bolt_status* st);

// Enqueues passes A, B1, S, B2 and C of one query whose compact group array
// (prm.gtab, cap + 2 slots with the two special slots zeroed), words and
// finalize buffers (fin.order_keys, fin.slots, fin.n_nonnull) are set up.
// pbits_override > 0 fixes the partition count (after a spill).
bolt_status gb_part_launch(bolt_ctx* ctx, GbPlan* pl, cudaStream_t s, uint32_t flags, int pbits_override);

}  // namespace bolt
