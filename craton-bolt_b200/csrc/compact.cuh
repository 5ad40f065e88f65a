// compact.cuh — order-preserving stream compaction (decoupled look-back).
#pragma once

#include "ctx.cuh"

namespace bolt {

struct CompactCol {
    const void* in;
    const uint8_t* in_valid;
    void* out;
    uint8_t* out_valid;
    int32_t width;  // bytes per row: 4, 8 or 16
};

constexpr int CP_MAX_COLS = 8;
constexpr int CP_MAX_PREDS = 4;

struct CompactPred {
    const void* col;
    const uint8_t* valid;
    int32_t dtype;
    int32_t cmp;
    ll lit_i;
    double lit_f;
    int32_t col_idx;  // index of the conjunct's column among the output columns
};

struct CompactSpec {
    uint64_t n = 0;
    CompactPred pred[CP_MAX_PREDS];
    int32_t n_pred = 0;
    const uint8_t* mask = nullptr;          // byte mask (keep when != 0)
    const uint8_t* keep_valid_of = nullptr; // keep rows whose bit is set (or clear, see invert)
    const uint32_t* ids_in = nullptr;       // element e stands for row ids_in[e] (validity test, row ids)
    int32_t invert = 0;                     // keep the complement of the selection
    CompactCol col[CP_MAX_COLS];
    int32_t n_cols = 0;
    uint32_t* row_ids = nullptr;            // selected row indices (+ row_id_base)
    uint32_t row_id_base = 0;
    uint64_t out_cap = UINT64_MAX;
    ull* n_out_dev = nullptr;               // device word receiving the count
};

// Enqueues one fused predicate-evaluation + scan + scatter pass.
// flags: BOLT_FLAG_PROFILE records the kernel's device time.
bolt_status compact_enqueue(bolt_ctx* ctx, cudaStream_t s, const CompactSpec& spec, uint32_t flags = 0);

}  // namespace bolt
