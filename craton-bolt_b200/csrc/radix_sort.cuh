// radix_sort.cuh — onesweep LSD radix sort (8-bit digits, decoupled look-back).
#pragma once

#include "ctx.cuh"

namespace bolt {

// Where the sort keys come from.
enum SortSrc : int32_t {
    SRC_U64_KEYS = 0,  // already order-transformed u64 keys (no transform)
    SRC_I32 = 1,
    SRC_I64 = 2,
    SRC_F32 = 3,
    SRC_F64 = 4,
    SRC_U32 = 5,
};

struct SortSpec {
    int32_t src = SRC_U64_KEYS;
    const void* keys = nullptr;         // raw column or u64 keys
    int32_t descending = 0;
    // Payload input: nullptr = row index (iota). When `indirect` is set the
    // keys are read as keys[payload_in[i]] (multi-key / NULL-partitioned sorts).
    const uint32_t* payload_in = nullptr;
    int32_t indirect = 0;
    uint64_t n = 0;                      // host row count (upper bound when n_dev is set)
    const ull* n_dev = nullptr;          // optional device row count
    uint32_t* payload_out = nullptr;     // sorted payload (required)
    ull* keys_out = nullptr;             // optional sorted u64 keys (SRC_U64_KEYS only)
};

// Enqueues the sort on `s`. Scratch comes from the context arena.
bolt_status radix_sort(bolt_ctx* ctx, cudaStream_t s, const SortSpec& spec);

// Scratch bytes radix_sort needs for n rows of the given source.
uint64_t radix_sort_scratch(uint64_t n, int32_t src);

}  // namespace bolt
