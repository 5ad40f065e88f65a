// radix_sort.cuh — onesweep LSD radix sort (8-bit digits, decoupled look-back)
// over one or many independent segments in the same launches.
#pragma once

#include <vector>

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

// One independent sort. Payload input nullptr = row index (iota). With
// `indirect` (a spec-wide flag) keys are read as keys[payload_in[i]].
struct SortSegment {
    const void* keys = nullptr;
    const uint32_t* payload_in = nullptr;
    uint32_t* payload_out = nullptr;   // sorted payload (required)
    const ull* n_dev = nullptr;        // optional device row count (n is then an upper bound)
    uint64_t n = 0;
};

struct SortSpec {
    int32_t src = SRC_U64_KEYS;
    int32_t descending = 0;
    int32_t indirect = 0;
    std::vector<SortSegment> segs;
};

// Enqueues the sort of every segment on `s`. Scratch comes from the arena.
bolt_status radix_sort(bolt_ctx* ctx, cudaStream_t s, const SortSpec& spec);

// Scratch bytes radix_sort needs for segments of the given sizes.
uint64_t radix_sort_scratch(uint64_t total_n, uint64_t nseg, int32_t src);

}  // namespace bolt
