// join.cuh — hash join table shared by the probe and the fused join GROUP BY.
#pragma once

#include "ctx.cuh"

// A build-side hash table in the context arena. Slot i holds two words:
//   word 0: bitwise NOT of the key (0 = empty; key -1 lives in slot `cap`),
//   word 1: (build row << 32) | u32 payload — or, in a multi-match table
//           (duplicate build keys), (first position in sorted_rows << 32) |
//           number of build rows with the key.
struct bolt_join_table {
    ull* slots = nullptr;
    int32_t log2cap = 0;
    int32_t key_dtype = BOLT_I64;
    int32_t has_payload = 0;
    int32_t multi = 0;                 // 1: duplicate build keys, word 1 as above
    uint32_t* sorted_rows = nullptr;   // multi: the non-NULL build rows, stably sorted by key
    uint64_t n_build = 0;
    uint64_t pinned_mark = 0;  // arena_pinned before this table was placed
    bolt_ctx* owner = nullptr;
};

namespace bolt {

constexpr ull JOIN_HASH = 0x9E3779B97F4A7C15ull;

// Looks up `key` (already widened to 64 bits); returns word 1 of the slot or
// ~0 when absent. Probes are bounded by the table size.
__device__ __forceinline__ ull join_lookup(const ull* slots, int log2cap, ull key) {
    const ull cap = 1ull << log2cap;
    const ull stored = ~key;
    if (stored == 0) {
        const ull* sp = slots + 2 * cap;
        return sp[0] ? sp[1] : ~0ull;
    }
    ull h = (stored * JOIN_HASH) >> (64 - log2cap);
    for (ull i = 0; i < cap; ++i) {
        const ulonglong2 s = __ldg(reinterpret_cast<const ulonglong2*>(slots) + h);
        if (s.x == stored) return s.y;
        if (s.x == 0) return ~0ull;
        h = (h + 1) & (cap - 1);
    }
    return ~0ull;
}

}  // namespace bolt
