// gb_device.cuh — device-side building blocks of the GROUP BY kernels:
// hashing, row loading, per-state contributions, merges into the shared and
// global tables, table probes and the aggregate-state layouts the row loops
// are compiled for. Included by groupby.cu and groupby_part.cu.
#pragma once

#include "groupby.cuh"
#include "join.cuh"

namespace bolt {
namespace {

constexpr int SMEM_PROBES = 16;
constexpr int SMALL_FINAL_MAX = 8192;
constexpr ull HASH_G = 0x9E3779B97F4A7C15ull;
constexpr ull HASH_S = 0xD6E8FEB86659FD93ull;

// ---------------------------------------------------------------------------
// Row loading
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t key_bits32(const void* c, int dt, uint64_t r) {
    if (dt == BOLT_F32) return canon_f32_bits(ld_stream((const float*)c + r));
    return (uint32_t)ld_stream((const int32_t*)c + r);
}

__device__ __forceinline__ ull pack_key(const GbParams& p, uint64_t r) {
    if (p.n_keys == 1) {
        const void* c = p.kcol[0];
        switch (p.kdtype[0]) {
        case BOLT_I32: return (ull)(ll)ld_stream((const int32_t*)c + r);
        case BOLT_I64: return (ull)ld_stream((const ll*)c + r);
        case BOLT_F32: return (ull)canon_f32_bits(ld_stream((const float*)c + r));
        default: return canon_f64_bits(ld_stream((const double*)c + r));
        }
    }
    ull hi = key_bits32(p.kcol[0], p.kdtype[0], r);
    ull lo = key_bits32(p.kcol[1], p.kdtype[1], r);
    return (hi << 32) | lo;
}

__device__ __forceinline__ bool cmp_i(ll v, int cmp, ll lit) {
    switch (cmp) {
    case BOLT_CMP_LT: return v < lit;
    case BOLT_CMP_LE: return v <= lit;
    case BOLT_CMP_GT: return v > lit;
    case BOLT_CMP_GE: return v >= lit;
    case BOLT_CMP_EQ: return v == lit;
    default: return v != lit;
    }
}

__device__ __forceinline__ bool cmp_f(double v, int cmp, double lit) {
    switch (cmp) {
    case BOLT_CMP_LT: return v < lit;
    case BOLT_CMP_LE: return v <= lit;
    case BOLT_CMP_GT: return v > lit;
    case BOLT_CMP_GE: return v >= lit;
    case BOLT_CMP_EQ: return v == lit;
    default: return v != lit;
    }
}

__device__ __forceinline__ bool eval_pred(const PredDesc& d, uint64_t r) {
    if (!bit_valid(d.valid, r)) return false;
    switch (d.dtype) {
    case BOLT_F64: return cmp_f(ld_stream((const double*)d.col + r), d.cmp, d.lit_f);
    case BOLT_F32: return cmp_f((double)ld_stream((const float*)d.col + r), d.cmp, d.lit_f);
    case BOLT_I64: return cmp_i(ld_stream((const ll*)d.col + r), d.cmp, d.lit_i);
    default: return cmp_i((ll)ld_stream((const int32_t*)d.col + r), d.cmp, d.lit_i);
    }
}

// Raw 64-bit image of a state's input (sign-extended ints, f64 bits,
// f32 widened to f64 bits, low word of a Decimal128).
__device__ __forceinline__ ull load_raw(const StateDesc& s, uint64_t r, bool& dec_fits) {
    switch (s.dtype) {
    case BOLT_I32: return (ull)(ll)ld_stream((const int32_t*)s.col + r);
    case BOLT_I64: return (ull)ld_stream((const ll*)s.col + r);
    case BOLT_F32: return (ull)__double_as_longlong((double)ld_stream((const float*)s.col + r));
    case BOLT_F64: return (ull)__double_as_longlong(ld_stream((const double*)s.col + r));
    default: {  // DEC128
        const ulonglong2 v = ld_stream((const ulonglong2*)s.col + r);
        dec_fits = (ll)v.y == ((ll)v.x >> 63);
        return v.x;
    }
    }
}

__device__ __forceinline__ ull order_key(ull raw, int dt) {
    if (dt == BOLT_F32 || dt == BOLT_F64) return f64_order_key(__longlong_as_double((ll)raw));
    return raw ^ 0x8000000000000000ull;
}

// Contribution (c0, c1) of one row to one state; zero words are the identity.
__device__ __forceinline__ void contribution(const GbParams& p, const StateDesc& s, int kind, ull raw, bool valid,
                                             bool dec_fits, uint64_t r, ull& c0, ull& c1) {
    c0 = 0;
    c1 = 0;
    if (!valid) return;
    switch (kind) {
    case K_COUNT: c0 = 1; break;
    case K_SUM_I32: c0 = raw; break;
    case K_SUM_D64:
        if (!dec_fits) { atomicOr(p.status, ST_FLAG_DECRANGE); return; }
        // fallthrough
    case K_SUM_I64:
        c0 = raw & 0xFFFFFFFFull;
        c1 = (ull)((ll)raw >> 32);
        break;
    case K_SUM_D128:
        c0 = raw;
        c1 = ld_stream((const ull*)s.col + 2 * r + 1);
        break;
    case K_SUM_FX: {
        ll hi;
        if (!f64_to_fixed(__longlong_as_double((ll)raw), p.fx_e, c0, hi)) {
            atomicOr(p.status, ST_FLAG_RANGE);
            c0 = 0;
            return;
        }
        c1 = (ull)hi;
        break;
    }
    case K_SUM_FATOM: c0 = raw; break;
    case K_MAX_ORD: c0 = order_key(raw, s.dtype); break;
    default: c0 = ~order_key(raw, s.dtype); break;  // K_MIN_ORD
    }
}

// Combines two contributions of the same state (register-side pre-aggregation).
__device__ __forceinline__ void combine(int kind, ull& a0, ull& a1, ull b0, ull b1) {
    switch (kind) {
    case K_COUNT:
    case K_SUM_I32: a0 += b0; break;
    case K_SUM_I64:
    case K_SUM_D64: a0 += b0; a1 += b1; break;
    case K_SUM_FX:
    case K_SUM_D128: {  // (warp pre-aggregation is off when a D128 state exists)
        ull lo = a0 + b0;
        a1 = a1 + b1 + (lo < a0 ? 1ull : 0ull);
        a0 = lo;
        break;
    }
    case K_SUM_FATOM:
        a0 = (ull)__double_as_longlong(__longlong_as_double((ll)a0) + __longlong_as_double((ll)b0));
        break;
    default: a0 = a0 > b0 ? a0 : b0; break;
    }
}

// Folds a contribution (or a partial state) into state words w (shared or
// global memory; the address space is resolved after inlining).
__device__ __forceinline__ void merge_words(ull* w, int kind, ull c0, ull c1) {
    if ((c0 | c1) == 0) return;
    switch (kind) {
    case K_COUNT:
    case K_SUM_I32: atomicAdd(w, c0); break;
    case K_SUM_I64:
    case K_SUM_D64:
        if (c0) atomicAdd(w, c0);
        if (c1) atomicAdd(w + 1, c1);
        break;
    case K_SUM_FX:
        // Global layout: bits 0-31 and 32-63 of the low word and the signed
        // high word accumulate in separate words, so no add waits for a
        // result (a 128-bit add would need the low word's old value for its
        // carry, one more round trip for every row that misses the shared
        // tier). The sums stay exact: the first two are below n * 2^32, the
        // third below 2^62 in magnitude (the fixed-point window shrinks as
        // the row count grows, see f64_to_fixed's scale).
        if (c0 & 0xFFFFFFFFull) atomicAdd(w, c0 & 0xFFFFFFFFull);
        if (c0 >> 32) atomicAdd(w + 1, c0 >> 32);
        if (c1) atomicAdd(w + 2, c1);
        break;
    case K_SUM_D128: {
        ull old = c0 ? atomicAdd(w, c0) : 0ull;
        ull carry = (c0 && old + c0 < old) ? 1ull : 0ull;
        ull mid = (c1 & 0xFFFFFFFFull) + carry;
        if (mid) atomicAdd(w + 1, mid);
        ull top = (ull)((ll)c1 >> 32);
        if (top) atomicAdd(w + 2, top);
        break;
    }
    case K_SUM_FATOM: atomicAdd(reinterpret_cast<double*>(w), __longlong_as_double((ll)c0)); break;
    default: atomicMax(w, c0); break;
    }
}

// Exact 64-bit add into a shared-memory word through native 32-bit atomics.
// A 64-bit shared atomic add is a compare-and-swap loop: about 6x the cost
// of a 32-bit add when uncontended and thousands of cycles when a warp or
// several warps hit one hot group. Here the low half takes the value's low
// 32 bits and its returned old value says whether it wrapped; the high half
// takes the high 32 bits plus that carry. The adds are linearisable, so the
// carries sum to exactly the wraps of the low half and the word ends equal
// to the 64-bit sum (it is only read after the CTA's final barrier).
__device__ __forceinline__ void smem_add64(ull* w, ull v) {
    uint32_t* h = reinterpret_cast<uint32_t*>(w);
    const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
    uint32_t c = 0;
    if (lo) {
        const uint32_t o = atomicAdd(h, lo);
        c = (o + lo < o) ? 1u : 0u;
    }
    if (hi + c) atomicAdd(h + 1, hi + c);
}

// The same, returning the carry out of bit 63 (the high half's add then
// returns its old value), for the low word of a 128-bit sum.
__device__ __forceinline__ uint32_t smem_add64_carry(ull* w, ull v) {
    uint32_t* h = reinterpret_cast<uint32_t*>(w);
    const uint32_t lo = (uint32_t)v, hi = (uint32_t)(v >> 32);
    uint32_t c = 0;
    if (lo) {
        const uint32_t o = atomicAdd(h, lo);
        c = (o + lo < o) ? 1u : 0u;
    }
    const uint32_t up = hi + c;
    uint32_t out = (up < hi) ? 1u : 0u;  // hi + c wrapped to 0: carry out, nothing to add
    if (up) {
        const uint32_t o = atomicAdd(h + 1, up);
        out += (o + up < o) ? 1u : 0u;
    }
    return out;
}

// Row-path merge into the shared-memory tier. Sums go through 32-bit
// atomics (smem_add64); COUNT accumulates in the low 32 bits of its word
// (exact while a CTA's table sees fewer than 2^32 rows: cnt32), and MIN /
// MAX read the word first and only use the (native) 64-bit atomic max when
// the row would win, which for a hot group is rarely after its first rows.
__device__ __forceinline__ void merge_words_smem(ull* w, int kind, ull c0, ull c1, bool cnt32) {
    if ((c0 | c1) == 0) return;
    switch (kind) {
    case K_COUNT:
        if (cnt32) atomicAdd(reinterpret_cast<uint32_t*>(w), (uint32_t)c0);
        else smem_add64(w, c0);
        break;
    case K_SUM_I32: smem_add64(w, c0); break;
    case K_SUM_I64:
    case K_SUM_D64:
        if (c0) smem_add64(w, c0);
        if (c1) smem_add64(w + 1, c1);
        break;
    case K_SUM_FX: {
        const uint32_t carry = c0 ? smem_add64_carry(w, c0) : 0u;
        if (c1 + carry) smem_add64(w + 1, c1 + carry);
        break;
    }
    case K_MAX_ORD:
    case K_MIN_ORD:
        if (c0 > *reinterpret_cast<volatile ull*>(w)) atomicMax(w, c0);
        break;
    default: merge_words(w, kind, c0, c1); break;  // D128, f64 atomics: rare modes
    }
}

// Folds a shared-table state (its words at src) into global-table state
// words w. A shared K_SUM_FX state is the 128-bit sum (lo, hi), which
// merge_words splits into the global layout.
__device__ __forceinline__ void merge_partial(ull* w, int kind, const ull* src) {
    if (kind == K_SUM_D128) {
        const ull s0 = src[0];
        ull old = s0 ? atomicAdd(w, s0) : 0ull;
        ull carry = (s0 && old + s0 < old) ? 1ull : 0ull;
        if (src[1] + carry) atomicAdd(w + 1, src[1] + carry);
        if (src[2]) atomicAdd(w + 2, src[2]);
        return;
    }
    const bool two = kind == K_SUM_I64 || kind == K_SUM_D64 || kind == K_SUM_FX;
    merge_words(w, kind, src[0], two ? src[1] : 0ull);
}

// Exact signed value of a K_SUM_D128 state; false when outside i128.
__device__ __forceinline__ bool d128_value(const ull* w, __int128& v) {
    const unsigned __int128 low = ((unsigned __int128)w[1] << 64) | w[0];
    const __int128 t = (__int128)(ll)w[2] + (__int128)(ull)(low >> 96);
    if (t < -((__int128)1 << 31) || t >= ((__int128)1 << 31)) return false;
    const unsigned __int128 r = low & ((((unsigned __int128)1) << 96) - 1);
    v = (__int128)(((unsigned __int128)t << 96) | r);
    return true;
}

// Global table find-or-insert; -1 (and SPILL) when the probe limit is hit.
__device__ __forceinline__ int64_t g_find_insert(const GbParams& p, ull stored, uint32_t& inserts) {
    const ull mask = (1ull << p.log2cap) - 1;
    ull h = (stored * HASH_G) >> (64 - p.log2cap);
    for (uint32_t i = 0; i < p.max_probe; ++i) {
        ull* kp = p.gtab + h * (ull)p.slot_words;
        ull k = ld_volatile(kp);
        if (k == stored) return (int64_t)h;
        if (k == 0) {
            ull old = atomicCAS(kp, 0ull, stored);
            if (old == 0) { ++inserts; return (int64_t)h; }
            if (old == stored) return (int64_t)h;
        }
        h = (h + 1) & mask;
    }
    atomicOr(p.status, ST_FLAG_SPILL);
    return -1;
}

// Shared-tier find-or-insert. New keys are admitted only while the table
// holds fewer than `limit` keys (counted in *fill), so the table never fills
// up: a key that is absent meets an empty slot after a few probes and goes to
// the global table, instead of scanning the whole probe window. The first
// keys a CTA meets are admitted, which under skew are the frequent ones.
__device__ __forceinline__ int s_find_insert(ull* sk, int log2, ull stored, uint32_t* fill, uint32_t limit) {
    const uint32_t mask = (1u << log2) - 1;
    uint32_t h = (uint32_t)((stored * HASH_S) >> (64 - log2));
    volatile ull* vk = sk;
    for (int i = 0; i < SMEM_PROBES; ++i) {
        ull k = vk[h];
        if (k == stored) return (int)h;
        if (k == 0) {
            if (*reinterpret_cast<volatile uint32_t*>(fill) >= limit) return -1;
            ull old = atomicCAS(&sk[h], 0ull, stored);
            if (old == 0) {
                atomicAdd(fill, 1u);
                return (int)h;
            }
            if (old == stored) return (int)h;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// Aggregation kernel
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// Aggregate-state layouts the row loop is compiled for. A runtime switch over
// state kinds inside the unrolled row loop costs ~1,500 instructions per row
// and thrashes the instruction cache; the common layouts (states sorted by
// kind, see gb_plan) get a loop with the kinds known at compile time, and
// everything else runs the generic loop.
// ---------------------------------------------------------------------------
struct SpecGeneric {
    static constexpr bool generic = true;
};
template <int N, int K0, int K1 = 0, int K2 = 0, int K3 = 0>
struct SpecK {
    static constexpr bool generic = false;
    static constexpr int n = N;
    __host__ __device__ static constexpr int kind(int s) { return s == 0 ? K0 : s == 1 ? K1 : s == 2 ? K2 : K3; }
};
// Spec ids shared with the planner (gb_spec_of).
using Spec1 = SpecK<4, K_COUNT, K_SUM_FX, K_MAX_ORD, K_MIN_ORD>;   // COUNT, SUM/AVG f64, MAX, MIN
using Spec2 = SpecK<4, K_COUNT, K_SUM_I64, K_MAX_ORD, K_MIN_ORD>;  // COUNT, SUM i64, MAX, MIN
using Spec3 = SpecK<2, K_COUNT, K_SUM_D64>;                        // COUNT, SUM Decimal128
using Spec4 = SpecK<2, K_COUNT, K_SUM_I64>;                        // COUNT, SUM i64
using Spec5 = SpecK<2, K_COUNT, K_SUM_FX>;                         // COUNT, SUM f64
using Spec6 = SpecK<1, K_COUNT>;                                   // COUNT
using Spec7 = SpecK<2, K_COUNT, K_SUM_I32>;                        // COUNT, SUM i32

template <class SP>
__device__ __forceinline__ int skind(const GbParams& p, int s) {
    if constexpr (SP::generic) return p.st[s].kind;
    else return SP::kind(s);
}
template <class SP>
__device__ __forceinline__ int snum(const GbParams& p) {
    if constexpr (SP::generic) return p.n_st;
    else return SP::n;
}


// Publishes the warp's largest |v| bit length for int64 SUMs (whole warp).
__device__ __forceinline__ void gb_flush_absbits(const GbParams& p, uint32_t& absbits) {
    const uint32_t m = __reduce_max_sync(0xffffffffu, absbits);
    if (p.i64_bits && m && lane_id() == 0) atomicMax(p.i64_bits, m);
    absbits = 0;
}

// Per-warp occupancy accounting after a tile (whole warp, no block barrier):
// new keys are added to the query's counter in batches, and the warp learns
// whether the query already flagged growth or a spill (then it stops).
__device__ __forceinline__ bool gb_warp_epilogue(const GbParams& p, uint32_t& inserts, uint32_t& pending) {
    pending += __reduce_add_sync(0xffffffffu, inserts);
    inserts = 0;
    const uint32_t batch = p.log2cap > 20 ? 256u : (p.log2cap > 12 ? (1u << (p.log2cap - 12)) : 1u);
    uint32_t stop = 0;
    if (lane_id() == 0) {
        if (pending >= batch) {
            const ull tot = atomicAdd(p.occupancy, (ull)pending) + pending;
            if (tot > p.grow_limit) atomicOr(p.status, ST_FLAG_GROW);
        }
        stop = (*reinterpret_cast<volatile uint32_t*>(p.status) & (ST_FLAG_GROW | ST_FLAG_SPILL)) != 0;
    }
    if (pending >= batch) pending = 0;
    return __shfl_sync(0xffffffffu, stop, 0) != 0;
}

// Adds a warp's not yet published key count to the query's counter.
__device__ __forceinline__ void gb_warp_flush_pending(const GbParams& p, uint32_t& pending) {
    if (lane_id() == 0 && pending) {
        const ull tot = atomicAdd(p.occupancy, (ull)pending) + pending;
        if (tot > p.grow_limit) atomicOr(p.status, ST_FLAG_GROW);
    }
    pending = 0;
}

// Merges a CTA's shared table into the query's global table (whole CTA,
// after a __syncthreads()).
__device__ __forceinline__ void gb_flush_shared(const GbParams& p, const ull* sk, const ull* sw, int C) {
    const int SW = p.sslot_words - 1;
    uint32_t inserts = 0;
    for (int i = threadIdx.x; i < C; i += blockDim.x) {
        const ull key = sk[i];
        if (key == 0) continue;
        const int64_t g = g_find_insert(p, key, inserts);
        if (g < 0) continue;
        ull* w = p.gtab + (ull)g * p.slot_words;
        const ull* src = sw + (ull)i * SW - 1;
        for (int s = 0; s < p.n_st; ++s) {
            const StateDesc& d = p.st[s];
            merge_partial(w + d.word, d.kind, src + d.sword);
        }
    }
    if (inserts) {
        const ull tot = atomicAdd(p.occupancy, (ull)inserts) + inserts;
        if (tot > p.grow_limit) atomicOr(p.status, ST_FLAG_GROW);
    }
}

// ---------------------------------------------------------------------------
// Reads from a staged tile (shared memory) or straight from the columns
// ---------------------------------------------------------------------------
template <bool STAGED>
__device__ __forceinline__ const unsigned char* sc_base(const GbParams& p, int c, const unsigned char* stage,
                                                       uint64_t tile_row0) {
    if (STAGED) return stage + p.sc_off[c];
    return static_cast<const unsigned char*>(p.sc_col[c]) + (p.row_begin + tile_row0) * (uint64_t)p.sc_w[c];
}

__device__ __forceinline__ bool pred_at(const GbParams& p, int q, const unsigned char* base, uint32_t i) {
    const PredDesc& d = p.pred[q];
    switch (d.dtype) {
    case BOLT_F64: return cmp_f(reinterpret_cast<const double*>(base)[i], d.cmp, d.lit_f);
    case BOLT_F32: return cmp_f((double)reinterpret_cast<const float*>(base)[i], d.cmp, d.lit_f);
    case BOLT_I64: return cmp_i(reinterpret_cast<const ll*>(base)[i], d.cmp, d.lit_i);
    default: return cmp_i((ll)reinterpret_cast<const int32_t*>(base)[i], d.cmp, d.lit_i);
    }
}

__device__ __forceinline__ uint32_t key32_at(int dt, const unsigned char* base, uint32_t i) {
    if (dt == BOLT_F32) return canon_f32_bits(reinterpret_cast<const float*>(base)[i]);
    return (uint32_t)reinterpret_cast<const int32_t*>(base)[i];
}

__device__ __forceinline__ ull key_at(const GbParams& p, const unsigned char* b0, const unsigned char* b1,
                                      uint32_t i) {
    if (p.n_keys == 1) {
        switch (p.kdtype[0]) {
        case BOLT_I32: return (ull)(ll)reinterpret_cast<const int32_t*>(b0)[i];
        case BOLT_I64: return (ull)reinterpret_cast<const ll*>(b0)[i];
        case BOLT_F32: return (ull)canon_f32_bits(reinterpret_cast<const float*>(b0)[i]);
        default: return canon_f64_bits(reinterpret_cast<const double*>(b0)[i]);
        }
    }
    return ((ull)key32_at(p.kdtype[0], b0, i) << 32) | (ull)key32_at(p.kdtype[1], b1, i);
}

__device__ __forceinline__ ull raw_at(int dt, const unsigned char* base, uint32_t i, bool& dec_fits) {
    switch (dt) {
    case BOLT_I32: return (ull)(ll)reinterpret_cast<const int32_t*>(base)[i];
    case BOLT_I64: return (ull)reinterpret_cast<const ll*>(base)[i];
    case BOLT_F32: return (ull)__double_as_longlong((double)reinterpret_cast<const float*>(base)[i]);
    case BOLT_F64: return (ull)__double_as_longlong(reinterpret_cast<const double*>(base)[i]);
    default: {  // DEC128
        const ulonglong2 v = reinterpret_cast<const ulonglong2*>(base)[i];
        dec_fits = (ll)v.y == ((ll)v.x >> 63);
        return v.x;
    }
    }
}


}  // namespace
}  // namespace bolt
