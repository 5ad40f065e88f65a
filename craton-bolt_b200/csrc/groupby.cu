// groupby.cu — fused filter + hash GROUP BY for sm_100a.
//
// Replaces the reference's GROUP BY executors (src/exec/groupby.rs:295-833,
// groupby_shmem_exec.rs, groupby_tier2_*.rs, groupby_with_pre.rs:222) whose
// kernels are runtime-emitted sm_70 PTX (hash_kernels.rs:246,764,
// shmem_*_kernel.rs, partition_*_kernel.rs): one keys launch plus one launch
// per aggregate, host key packing, host unique-count, host overflow re-fold
// and a host sort of the groups.
//
// Here one kernel streams every input column once (evict-first loads so the
// hash table keeps L2), evaluates the WHERE conjunction, packs the key
// (pack_keys semantics, groupby_common.rs:352) and folds every aggregate:
//   tier 1: a per-CTA open-addressing table in shared memory sized to the
//           227 KB opt-in limit (insert-if-room, bounded probes), optionally
//           fed by warp-level __match_any_sync pre-aggregation;
//   tier 2: rows whose key finds no room there go to a global open-addressing
//           table (64-bit CAS claim, linear probing, bounded probes -> spill);
//           the shared tables are merged into it when a CTA finishes.
// A finalize step compacts the occupied slots, sorts them by the packed key
// as a signed 64-bit integer (groupby.rs:789-800; onesweep radix sort, or a
// one-CTA bitonic sort for small tables) and writes the typed output columns.
//
// Exactness: integer SUMs are kept as split 32-bit partial sums that cannot
// overflow before 2^32 rows, then checked against the i64 range once
// (BOLT_ERR_OVERFLOW). float64 SUM/AVG use a 128-bit fixed-point accumulator
// whose scale follows from the row count, so the result is independent of
// the order of the atomics (identical alone or in a batch) and within
// n * 2^-(e+1) of the exact sum. Non-finite or |v| >= 2^32 inputs flag the
// call and it is re-run with plain f64 atomics (the reference's own method).
#include "groupby.cuh"
#include "radix_sort.cuh"

#include <algorithm>
#include <cstring>

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

__device__ __forceinline__ bool eval_pred(const PredDesc& d, uint64_t r) {
    if (!bit_valid(d.valid, r)) return false;
    if (d.dtype == BOLT_F64 || d.dtype == BOLT_F32) {
        double v = d.dtype == BOLT_F64 ? ld_stream((const double*)d.col + r)
                                       : (double)ld_stream((const float*)d.col + r);
        switch (d.cmp) {
        case BOLT_CMP_LT: return v < d.lit_f;
        case BOLT_CMP_LE: return v <= d.lit_f;
        case BOLT_CMP_GT: return v > d.lit_f;
        case BOLT_CMP_GE: return v >= d.lit_f;
        case BOLT_CMP_EQ: return v == d.lit_f;
        default: return v != d.lit_f;
        }
    }
    ll v = d.dtype == BOLT_I32 ? (ll)ld_stream((const int32_t*)d.col + r) : ld_stream((const ll*)d.col + r);
    switch (d.cmp) {
    case BOLT_CMP_LT: return v < d.lit_i;
    case BOLT_CMP_LE: return v <= d.lit_i;
    case BOLT_CMP_GT: return v > d.lit_i;
    case BOLT_CMP_GE: return v >= d.lit_i;
    case BOLT_CMP_EQ: return v == d.lit_i;
    default: return v != d.lit_i;
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
__device__ __forceinline__ void contribution(const GbParams& p, const StateDesc& s, ull raw, bool valid,
                                             bool dec_fits, uint64_t r, ull& c0, ull& c1) {
    c0 = 0;
    c1 = 0;
    if (!valid) return;
    switch (s.kind) {
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
    case K_SUM_FX: {
        ull old = c0 ? atomicAdd(w, c0) : 0ull;
        ull carry = (c0 && old + c0 < old) ? 1ull : 0ull;
        if (c1 + carry) atomicAdd(w + 1, c1 + carry);
        break;
    }
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

// Folds a partial state (all of its words) into state words w.
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

__device__ __forceinline__ int s_find_insert(ull* sk, int log2, ull stored) {
    const uint32_t mask = (1u << log2) - 1;
    uint32_t h = (uint32_t)((stored * HASH_S) >> (64 - log2));
    volatile ull* vk = sk;
    for (int i = 0; i < SMEM_PROBES; ++i) {
        ull k = vk[h];
        if (k == stored) return (int)h;
        if (k == 0) {
            ull old = atomicCAS(&sk[h], 0ull, stored);
            if (old == 0 || old == stored) return (int)h;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

// ---------------------------------------------------------------------------
// Aggregation kernel
// ---------------------------------------------------------------------------
template <int U, int MAXS>
__global__ void __launch_bounds__(512) gb_agg_kernel(const __grid_constant__ GbParams p) {
    extern __shared__ __align__(16) ull smem[];
    __shared__ uint32_t s_ins;
    __shared__ int s_stop;
    const int SW = p.slot_words - 1;
    const int C = p.smem_log2 ? (1 << p.smem_log2) : 0;
    ull* sk = smem;
    ull* sw = smem + C;
    for (int i = threadIdx.x; i < C * (SW + 1); i += blockDim.x) smem[i] = 0;
    if (threadIdx.x == 0) { s_ins = 0; s_stop = 0; }
    __syncthreads();

    const uint32_t lane = lane_id();
    const uint64_t n = p.n_rows;
    const uint64_t tile = (uint64_t)blockDim.x * U;
    uint32_t inserts = 0;

    for (uint64_t base = (uint64_t)blockIdx.x * tile; base < n; base += (uint64_t)gridDim.x * tile) {
        bool has[U];
        bool knull[U];
        ull stored[U];
        ull raw[U][MAXS];
        uint32_t vbits[U];
        uint32_t dfit[U];
        // Issue every column load of the tile before any predicate resolves:
        // all sectors are read anyway at the selectivities of interest, and
        // independent loads keep more bytes in flight per SM.
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint64_t i = base + (uint64_t)u * blockDim.x + threadIdx.x;
            const uint64_t r = p.row_begin + i;
            has[u] = i < n;
            knull[u] = false;
            stored[u] = 0;
            vbits[u] = 0;
            dfit[u] = 0;
#pragma unroll
            for (int s = 0; s < MAXS; ++s) raw[u][s] = 0;
            if (!has[u]) continue;
            stored[u] = ~pack_key(p, r);
#pragma unroll
            for (int s = 0; s < MAXS; ++s) {
                if (s < p.n_st && p.st[s].col) {
                    bool fits = true;
                    raw[u][s] = load_raw(p.st[s], r, fits);
                    if (bit_valid(p.st[s].valid, r)) vbits[u] |= 1u << s;
                    if (fits) dfit[u] |= 1u << s;
                } else if (s < p.n_st) {
                    vbits[u] |= 1u << s;  // COUNT(*)
                    dfit[u] |= 1u << s;
                }
            }
            for (int q = 0; q < p.n_pred; ++q) has[u] = has[u] && eval_pred(p.pred[q], r);
            for (int k = 0; k < p.n_keys; ++k) knull[u] = knull[u] || !bit_valid(p.kvalid[k], r);
            if (knull[u] && p.n_keys > 1) has[u] = false;  // multi-key: NULL-key rows are dropped
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            bool row = has[u];
            ull c0[MAXS], c1[MAXS];
#pragma unroll
            for (int s = 0; s < MAXS; ++s) {
                c0[s] = 0;
                c1[s] = 0;
                if (row && s < p.n_st)
                    contribution(p, p.st[s], raw[u][s], (vbits[u] >> s) & 1, (dfit[u] >> s) & 1,
                                 p.row_begin + base + (uint64_t)u * blockDim.x + threadIdx.x, c0[s], c1[s]);
            }
            // Special groups: the NULL key and the key whose complement is 0.
            const bool special = row && (knull[u] || stored[u] == 0);
            if (special) {
                const ull slot = (1ull << p.log2cap) + (knull[u] ? 1 : 0);
                ull* w = p.gtab + slot * (ull)p.slot_words;
                if (ld_volatile(w) == 0) *reinterpret_cast<volatile ull*>(w) = 1ull;
#pragma unroll
                for (int s = 0; s < MAXS; ++s)
                    if (s < p.n_st) merge_words(w + p.st[s].word, p.st[s].kind, c0[s], c1[s]);
                row = false;
            }
            // Warp-level pre-aggregation of duplicate keys.
            if (p.warp_agg) {
                const uint32_t act = __ballot_sync(0xffffffffu, row);
                uint32_t peers = 0;
                if (row) peers = __match_any_sync(act, stored[u]);
                const bool leader = row && (uint32_t)(__ffs(peers) - 1) == lane;
                uint32_t others = leader ? (peers & ~(1u << lane)) : 0u;
                const int rounds = __reduce_max_sync(0xffffffffu, (uint32_t)__popc(others));
                for (int it = 0; it < rounds; ++it) {
                    int src = (int)lane;
                    if (others) {
                        src = __ffs(others) - 1;
                        others &= others - 1;
                    }
#pragma unroll
                    for (int s = 0; s < MAXS; ++s) {
                        if (s < p.n_st) {
                            ull b0 = __shfl_sync(0xffffffffu, c0[s], src);
                            ull b1 = __shfl_sync(0xffffffffu, c1[s], src);
                            if (leader && src != (int)lane) combine(p.st[s].kind, c0[s], c1[s], b0, b1);
                        }
                    }
                }
                row = leader;
            }
            if (!row) continue;
            int sl = -1;
            if (C) sl = s_find_insert(sk, p.smem_log2, stored[u]);
            if (sl >= 0) {
                ull* w = sw + (ull)sl * SW - 1;  // state word offsets count the key word
#pragma unroll
                for (int s = 0; s < MAXS; ++s)
                    if (s < p.n_st) merge_words(w + p.st[s].word, p.st[s].kind, c0[s], c1[s]);
            } else {
                int64_t g = g_find_insert(p, stored[u], inserts);
                if (g >= 0) {
                    ull* w = p.gtab + (ull)g * p.slot_words;
#pragma unroll
                    for (int s = 0; s < MAXS; ++s)
                        if (s < p.n_st) merge_words(w + p.st[s].word, p.st[s].kind, c0[s], c1[s]);
                }
            }
        }
        // Occupancy accounting: stop early once the table must grow.
        if (inserts) {
            atomicAdd(&s_ins, inserts);
            inserts = 0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (s_ins) {
                ull tot = atomicAdd(p.occupancy, (ull)s_ins) + s_ins;
                s_ins = 0;
                if (tot > p.grow_limit) atomicOr(p.status, ST_FLAG_GROW);
            }
            s_stop = (*reinterpret_cast<volatile uint32_t*>(p.status) & (ST_FLAG_GROW | ST_FLAG_SPILL)) != 0;
        }
        __syncthreads();
        if (s_stop) break;
    }
    if (s_stop) return;

    // Merge the shared-memory table into the global table.
    __syncthreads();
    for (int i = threadIdx.x; i < C; i += blockDim.x) {
        const ull key = sk[i];
        if (key == 0) continue;
        int64_t g = g_find_insert(p, key, inserts);
        if (g < 0) continue;
        ull* w = p.gtab + (ull)g * p.slot_words;
        const ull* src = sw + (ull)i * SW - 1;
        for (int s = 0; s < p.n_st; ++s) {
            const StateDesc& d = p.st[s];
            merge_partial(w + d.word, d.kind, src + d.word);
        }
    }
    if (inserts) {
        ull tot = atomicAdd(p.occupancy, (ull)inserts) + inserts;
        if (tot > p.grow_limit) atomicOr(p.status, ST_FLAG_GROW);
    }
}

// ---------------------------------------------------------------------------
// Finalize
// ---------------------------------------------------------------------------
__device__ __forceinline__ void write_bit(uint8_t* bm, uint64_t i, bool on) {
    if (bm) set_bit_atomic(bm, i, on);
}

__device__ __forceinline__ double sum_as_double(const GbFinal& f, const StateDesc& s, const ull* w) {
    switch (s.kind) {
    case K_SUM_I32: return (double)(ll)w[0];
    case K_SUM_I64:
    case K_SUM_D64: {
        __int128 v = ((__int128)(ll)w[1] << 32) + (__int128)w[0];
        return i128_to_double_scaled((ull)v, (ll)(v >> 64), 0);
    }
    case K_SUM_FX: return i128_to_double_scaled(w[0], (ll)w[1], f.fx_e);
    default: return __longlong_as_double((ll)w[0]);
    }
}

// Writes output row o from slot `slot` (slot == cap + 1 is the NULL group).
__device__ void emit_group(const GbFinal& f, uint64_t o, uint64_t slot) {
    const ull cap = 1ull << f.log2cap;
    const ull* w = f.gtab + slot * (ull)f.slot_words;
    const bool null_key = slot == cap + 1;
    const ull packed = slot == cap ? ~0ull : ~w[0];
    for (int k = 0; k < f.n_keys; ++k) {
        void* out = f.out_key[k];
        ull bits = f.n_keys == 1 ? packed : (k == 0 ? (packed >> 32) : (packed & 0xFFFFFFFFull));
        if (null_key) bits = 0;
        switch (f.kdtype[k]) {
        case BOLT_I32:
        case BOLT_F32: ((uint32_t*)out)[o] = (uint32_t)bits; break;
        default: ((ull*)out)[o] = bits; break;
        }
        write_bit(f.out_key_valid[k], o, !null_key);
    }
    for (int a = 0; a < f.n_aggs; ++a) {
        const AggOut& g = f.agg[a];
        ull cnt = g.cnt_state >= 0 ? w[f.st[g.cnt_state].word] : 1ull;
        bool valid = !g.nullable || cnt > 0;
        switch (g.op) {
        case BOLT_AGG_COUNT_STAR:
        case BOLT_AGG_COUNT:
            ((ll*)g.out)[o] = (ll)cnt;
            valid = true;
            break;
        case BOLT_AGG_SUM: {
            const StateDesc& s = f.st[g.sum_state];
            const ull* sw = w + s.word;
            if (s.kind == K_SUM_I32) {
                ((ll*)g.out)[o] = (ll)sw[0];
            } else if (s.kind == K_SUM_I64) {
                __int128 v = ((__int128)(ll)sw[1] << 32) + (__int128)sw[0];
                if (v > (__int128)0x7FFFFFFFFFFFFFFFll || v < -(__int128)0x7FFFFFFFFFFFFFFFll - 1)
                    atomicOr(f.status, ST_FLAG_OVERFLOW);
                ((ll*)g.out)[o] = (ll)v;
            } else if (s.kind == K_SUM_D64 || s.kind == K_SUM_D128) {
                __int128 v = 0;
                if (s.kind == K_SUM_D64) v = ((__int128)(ll)sw[1] << 32) + (__int128)sw[0];
                else if (!d128_value(sw, v)) atomicOr(f.status, ST_FLAG_DECOVERFLOW);
                if (!valid) v = 0;
                ((ull*)g.out)[2 * o] = (ull)v;
                ((ull*)g.out)[2 * o + 1] = (ull)(v >> 64);
            } else {
                ((double*)g.out)[o] = valid ? sum_as_double(f, s, sw) : 0.0;
            }
            break;
        }
        case BOLT_AGG_AVG: {
            const StateDesc& s = f.st[g.sum_state];
            ((double*)g.out)[o] = (valid && cnt) ? sum_as_double(f, s, w + s.word) / (double)cnt : 0.0;
            break;
        }
        default: {  // MIN / MAX
            const StateDesc& s = f.st[g.mm_state];
            ull k = w[s.word];
            if (s.kind == K_MIN_ORD) k = ~k;
            if (!valid) k = 0x8000000000000000ull;
            switch (g.out_dtype) {
            case BOLT_I32: ((int32_t*)g.out)[o] = (int32_t)(ll)(k ^ 0x8000000000000000ull); break;
            case BOLT_I64: ((ll*)g.out)[o] = (ll)(k ^ 0x8000000000000000ull); break;
            case BOLT_F32: ((float*)g.out)[o] = valid ? (float)f64_from_order_key(k) : 0.f; break;
            default: ((double*)g.out)[o] = valid ? f64_from_order_key(k) : 0.0; break;
            }
        }
        }
        write_bit(g.out_valid, o, valid);
    }
}

// Occupied-slot compaction for the large path; order key = packed ^ sign bit.
__global__ void __launch_bounds__(256) gb_compact_kernel(GbFinal f) {
    const ull cap = 1ull << f.log2cap;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base <= cap; base += stride) {
        const uint64_t i = base + threadIdx.x;
        bool occ = false;
        ull ok = 0;
        if (i < cap) {
            ull k = ld_volatile(f.gtab + i * (ull)f.slot_words);
            occ = k != 0;
            ok = ~k ^ 0x8000000000000000ull;
        } else if (i == cap) {
            occ = f.gtab[cap * (ull)f.slot_words] != 0;
            ok = ~0ull ^ 0x8000000000000000ull;
        }
        const uint32_t m = __ballot_sync(0xffffffffu, occ);
        if (!m) continue;
        ull pos = 0;
        if (lane_id() == (uint32_t)(__ffs(m) - 1)) pos = atomicAdd(f.n_nonnull, (ull)__popc(m));
        pos = __shfl_sync(0xffffffffu, pos, __ffs(m) - 1);
        if (occ) {
            pos += __popc(m & lanemask_lt());
            f.order_keys[pos] = ok;
            f.slots[pos] = (uint32_t)i;
        }
    }
}

__global__ void __launch_bounds__(256) gb_gather_kernel(GbFinal f) {
    const ull cap = 1ull << f.log2cap;
    const ull G = *f.n_nonnull;
    const bool has_null = f.gtab[(cap + 1) * (ull)f.slot_words] != 0;
    const ull total = G + (has_null ? 1 : 0);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *f.n_groups = total;
        if (f.n_groups_user) *f.n_groups_user = total;
        if (total > f.out_cap) atomicOr(f.status, ST_FLAG_CAPACITY);
    }
    const ull lim = total < f.out_cap ? total : f.out_cap;
    for (uint64_t o = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; o < lim; o += (uint64_t)gridDim.x * blockDim.x)
        emit_group(f, o, o < G ? f.sorted[o] : cap + 1);
}

// One CTA: compact + bitonic sort in shared memory + emit (tables <= 8192 slots).
__global__ void __launch_bounds__(1024) gb_small_final_kernel(GbFinal f) {
    extern __shared__ __align__(16) ull sm[];
    __shared__ uint32_t s_n;
    const ull cap = 1ull << f.log2cap;
    const uint32_t P = (uint32_t)cap * 2;  // power of two >= cap + 1
    ull* key = sm;
    uint32_t* slot = reinterpret_cast<uint32_t*>(sm + P);
    if (threadIdx.x == 0) s_n = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i <= cap; i += blockDim.x) {
        ull k = f.gtab[(ull)i * f.slot_words];
        if (k == 0) continue;
        uint32_t pos = atomicAdd(&s_n, 1u);
        key[pos] = (i == cap ? ~0ull : ~k) ^ 0x8000000000000000ull;
        slot[pos] = i;
    }
    __syncthreads();
    const uint32_t G = s_n;
    uint32_t Pn = 1;
    while (Pn < G) Pn <<= 1;
    for (uint32_t i = G + threadIdx.x; i < Pn; i += blockDim.x) {
        key[i] = ~0ull;
        slot[i] = 0xFFFFFFFFu;
    }
    __syncthreads();
    for (uint32_t k = 2; k <= Pn; k <<= 1) {
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < Pn; i += blockDim.x) {
                const uint32_t x = i ^ j;
                if (x > i) {
                    const bool asc = (i & k) == 0;
                    const ull a = key[i], b = key[x];
                    // Padding (slot ~0) always sorts last; keys are unique.
                    const bool gt = (slot[i] == 0xFFFFFFFFu) ? (slot[x] != 0xFFFFFFFFu)
                                  : (slot[x] == 0xFFFFFFFFu) ? false : a > b;
                    if (gt == asc) {
                        key[i] = b; key[x] = a;
                        const uint32_t t = slot[i]; slot[i] = slot[x]; slot[x] = t;
                    }
                }
            }
            __syncthreads();
        }
    }
    const bool has_null = f.gtab[(cap + 1) * (ull)f.slot_words] != 0;
    const ull total = (ull)G + (has_null ? 1 : 0);
    if (threadIdx.x == 0) {
        *f.n_groups = total;
        *f.n_nonnull = G;
        if (f.n_groups_user) *f.n_groups_user = total;
        if (total > f.out_cap) atomicOr(f.status, ST_FLAG_CAPACITY);
    }
    const ull lim = total < f.out_cap ? total : f.out_cap;
    for (uint64_t o = threadIdx.x; o < lim; o += blockDim.x) emit_group(f, o, o < G ? slot[o] : cap + 1);
}

template <int U, int MAXS>
bolt_status launch_agg(bolt_ctx* ctx, const GbPlan& pl, cudaStream_t s, size_t smem) {
    auto kfn = gb_agg_kernel<U, MAXS>;
    BOLT_CUDA(ctx, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kfn<<<pl.grid, pl.block, smem, s>>>(pl.prm);
    ctx->last_launches++;
    return BOLT_OK;
}

int dtype_size(int dt) {
    switch (dt) {
    case BOLT_I32: case BOLT_F32: case BOLT_U32: return 4;
    case BOLT_DEC128: return 16;
    default: return 8;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Planning
// ---------------------------------------------------------------------------
bolt_status gb_plan(bolt_ctx* ctx, const bolt_groupby_desc* d, const bolt_groupby_out* out,
                    uint64_t row_begin, uint64_t row_end, uint32_t flags, int mode,
                    uint64_t cap_override, GbPlan* pl) {
    if (!d || !out || !d->cols || d->n_cols <= 0) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: missing table");
    if (d->n_keys < 1 || d->n_keys > 2 || !d->key_cols)
        return fail(ctx, BOLT_DECLINE, "GROUP BY: %d key columns (1 or 2 supported)", d->n_keys);
    if (d->n_aggs < 1 || d->n_aggs > GB_MAX_AGGS || !d->aggs)
        return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: %d aggregates", d->n_aggs);
    if (d->n_preds < 0 || d->n_preds > GB_MAX_PREDS)
        return fail(ctx, BOLT_DECLINE, "GROUP BY: %d WHERE conjuncts (max %d)", d->n_preds, GB_MAX_PREDS);
    *pl = GbPlan();
    GbParams& p = pl->prm;
    GbFinal& f = pl->fin;
    pl->flags = flags;
    pl->mode = mode;
    const uint64_t n = row_end > row_begin ? row_end - row_begin : 0;
    auto col = [&](int i) -> const bolt_col_view* {
        return (i >= 0 && i < d->n_cols) ? &d->cols[i] : nullptr;
    };
    for (int k = 0; k < d->n_keys; ++k) {
        const bolt_col_view* c = col(d->key_cols[k]);
        if (!c) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: key column %d out of range", d->key_cols[k]);
        if (c->len < row_end) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: key column shorter than the rows");
        const int dt = c->dtype;
        const bool ok = d->n_keys == 1 ? (dt == BOLT_I32 || dt == BOLT_I64 || dt == BOLT_F32 || dt == BOLT_F64)
                                       : (dt == BOLT_I32 || dt == BOLT_F32);
        if (!ok) return fail(ctx, BOLT_DECLINE, "GROUP BY: key dtype %d not packable into 64 bits", dt);
        p.kcol[k] = c->data;
        p.kvalid[k] = c->validity;
        p.kdtype[k] = dt;
        f.kdtype[k] = dt;
        if (!out->keys || out->keys[k].dtype != dt)
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output key column %d dtype mismatch", k);
        f.out_key[k] = out->keys[k].data;
        f.out_key_valid[k] = out->keys[k].validity;
    }
    p.n_keys = f.n_keys = d->n_keys;
    for (int q = 0; q < d->n_preds; ++q) {
        const bolt_col_view* c = col(d->preds[q].col);
        if (!c) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: WHERE column out of range");
        if (c->dtype == BOLT_DEC128 || c->dtype == BOLT_U32)
            return fail(ctx, BOLT_DECLINE, "GROUP BY: WHERE on dtype %d", c->dtype);
        p.pred[q] = PredDesc{c->data, c->validity, c->dtype, d->preds[q].cmp, d->preds[q].lit_i, d->preds[q].lit_f};
    }
    p.n_pred = d->n_preds;

    // States, deduplicated by (kind, column).
    int n_st = 0;
    int word = 1;
    auto add_state = [&](int kind, int ci) -> int {
        const bolt_col_view* c = ci >= 0 ? col(ci) : nullptr;
        const void* data = c ? c->data : nullptr;
        // COUNT(col) of a column without NULLs is COUNT(*).
        if (kind == K_COUNT && c && !c->validity) data = nullptr, c = nullptr;
        for (int s = 0; s < n_st; ++s)
            if (p.st[s].kind == kind && p.st[s].col == data &&
                p.st[s].valid == (c ? c->validity : nullptr))
                return s;
        if (n_st == GB_MAX_STATES) return -1;
        StateDesc& sd = p.st[n_st];
        sd.col = data;
        sd.valid = c ? c->validity : nullptr;
        sd.kind = kind;
        sd.dtype = c ? c->dtype : BOLT_I64;
        sd.word = word;
        sd.nwords = (kind == K_SUM_I64 || kind == K_SUM_FX || kind == K_SUM_D64) ? 2 : (kind == K_SUM_D128 ? 3 : 1);
        word += sd.nwords;
        return n_st++;
    };
    for (int a = 0; a < d->n_aggs; ++a) {
        const bolt_agg_spec& sp = d->aggs[a];
        AggOut& g = f.agg[a];
        g.op = sp.op;
        g.sum_state = g.cnt_state = g.mm_state = -1;
        const bolt_col_view* c = sp.op == BOLT_AGG_COUNT_STAR ? nullptr : col(sp.input_col);
        if (sp.op != BOLT_AGG_COUNT_STAR && !c)
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: aggregate %d input column out of range", a);
        if (c && c->len < row_end) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: value column shorter than the rows");
        const int dt = c ? c->dtype : BOLT_I64;
        g.in_dtype = dt;
        g.nullable = c && c->validity ? 1 : 0;
        int need_cnt = g.nullable;
        switch (sp.op) {
        case BOLT_AGG_COUNT_STAR:
            g.out_dtype = BOLT_I64;
            g.cnt_state = add_state(K_COUNT, -1);
            break;
        case BOLT_AGG_COUNT:
            g.out_dtype = BOLT_I64;
            g.cnt_state = add_state(K_COUNT, sp.input_col);
            need_cnt = 0;
            break;
        case BOLT_AGG_SUM:
        case BOLT_AGG_AVG: {
            int kind;
            if (dt == BOLT_I32) kind = K_SUM_I32;
            else if (dt == BOLT_I64) kind = K_SUM_I64;
            else if (dt == BOLT_F64) kind = (mode & GB_MODE_F64_ATOMIC) ? K_SUM_FATOM : K_SUM_FX;
            else if (dt == BOLT_DEC128 && sp.op == BOLT_AGG_SUM) kind = (mode & GB_MODE_WIDE_DEC) ? K_SUM_D128 : K_SUM_D64;
            else return fail(ctx, BOLT_DECLINE, "GROUP BY: %s over dtype %d", sp.op == BOLT_AGG_SUM ? "SUM" : "AVG", dt);
            g.sum_state = add_state(kind, sp.input_col);
            if (sp.op == BOLT_AGG_AVG) {
                g.out_dtype = BOLT_F64;
                g.cnt_state = add_state(K_COUNT, sp.input_col);
                need_cnt = 0;
            } else {
                g.out_dtype = dt == BOLT_I32 ? BOLT_I64 : dt;
            }
            break;
        }
        case BOLT_AGG_MIN:
        case BOLT_AGG_MAX:
            if (dt == BOLT_DEC128 || dt == BOLT_U32)
                return fail(ctx, BOLT_DECLINE, "GROUP BY: MIN/MAX over dtype %d", dt);
            g.out_dtype = dt;
            g.mm_state = add_state(sp.op == BOLT_AGG_MIN ? K_MIN_ORD : K_MAX_ORD, sp.input_col);
            break;
        default:
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: unknown aggregate op %d", sp.op);
        }
        if (need_cnt) g.cnt_state = add_state(K_COUNT, sp.input_col);
        const bool is_count = sp.op == BOLT_AGG_COUNT || sp.op == BOLT_AGG_COUNT_STAR;
        const bool missing = is_count ? g.cnt_state < 0
                           : ((g.sum_state < 0 && g.mm_state < 0) || ((g.nullable || sp.op == BOLT_AGG_AVG) && g.cnt_state < 0));
        if (missing) return fail(ctx, BOLT_DECLINE, "GROUP BY: more than %d aggregate states", GB_MAX_STATES);
        if (!out->aggs || out->aggs[a].dtype != g.out_dtype)
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output column %d must have dtype %d", a, g.out_dtype);
        g.out = out->aggs[a].data;
        g.out_valid = out->aggs[a].validity;
    }
    p.n_st = n_st;
    p.slot_words = word;
    f.slot_words = word;
    f.n_aggs = d->n_aggs;
    std::memcpy(f.st, p.st, sizeof(p.st));
    pl->n_aggs = d->n_aggs;

    uint64_t out_cap = UINT64_MAX;
    for (int k = 0; k < d->n_keys; ++k) out_cap = std::min<uint64_t>(out_cap, out->keys[k].cap);
    for (int a = 0; a < d->n_aggs; ++a) out_cap = std::min<uint64_t>(out_cap, out->aggs[a].cap);
    f.out_cap = out_cap;

    // Table sizing: 2x the expected groups (load <= 0.5), grown on demand.
    uint64_t cap;
    if (cap_override) cap = cap_override;
    else if (d->groups_hint) cap = 1ull << ceil_log2_u64(std::max<uint64_t>(2 * d->groups_hint + 16, 64));
    else cap = 1ull << ceil_log2_u64(std::max<uint64_t>(std::min<uint64_t>(2 * n + 16, 1ull << 16), 64));
    pl->cap = cap;
    p.log2cap = f.log2cap = ceil_log2_u64(cap);
    p.max_probe = (uint32_t)std::min<uint64_t>(cap, 1u << 14);
    p.grow_limit = cap - cap / 4;
    p.row_begin = row_begin;
    p.n_rows = n;
    p.fx_e = 126 - 32 - ceil_log2_u64(n + 1);
    f.fx_e = p.fx_e;
    p.warp_agg = 0;

    // Shared-memory tier: the largest power of two of slots that fits the
    // opt-in limit, no larger than 2x the expected groups.
    const size_t entry = 8ull * (size_t)word;
    const size_t budget = (size_t)std::max(ctx->max_smem_optin - 2048, 0);
    int sl = 0;
    if (!(flags & BOLT_FLAG_FORCE_GLOBAL)) {
        while (((size_t)2 << sl) * entry <= budget && sl < 16) ++sl;
        const uint64_t want = 1ull << ceil_log2_u64(std::max<uint64_t>(2 * (d->groups_hint ? d->groups_hint : cap), 256));
        while (sl > 8 && (1ull << sl) > want) --sl;
        if (((size_t)1 << sl) * entry > budget) sl = 0;
    }
    p.smem_log2 = sl;
    pl->smem_entries = sl ? (1 << sl) : 0;
    pl->u = n_st <= 4 ? 4 : 2;
    pl->block = 512;
    pl->small_final = cap <= SMALL_FINAL_MAX;
    p.status = ctx->d_status;
    f.status = ctx->d_status;
    return BOLT_OK;
}

uint64_t gb_plan_scratch(const GbPlan& pl) {
    const uint64_t table = (pl.cap + 2) * (uint64_t)pl.prm.slot_words * 8 + 256;
    if (pl.small_final) return table + 1024;
    const uint64_t g = pl.cap + 1;
    return table + g * 8 + g * 4 + g * 4 + radix_sort_scratch(g, SRC_U64_KEYS) + 4096;
}

bolt_status gb_enqueue(bolt_ctx* ctx, GbPlan* pl, cudaStream_t s) {
    GbParams& p = pl->prm;
    GbFinal& f = pl->fin;
    const uint64_t table_bytes = (pl->cap + 2) * (uint64_t)p.slot_words * 8;
    p.gtab = (ull*)arena_alloc(ctx, table_bytes);
    ull* words = (ull*)arena_alloc(ctx, 256);
    if (!p.gtab || !words)
        return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for a %llu-slot table",
                    (ull)pl->cap);
    p.occupancy = words;
    f.gtab = p.gtab;
    f.n_nonnull = words + 1;
    f.n_groups = words + 2;
    BOLT_CUDA(ctx, cudaMemsetAsync(p.gtab, 0, table_bytes, s));
    BOLT_CUDA(ctx, cudaMemsetAsync(words, 0, 256, s));

    const size_t smem = (size_t)pl->smem_entries * 8ull * (size_t)p.slot_words;
    // Grid: resident CTAs on every SM, no more than the tiles.
    const uint64_t tile = (uint64_t)pl->block * pl->u;
    const uint64_t tiles = (p.n_rows + tile - 1) / tile;
    int per_sm = 1;
    {
        cudaError_t e;
        if (pl->u == 4) {
            BOLT_CUDA(ctx, cudaFuncSetAttribute(gb_agg_kernel<4, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb_agg_kernel<4, 4>, pl->block, smem);
        } else {
            BOLT_CUDA(ctx, cudaFuncSetAttribute(gb_agg_kernel<2, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, gb_agg_kernel<2, 8>, pl->block, smem);
        }
        if (e != cudaSuccess || per_sm < 1) per_sm = 1;
    }
    uint64_t grid = std::min<uint64_t>((uint64_t)per_sm * ctx->num_sms, std::max<uint64_t>(tiles, 1));
    if (pl->grid > 0) grid = std::min<uint64_t>(grid, (uint64_t)pl->grid);
    pl->grid = (int)grid;
    if (p.n_rows > 0) {
        kernel_mark_begin(ctx, pl->flags, s);
        bolt_status st = pl->u == 4 ? launch_agg<4, 4>(ctx, *pl, s, smem) : launch_agg<2, 8>(ctx, *pl, s, smem);
        kernel_mark_end(ctx, pl->flags, s);
        if (st != BOLT_OK) return st;
    }

    if (pl->small_final) {
        const size_t fsm = (size_t)pl->cap * 2 * 12;
        BOLT_CUDA(ctx, cudaFuncSetAttribute(gb_small_final_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fsm));
        gb_small_final_kernel<<<1, 1024, fsm, s>>>(f);
        ctx->last_launches++;
    } else {
        const uint64_t g = pl->cap + 1;
        f.order_keys = (ull*)arena_alloc(ctx, g * 8);
        f.slots = (uint32_t*)arena_alloc(ctx, g * 4);
        f.sorted = (uint32_t*)arena_alloc(ctx, g * 4);
        if (!f.order_keys || !f.slots || !f.sorted)
            return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the finalize");
        gb_compact_kernel<<<grid_for(g, 256, ctx->num_sms * 8), 256, 0, s>>>(f);
        ctx->last_launches++;
        SortSpec sp;
        sp.src = SRC_U64_KEYS;
        sp.keys = f.order_keys;
        sp.payload_in = f.slots;
        sp.n = g;
        sp.n_dev = f.n_nonnull;
        sp.payload_out = f.sorted;
        bolt_status st = radix_sort(ctx, s, sp);
        if (st != BOLT_OK) return st;
        gb_gather_kernel<<<grid_for(g, 256, ctx->num_sms * 8), 256, 0, s>>>(f);
        ctx->last_launches++;
    }
    BOLT_CUDA(ctx, cudaGetLastError());
    return BOLT_OK;
}

}  // namespace bolt

using namespace bolt;

extern "C" uint64_t bolt_groupby_footprint(const bolt_groupby_desc* desc, uint64_t n_rows) {
    if (!desc) return 0;
    // Table words per slot: key + up to two words per aggregate state.
    const uint64_t words = 1 + 2ull * (uint64_t)(desc->n_aggs > 0 ? desc->n_aggs : 1);
    const uint64_t groups = desc->groups_hint ? desc->groups_hint : std::min<uint64_t>(n_rows, 1ull << 15);
    const uint64_t cap = 1ull << ceil_log2_u64(std::max<uint64_t>(2 * groups + 16, 64));
    uint64_t bytes = (cap + 2) * words * 8 + 4096;
    if (cap > 8192) bytes += (cap + 1) * 16 + radix_sort_scratch(cap + 1, SRC_U64_KEYS);
    return bytes;
}

extern "C" bolt_status bolt_groupby(bolt_ctx* ctx, const bolt_groupby_desc* desc, bolt_groupby_out* out,
                                    uint32_t flags, bolt_stream stream) {
    if (!ctx || !desc || !out) return BOLT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t nrows = 0;
    if (desc->n_keys >= 1 && desc->key_cols && desc->cols && desc->key_cols[0] >= 0 && desc->key_cols[0] < desc->n_cols)
        nrows = desc->cols[desc->key_cols[0]].len;
    int mode = 0;
    uint64_t cap_override = 0;
    for (int attempt = 0; attempt < 6; ++attempt) {
        bolt_status st = call_begin(ctx, flags, s);
        if (st != BOLT_OK) return st;
        GbPlan pl;
        st = gb_plan(ctx, desc, out, 0, nrows, flags, mode, cap_override, &pl);
        if (st != BOLT_OK) return st;
        pl.fin.n_groups_user = (flags & BOLT_FLAG_ASYNC) ? (ull*)out->n_groups_dev : nullptr;
        st = gb_enqueue(ctx, &pl, s);
        if (st != BOLT_OK) return st;
        st = call_end(ctx, flags, s);
        if (st != BOLT_OK) return st;
        if (flags & BOLT_FLAG_ASYNC) return BOLT_OK;
        uint32_t f = 0;
        st = read_status(ctx, s, 0, &f);
        if (st != BOLT_OK) return st;
        ull ng = 0;
        BOLT_CUDA(ctx, cudaMemcpy(&ng, pl.fin.n_groups, 8, cudaMemcpyDeviceToHost));
        out->n_groups = ng;
        if (f & (ST_FLAG_GROW | ST_FLAG_SPILL)) {
            if (flags & BOLT_FLAG_FORCE_SHMEM) return fail(ctx, BOLT_ERR_SPILL, "partition_reduce spill: shared-memory tier overflow");
            cap_override = pl.cap * 8;
            continue;
        }
        if (f & (ST_FLAG_RANGE | ST_FLAG_DECRANGE)) {
            if (f & ST_FLAG_RANGE) mode |= GB_MODE_F64_ATOMIC;
            if (f & ST_FLAG_DECRANGE) mode |= GB_MODE_WIDE_DEC;
            continue;
        }
        if (f & ST_FLAG_DECOVERFLOW)
            return fail(ctx, BOLT_ERR_OVERFLOW, "SUM(Decimal128) precision overflow: accumulator exceeds i128 range");
        return flags_to_status(ctx, f, "GROUP BY");
    }
    return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: table growth did not converge");
}
