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
#include "gb_device.cuh"
#include "groupby_part.cuh"
#include "join.cuh"
#include "radix_sort.cuh"
#include "bulk.cuh"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace bolt {
namespace {

// Folds one row (already loaded and filtered: row_in) into the shared or
// global table. Every lane of the warp calls it together (the warp-level
// pre-aggregation is collective); lanes without a row pass row_in = false.
template <int MAXS, class SP>
__device__ __forceinline__ void row_fold(const GbParams& p, ull* sk, ull* sw, int C, uint32_t* fill, bool row_in,
                                         bool knull, ull stored, const ull (&raw)[MAXS], uint32_t vbits,
                                         uint32_t dfit, uint64_t r, uint32_t& inserts, uint32_t& absbits) {
    const int SW = p.sslot_words - 1;
    const uint32_t lane = lane_id();
    const int NS = snum<SP>(p);
    bool row = row_in;
    ull c0[MAXS], c1[MAXS];
#pragma unroll
    for (int s = 0; s < MAXS; ++s) {
        c0[s] = 0;
        c1[s] = 0;
        if (row && s < NS)
            contribution(p, p.st[s], skind<SP>(p, s), raw[s], (vbits >> s) & 1, (dfit >> s) & 1,
                         r, c0[s], c1[s]);
    }
    // Bit length of the largest |v| fed to an int64 SUM: decides whether
    // a row-order prefix of some group could leave the i64 range (then
    // the exact row-order check runs after the query).
    if (row && p.i64_bits) {
#pragma unroll
        for (int s = 0; s < MAXS; ++s) {
            if (s < NS && skind<SP>(p, s) == K_SUM_I64 && ((vbits >> s) & 1)) {
                const ll v = (ll)raw[s];
                const ull a = v < 0 ? (ull)(-(v + 1)) + 1ull : (ull)v;
                const uint32_t b = a ? 64u - (uint32_t)__clzll((ll)a) : 0u;
                absbits = b > absbits ? b : absbits;
            }
        }
    }
    // Special groups: the NULL key and the key whose complement is 0.
    const bool special = row && (knull || stored == 0);
    if (special) {
        const ull slot = (1ull << p.log2cap) + (knull ? 1 : 0);
        ull* w = p.gtab + slot * (ull)p.slot_words;
        if (ld_volatile(w) == 0) *reinterpret_cast<volatile ull*>(w) = 1ull;
#pragma unroll
        for (int s = 0; s < MAXS; ++s)
            if (s < NS) merge_words(w + p.st[s].word, skind<SP>(p, s), c0[s], c1[s]);
        row = false;
    }
    // Warp-level pre-aggregation of duplicate keys.
    if (p.warp_agg) {
        const uint32_t act = __ballot_sync(0xffffffffu, row);
        uint32_t peers = 0;
        if (row) peers = __match_any_sync(act, stored);
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
                if (s < NS) {
                    const ull b0 = __shfl_sync(0xffffffffu, c0[s], src);
                    const ull b1 = __shfl_sync(0xffffffffu, c1[s], src);
                    if (leader && src != (int)lane) combine(skind<SP>(p, s), c0[s], c1[s], b0, b1);
                }
            }
        }
        row = leader;
    }
    if (!row) return;
    int sl = -1;
    if (C) sl = s_find_insert(sk, p.smem_log2, stored, fill, p.smem_fill);
    if (sl >= 0) {
        ull* w = sw + (ull)sl * SW - 1;  // state word offsets count the key word
#pragma unroll
        for (int s = 0; s < MAXS; ++s)
            if (s < NS) merge_words_smem(w + p.st[s].sword, skind<SP>(p, s), c0[s], c1[s], p.cnt32);
    } else {
        const int64_t g = g_find_insert(p, stored, inserts);
        if (g >= 0) {
            ull* w = p.gtab + (ull)g * p.slot_words;
#pragma unroll
            for (int s = 0; s < MAXS; ++s)
                if (s < NS) merge_words(w + p.st[s].word, skind<SP>(p, s), c0[s], c1[s]);
        }
    }
}

// One tile of blockDim.x * U rows starting at row `base` of the query:
// load, filter, key, pre-aggregate and fold into the shared or global table.
// `sk` / `sw` are the shared table's keys and state words (C slots, C may be 0).
template <int U, int MAXS, class SP>
__device__ __forceinline__ void gb_process_tile(const GbParams& p, ull* sk, ull* sw, int C, uint32_t* fill,
                                                uint64_t base, uint32_t& inserts, uint32_t& absbits) {
    const uint64_t n = p.n_rows;
    const int NS = snum<SP>(p);
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
        if (p.jslots) {
            if (bit_valid(p.jkvalid, r))
                stored[u] = p.jkdt == BOLT_I32 ? (ull)(ll)ld_stream((const int32_t*)p.jkey + r)
                                               : (ull)ld_stream((const ll*)p.jkey + r);
            else
                has[u] = false;
        } else {
            stored[u] = ~pack_key(p, r);
        }
#pragma unroll
        for (int s = 0; s < MAXS; ++s) {
            if (s < NS && p.st[s].col) {
                bool fits = true;
                raw[u][s] = load_raw(p.st[s], r, fits);
                if (bit_valid(p.st[s].valid, r)) vbits[u] |= 1u << s;
                if (fits) dfit[u] |= 1u << s;
            } else if (s < NS) {
                vbits[u] |= 1u << s;  // COUNT(*)
                dfit[u] |= 1u << s;
            }
        }
        for (int q = 0; q < p.n_pred; ++q) has[u] = has[u] && eval_pred(p.pred[q], r);
        if (!p.jslots)
            for (int k = 0; k < p.n_keys; ++k) knull[u] = knull[u] || !bit_valid(p.kvalid[k], r);
        if (knull[u] && p.n_keys > 1) has[u] = false;  // multi-key: NULL-key rows are dropped
    }
    if (p.jslots) {
        // Join source: stored[u] holds the probe key; its group key is the
        // matched build row's payload. All U lookups are issued together.
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (!has[u]) continue;
            const ull w1 = join_lookup(p.jslots, p.jlog2cap, stored[u]);
            if (w1 == ~0ull) has[u] = false;
            stored[u] = ~(ull)(ll)(int32_t)(uint32_t)w1;
        }
    }
    // Rows are folded one at a time in a rolled loop (one copy of the code,
    // which keeps the kernel inside the instruction cache): row u sits in
    // slot 0 and the later rows move down one slot after each iteration.
#pragma unroll 1
    for (int u = 0; u < U; ++u) {
        row_fold<MAXS, SP>(p, sk, sw, C, fill, has[0], knull[0], stored[0], raw[0], vbits[0], dfit[0],
                           p.row_begin + base + (uint64_t)u * blockDim.x + threadIdx.x, inserts, absbits);
#pragma unroll
        for (int v = 0; v + 1 < U; ++v) {
            has[v] = has[v + 1];
            knull[v] = knull[v + 1];
            stored[v] = stored[v + 1];
            vbits[v] = vbits[v + 1];
            dfit[v] = dfit[v + 1];
#pragma unroll
            for (int s = 0; s < MAXS; ++s) raw[v][s] = raw[v + 1][s];
        }
    }
}

template <int U, int MAXS, class SP>
__global__ void __launch_bounds__(512, SP::generic ? 1 : 2) gb_agg_kernel(const __grid_constant__ GbParams p) {
    extern __shared__ __align__(16) ull smem[];
    __shared__ uint32_t s_fill;
    const int SW = p.sslot_words - 1;
    const int C = p.smem_log2 ? (1 << p.smem_log2) : 0;
    ull* sk = smem;
    ull* sw = smem + C;
    for (int i = threadIdx.x; i < C * (SW + 1); i += blockDim.x) smem[i] = 0;
    if (threadIdx.x == 0) s_fill = 0;
    __syncthreads();
    const uint64_t tile = (uint64_t)blockDim.x * U;
    uint32_t inserts = 0, pending = 0, absbits = 0;
    for (uint64_t base = (uint64_t)blockIdx.x * tile; base < p.n_rows; base += (uint64_t)gridDim.x * tile) {
        gb_process_tile<U, MAXS, SP>(p, sk, sw, C, &s_fill, base, inserts, absbits);
        if (gb_warp_epilogue(p, inserts, pending)) break;
    }
    gb_warp_flush_pending(p, pending);
    gb_flush_absbits(p, absbits);
    __syncthreads();
    gb_flush_shared(p, sk, sw, C);
}

// ---------------------------------------------------------------------------
// Staged aggregation kernel.
//
// Warp 0 of the CTA is the producer: its lane 0 streams tiles of tile_rows
// rows of every input column into a ring of n_stages shared-memory stages
// with bulk copies (cp.async.bulk) that complete on the stage's `full`
// mbarrier. The other warps are consumers: each takes its `chunks` x 32
// contiguous rows of the tile, evaluates the WHERE conjuncts, compacts the
// surviving row numbers into a per-warp list, and folds the survivors 32 to
// a warp step, so filtered-out rows cost no aggregation work. A consumer
// releases the stage on its `empty` mbarrier (count: consumer warps).
//
// Only whole tiles are staged; the last n_rows % tile_rows rows are folded
// from global memory after the ring drains. All waits are bounded.
// ---------------------------------------------------------------------------
// Filters, compacts and folds the rows [first, first + 32 * nchunks) of one
// tile (tile-relative numbers, below `limit`) for the calling warp. `list` is
// the warp's compaction buffer of 32 * nchunks entries.
template <class SP, bool STAGED>
__device__ __forceinline__ void staged_rows(const GbParams& p, ull* sk, ull* sw, int C, uint32_t* fill,
                                            const unsigned char* stage, uint64_t tile_row0, uint32_t first,
                                            int nchunks, uint32_t limit, uint16_t* list, uint32_t& inserts,
                                            uint32_t& absbits) {
    constexpr int MAXS = SP::n;
    const uint32_t lane = lane_id();
    uint32_t cnt = 0;
    for (int c = 0; c < nchunks; ++c) {
        const uint32_t i = first + (uint32_t)c * 32u + lane;
        const uint64_t r = p.row_begin + tile_row0 + i;
        bool ok = i < limit;
        if (ok) {
            for (int q = 0; q < p.n_pred; ++q)
                ok = ok && bit_valid(p.pred[q].valid, r) &&
                     pred_at(p, q, sc_base<STAGED>(p, p.pr_sc[q], stage, tile_row0), i);
            if (p.n_keys > 1)
                for (int k = 0; k < p.n_keys; ++k) ok = ok && bit_valid(p.kvalid[k], r);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        if (ok) list[cnt + __popc(m & lanemask_lt())] = (uint16_t)(i - first);
        cnt += __popc(m);
    }
    __syncwarp();
    const unsigned char* kb0 = sc_base<STAGED>(p, p.k_sc[0], stage, tile_row0);
    const unsigned char* kb1 = p.n_keys > 1 ? sc_base<STAGED>(p, p.k_sc[1], stage, tile_row0) : kb0;
    for (uint32_t b = 0; b < cnt; b += 32) {
        const bool has = b + lane < cnt;
        const uint32_t i = first + (has ? (uint32_t)list[b + lane] : 0u);
        const uint64_t r = p.row_begin + tile_row0 + i;
        ull raw[MAXS];
        uint32_t vbits = 0, dfit = 0;
        bool knull = false;
        ull stored = 0;
        if (has) {
            stored = ~key_at(p, kb0, kb1, i);
            if (p.n_keys == 1) knull = !bit_valid(p.kvalid[0], r);
        }
#pragma unroll
        for (int s = 0; s < MAXS; ++s) {
            raw[s] = 0;
            if (!has) continue;
            if (p.st_sc[s] >= 0) {
                bool fits = true;
                raw[s] = raw_at(p.st[s].dtype, sc_base<STAGED>(p, p.st_sc[s], stage, tile_row0), i, fits);
                if (bit_valid(p.st[s].valid, r)) vbits |= 1u << s;
                if (fits) dfit |= 1u << s;
            } else {
                vbits |= 1u << s;  // COUNT(*)
                dfit |= 1u << s;
            }
        }
        row_fold<MAXS, SP>(p, sk, sw, C, fill, has, knull, stored, raw, vbits, dfit, r, inserts, absbits);
    }
    __syncwarp();
}

template <class SP>
__global__ void __launch_bounds__(1024, 1) gb_staged_kernel(const __grid_constant__ GbParams p) {
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ __align__(8) uint64_t full[4], empty[4];
    __shared__ uint32_t s_fill;
    const int S = p.n_stages;
    const int NW = (int)(blockDim.x >> 5) - 1;  // consumer warps
    const int warp = (int)(threadIdx.x >> 5);
    const uint32_t lane = lane_id();
    const int SW = p.sslot_words - 1;
    const int C = p.smem_log2 ? (1 << p.smem_log2) : 0;
    unsigned char* stages = dsm;
    ull* sk = reinterpret_cast<ull*>(dsm + (size_t)S * p.stage_bytes);
    ull* sw = sk + C;
    uint16_t* lists = reinterpret_cast<uint16_t*>(sw + (size_t)C * SW);
    const uint32_t T = p.tile_rows;
    const uint64_t ntiles = p.n_rows / T;

    for (int i = threadIdx.x; i < C * (SW + 1); i += blockDim.x) sk[i] = 0;
    if (threadIdx.x == 0) {
        s_fill = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], (uint32_t)NW);
        }
        mbar_init_fence();
    }
    __syncthreads();

    uint32_t inserts = 0, pending = 0, absbits = 0;
    if (warp == 0) {
        if (lane == 0) {
            const uint64_t pol = l2_evict_first_policy();
            uint32_t j = 0;
            bool ok = true;
            for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++j) {
                const int st = (int)(j % (uint32_t)S);
                const uint32_t use = j / (uint32_t)S;
                if (use > 0 && !mbar_wait(&empty[st], (use - 1) & 1u)) {
                    ok = false;
                    break;
                }
                const bool stop = (*reinterpret_cast<volatile uint32_t*>(p.status) &
                                   (ST_FLAG_GROW | ST_FLAG_SPILL | ST_FLAG_TIMEOUT)) != 0;
                if (stop) {
                    mbar_arrive(&full[st]);  // completes the phase with no data
                } else {
                    mbar_arrive_expect_tx(&full[st], p.stage_bytes);
                    unsigned char* dst = stages + (size_t)st * p.stage_bytes;
                    for (int c = 0; c < p.n_sc; ++c) {
                        const uint32_t w = (uint32_t)p.sc_w[c];
                        const unsigned char* src =
                            static_cast<const unsigned char*>(p.sc_col[c]) + (p.row_begin + t * T) * (uint64_t)w;
                        bulk_load(dst + p.sc_off[c], src, T * w, &full[st], pol);
                    }
                }
            }
            // The copies of the last (up to S) tiles may still be landing if a
            // consumer gave up early: wait for them before the CTA can exit.
            const uint32_t issued = j;
            for (uint32_t k = issued > (uint32_t)S ? issued - (uint32_t)S : 0u; k < issued; ++k)
                if (!mbar_wait(&full[k % (uint32_t)S], (k / (uint32_t)S) & 1u)) ok = false;
            if (!ok) atomicOr(p.status, ST_FLAG_TIMEOUT);
        }
        __syncwarp();
    } else {
        const int cw = warp - 1;
        uint16_t* list = lists + (size_t)cw * 32 * p.chunks;
        uint32_t j = 0;
        for (uint64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++j) {
            const int st = (int)(j % (uint32_t)S);
            const bool ready = mbar_wait(&full[st], (j / (uint32_t)S) & 1u);
            if (!__all_sync(0xffffffffu, ready)) {
                if (lane == 0) atomicOr(p.status, ST_FLAG_TIMEOUT);
                break;
            }
            uint32_t stop = 0;
            if (lane == 0)
                stop = (*reinterpret_cast<volatile uint32_t*>(p.status) &
                        (ST_FLAG_GROW | ST_FLAG_SPILL | ST_FLAG_TIMEOUT)) != 0;
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (!stop)
                staged_rows<SP, true>(p, sk, sw, C, &s_fill, stages + (size_t)st * p.stage_bytes, t * T,
                                      (uint32_t)cw * 32u * (uint32_t)p.chunks, p.chunks, T, list, inserts, absbits);
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
            gb_warp_epilogue(p, inserts, pending);
        }
        // Rows after the last whole tile, 32 per consumer warp, from global memory.
        const uint64_t rem0 = ntiles * T;
        const uint32_t rem = (uint32_t)(p.n_rows - rem0);
        for (uint32_t c = (uint32_t)(blockIdx.x * NW + cw) * 32u; c < rem; c += gridDim.x * (uint32_t)NW * 32u)
            staged_rows<SP, false>(p, sk, sw, C, &s_fill, nullptr, rem0, c, 1, rem, list, inserts, absbits);
    }
    gb_warp_flush_pending(p, pending);
    gb_flush_absbits(p, absbits);
    __syncthreads();
    gb_flush_shared(p, sk, sw, C);
}

// ---------------------------------------------------------------------------
// Finalize
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sum_as_double(const GbFinal& f, const StateDesc& s, const ull* w) {
    switch (s.kind) {
    case K_SUM_I32: return (double)(ll)w[0];
    case K_SUM_I64:
    case K_SUM_D64: {
        __int128 v = ((__int128)(ll)w[1] << 32) + (__int128)w[0];
        return i128_to_double_scaled((ull)v, (ll)(v >> 64), 0);
    }
    case K_SUM_FX: {  // global layout: w0 + w1 * 2^32 + w2 * 2^64, mod 2^128
        const unsigned __int128 v =
            (unsigned __int128)w[0] + ((unsigned __int128)w[1] << 32) + ((unsigned __int128)w[2] << 64);
        return i128_to_double_scaled((ull)v, (ll)(ull)(v >> 64), f.fx_e);
    }
    default: return __longlong_as_double((ll)w[0]);
    }
}

// Writes output row o from slot `slot` (slot == cap + 1 is the NULL group)
// and returns its validity bits: bit k for key column k, bit n_keys + a for
// aggregate column a (write_valid_words stores them).
__device__ __forceinline__ uint32_t emit_group(const GbFinal& f, uint64_t o, uint64_t slot) {
    uint32_t vbits = 0;
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
        if (!null_key) vbits |= 1u << k;
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
        if (valid) vbits |= 1u << (f.n_keys + a);
    }
    return vbits;
}

// Validity bitmaps of output rows [o0, o0 + 32) from one warp (o0 a multiple
// of 32, lanes past the rows pass row = false): one ballot per column and
// byte stores by lane 0, so no two warps share a byte and no atomics are
// needed; bytes past the last output row are not written.
__device__ __forceinline__ void write_valid_words(const GbFinal& f, uint64_t o0, uint64_t lim, uint32_t vbits,
                                                  bool row) {
    const uint64_t nbytes = (lim + 7) / 8;
    const int nc = f.n_keys + f.n_aggs;
    for (int c = 0; c < nc; ++c) {
        uint8_t* bm = c < f.n_keys ? f.out_key_valid[c] : f.agg[c - f.n_keys].out_valid;
        const uint32_t m = __ballot_sync(0xffffffffu, row && ((vbits >> c) & 1u));
        if (bm && lane_id() == 0) {
#pragma unroll
            for (int b = 0; b < 4; ++b)
                if (o0 / 8 + b < nbytes) bm[o0 / 8 + b] = (uint8_t)(m >> (8 * b));
        }
    }
}

// Copies query q's finalize descriptor into shared memory (whole CTA).
__device__ __forceinline__ void load_final(GbFinal& dst, const GbFinal* src) {
    const int4* s = reinterpret_cast<const int4*>(src);
    int4* d = reinterpret_cast<int4*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(GbFinal) / 16); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

// Index of the query owning flattened work item `item`.
__device__ __forceinline__ int query_of(const uint32_t* begins, int nq, uint32_t item) {
    int lo = 0, hi = nq;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(begins + mid) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

constexpr int FIN_CHUNK = 4096;
// Output rows per gather work item (a multiple of 32: each warp owns whole
// validity words); smaller than FIN_CHUNK so the rows spread over every CTA.
constexpr int GATHER_CHUNK = 1024;

// Occupied-slot compaction of the large-table queries: work items are
// (query, chunk of 4096 slots); order key = packed key ^ sign bit.
__global__ void __launch_bounds__(256) gb_compact_batch_kernel(const GbFinal* fins, const uint32_t* begins, int nq,
                                                                uint32_t total_items) {
    // Each warp takes runs of 32 x CMP_ROUNDS slots: it reads their keys,
    // counts the occupied ones with ballots, claims that many output rows
    // with one atomic, then writes them (one atomic per 512 slots instead of
    // per 32 keeps the shared counter out of the way).
    constexpr int CMP_ROUNDS = 16;
    __shared__ __align__(16) GbFinal f;
    const uint32_t lane = lane_id();
    const int warp = (int)(threadIdx.x >> 5), nwarps = (int)(blockDim.x >> 5);
    for (uint32_t item = blockIdx.x; item < total_items; item += gridDim.x) {
        const int q = query_of(begins, nq, item);
        __syncthreads();
        load_final(f, fins + q);
        const ull cap = 1ull << f.log2cap;
        const uint64_t c0 = (uint64_t)(item - begins[q]) * FIN_CHUNK;
        const uint64_t c1 = c0 + FIN_CHUNK < cap + 1 ? c0 + FIN_CHUNK : cap + 1;
        for (uint64_t run = c0 + (uint64_t)warp * 32 * CMP_ROUNDS; run < c1;
             run += (uint64_t)nwarps * 32 * CMP_ROUNDS) {
            ull ok[CMP_ROUNDS];
            uint32_t occ = 0, total = 0;
#pragma unroll
            for (int j = 0; j < CMP_ROUNDS; ++j) {
                const uint64_t i = run + (uint64_t)j * 32 + lane;
                bool o = false;
                ok[j] = 0;
                if (i < c1) {
                    if (i < cap) {
                        const ull k = ld_volatile(f.gtab + i * (ull)f.slot_words);
                        o = k != 0;
                        ok[j] = ~k ^ 0x8000000000000000ull;
                    } else {  // i == cap: the key whose complement is 0
                        o = f.gtab[cap * (ull)f.slot_words] != 0;
                        ok[j] = ~0ull ^ 0x8000000000000000ull;
                    }
                }
                total += __popc(__ballot_sync(0xffffffffu, o));
                if (o) occ |= 1u << j;
            }
            if (!total) continue;
            ull pos = 0;
            if (lane == 0) pos = atomicAdd(f.n_nonnull, (ull)total);
            pos = __shfl_sync(0xffffffffu, pos, 0);
#pragma unroll
            for (int j = 0; j < CMP_ROUNDS; ++j) {
                const bool o = (occ >> j) & 1u;
                const uint32_t m = __ballot_sync(0xffffffffu, o);
                if (o) {
                    const ull at = pos + __popc(m & lanemask_lt());
                    f.order_keys[at] = ok[j];
                    f.slots[at] = (uint32_t)(run + (uint64_t)j * 32 + lane);
                }
                pos += __popc(m);
            }
        }
    }
}

// Output rows of the large-table queries: work items are (query, chunk of
// GATHER_CHUNK output rows) up to cap + 1 rows; rows past the group count exit.
__global__ void __launch_bounds__(256) gb_gather_batch_kernel(const GbFinal* fins, const uint32_t* begins, int nq,
                                                               uint32_t total_items) {
    __shared__ __align__(16) GbFinal f;
    for (uint32_t item = blockIdx.x; item < total_items; item += gridDim.x) {
        const int q = query_of(begins, nq, item);
        __syncthreads();
        load_final(f, fins + q);
        const ull cap = 1ull << f.log2cap;
        const ull G = min(*f.n_nonnull, f.n_max);  // (a counter that ran past the table flagged GROW)
        const bool has_null = f.gtab[(cap + 1) * (ull)f.slot_words] != 0;
        const ull total = G + (has_null ? 1 : 0);
        const uint64_t c0 = (uint64_t)(item - begins[q]) * GATHER_CHUNK;
        if (c0 == 0 && threadIdx.x == 0) {
            *f.n_groups = total;
            if (f.n_groups_user) *f.n_groups_user = total;
            if (total > f.out_cap) atomicOr(f.status, ST_FLAG_CAPACITY);
        }
        const ull lim = total < f.out_cap ? total : f.out_cap;
        const uint64_t c1 = c0 + GATHER_CHUNK < lim ? c0 + GATHER_CHUNK : lim;
        // Warp-uniform rows of 32 (c0 and blockDim are multiples of 32).
        for (uint64_t o0 = c0 + (threadIdx.x & ~31u); o0 < c1; o0 += blockDim.x) {
            const uint64_t o = o0 + lane_id();
            bool row = o < c1;
            uint32_t vb = 0;
            if (row) {
                const uint64_t slot = o < G ? f.sorted[o] : cap + 1;
                if (slot > cap + 1) {  // (a sort entry nobody wrote: never read past the table)
                    atomicOr(f.status, ST_FLAG_INTERNAL);
                    row = false;
                } else {
                    vb = emit_group(f, o, slot);
                }
            }
            write_valid_words(f, o0, lim, vb, row);
        }
    }
}

// One CTA per small-table query (<= 8192 slots): compacts the occupied
// slots, sorts their (order key, slot) pairs by key in shared memory and
// emits the groups. The sort is a stable LSD radix sort over only the key
// bytes that differ between the groups (two passes for keys below 2^16),
// ranked per warp like the global radix sort.
constexpr int SF_BLOCK = 512;
constexpr int SF_NW = SF_BLOCK / 32;

// Dynamic shared memory of gb_small_final_kernel for tables of `cap` slots:
// two (key, slot) buffers of cap + 1 entries.
inline size_t small_final_smem(uint64_t cap) { return (size_t)(cap + 1) * 2 * 12; }

__device__ __forceinline__ void small_final_body(const GbFinal& f) {
    extern __shared__ __align__(16) ull sm[];
    __shared__ uint32_t s_n;
    __shared__ ull s_vary;
    __shared__ uint32_t warp_pos[SF_NW][256];
    __shared__ uint32_t wsum[8];
    const ull cap = 1ull << f.log2cap;
    const uint32_t M = (uint32_t)cap + 1;
    ull* const key0 = sm;
    ull* const key1 = sm + M;
    uint32_t* const slot0 = reinterpret_cast<uint32_t*>(sm + 2 * (size_t)M);
    uint32_t* const slot1 = slot0 + M;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        s_n = 0;
        s_vary = 0;
    }
    __syncthreads();
    // Occupied slots, 8 loads in flight per thread, one counter update per
    // warp and load round.
    constexpr int SF_U = 8;
    for (uint32_t w0 = (threadIdx.x & ~31u) * SF_U; w0 <= cap; w0 += blockDim.x * SF_U) {  // (warp-uniform)
        const uint32_t i0 = w0 + lane;
        ull kk[SF_U];
#pragma unroll
        for (int u = 0; u < SF_U; ++u) {
            const uint32_t i = i0 + 32u * u;
            kk[u] = i <= cap ? f.gtab[(ull)i * f.slot_words] : 0ull;
        }
#pragma unroll
        for (int u = 0; u < SF_U; ++u) {
            const uint32_t i = i0 + 32u * u;
            const uint32_t m = __ballot_sync(0xffffffffu, kk[u] != 0);
            if (m == 0) continue;
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&s_n, (uint32_t)__popc(m));
            base = __shfl_sync(0xffffffffu, base, 0);
            if (kk[u] != 0) {
                const uint32_t pos = base + __popc(m & lanemask_lt());
                key0[pos] = (i == cap ? ~0ull : ~kk[u]) ^ 0x8000000000000000ull;
                slot0[pos] = i;
            }
        }
    }
    __syncthreads();
    const uint32_t G = s_n;
    // Bits in which some group's key differs from the first one's.
    if (G > 1) {
        const ull k0 = key0[0];
        ull v = 0;
        for (uint32_t i = threadIdx.x; i < G; i += blockDim.x) v |= key0[i] ^ k0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicOr(&s_vary, v);
    }
    __syncthreads();
    const ull vary = s_vary;
    // Each warp ranks a contiguous run of the entries, so the passes keep
    // the order of equal digits.
    const uint32_t per = (((G + SF_NW - 1) / SF_NW) + 31) & ~31u;
    const uint32_t lo = min((uint32_t)w * per, G), hi = min(lo + per, G);
    int cur = 0;
    for (int byte = 0; byte < 8; ++byte) {
        if (((vary >> (8 * byte)) & 0xFFull) == 0) continue;  // (uniform over the CTA)
        const int sh = 8 * byte;
        const ull* ka = cur ? key1 : key0;
        const uint32_t* sa = cur ? slot1 : slot0;
        ull* kb = cur ? key0 : key1;
        uint32_t* sb = cur ? slot0 : slot1;
        for (int i = threadIdx.x; i < SF_NW * 256; i += blockDim.x) (&warp_pos[0][0])[i] = 0;
        __syncthreads();
        for (uint32_t i = lo + lane; i < hi; i += 32) atomicAdd(&warp_pos[w][(uint32_t)(ka[i] >> sh) & 0xFFu], 1u);
        __syncthreads();
        // Digit-major, then warp order: each warp's first position per digit.
        uint32_t cnt[SF_NW];
        uint32_t run = 0, x = 0;
        if (threadIdx.x < 256) {
#pragma unroll
            for (int ww = 0; ww < SF_NW; ++ww) {
                cnt[ww] = warp_pos[ww][threadIdx.x];
                run += cnt[ww];
            }
            x = run;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) wsum[w] = x;
        }
        __syncthreads();
        if (threadIdx.x < 256) {
            uint32_t off = x - run;
            for (int i = 0; i < w; ++i) off += wsum[i];
#pragma unroll
            for (int ww = 0; ww < SF_NW; ++ww) {
                warp_pos[ww][threadIdx.x] = off;
                off += cnt[ww];
            }
        }
        __syncthreads();
        for (uint32_t b0 = lo; b0 < hi; b0 += 32) {  // (warp-uniform)
            const uint32_t i = b0 + lane;
            const bool valid = i < hi;
            const ull k = valid ? ka[i] : 0ull;
            const uint32_t dg = (uint32_t)(k >> sh) & 0xFFu;
            uint32_t peers = __ballot_sync(0xffffffffu, valid);
#pragma unroll
            for (int bit = 0; bit < 8; ++bit) {
                const uint32_t on = (dg >> bit) & 1u;
                const uint32_t bal = __ballot_sync(0xffffffffu, on);
                peers &= on ? bal : ~bal;
            }
            if (!valid) peers = 1u << lane;
            const int leader = 31 - __clz(peers);
            uint32_t bpos = 0;
            if (valid && lane == leader) {
                bpos = warp_pos[w][dg];
                warp_pos[w][dg] = bpos + __popc(peers);
            }
            bpos = __shfl_sync(0xffffffffu, bpos, leader);
            if (valid) {
                const uint32_t pos = bpos + __popc(peers & lanemask_lt());
                kb[pos] = k;
                sb[pos] = sa[i];
            }
            __syncwarp();
        }
        __syncthreads();
        cur ^= 1;
    }
    const uint32_t* sorted = cur ? slot1 : slot0;
    const bool has_null = f.gtab[(cap + 1) * (ull)f.slot_words] != 0;
    const ull total = (ull)G + (has_null ? 1 : 0);
    if (threadIdx.x == 0) {
        *f.n_groups = total;
        *f.n_nonnull = G;
        if (f.n_groups_user) *f.n_groups_user = total;
        if (total > f.out_cap) atomicOr(f.status, ST_FLAG_CAPACITY);
    }
    const ull lim = total < f.out_cap ? total : f.out_cap;
    for (uint64_t o0 = threadIdx.x & ~31u; o0 < lim; o0 += blockDim.x) {  // (warp-uniform)
        const uint64_t o = o0 + lane;
        const bool row = o < lim;
        const uint32_t vb = row ? emit_group(f, o, o < G ? sorted[o] : cap + 1) : 0u;
        write_valid_words(f, o0, lim, vb, row);
    }
}

// Several queries, one CTA each (descriptors in device memory).
__global__ void __launch_bounds__(SF_BLOCK) gb_small_final_kernel(const GbFinal* fins) {
    __shared__ __align__(16) GbFinal f;
    load_final(f, fins + blockIdx.x);
    small_final_body(f);
}

// One query, its descriptor passed by value (no upload before the launch).
__global__ void __launch_bounds__(SF_BLOCK) gb_small_final1_kernel(const __grid_constant__ GbFinal f) {
    small_final_body(f);
}

// ---------------------------------------------------------------------------
// Exact row-order check of int64 SUM (checked_group_sum, groupby.rs:1775):
// only run when some group's partial sums could leave the i64 range.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int64_t g_find(const GbParams& p, ull stored) {
    const ull mask = (1ull << p.log2cap) - 1;
    ull h = (stored * HASH_G) >> (64 - p.log2cap);
    for (uint32_t i = 0; i < p.max_probe; ++i) {
        const ull k = ld_volatile(p.gtab + h * (ull)p.slot_words);
        if (k == stored) return (int64_t)h;
        if (k == 0) return -1;
        h = (h + 1) & mask;
    }
    return -1;
}

// Row -> group slot; rows that reach no group get ~0u.
__global__ void __launch_bounds__(256) gb_row_slot_kernel(const __grid_constant__ GbParams p, uint32_t* slot_of_row) {
    const ull cap = 1ull << p.log2cap;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < p.n_rows;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = p.row_begin + i;
        bool has = true;
        for (int q = 0; q < p.n_pred; ++q) has = has && eval_pred(p.pred[q], r);
        bool knull = false;
        ull stored = 0;
        if (p.jslots) {
            if (!bit_valid(p.jkvalid, r)) has = false;
            if (has) {
                const ull k = p.jkdt == BOLT_I32 ? (ull)(ll)__ldg((const int32_t*)p.jkey + r) : (ull)__ldg((const ll*)p.jkey + r);
                const ull w1 = join_lookup(p.jslots, p.jlog2cap, k);
                if (w1 == ~0ull) has = false;
                stored = ~(ull)(ll)(int32_t)(uint32_t)w1;
            }
        } else {
            for (int k = 0; k < p.n_keys; ++k) knull = knull || !bit_valid(p.kvalid[k], r);
            if (knull && p.n_keys > 1) has = false;
            if (has && !knull) stored = ~pack_key(p, r);
        }
        uint32_t slot = 0xFFFFFFFFu;
        if (has) {
            if (knull) slot = (uint32_t)(cap + 1);
            else if (stored == 0) slot = (uint32_t)cap;
            else {
                const int64_t g = g_find(p, stored);
                if (g >= 0) slot = (uint32_t)g;
            }
        }
        slot_of_row[i] = slot;
    }
}

// One thread per run of equal slots in the stable (slot, row) order: replays
// the group's int64 SUMs in row order and flags any prefix outside i64.
__global__ void __launch_bounds__(256) gb_prefix_check_kernel(const __grid_constant__ GbParams p,
                                                               const uint32_t* slot_of_row, const uint32_t* sorted) {
    const uint64_t n = p.n_rows;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = slot_of_row[sorted[i]];
        if (s == 0xFFFFFFFFu) continue;
        if (i > 0 && slot_of_row[sorted[i - 1]] == s) continue;  // not the head of its run
        for (int st = 0; st < p.n_st; ++st) {
            const StateDesc& d = p.st[st];
            if (d.kind != K_SUM_I64) continue;
            ll acc = 0;
            for (uint64_t j = i; j < n; ++j) {
                const uint32_t row = sorted[j];
                if (slot_of_row[row] != s) break;
                const uint64_t r = p.row_begin + row;
                if (!bit_valid(d.valid, r)) continue;
                const ll v = __ldg((const ll*)d.col + r);
                const ll nx = (ll)((ull)acc + (ull)v);
                if ((v > 0 && nx < acc) || (v < 0 && nx > acc)) {
                    atomicOr(p.status, ST_FLAG_OVERFLOW);
                    break;
                }
                acc = nx;
            }
        }
    }
}

// Items one CTA of the multi-query kernel takes before it exits: CTAs of
// bounded length (about 130K rows) let the scheduler interleave other
// streams' higher-priority blocks between them.
constexpr uint32_t BATCH_CTA_ITEMS = 16;

// Persistent multi-query aggregation: work items are (query, run of
// item_tiles tiles of blockDim.x * U rows) handed out in order from one
// counter. A CTA keeps one query's shared table while its items stay on that
// query and merges it into that query's global table when it moves on. Each
// query has its own table, occupancy and status words, so one query's spill
// never touches another's. One block barrier per item (the hand-out).
template <int U, int MAXS, class SP>
__global__ void __launch_bounds__(512, SP::generic ? 1 : 2) gb_batch_agg_kernel(const GbParams* prms, const uint32_t* begins, int nq,
                                                           uint32_t total_items, uint32_t item_tiles,
                                                           uint32_t* counter) {
    extern __shared__ __align__(16) ull smem[];
    __shared__ __align__(16) GbParams p;
    __shared__ uint32_t s_item[2];  // alternating: a slot is rewritten only after everyone read it
    __shared__ uint32_t s_fill;
    int cur = -1, stopped = -1;
    int C = 0;
    uint32_t inserts = 0, pending = 0, absbits = 0;
    for (uint32_t it = 0; it < BATCH_CTA_ITEMS; ++it) {
        if (threadIdx.x == 0) s_item[it & 1] = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t item = s_item[it & 1];
        if (item >= total_items) break;
        const int q = query_of(begins, nq, item);
        if (q != cur) {
            if (cur >= 0) {
                gb_warp_flush_pending(p, pending);
                gb_flush_absbits(p, absbits);
                gb_flush_shared(p, smem, smem + C, C);
                __syncthreads();
            }
            const int4* src = reinterpret_cast<const int4*>(prms + q);
            int4* dst = reinterpret_cast<int4*>(&p);
            for (int i = threadIdx.x; i < (int)(sizeof(GbParams) / 16); i += blockDim.x) dst[i] = src[i];
            __syncthreads();
            C = p.smem_log2 ? (1 << p.smem_log2) : 0;
            for (int i = threadIdx.x; i < C * p.sslot_words; i += blockDim.x) smem[i] = 0;
            if (threadIdx.x == 0) s_fill = 0;
            __syncthreads();
            cur = q;
        }
        if (stopped == q) continue;  // the query already flagged growth; the host re-runs it
        const uint64_t tile = (uint64_t)blockDim.x * U;
        const uint64_t first = (uint64_t)(item - begins[q]) * item_tiles * tile;
        for (uint32_t t = 0; t < item_tiles; ++t) {
            const uint64_t base = first + (uint64_t)t * tile;
            if (base >= p.n_rows) break;
            gb_process_tile<U, MAXS, SP>(p, smem, smem + C, C, &s_fill, base, inserts, absbits);
            if (gb_warp_epilogue(p, inserts, pending)) {
                stopped = q;
                break;
            }
        }
    }
    if (cur >= 0) {
        gb_warp_flush_pending(p, pending);
        gb_flush_absbits(p, absbits);
        __syncthreads();
        gb_flush_shared(p, smem, smem + C, C);
    }
}

using AggKernel = void (*)(GbParams);
using BatchKernel = void (*)(const GbParams*, const uint32_t*, int, uint32_t, uint32_t, uint32_t*);

// Kernel instantiation for a compiled state layout (gb_spec_of); the generic
// loop handles up to 4 states at 4 rows per thread or 8 states at 2.
AggKernel agg_kernel_for(int spec, int n_st) {
    switch (spec) {
    case 1: return gb_agg_kernel<4, 4, Spec1>;
    case 2: return gb_agg_kernel<4, 4, Spec2>;
    case 3: return gb_agg_kernel<4, 2, Spec3>;
    case 4: return gb_agg_kernel<4, 2, Spec4>;
    case 5: return gb_agg_kernel<4, 2, Spec5>;
    case 6: return gb_agg_kernel<4, 1, Spec6>;
    case 7: return gb_agg_kernel<4, 2, Spec7>;
    default: return n_st <= 4 ? gb_agg_kernel<4, 4, SpecGeneric> : gb_agg_kernel<2, 8, SpecGeneric>;
    }
}

BatchKernel batch_kernel_for(int spec, int max_st) {
    switch (spec) {
    case 1: return gb_batch_agg_kernel<4, 4, Spec1>;
    case 2: return gb_batch_agg_kernel<4, 4, Spec2>;
    case 3: return gb_batch_agg_kernel<4, 2, Spec3>;
    case 4: return gb_batch_agg_kernel<4, 2, Spec4>;
    case 5: return gb_batch_agg_kernel<4, 2, Spec5>;
    case 6: return gb_batch_agg_kernel<4, 1, Spec6>;
    case 7: return gb_batch_agg_kernel<4, 2, Spec7>;
    default: return max_st <= 4 ? gb_batch_agg_kernel<4, 4, SpecGeneric> : gb_batch_agg_kernel<2, 8, SpecGeneric>;
    }
}

AggKernel staged_kernel_for(int spec) {
    switch (spec) {
    case 1: return gb_staged_kernel<Spec1>;
    case 2: return gb_staged_kernel<Spec2>;
    case 3: return gb_staged_kernel<Spec3>;
    case 4: return gb_staged_kernel<Spec4>;
    case 5: return gb_staged_kernel<Spec5>;
    case 6: return gb_staged_kernel<Spec6>;
    default: return gb_staged_kernel<Spec7>;
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Planning
// ---------------------------------------------------------------------------
namespace {
template <class SP>
bool spec_matches(const StateDesc* st, int n) {
    if (n != SP::n) return false;
    for (int s = 0; s < n; ++s)
        if (st[s].kind != SP::kind(s)) return false;
    return true;
}
}  // namespace

// Which compiled row loop serves these (canonically ordered) states.
int gb_spec_of(const StateDesc* st, int n) {
    if (spec_matches<Spec1>(st, n)) return 1;
    if (spec_matches<Spec2>(st, n)) return 2;
    if (spec_matches<Spec3>(st, n)) return 3;
    if (spec_matches<Spec4>(st, n)) return 4;
    if (spec_matches<Spec5>(st, n)) return 5;
    if (spec_matches<Spec6>(st, n)) return 6;
    if (spec_matches<Spec7>(st, n)) return 7;
    return 0;
}

uint64_t gb_shape_key(const GbParams& p, uint64_t n_rows, uint64_t groups_hint) {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        h ^= v;
        h *= 1099511628211ull;
    };
    mix((uint64_t)p.n_keys);
    for (int k = 0; k < p.n_keys; ++k) mix((uint64_t)p.kdtype[k]);
    mix((uint64_t)p.n_pred);
    mix(p.jslots ? 1 : 0);
    for (int s = 0; s < p.n_st; ++s) mix(((uint64_t)p.st[s].kind << 8) | (uint64_t)p.st[s].dtype);
    mix((uint64_t)ceil_log2_u64(n_rows + 1));
    mix((uint64_t)ceil_log2_u64(groups_hint + 1));
    return h;
}

bolt_status gb_plan(bolt_ctx* ctx, const bolt_groupby_desc* d, const bolt_groupby_out* out,
                    uint64_t row_begin, uint64_t row_end, uint32_t flags, int mode,
                    uint64_t cap_override, GbPlan* pl, const bolt_ctx::GbTune* force_tune) {
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
        if (!col_aligned(c->data, c->dtype))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: key column %d is not aligned to its element width", k);
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
        if (!col_aligned(out->keys[k].data, dt))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output key column %d is not aligned", k);
        f.out_key[k] = out->keys[k].data;
        f.out_key_valid[k] = out->keys[k].validity;
    }
    p.n_keys = f.n_keys = d->n_keys;
    for (int q = 0; q < d->n_preds; ++q) {
        const bolt_col_view* c = col(d->preds[q].col);
        if (!c) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: WHERE column out of range");
        if (c->dtype == BOLT_DEC128 || c->dtype == BOLT_U32)
            return fail(ctx, BOLT_DECLINE, "GROUP BY: WHERE on dtype %d", c->dtype);
        if (!col_aligned(c->data, c->dtype))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: WHERE column %d is not aligned to its element width", q);
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
        sd.nwords = (kind == K_SUM_I64 || kind == K_SUM_D64) ? 2 : (kind == K_SUM_D128 || kind == K_SUM_FX ? 3 : 1);
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
        if (c && !col_aligned(c->data, c->dtype))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: aggregate %d input is not aligned to its element width", a);
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
        if (!col_aligned(out->aggs[a].data, g.out_dtype))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output column %d is not aligned to its element width", a);
        g.out = out->aggs[a].data;
        g.out_valid = out->aggs[a].validity;
    }
    // Canonical state order (COUNT, SUMs, MAX, MIN, the rest; stable), so the
    // common layouts hit a row loop compiled for them.
    {
        auto rank = [](int k) {
            return k == K_COUNT ? 0 : (k == K_SUM_I32 || k == K_SUM_I64 || k == K_SUM_FX || k == K_SUM_D64) ? 1
                 : k == K_MAX_ORD ? 2 : k == K_MIN_ORD ? 3 : 4;
        };
        int order[GB_MAX_STATES], where[GB_MAX_STATES];
        for (int s = 0; s < n_st; ++s) order[s] = s;
        std::stable_sort(order, order + n_st, [&](int a, int b) { return rank(p.st[a].kind) < rank(p.st[b].kind); });
        StateDesc sorted[GB_MAX_STATES];
        word = 1;
        int sword = 1;
        for (int i = 0; i < n_st; ++i) {
            sorted[i] = p.st[order[i]];
            sorted[i].word = word;
            sorted[i].sword = sword;
            word += sorted[i].nwords;
            sword += sorted[i].nwords - (sorted[i].kind == K_SUM_FX ? 1 : 0);
            where[order[i]] = i;
        }
        p.sslot_words = sword;
        for (int i = 0; i < n_st; ++i) p.st[i] = sorted[i];
        for (int a = 0; a < d->n_aggs; ++a) {
            AggOut& g = f.agg[a];
            if (g.sum_state >= 0) g.sum_state = where[g.sum_state];
            if (g.cnt_state >= 0) g.cnt_state = where[g.cnt_state];
            if (g.mm_state >= 0) g.mm_state = where[g.mm_state];
        }
        p.spec = gb_spec_of(p.st, n_st);
    }
    p.n_st = n_st;
    // Staged kernel column map: each distinct input column once.
    p.n_sc = 0;
    auto sc_of = [&](const void* colp, int dt) -> int8_t {
        if (!colp) return -1;
        const int w = dtype_width(dt);
        for (int c = 0; c < p.n_sc; ++c)
            if (p.sc_col[c] == colp && p.sc_w[c] == w) return (int8_t)c;
        p.sc_col[p.n_sc] = colp;
        p.sc_w[p.n_sc] = w;
        return (int8_t)p.n_sc++;
    };
    for (int k = 0; k < 2; ++k) p.k_sc[k] = k < p.n_keys ? sc_of(p.kcol[k], p.kdtype[k]) : -1;
    for (int q = 0; q < GB_MAX_PREDS; ++q) p.pr_sc[q] = q < p.n_pred ? sc_of(p.pred[q].col, p.pred[q].dtype) : -1;
    for (int s2 = 0; s2 < GB_MAX_STATES; ++s2) p.st_sc[s2] = s2 < n_st ? sc_of(p.st[s2].col, p.st[s2].dtype) : -1;
    p.slot_words = word;
    f.slot_words = word;
    f.n_aggs = d->n_aggs;
    std::memcpy(f.st, p.st, sizeof(p.st));
    pl->n_aggs = d->n_aggs;

    uint64_t out_cap = UINT64_MAX;
    for (int k = 0; k < d->n_keys; ++k) out_cap = std::min<uint64_t>(out_cap, out->keys[k].cap);
    for (int a = 0; a < d->n_aggs; ++a) out_cap = std::min<uint64_t>(out_cap, out->aggs[a].cap);
    f.out_cap = out_cap;

    // A query has at most as many groups as rows (plus the NULL group), so a
    // hint above the row count sizes nothing larger than the rows need: a
    // 10K-row query hinted at 1M groups would otherwise clear and scan an
    // 8M-slot table.
    const uint64_t hint = d->groups_hint ? std::min<uint64_t>(d->groups_hint, n + 2) : 0;
    pl->groups_hint = hint;
    // Autotuned choices for this query shape, if any (bolt_groupby_autotune).
    pl->shape = gb_shape_key(p, n, hint);
    // Untuned default: the register kernel for small inputs; from 256K rows
    // the streaming kernel compiled for the query's layout where it applies
    // (measured faster from there: 1M rows, 1,024 groups 0.071 -> 0.058 ms
    // per query), else the staged kernel (2 chunks per consumer warp) from
    // 4M rows, where its pipeline fills.
    // Shared-tier admission cap in eighths of the table: half full when the
    // expected groups fit in it; 3/8 when they outnumber it, so keys that miss
    // meet an empty slot sooner (shorter divergent probe loops; measured
    // 3.05 -> 2.95 ms at 100M rows and 3.28M groups).
    const int fill = (hint && hint <= 1024) ? 4 : 3;
    bolt_ctx::GbTune tn{512, 1, 0, 1, fill, n >= GB_LEAN_MIN_ROWS ? 2 : 0, 0.0};
    if (!(flags & BOLT_FLAG_NO_TUNE)) {
        auto it = ctx->tune.find(pl->shape);
        if (it != ctx->tune.end()) tn = it->second;
    }
    if (force_tune) tn = *force_tune;
    if (flags & BOLT_FLAG_KERNEL_REGS) tn.staged = 0;
    if ((flags & BOLT_FLAG_KERNEL_STAGED) && tn.staged == 0) tn.staged = 2;
    pl->tune = tn;

    // Table sizing: the next power of two of (groups_hint << load_shift),
    // load_shift 0..2 (autotuned; untuned 1), grown x8 when occupancy
    // passes 3/4.
    uint64_t cap;
    if (cap_override) cap = cap_override;
    else if (hint)
        cap = 1ull << ceil_log2_u64(std::max<uint64_t>((hint << tn.load_shift) + 16, 64));
    else cap = 1ull << ceil_log2_u64(std::max<uint64_t>(std::min<uint64_t>(2 * n + 16, 1ull << 16), 64));
    pl->cap = cap;
    p.log2cap = f.log2cap = ceil_log2_u64(cap);
    f.n_max = cap + 1;
    p.max_probe = (uint32_t)std::min<uint64_t>(cap, 1u << 14);
    p.grow_limit = cap - cap / 4;
    p.row_begin = row_begin;
    p.n_rows = n;
    p.fx_e = 126 - 32 - ceil_log2_u64(n + 1);
    f.fx_e = p.fx_e;
    p.warp_agg = tn.warp_agg;
    // A CTA's shared table sees at most n rows: COUNT fits its low 32 bits.
    p.cnt32 = n < 0xFFFFFFFFull ? 1 : 0;
    for (int s = 0; s < n_st; ++s)
        if (p.st[s].kind == K_SUM_D128) p.warp_agg = 0;  // D128 partials do not combine in registers

    // Shared-memory tier: the largest power of two of slots that fits the
    // opt-in limit, no larger than 2x the expected groups.
    const size_t entry = 8ull * (size_t)p.sslot_words;
    const size_t budget = (size_t)std::max(ctx->max_smem_optin - 2048, 0);
    int sl = 0;
    if (!(flags & BOLT_FLAG_FORCE_GLOBAL)) {
        while (((size_t)2 << sl) * entry <= budget && sl < 16) ++sl;
        const uint64_t want = 1ull << ceil_log2_u64(std::max<uint64_t>(2 * (hint ? hint : cap), 256));
        while (sl > 8 && (1ull << sl) > want) --sl;
        if (((size_t)1 << sl) * entry > budget) sl = 0;
        // The tuned shrink (more CTAs per SM) applies when the expected
        // groups outgrow the table anyway; a table that holds them all at
        // the admission limit keeps its size.
        if (tn.smem_shift >= 8) sl = 0;
        else if (sl && (1ull << sl) < want) sl = std::max(sl - tn.smem_shift, 6);
    }
    p.smem_log2 = sl;
    p.smem_fill = sl ? (uint32_t)(((1ull << sl) * (uint64_t)tn.smem_fill) / 8) : 0;
    pl->smem_entries = sl ? (1 << sl) : 0;
    pl->u = n_st <= 4 ? 4 : 2;
    pl->block = tn.block;
    pl->small_final = cap <= SMALL_FINAL_MAX;
    p.status = ctx->d_status;
    f.status = ctx->d_status;
    return BOLT_OK;
}

uint64_t gb_plan_scratch(const GbPlan& pl) {
    const uint64_t table = (pl.cap + 2) * (uint64_t)pl.prm.slot_words * 8 + 256 + 64;
    if (pl.small_final) return table + sizeof(GbFinal) + 512;
    const uint64_t g = pl.cap + 1;
    return table + g * 16 + 1024 + sizeof(GbFinal) + radix_sort_scratch(g, 1, SRC_U64_KEYS);
}

namespace {

bolt_status launch_batch_agg(bolt_ctx* ctx, cudaStream_t s, BatchKernel kfn, const GbParams* d_prms,
                             const uint32_t* d_begins, int nq, uint32_t items, uint32_t item_tiles, uint32_t* counter,
                             size_t smem, int block) {
    BOLT_CUDA(ctx, smem_optin(kfn, ctx));
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, block, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    // Enough CTAs for every item at BATCH_CTA_ITEMS each, and at least a
    // full wave.
    const uint64_t need = ((uint64_t)items + BATCH_CTA_ITEMS - 1) / BATCH_CTA_ITEMS;
    const unsigned grid =
        (unsigned)std::max<uint64_t>(need, std::min<uint64_t>((uint64_t)per_sm * ctx->num_sms, items));
    kfn<<<grid, block, smem, s>>>(d_prms, d_begins, nq, items, item_tiles, counter);
    ctx->last_launches++;
    return BOLT_OK;
}

}  // namespace

// Whether the staged kernel serves this plan, and its launch shape: one
// producer warp plus 31 (chunks <= 2) or 15 consumer warps, tiles of
// consumers x 32 x chunks rows, as many stages (2..4) as fit beside the
// shared table (which shrinks when two stages do not fit).
bool gb_staged_layout(const bolt_ctx* ctx, const GbPlan& pl, GbStagedLaunch* out) {
    const GbParams& p = pl.prm;
    const int chunks = pl.tune.staged;
    if (chunks <= 0 || p.spec == 0 || p.jslots || p.n_sc == 0) return false;
    const int block = chunks <= 2 ? 1024 : 512;
    const int nw = block / 32 - 1;
    const uint32_t T = (uint32_t)(nw * 32 * chunks);
    if (p.n_rows < (uint64_t)T) return false;
    uint64_t row_w = 0;
    for (int c = 0; c < p.n_sc; ++c) {
        // Bulk copies need 16-byte aligned tile starts.
        if (((uintptr_t)p.sc_col[c] + p.row_begin * (uint64_t)p.sc_w[c]) % 16 != 0) return false;
        row_w += (uint64_t)p.sc_w[c];
    }
    const size_t stage = (size_t)T * row_w;
    const size_t lists = (size_t)nw * 32 * chunks * 2;
    const size_t budget = (size_t)std::max(ctx->max_smem_optin - 1024, 0);
    int sl = p.smem_log2;
    for (;;) {
        const size_t table = sl ? ((size_t)1 << sl) * 8 * (size_t)p.sslot_words : 0;
        if (table + lists + 2 * stage <= budget) {
            const int S = (int)std::min<size_t>(4, (budget - table - lists) / stage);
            if (out) *out = GbStagedLaunch{block, T, S, (uint32_t)stage, sl, (size_t)S * stage + table + lists};
            return true;
        }
        if (sl == 0) return false;
        sl = sl > 7 ? sl - 1 : 0;
    }
}

// Allocates and zeroes the queries' tables and words and points the plans at them.
static bolt_status gb_run_tables(bolt_ctx* ctx, GbPlan** pls, int nq, cudaStream_t s, bool query_status) {
    if (nq <= 0) return BOLT_OK;
    // Tables and per-query words (occupancy, groups, status) in one zeroed region.
    std::vector<uint64_t> toff(nq);
    uint64_t tot = 0;
    for (int q = 0; q < nq; ++q) {
        toff[q] = tot;
        tot += ((pls[q]->cap + 2) * (uint64_t)pls[q]->prm.slot_words * 8 + 255) & ~uint64_t(255);
    }
    const uint64_t words_off = tot;
    tot += (uint64_t)nq * 64;
    char* region = (char*)arena_alloc(ctx, tot);
    if (!region)
        return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for %d table(s) of %llu bytes", nq,
                    (ull)tot);
    BOLT_CUDA(ctx, cudaMemsetAsync(region, 0, tot, s));
    for (int q = 0; q < nq; ++q) {
        GbParams& p = pls[q]->prm;
        GbFinal& f = pls[q]->fin;
        ull* w = (ull*)(region + words_off) + 8 * q;
        p.gtab = (ull*)(region + toff[q]);
        p.occupancy = w;
        // A single query reports through the context's status word (so
        // bolt_ctx_sync_status sees it); batched queries each get their own,
        // also in a batch of one.
        p.status = (nq == 1 && !query_status) ? ctx->d_status : (uint32_t*)(w + 3);
        f.gtab = p.gtab;
        f.n_nonnull = w + 1;
        f.n_groups = w + 2;
        f.status = p.status;
        pls[q]->words = w;
        p.i64_bits = nullptr;
        for (int s2 = 0; s2 < p.n_st; ++s2)
            if (p.st[s2].kind == K_SUM_I64) p.i64_bits = (uint32_t*)(w + 4);
    }
    return BOLT_OK;
}

// Launches the aggregation of one query (the single-query kernels).
static bolt_status gb_agg_one(bolt_ctx* ctx, GbPlan* pl, cudaStream_t s, uint32_t flags) {
    // Dense shapes of 4M+ rows: the streaming kernel compiled for the key,
    // WHERE and state layouts (groupby_part.cu), misses to the global table.
    if (!(flags & BOLT_FLAG_KERNEL_STAGED) && pl->tune.staged != 0) {
        bolt_status st = BOLT_OK;
        if (gb_lean_global(ctx, pl, s, flags, &st)) return st;
    }
    GbParams& p = pl->prm;
    size_t smem = (size_t)pl->smem_entries * 8ull * (size_t)p.sslot_words;
    const uint64_t tile = (uint64_t)pl->block * pl->u;
    GbStagedLaunch stg;
    const bool staged = (p.n_rows >= GB_STAGED_MIN_ROWS || (flags & BOLT_FLAG_KERNEL_STAGED)) &&
                        gb_staged_layout(ctx, *pl, &stg);
    AggKernel kfn;
    int block = pl->block;
    uint64_t tiles;
    if (staged) {
        kfn = staged_kernel_for(p.spec);
        block = stg.block;
        smem = stg.smem;
        p.smem_log2 = stg.smem_log2;
        p.smem_fill = stg.smem_log2 ? (uint32_t)(((1ull << stg.smem_log2) * (uint64_t)pl->tune.smem_fill) / 8) : 0;
        p.tile_rows = stg.tile_rows;
        p.n_stages = stg.n_stages;
        p.stage_bytes = stg.stage_bytes;
        p.chunks = pl->tune.staged;
        uint32_t off = 0;
        for (int c = 0; c < p.n_sc; ++c) {
            p.sc_off[c] = off;
            off += stg.tile_rows * (uint32_t)p.sc_w[c];
        }
        tiles = std::max<uint64_t>(p.n_rows / stg.tile_rows, 1);
    } else {
        kfn = agg_kernel_for(p.spec, p.n_st);
        tiles = (p.n_rows + tile - 1) / tile;
    }
    int per_sm = 1;
    BOLT_CUDA(ctx, smem_optin(kfn, ctx));
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, block, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    uint64_t grid = std::min<uint64_t>((uint64_t)per_sm * ctx->num_sms, std::max<uint64_t>(tiles, 1));
    if (pl->grid > 0) grid = std::min<uint64_t>(grid, (uint64_t)pl->grid);
    pl->grid = (int)grid;
    if (p.n_rows > 0) {
        kernel_mark_begin(ctx, flags, s);
        kfn<<<pl->grid, block, smem, s>>>(p);
        BOLT_CUDA(ctx, cudaGetLastError());
        ctx->last_launches++;
        kernel_mark_end(ctx, flags, s);
    }
    return BOLT_OK;
}

// One persistent launch over a group of queries that share a compiled layout.
static bolt_status gb_agg_batch(bolt_ctx* ctx, GbPlan** pls, int nq, cudaStream_t s, uint32_t flags) {
    // One compiled row loop for the whole batch: the queries' common
    // layout, else the generic loop.
    int u = 4, max_st = 0, spec = pls[0]->prm.spec;
    size_t smem = 0;
    for (int q = 0; q < nq; ++q) {
        max_st = std::max(max_st, (int)pls[q]->prm.n_st);
        if (pls[q]->prm.spec != spec) spec = 0;
        smem = std::max<size_t>(smem, (size_t)pls[q]->smem_entries * 8 * (size_t)pls[q]->prm.sslot_words);
    }
    if (spec == 0 && max_st > 4) u = 2;
    const BatchKernel kfn = batch_kernel_for(spec, max_st);
    const uint32_t item_tiles = 4;
    std::vector<GbParams> prms(nq);
    std::vector<uint32_t> begins(nq + 1);
    uint64_t items = 0;
    const uint64_t tile = 512ull * u * item_tiles;
    for (int q = 0; q < nq; ++q) {
        prms[q] = pls[q]->prm;
        begins[q] = (uint32_t)items;
        items += (pls[q]->prm.n_rows + tile - 1) / tile;
    }
    begins[nq] = (uint32_t)items;
    if (items >= (1ull << 32)) return fail(ctx, BOLT_DECLINE, "batched GROUP BY: too many row tiles");
    GbParams* d_prms = (GbParams*)arena_alloc(ctx, sizeof(GbParams) * nq);
    uint32_t* d_begins = (uint32_t*)arena_alloc(ctx, 4ull * (nq + 1) + 64);
    if (!d_prms || !d_begins) return fail(ctx, BOLT_ERR_CAPACITY, "batched GROUP BY: scratch arena too small");
    uint32_t* counter = d_begins + nq + 1;
    bolt_status st = stage_upload(ctx, s, d_prms, prms.data(), sizeof(GbParams) * nq);
    if (st == BOLT_OK) st = stage_upload(ctx, s, d_begins, begins.data(), 4ull * (nq + 1));
    if (st != BOLT_OK) return st;
    BOLT_CUDA(ctx, cudaMemsetAsync(counter, 0, 4, s));
    if (items) {
        kernel_mark_begin(ctx, flags, s);
        st = launch_batch_agg(ctx, s, kfn, d_prms, d_begins, nq, (uint32_t)items, item_tiles, counter, smem, 512);
        kernel_mark_end(ctx, flags, s);
        if (st != BOLT_OK) return st;
    }
    return BOLT_OK;
}

// Queries with at least this many rows are launched alone in a batch: at that
// size a launch of their own costs little, and they get the single-query
// kernels (the staged kernel among them).
constexpr uint64_t BATCH_ALONE_ROWS = 1ull << 21;

// Launches the aggregation of every query into its table: one query alone;
// in a batch, large queries alone and the others grouped by compiled layout,
// one persistent launch per group.
static bolt_status gb_run_aggregate(bolt_ctx* ctx, GbPlan** pls, int nq, cudaStream_t s, uint32_t flags) {
    if (nq == 1) return gb_agg_one(ctx, pls[0], s, flags);
    std::vector<GbPlan*> groups[8];
    for (int q = 0; q < nq; ++q) {
        if (pls[q]->prm.n_rows >= BATCH_ALONE_ROWS) {
            bolt_status st = gb_agg_one(ctx, pls[q], s, flags);
            if (st != BOLT_OK) return st;
        } else {
            groups[std::min(std::max(pls[q]->prm.spec, 0), 7)].push_back(pls[q]);
        }
    }
    for (auto& g : groups) {
        if (g.empty()) continue;
        bolt_status st = gb_agg_batch(ctx, g.data(), (int)g.size(), s, flags);
        if (st != BOLT_OK) return st;
    }
    return BOLT_OK;
}

// Finalizes every query's table into its output columns.
static bolt_status gb_run_finalize(bolt_ctx* ctx, GbPlan** pls, int nq, cudaStream_t s) {
    // Finalize: small tables one CTA each; large tables through batched
    // compaction, a segmented radix sort and a batched gather.
    std::vector<GbFinal> small, large;
    std::vector<int> large_q;
    uint64_t small_cap = 0;
    for (int q = 0; q < nq; ++q) {
        if (pls[q]->small_final) {
            small.push_back(pls[q]->fin);
            small_cap = std::max<uint64_t>(small_cap, pls[q]->cap);
        } else {
            large_q.push_back(q);
        }
    }
    if (small.size() == 1) {
        BOLT_CUDA(ctx, smem_optin(gb_small_final1_kernel, ctx));
        gb_small_final1_kernel<<<1, SF_BLOCK, small_final_smem(small_cap), s>>>(small[0]);
        ctx->last_launches++;
    } else if (!small.empty()) {
        GbFinal* d_f = (GbFinal*)arena_alloc(ctx, sizeof(GbFinal) * small.size());
        if (!d_f) return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the finalize");
        bolt_status st = stage_upload(ctx, s, d_f, small.data(), sizeof(GbFinal) * small.size());
        if (st != BOLT_OK) return st;
        const size_t fsm = small_final_smem(small_cap);
        BOLT_CUDA(ctx, smem_optin(gb_small_final_kernel, ctx));
        gb_small_final_kernel<<<(unsigned)small.size(), SF_BLOCK, fsm, s>>>(d_f);
        ctx->last_launches++;
    }
    if (!large_q.empty()) {
        const int nl = (int)large_q.size();
        std::vector<uint32_t> cbeg(nl + 1), gbeg(nl + 1);
        uint64_t citems = 0, gitems = 0;
        SortSpec sp;
        sp.src = SRC_U64_KEYS;
        for (int i = 0; i < nl; ++i) {
            GbPlan* pl = pls[large_q[i]];
            GbFinal& f = pl->fin;
            const uint64_t g = pl->cap + 1;
            if (!pl->precompacted) {  // (the partitioned tier wrote the sort keys itself)
                f.order_keys = (ull*)arena_alloc(ctx, g * 8);
                f.slots = (uint32_t*)arena_alloc(ctx, g * 4);
                f.sorted = (uint32_t*)arena_alloc(ctx, g * 4);
            }
            if (!f.order_keys || !f.slots || !f.sorted)
                return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the finalize");
            large.push_back(f);
            cbeg[i] = (uint32_t)citems;
            citems += (g + FIN_CHUNK - 1) / FIN_CHUNK;
            gbeg[i] = (uint32_t)gitems;
            gitems += (g + GATHER_CHUNK - 1) / GATHER_CHUNK;
            SortSegment seg;
            seg.keys = f.order_keys;
            seg.payload_in = f.slots;
            seg.payload_out = f.sorted;
            seg.n_dev = f.n_nonnull;
            seg.n = f.n_max;
            sp.segs.push_back(seg);
        }
        cbeg[nl] = (uint32_t)citems;
        gbeg[nl] = (uint32_t)gitems;
        GbFinal* d_f = (GbFinal*)arena_alloc(ctx, sizeof(GbFinal) * nl);
        uint32_t* d_beg = (uint32_t*)arena_alloc(ctx, 4ull * (nl + 1));
        uint32_t* d_gbeg = (uint32_t*)arena_alloc(ctx, 4ull * (nl + 1));
        if (!d_f || !d_beg || !d_gbeg)
            return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the finalize");
        bolt_status st = stage_upload(ctx, s, d_f, large.data(), sizeof(GbFinal) * nl);
        if (st == BOLT_OK) st = stage_upload(ctx, s, d_beg, cbeg.data(), 4ull * (nl + 1));
        if (st == BOLT_OK) st = stage_upload(ctx, s, d_gbeg, gbeg.data(), 4ull * (nl + 1));
        if (st != BOLT_OK) return st;
        const unsigned cg = (unsigned)std::min<uint64_t>(citems, (uint64_t)ctx->num_sms * 8);
        if (!pls[large_q[0]]->precompacted) {  // (a precompacted query is finalized alone)
            gb_compact_batch_kernel<<<cg, 256, 0, s>>>(d_f, d_beg, nl, (uint32_t)citems);
            ctx->last_launches++;
        }
        st = radix_sort(ctx, s, sp);
        if (st != BOLT_OK) return st;
        const unsigned gg = (unsigned)std::min<uint64_t>(gitems, (uint64_t)ctx->num_sms * 8);
        gb_gather_batch_kernel<<<gg, 256, 0, s>>>(d_f, d_gbeg, nl, (uint32_t)gitems);
        ctx->last_launches++;
    }
    BOLT_CUDA(ctx, cudaGetLastError());
    return BOLT_OK;
}

bolt_status gb_run(bolt_ctx* ctx, GbPlan** pls, int nq, cudaStream_t s, uint32_t flags, bool query_status) {
    if (nq <= 0) return BOLT_OK;
    bolt_status st = gb_run_tables(ctx, pls, nq, s, query_status);
    if (st == BOLT_OK) st = gb_run_aggregate(ctx, pls, nq, s, flags);
    if (st == BOLT_OK) st = gb_run_finalize(ctx, pls, nq, s);
    return st;
}

}  // namespace bolt

using namespace bolt;

extern "C" uint64_t bolt_groupby_footprint(const bolt_groupby_desc* desc, uint64_t n_rows) {
    if (!desc) return 0;
    // Table words per slot: key + at most four words per aggregate (AVG: a
    // three-word sum and a count); slots as the planner sizes them untuned
    // (2x the expected groups, or 2x the rows up to 64K without a hint).
    const uint64_t words = 1 + 4ull * (uint64_t)(desc->n_aggs > 0 ? desc->n_aggs : 1);
    const uint64_t hint = desc->groups_hint ? std::min<uint64_t>(desc->groups_hint, n_rows + 2) : 0;
    const uint64_t want = hint ? (hint << 1) + 16 : std::min<uint64_t>(2 * n_rows + 16, 1ull << 16);
    const uint64_t cap = 1ull << ceil_log2_u64(std::max<uint64_t>(want, 64));
    uint64_t bytes = (cap + 2) * words * 8 + 4096;
    if (cap > 8192) bytes += (cap + 1) * 16 + radix_sort_scratch(cap + 1, 1, SRC_U64_KEYS);
    return bytes;
}

namespace bolt {

// Runs one query on the hash-partitioned tier: the compact group array
// (cap + 2 slots; only the two special slots start at zero, pass C writes
// every other slot it uses), the per-query words, the finalize buffers that
// pass C fills with the groups' sort keys, the partitioned passes and the
// finalize.
static bolt_status gb_run_part(bolt_ctx* ctx, GbPlan* pl, cudaStream_t s, uint32_t flags, int pbits) {
    GbParams& p = pl->prm;
    GbFinal& f = pl->fin;
    const uint64_t slot_bytes = (uint64_t)p.slot_words * 8;
    const uint64_t table = ((pl->cap + 2) * slot_bytes + 255) & ~uint64_t(255);
    char* region = (char*)arena_alloc(ctx, table + 256);
    const uint64_t g = pl->cap + 1;
    f.order_keys = (ull*)arena_alloc(ctx, g * 8);
    f.slots = (uint32_t*)arena_alloc(ctx, g * 4);
    f.sorted = (uint32_t*)arena_alloc(ctx, g * 4);
    if (!region || !f.order_keys || !f.slots || !f.sorted)
        return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the group array");
    ull* w = (ull*)(region + table);
    BOLT_CUDA(ctx, cudaMemsetAsync(region + pl->cap * slot_bytes, 0, 2 * slot_bytes, s));
    BOLT_CUDA(ctx, cudaMemsetAsync(w, 0, 256, s));
    p.gtab = (ull*)region;
    p.occupancy = w;
    p.status = ctx->d_status;
    p.i64_bits = nullptr;
    for (int s2 = 0; s2 < p.n_st; ++s2)
        if (p.st[s2].kind == K_SUM_I64) p.i64_bits = (uint32_t*)(w + 4);
    f.gtab = p.gtab;
    f.n_nonnull = w + 1;
    f.n_groups = w + 2;
    f.status = p.status;
    f.n_max = pl->cap;
    pl->words = w;
    pl->precompacted = true;
    pl->small_final = false;
    bolt_status st = gb_part_launch(ctx, pl, s, flags, pbits);
    if (st != BOLT_OK) return st;
    GbPlan* one = pl;
    return gb_run_finalize(ctx, &one, 1, s);
}

// The reference checks SUM(Int64) with a checked add in row order per group
// (checked_group_sum, groupby.rs:1775-1798), so a prefix that leaves the
// i64 range errors even when the final sum fits. When the largest |v| and
// the row count allow such a prefix, replay every group's rows in row order
// (stable radix sort of (slot, row), then one sequential fold per group).
static bolt_status gb_exact_i64_check(bolt_ctx* ctx, GbPlan& pl, cudaStream_t s) {
    const uint64_t n = pl.prm.n_rows;
    if (n >= (1ull << 30))
        return fail(ctx, BOLT_DECLINE, "GROUP BY: SUM(Int64) row-order overflow check needs < 2^30 rows");
    uint32_t* slot_of_row = (uint32_t*)arena_alloc(ctx, n * 4 + 16);
    uint32_t* sorted = (uint32_t*)arena_alloc(ctx, n * 4 + 16);
    if (!slot_of_row || !sorted) return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the SUM check");
    const unsigned g = grid_for(n, 256, ctx->num_sms * 8);
    gb_row_slot_kernel<<<g, 256, 0, s>>>(pl.prm, slot_of_row);
    SortSpec sp;
    sp.src = SRC_U32;
    SortSegment seg;
    seg.keys = slot_of_row;
    seg.n = n;
    seg.payload_out = sorted;
    sp.segs.push_back(seg);
    bolt_status st = radix_sort(ctx, s, sp);
    if (st != BOLT_OK) return st;
    gb_prefix_check_kernel<<<g, 256, 0, s>>>(pl.prm, slot_of_row, sorted);
    BOLT_CUDA(ctx, cudaGetLastError());
    uint32_t f = 0;
    st = read_status(ctx, s, 0, &f);
    if (st != BOLT_OK) return st;
    return flags_to_status(ctx, f, "GROUP BY");
}

// Runs one query (optionally with a join table as its key source) with the
// retry policy: grow the table on GROW / SPILL, switch the f64 SUM to atomics
// on RANGE, switch Decimal128 SUM to the wide state on DECRANGE.
static bolt_status gb_single(bolt_ctx* ctx, const bolt_groupby_desc* d, bolt_groupby_out* out, uint64_t rb,
                             uint64_t re, uint32_t flags, cudaStream_t s, const bolt_join_table* jt,
                             const bolt_col_view* jkey, const char* op) {
    int mode = 0;
    uint64_t cap_override = 0;
    int part_pbits = 0;       // partitions (log2) after a partition spilled
    bool no_part = false;     // the partitioned tier gave way to the global table
    uint64_t groups_seen = 0; // groups an earlier attempt counted (sizes the next one)
    for (int attempt = 0; attempt < 8; ++attempt) {
        bolt_status st = call_begin(ctx, flags, s);
        if (st != BOLT_OK) return st;
        GbPlan pl;
        st = gb_plan(ctx, d, out, rb, re, flags, mode, cap_override, &pl);
        if (st != BOLT_OK) return st;
        pl.groups_hint = std::max<uint64_t>(pl.groups_hint, groups_seen);
        if (!jt && !no_part && gb_part_applies(ctx, pl, flags)) {
            ctx->last_tier = 2;
            pl.fin.n_groups_user = (flags & BOLT_FLAG_ASYNC) ? (ull*)out->n_groups_dev : nullptr;
            st = gb_run_part(ctx, &pl, s, flags, part_pbits);
            if (st == BOLT_DECLINE || st == BOLT_ERR_CAPACITY) {
                // No kernel for this layout, or no room for the spill
                // segments: the global-table path serves the query.
                ctx->last_error.clear();
                no_part = true;
                continue;
            }
            if (st != BOLT_OK) return st;
            st = call_end(ctx, flags, s);
            if (st != BOLT_OK) return st;
            if (flags & BOLT_FLAG_ASYNC) return BOLT_OK;
            uint32_t f = 0;
            st = read_status(ctx, s, 0, &f);
            if (st != BOLT_OK) return st;
            ull w[5] = {0, 0, 0, 0, 0};
            BOLT_CUDA(ctx, cudaMemcpy(w, pl.words, sizeof w, cudaMemcpyDeviceToHost));
            out->n_groups = w[2];
            const uint32_t bits = (uint32_t)w[4];
            if (f == 0 && pl.prm.i64_bits && bits + (uint32_t)ceil_log2_u64(pl.prm.n_rows + 1) >= 63) {
                // The row-order SUM(Int64) check replays rows against a hash
                // table of the groups: run the query on the global table.
                no_part = true;
                continue;
            }
            // The group counter (w[1]) counts past the array, so it sizes the
            // retry; after a spill it is a lower bound.
            if (f & ST_FLAG_SPILL) {
                // A partition outgrew its table (or a segment its room):
                // 4x the partitions, then the global table.
                groups_seen = std::max<uint64_t>(groups_seen, 2 * w[1]);
                if (pl.part_pbits + 2 <= GB_PART_MAX_PBITS) part_pbits = pl.part_pbits + 2;
                else no_part = true;
                continue;
            }
            if (f & ST_FLAG_GROW) {
                groups_seen = std::max<uint64_t>(groups_seen, w[1]);
                cap_override = std::max<uint64_t>(pl.cap * 2, 1ull << ceil_log2_u64(w[1] + w[1] / 4 + 16));
                continue;
            }
            if (f & (ST_FLAG_RANGE | ST_FLAG_DECRANGE)) {
                if (f & ST_FLAG_RANGE) mode |= GB_MODE_F64_ATOMIC;
                if (f & ST_FLAG_DECRANGE) mode |= GB_MODE_WIDE_DEC;
                continue;
            }
            if (f & ST_FLAG_DECOVERFLOW)
                return fail(ctx, BOLT_ERR_OVERFLOW, "SUM(Decimal128) precision overflow: accumulator exceeds i128 range");
            return flags_to_status(ctx, f, op);
        }
        ctx->last_tier = 1;
        if (jt) {
            pl.prm.jslots = jt->slots;
            pl.prm.jlog2cap = jt->log2cap;
            pl.prm.jkdt = jkey->dtype;
            pl.prm.jkey = jkey->data;
            pl.prm.jkvalid = jkey->validity;
        }
        pl.fin.n_groups_user = (flags & BOLT_FLAG_ASYNC) ? (ull*)out->n_groups_dev : nullptr;
        GbPlan* one = &pl;
        st = gb_run(ctx, &one, 1, s, flags);
        if (st != BOLT_OK) return st;
        st = call_end(ctx, flags, s);
        if (st != BOLT_OK) return st;
        if (flags & BOLT_FLAG_ASYNC) return BOLT_OK;
        uint32_t f = 0;
        st = read_status(ctx, s, 0, &f);
        if (st != BOLT_OK) return st;
        ull w[5] = {0, 0, 0, 0, 0};
        BOLT_CUDA(ctx, cudaMemcpy(w, pl.words, sizeof w, cudaMemcpyDeviceToHost));
        out->n_groups = w[2];
        const uint32_t bits = (uint32_t)w[4];
        if (f == 0 && pl.prm.i64_bits && bits + (uint32_t)ceil_log2_u64(pl.prm.n_rows + 1) >= 63)
            return gb_exact_i64_check(ctx, pl, s);
        if (f & (ST_FLAG_GROW | ST_FLAG_SPILL)) {
            if (flags & BOLT_FLAG_FORCE_SHMEM)
                return fail(ctx, BOLT_ERR_SPILL, "partition_reduce spill: shared-memory tier overflow");
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
        return flags_to_status(ctx, f, op);
    }
    return fail(ctx, BOLT_ERR_CAPACITY, "%s: table growth did not converge", op);
}

// Adds `delta` to every column pointer of `p` that lies in [lo, hi).
static void gb_rebase(GbParams& p, uintptr_t lo, uintptr_t hi, ptrdiff_t delta) {
    auto fix = [&](const void*& q) {
        const uintptr_t v = reinterpret_cast<uintptr_t>(q);
        if (v >= lo && v < hi) q = reinterpret_cast<const void*>(v + delta);
    };
    auto fixv = [&](const uint8_t*& q) {
        const void* t = q;
        fix(t);
        q = static_cast<const uint8_t*>(t);
    };
    for (int k = 0; k < 2; ++k) {
        fix(p.kcol[k]);
        fixv(p.kvalid[k]);
    }
    for (int q = 0; q < GB_MAX_PREDS; ++q) {
        fix(p.pred[q].col);
        fixv(p.pred[q].valid);
    }
    for (int s2 = 0; s2 < GB_MAX_STATES; ++s2) {
        fix(p.st[s2].col);
        fixv(p.st[s2].valid);
    }
    for (int c = 0; c < GB_MAX_SC; ++c) fix(p.sc_col[c]);
}

// GROUP BY over host-resident columns. The rows go to the device in chunks
// on the context's copy stream, into a ring of staging slots in the scratch
// arena, while the aggregation kernel folds the previous chunks into the one
// table on the caller's stream: the host -> device transfer and the
// aggregation overlap, and no column is ever resident in full.
static bolt_status gb_host(bolt_ctx* ctx, const bolt_groupby_desc* d, bolt_groupby_out* out, uint32_t flags,
                           cudaStream_t s) {
    const char* op = "GROUP BY (host columns)";
    if (flags & BOLT_FLAG_ASYNC) return fail(ctx, BOLT_ERR_INVALID, "%s: BOLT_FLAG_ASYNC is not supported", op);
    if (!d->cols || d->n_cols <= 0 || d->n_cols > 64 || !d->key_cols || d->n_keys < 1 || d->n_keys > 2 ||
        d->n_preds < 0 || d->n_preds > GB_MAX_PREDS || d->n_aggs < 0 || (d->n_preds && !d->preds) ||
        (d->n_aggs && !d->aggs))
        return fail(ctx, BOLT_ERR_INVALID, "%s: bad descriptor", op);
    bool used[64] = {};
    auto use = [&](int i) {
        if (i < 0 || i >= d->n_cols) return false;
        used[i] = true;
        return true;
    };
    for (int k = 0; k < d->n_keys; ++k)
        if (!use(d->key_cols[k])) return fail(ctx, BOLT_ERR_INVALID, "%s: key column out of range", op);
    for (int q = 0; q < d->n_preds; ++q)
        if (!use(d->preds[q].col)) return fail(ctx, BOLT_ERR_INVALID, "%s: WHERE column out of range", op);
    for (int a = 0; a < d->n_aggs; ++a)
        if (d->aggs[a].op != BOLT_AGG_COUNT_STAR && !use(d->aggs[a].input_col))
            return fail(ctx, BOLT_ERR_INVALID, "%s: aggregate column out of range", op);
    const uint64_t n = d->cols[d->key_cols[0]].len;
    uint64_t row_bytes = 0;
    for (int i = 0; i < d->n_cols; ++i) {
        if (!used[i]) continue;
        const int w = dtype_width(d->cols[i].dtype);
        if (w == 0 || !d->cols[i].data) return fail(ctx, BOLT_ERR_INVALID, "%s: column %d has no data", op, i);
        if (d->cols[i].len < n) return fail(ctx, BOLT_ERR_INVALID, "%s: column %d shorter than the key", op, i);
        row_bytes += (uint64_t)w + (d->cols[i].validity ? 1 : 0);
    }
    if (gb_wide_applies(d)) {
        // Keys wider than 64 bits: the sort-based path needs every row at
        // once, so the used columns are uploaded whole into the arena, held
        // there (pinned) while the wide path runs on the device copies.
        const uint64_t pinned0 = ctx->arena_pinned;
        ctx->arena_used = pinned0;
        std::vector<bolt_col_view> dev(d->cols, d->cols + d->n_cols);
        for (int i = 0; i < d->n_cols; ++i) {
            if (!used[i]) continue;
            const uint64_t db = n * (uint64_t)dtype_width(d->cols[i].dtype);
            const uint64_t vb = (n + 7) / 8;
            void* dd = arena_alloc(ctx, db ? db : 1);
            uint8_t* dv = d->cols[i].validity ? (uint8_t*)arena_alloc(ctx, vb ? vb : 1) : nullptr;
            if (!dd || (d->cols[i].validity && !dv))
                return fail(ctx, BOLT_ERR_CAPACITY, "%s: scratch arena too small for the wide-key columns", op);
            if (db) BOLT_CUDA(ctx, cudaMemcpyAsync(dd, d->cols[i].data, db, cudaMemcpyHostToDevice, s));
            if (dv && vb) BOLT_CUDA(ctx, cudaMemcpyAsync(dv, d->cols[i].validity, vb, cudaMemcpyHostToDevice, s));
            dev[i].data = dd;
            dev[i].validity = dv;
            dev[i].len = n;
        }
        bolt_groupby_desc dd = *d;
        dd.cols = dev.data();
        ctx->arena_pinned = ctx->arena_used;
        const bolt_status st = gb_wide(ctx, &dd, out, flags, s);
        // The copies and kernels are done before the columns are unpinned
        // and before the caller's host buffers may be reused.
        const cudaError_t e = cudaStreamSynchronize(s);
        ctx->arena_pinned = pinned0;
        if (st == BOLT_OK && e != cudaSuccess) return cuda_fail(ctx, e, "cudaStreamSynchronize");
        return st;
    }
    constexpr int NB = bolt_ctx::HOST_SLOTS;
    if (!ctx->copy_stream) {
        BOLT_CUDA(ctx, cudaSetDevice(ctx->device));
        BOLT_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
        for (int i = 0; i < 2 * NB + 1; ++i)
            BOLT_CUDA(ctx, cudaEventCreateWithFlags(&ctx->host_ev[i], cudaEventDisableTiming));
    }
    cudaEvent_t* copied = ctx->host_ev;
    cudaEvent_t* consumed = ctx->host_ev + NB;
    cudaEvent_t start = ctx->host_ev[2 * NB];
    // Whatever leaves this function, the copies that read the caller's host
    // buffers have finished.
    struct CopyDrain {
        cudaStream_t cs;
        ~CopyDrain() { cudaStreamSynchronize(cs); }
    } drain{ctx->copy_stream};

    int mode = 0;
    uint64_t cap_override = 0;
    for (int attempt = 0; attempt < 6; ++attempt) {
        bolt_status st = call_begin(ctx, flags, s);
        if (st != BOLT_OK) return st;
        // Chunk rows: a multiple of 64 (whole validity bytes), 4M at most,
        // the ring using at most a quarter of the free arena.
        const uint64_t free_b = ctx->arena_bytes - ctx->arena_used;
        uint64_t R = std::min<uint64_t>(4ull << 20, (n + 63) & ~63ull);
        while (R > 64 && (uint64_t)NB * (R * row_bytes + 256ull * 2 * d->n_cols) > free_b / 4) R = (R / 2 + 63) & ~63ull;
        R = std::max<uint64_t>(R, 64);
        // Slot layout: every used column's data and validity at fixed offsets.
        std::vector<uint64_t> doff(d->n_cols, 0), voff(d->n_cols, 0);
        uint64_t stride = 0;
        for (int i = 0; i < d->n_cols; ++i) {
            if (!used[i]) continue;
            doff[i] = stride;
            stride += (R * (uint64_t)dtype_width(d->cols[i].dtype) + 255) & ~255ull;
            if (d->cols[i].validity) {
                voff[i] = stride;
                stride += (R / 8 + 255) & ~255ull;
            }
        }
        char* ring = (char*)arena_alloc(ctx, stride * NB);
        if (!ring) return fail(ctx, BOLT_ERR_CAPACITY, "%s: scratch arena too small for the staging ring", op);
        std::vector<bolt_col_view> dcols(d->cols, d->cols + d->n_cols);
        for (int i = 0; i < d->n_cols; ++i) {
            if (!used[i]) continue;
            dcols[i].data = ring + doff[i];
            dcols[i].validity = d->cols[i].validity ? reinterpret_cast<const uint8_t*>(ring + voff[i]) : nullptr;
        }
        bolt_groupby_desc dd = *d;
        dd.cols = dcols.data();
        GbPlan pl;
        st = gb_plan(ctx, &dd, out, 0, n, flags, mode, cap_override, &pl);
        if (st != BOLT_OK) return st;
        pl.fin.n_groups_user = nullptr;
        GbPlan* one = &pl;
        st = gb_run_tables(ctx, &one, 1, s, false);
        if (st != BOLT_OK) return st;
        const GbParams base = pl.prm;
        // The ring may still be read by an earlier call's kernels on `s`.
        BOLT_CUDA(ctx, cudaEventRecord(start, s));
        BOLT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, start, 0));
        const uint64_t chunks = (n + R - 1) / R;
        for (uint64_t c = 0; c < chunks; ++c) {
            const int k = (int)(c % NB);
            const uint64_t r0 = c * R;
            const uint64_t rows = std::min<uint64_t>(R, n - r0);
            if (c >= (uint64_t)NB) BOLT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_stream, consumed[k], 0));
            char* slot = ring + (uint64_t)k * stride;
            for (int i = 0; i < d->n_cols; ++i) {
                if (!used[i]) continue;
                const uint64_t w = (uint64_t)dtype_width(d->cols[i].dtype);
                BOLT_CUDA(ctx, cudaMemcpyAsync(slot + doff[i], static_cast<const char*>(d->cols[i].data) + r0 * w,
                                               rows * w, cudaMemcpyHostToDevice, ctx->copy_stream));
                if (d->cols[i].validity)
                    BOLT_CUDA(ctx, cudaMemcpyAsync(slot + voff[i], d->cols[i].validity + r0 / 8, (rows + 7) / 8,
                                                   cudaMemcpyHostToDevice, ctx->copy_stream));
            }
            BOLT_CUDA(ctx, cudaEventRecord(copied[k], ctx->copy_stream));
            BOLT_CUDA(ctx, cudaStreamWaitEvent(s, copied[k], 0));
            pl.prm = base;
            gb_rebase(pl.prm, reinterpret_cast<uintptr_t>(ring), reinterpret_cast<uintptr_t>(ring) + stride,
                      (ptrdiff_t)((uint64_t)k * stride));
            pl.prm.row_begin = 0;
            pl.prm.n_rows = rows;
            pl.grid = 0;
            st = gb_run_aggregate(ctx, &one, 1, s, flags);
            if (st != BOLT_OK) return st;
            BOLT_CUDA(ctx, cudaEventRecord(consumed[k], s));
        }
        pl.prm = base;
        st = gb_run_finalize(ctx, &one, 1, s);
        if (st != BOLT_OK) return st;
        st = call_end(ctx, flags, s);
        if (st != BOLT_OK) return st;
        uint32_t f = 0;
        st = read_status(ctx, s, 0, &f);
        if (st != BOLT_OK) return st;
        ull w[5] = {0, 0, 0, 0, 0};
        BOLT_CUDA(ctx, cudaMemcpy(w, pl.words, sizeof w, cudaMemcpyDeviceToHost));
        out->n_groups = w[2];
        if (f == 0 && base.i64_bits && (uint32_t)w[4] + (uint32_t)ceil_log2_u64(n + 1) >= 63)
            return fail(ctx, BOLT_DECLINE,
                        "%s: SUM(Int64) inputs large enough to need the row-order overflow check; run it on device "
                        "columns (bolt_groupby)", op);
        if (f & (ST_FLAG_GROW | ST_FLAG_SPILL)) {
            if (flags & BOLT_FLAG_FORCE_SHMEM)
                return fail(ctx, BOLT_ERR_SPILL, "partition_reduce spill: shared-memory tier overflow");
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
        return flags_to_status(ctx, f, op);
    }
    return fail(ctx, BOLT_ERR_CAPACITY, "%s: table growth did not converge", op);
}

}  // namespace bolt

extern "C" bolt_status bolt_groupby_host(bolt_ctx* ctx, const bolt_groupby_desc* desc, bolt_groupby_out* out,
                                         uint32_t flags, bolt_stream stream) {
    if (!ctx || !desc || !out) return BOLT_ERR_INVALID;
    return gb_host(ctx, desc, out, flags, (cudaStream_t)stream);
}

extern "C" bolt_status bolt_groupby(bolt_ctx* ctx, const bolt_groupby_desc* desc, bolt_groupby_out* out,
                                    uint32_t flags, bolt_stream stream) {
    if (!ctx || !desc || !out) return BOLT_ERR_INVALID;
    uint64_t nrows = 0;
    if (desc->n_keys >= 1 && desc->key_cols && desc->cols && desc->key_cols[0] >= 0 && desc->key_cols[0] < desc->n_cols)
        nrows = desc->cols[desc->key_cols[0]].len;
    if (gb_wide_applies(desc)) return gb_wide(ctx, desc, out, flags, (cudaStream_t)stream);
    return gb_single(ctx, desc, out, 0, nrows, flags, (cudaStream_t)stream, nullptr, nullptr, "GROUP BY");
}

// ---------------------------------------------------------------------------
// GROUP BY that allocates nothing (bolt_groupby_noalloc)
// ---------------------------------------------------------------------------
// Some callers may not allocate device memory at all: an engine whose own
// pool allocator owns every byte of HBM (a stray cudaMalloc there fails or
// fragments the pool), or a latency-critical loop in which cudaMalloc /
// cudaFree would synchronise the whole device. They cannot create a
// bolt_ctx, whose scratch arena is one cudaMalloc. bolt_groupby_noalloc
// serves them for small group counts: the hash table, the group counters and
// the finalize descriptor live in the fixed array below, which every GPU that
// loads this library holds until the process exits.
//
// In host code the array's name is only a stand-in for it, so the device
// address is resolved with cudaGetSymbolAddress: on the first call on each
// device, with that device current. Make that first call before any stream
// capture. Every call reuses the same array and clears the part that must
// start at zero, so calls that overlap on the GPU (different streams or
// host threads) race on it and corrupt each other: serialise them.
constexpr uint64_t NOALLOC_SCRATCH_BYTES = 2ull << 20;  // 2 MiB
constexpr uint64_t NOALLOC_MAX_SLOTS = 8192;            // table slots -> at most 6144 groups
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

namespace {

std::mutex g_noalloc_mu;
unsigned char* g_noalloc_addr[NOALLOC_MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on `dev`, which must be current.
bool noalloc_scratch(int dev, unsigned char** out) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return false;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return false;
        g_noalloc_addr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_noalloc_addr[dev];
    return true;
}

}  // namespace

extern "C" bolt_status bolt_groupby_noalloc(const bolt_groupby_desc* desc, bolt_groupby_out* out,
                                            bolt_stream stream, char* err, int32_t err_cap) {
    auto report = [&](bolt_status st, const char* msg) {
        if (err && err_cap > 0) std::snprintf(err, (size_t)err_cap, "%s", msg);
        return st;
    };
    if (!desc || !out) return report(BOLT_ERR_INVALID, "bolt_groupby_noalloc: null descriptor or output");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: no current device");
    unsigned char* base = nullptr;
    if (!noalloc_scratch(dev, &base))
        return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: cudaGetSymbolAddress of the static scratch failed");
    cudaStream_t s = (cudaStream_t)stream;

    // A host-only context: device attributes for the planner and a place for
    // its error text; it owns no device memory.
    bolt_ctx c;
    c.device = dev;
    if (cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&c.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
        return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: device attribute query failed");
    // Scratch layout: [0, 256) status word and counters, then the finalize
    // descriptor, then the hash table.
    ull* words = reinterpret_cast<ull*>(base);
    GbFinal* d_final = reinterpret_cast<GbFinal*>(base + 256);
    ull* table = reinterpret_cast<ull*>(base + 256 + ((sizeof(GbFinal) + 255) & ~size_t(255)));
    const uint64_t table_room = NOALLOC_SCRATCH_BYTES - (uint64_t)(reinterpret_cast<unsigned char*>(table) - base);

    uint64_t nrows = 0;
    if (desc->n_keys >= 1 && desc->key_cols && desc->cols && desc->key_cols[0] >= 0 && desc->key_cols[0] < desc->n_cols)
        nrows = desc->cols[desc->key_cols[0]].len;
    // Table slots: twice the hint (clamped before doubling), at most the
    // array's 8192; without a hint the largest table.
    const uint64_t hint = desc->groups_hint;
    const uint64_t want =
        (hint == 0 || hint >= NOALLOC_MAX_SLOTS) ? NOALLOC_MAX_SLOTS : 1ull << ceil_log2_u64(2 * hint + 16);
    uint64_t cap = std::max<uint64_t>(64, std::min<uint64_t>(want, NOALLOC_MAX_SLOTS));
    int mode = 0;
    // Up to three table sizes (x8 each, capped) and two accumulator-mode
    // switches can combine.
    for (int attempt = 0; attempt < 8; ++attempt) {
        GbPlan pl;
        bolt_status st = gb_plan(&c, desc, out, 0, nrows, BOLT_FLAG_NO_TUNE, mode, cap, &pl);
        if (st != BOLT_OK) return report(st, c.last_error.c_str());
        const uint64_t table_bytes = (pl.cap + 2) * (uint64_t)pl.prm.slot_words * 8;
        if (table_bytes > table_room)
            return report(BOLT_ERR_CAPACITY,
                          "bolt_groupby_noalloc: the hash table for this aggregate list exceeds the 2 MiB static scratch");
        GbParams& p = pl.prm;
        GbFinal& f = pl.fin;
        p.gtab = table;
        p.status = reinterpret_cast<uint32_t*>(words);
        p.occupancy = words + 1;
        p.i64_bits = nullptr;
        for (int s2 = 0; s2 < p.n_st; ++s2)
            if (p.st[s2].kind == K_SUM_I64) p.i64_bits = reinterpret_cast<uint32_t*>(words + 4);
        f.gtab = table;
        f.status = p.status;
        f.n_nonnull = words + 2;
        f.n_groups = words + 3;
        f.n_groups_user = nullptr;
        // The previous call left its table and counters in the array.
        if (cudaMemsetAsync(words, 0, 256, s) != cudaSuccess || cudaMemsetAsync(table, 0, table_bytes, s) != cudaSuccess)
            return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: clearing the static scratch failed");
        if (cudaMemcpyAsync(d_final, &f, sizeof(GbFinal), cudaMemcpyHostToDevice, s) != cudaSuccess)
            return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: descriptor upload failed");
        const size_t smem = (size_t)pl.smem_entries * 8ull * (size_t)p.sslot_words;
        const uint64_t tile = (uint64_t)pl.block * pl.u;
        const uint64_t tiles = (p.n_rows + tile - 1) / tile;
        const unsigned grid = (unsigned)std::min<uint64_t>((uint64_t)c.num_sms, std::max<uint64_t>(tiles, 1));
        if (p.n_rows > 0) {
            const AggKernel kfn = agg_kernel_for(p.spec, p.n_st);
            if (smem_optin(kfn, &c) != cudaSuccess)
                return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: shared-memory attribute failed");
            kfn<<<grid, pl.block, smem, s>>>(p);
            if (cudaGetLastError() != cudaSuccess)
                return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: aggregation launch failed");
        }
        const size_t fsm = small_final_smem(pl.cap);
        if (smem_optin(gb_small_final_kernel, &c) != cudaSuccess)
            return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: shared-memory attribute failed");
        gb_small_final_kernel<<<1, SF_BLOCK, fsm, s>>>(d_final);
        if (cudaGetLastError() != cudaSuccess) return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: finalize launch failed");
        ull w[5] = {0, 0, 0, 0, 0};
        if (cudaMemcpyAsync(w, words, sizeof w, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: kernel or readback failed");
        const uint32_t fl = (uint32_t)w[0];
        out->n_groups = w[3];
        if (fl & (ST_FLAG_GROW | ST_FLAG_SPILL)) {
            // More groups than the hint: a larger table while the array has room.
            if (pl.cap < NOALLOC_MAX_SLOTS) {
                cap = std::min<uint64_t>(pl.cap * 8, NOALLOC_MAX_SLOTS);
                continue;
            }
            return report(BOLT_ERR_CAPACITY,
                          "bolt_groupby_noalloc: more than 6144 groups (8192-slot table limit); use bolt_groupby");
        }
        if (fl & (ST_FLAG_RANGE | ST_FLAG_DECRANGE)) {
            if (fl & ST_FLAG_RANGE) mode |= GB_MODE_F64_ATOMIC;
            if (fl & ST_FLAG_DECRANGE) mode |= GB_MODE_WIDE_DEC;
            continue;
        }
        if (fl & ST_FLAG_DECOVERFLOW)
            return report(BOLT_ERR_OVERFLOW, "SUM(Decimal128) precision overflow: accumulator exceeds i128 range");
        if (fl & ST_FLAG_OVERFLOW)
            return report(BOLT_ERR_OVERFLOW, "SUM(integer) overflow: accumulator exceeds i64 range");
        if (fl & ST_FLAG_CAPACITY) return report(BOLT_ERR_CAPACITY, "bolt_groupby_noalloc: output capacity exceeded");
        if (fl) return report(BOLT_ERR_CUDA, "bolt_groupby_noalloc: unexpected device status");
        if (p.i64_bits && (uint32_t)w[4] + (uint32_t)ceil_log2_u64(p.n_rows + 1) >= 63)
            return report(BOLT_DECLINE, "bolt_groupby_noalloc: SUM(Int64) inputs large enough to need the row-order "
                                        "overflow check; use bolt_groupby");
        if (err && err_cap > 0) err[0] = 0;
        return BOLT_OK;
    }
    return report(BOLT_ERR_CAPACITY, "bolt_groupby_noalloc: table growth and accumulator mode retries did not converge");
}

// Fused probe -> GROUP BY <build payload>: the GROUP BY kernel with a join
// lookup as its key source; the joined rows are never materialised.
extern "C" bolt_status bolt_join_groupby(bolt_ctx* ctx, const bolt_join_table* t, const bolt_col_view* probe_key,
                                         const bolt_col_view* value, bolt_col_mut* out_group, bolt_col_mut* out_sum,
                                         bolt_col_mut* out_count, uint64_t* n_groups, uint32_t flags,
                                         bolt_stream stream) {
    if (!ctx) return BOLT_ERR_INVALID;
    if (!t || !probe_key || !value || !out_group || !out_sum || !out_count || !n_groups)
        return fail(ctx, BOLT_ERR_INVALID, "join GROUP BY: bad arguments");
    if (!t->has_payload) return fail(ctx, BOLT_ERR_INVALID, "join GROUP BY: the table was built without a payload");
    if (t->multi)  // one aggregation row per probe row: a key with several build rows does not fit
        return fail(ctx, BOLT_DECLINE, "join GROUP BY: duplicate build keys");
    if (probe_key->dtype != BOLT_I32 && probe_key->dtype != BOLT_I64)
        return fail(ctx, BOLT_DECLINE, "join GROUP BY: probe key dtype %d", probe_key->dtype);
    if (value->len != probe_key->len) return fail(ctx, BOLT_ERR_INVALID, "join GROUP BY: column lengths differ");
    if (!col_aligned(probe_key->data, probe_key->dtype))
        return fail(ctx, BOLT_ERR_INVALID, "join GROUP BY: probe key is not aligned to its element width");
    // Column 0 stands for the group key (its data is never read in join mode).
    bolt_col_view cols[2] = {*probe_key, *value};
    cols[0].dtype = BOLT_I32;
    cols[0].validity = nullptr;
    const int32_t key_cols[1] = {0};
    const bolt_agg_spec aggs[2] = {{BOLT_AGG_SUM, 1}, {BOLT_AGG_COUNT_STAR, -1}};
    bolt_groupby_desc d{};
    d.cols = cols;
    d.n_cols = 2;
    d.key_cols = key_cols;
    d.n_keys = 1;
    d.aggs = aggs;
    d.n_aggs = 2;
    // Sized for up to 1024 groups: the table (8192 slots) then finalizes in one
    // CTA; more groups grow it through the retry.
    d.groups_hint = std::min<uint64_t>(std::max<uint64_t>(t->n_build, 1), 1024);
    bolt_col_mut agg_out[2] = {*out_sum, *out_count};
    bolt_groupby_out o{};
    o.keys = out_group;
    o.aggs = agg_out;
    bolt_status st = gb_single(ctx, &d, &o, 0, probe_key->len, flags, (cudaStream_t)stream, t, probe_key,
                               "join GROUP BY");
    *n_groups = o.n_groups;
    return st;
}

// Many filter + GROUP BY queries: one persistent aggregation launch and one
// batched finalize for the whole batch; queries that need a bigger table or
// another accumulator mode are re-run alone afterwards.
extern "C" bolt_status bolt_batch_groupby(bolt_ctx* ctx, bolt_query* qs, int32_t n, uint32_t flags,
                                          bolt_stream stream) {
    if (!ctx) return BOLT_ERR_INVALID;
    if (!qs || n < 0) return fail(ctx, BOLT_ERR_INVALID, "batched GROUP BY: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    bolt_status st = call_begin(ctx, flags, s);
    if (st != BOLT_OK) return st;
    std::vector<GbPlan> plans(n);
    std::vector<GbPlan*> run;
    std::vector<int> idx;
    for (int i = 0; i < n; ++i) {
        bolt_query& q = qs[i];
        q.status = gb_plan(ctx, &q.desc, &q.out, q.row_begin, q.row_end, flags, 0, 0, &plans[i]);
        if (q.status != BOLT_OK) continue;
        plans[i].fin.n_groups_user = (ull*)q.out.n_groups_dev;
        run.push_back(&plans[i]);
        idx.push_back(i);
    }
    st = gb_run(ctx, run.data(), (int)run.size(), s, flags, true);
    if (st == BOLT_ERR_CAPACITY && run.size() > 1 && !(flags & BOLT_FLAG_ASYNC)) {
        // The batch's tables do not fit the arena together: run each query
        // alone (each call starts from an empty arena).
        BOLT_CUDA(ctx, cudaStreamSynchronize(s));
        ctx->last_error.clear();
        for (int i : idx)
            qs[i].status = gb_single(ctx, &qs[i].desc, &qs[i].out, qs[i].row_begin, qs[i].row_end,
                                     flags & ~(BOLT_FLAG_PROFILE | BOLT_FLAG_KERNEL_TIMES), s, nullptr, nullptr,
                                     "batched GROUP BY");
        for (int i = 0; i < n; ++i)
            if (qs[i].status != BOLT_OK)
                return fail(ctx, qs[i].status, "batched GROUP BY: query %d failed (%s)", i,
                            bolt_status_str(qs[i].status));
        return BOLT_OK;
    }
    if (st != BOLT_OK) return st;
    st = call_end(ctx, flags, s);
    if (st != BOLT_OK) return st;
    if (flags & BOLT_FLAG_ASYNC) return BOLT_OK;
    uint32_t gf = 0;
    st = read_status(ctx, s, 0, &gf);
    if (st != BOLT_OK) return st;
    if (gf & ST_FLAG_TIMEOUT) return flags_to_status(ctx, gf, "batched GROUP BY");
    const int m = (int)run.size();
    std::vector<ull> w((size_t)m * 8);
    if (m) BOLT_CUDA(ctx, cudaMemcpy(w.data(), run[0]->words, (size_t)m * 64, cudaMemcpyDeviceToHost));
    std::vector<int> redo;
    for (int j = 0; j < m; ++j) {
        bolt_query& q = qs[idx[j]];
        const uint32_t f = (uint32_t)w[(size_t)j * 8 + 3];
        q.out.n_groups = w[(size_t)j * 8 + 2];
        // Re-run alone: a bigger table or another accumulator mode, or a
        // SUM(Int64) whose row-order prefixes need the exact check.
        const bool i64_check = run[j]->prm.i64_bits &&
                               (uint32_t)w[(size_t)j * 8 + 4] + (uint32_t)ceil_log2_u64(run[j]->prm.n_rows + 1) >= 63;
        if ((f & (ST_FLAG_GROW | ST_FLAG_SPILL | ST_FLAG_RANGE | ST_FLAG_DECRANGE)) || (f == 0 && i64_check)) {
            redo.push_back(idx[j]);
            continue;
        }
        if (f & ST_FLAG_DECOVERFLOW) q.status = BOLT_ERR_OVERFLOW;
        else if (f & ST_FLAG_OVERFLOW) q.status = BOLT_ERR_OVERFLOW;
        else if (f & ST_FLAG_TIMEOUT) q.status = BOLT_ERR_TIMEOUT;
        else if (f & ST_FLAG_CAPACITY) q.status = BOLT_ERR_CAPACITY;
        else q.status = BOLT_OK;
    }
    for (int i : redo) {
        bolt_query& q = qs[i];
        q.status = gb_single(ctx, &q.desc, &q.out, q.row_begin, q.row_end,
                             flags & ~(BOLT_FLAG_PROFILE | BOLT_FLAG_KERNEL_TIMES), s, nullptr, nullptr,
                             "batched GROUP BY");
    }
    ctx->last_error.clear();
    for (int i = 0; i < n; ++i)
        if (qs[i].status != BOLT_OK)
            return fail(ctx, qs[i].status, "batched GROUP BY: query %d failed (%s)", i, bolt_status_str(qs[i].status));
    return BOLT_OK;
}

// ---------------------------------------------------------------------------
// Autotuner
// ---------------------------------------------------------------------------
extern "C" bolt_status bolt_groupby_autotune(bolt_ctx* ctx, const bolt_groupby_desc* desc, bolt_groupby_out* out,
                                             bolt_stream stream, double* best_ms) {
    if (!ctx || !desc || !out) return BOLT_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t nrows = 0;
    if (desc->n_keys >= 1 && desc->key_cols && desc->cols && desc->key_cols[0] >= 0 && desc->key_cols[0] < desc->n_cols)
        nrows = desc->cols[desc->key_cols[0]].len;
    // A plain run first: it settles the table size and accumulator modes.
    bolt_status st = gb_single(ctx, desc, out, 0, nrows, BOLT_FLAG_NO_TUNE, s, nullptr, nullptr, "GROUP BY autotune");
    if (st != BOLT_OK) return st;
    std::vector<bolt_ctx::GbTune> cands;
    for (int block : {256, 512})
        for (int smem_shift : {0, 1, 8})
            for (int warp_agg : {0, 1})
                for (int load_shift : {0, 1, 2})
                    for (int smem_fill : {4, 6}) {
                        if (smem_shift == 8 && smem_fill != 4) continue;  // no shared tier: the fill is moot
                        cands.push_back({block, smem_shift, warp_agg, load_shift, smem_fill, 0, 0.0});
                    }
    for (int staged : {1, 2, 4})
        for (int smem_shift : {0, 1})
            for (int warp_agg : {0, 1})
                for (int load_shift : {0, 1, 2})
                    for (int smem_fill : {2, 3, 4, 6}) cands.push_back({512, smem_shift, warp_agg, load_shift, smem_fill, staged, 0.0});
    // The hash-partitioned tier, with two admission caps of its shared table.
    for (int smem_fill : {3, 4}) {
        bolt_ctx::GbTune c{512, 0, 0, 1, smem_fill, 2, 0.0};
        c.part = 1;
        cands.push_back(c);
    }
    bolt_ctx::GbTune best{512, 1, 0, 1, 4, 0, 1e30};
    const bool verbose = std::getenv("BOLT_TUNE_VERBOSE") != nullptr;
    uint64_t shape = 0;
    for (auto& c : cands) {
        double tot = 0.0;
        bool ok = true;
        for (int rep = 0; rep < 3 && ok; ++rep) {
            st = call_begin(ctx, 0, s);
            if (st != BOLT_OK) return st;
            GbPlan pl;
            st = gb_plan(ctx, desc, out, 0, nrows, 0, 0, 0, &pl, &c);
            if (st != BOLT_OK) return st;
            shape = pl.shape;
            if (c.part ? !gb_part_applies(ctx, pl, BOLT_FLAG_FORCE_PART)
                       : (c.staged && !gb_staged_layout(ctx, pl, nullptr))) {
                ok = false;  // the candidate's kernels do not apply to this query
                break;
            }
            BOLT_CUDA(ctx, cudaEventRecord(ctx->ev0, s));
            GbPlan* one = &pl;
            st = c.part ? gb_run_part(ctx, &pl, s, 0, 0) : gb_run(ctx, &one, 1, s, 0);
            if (st == BOLT_DECLINE || st == BOLT_ERR_CAPACITY) {
                ctx->last_error.clear();
                ok = false;
                break;
            }
            if (st != BOLT_OK) return st;
            BOLT_CUDA(ctx, cudaEventRecord(ctx->ev1, s));
            uint32_t f = 0;
            st = read_status(ctx, s, 0, &f);
            if (st != BOLT_OK) return st;
            if (f) {
                ok = false;  // this candidate spilled / flagged: not eligible
                break;
            }
            float ms = 0.f;
            BOLT_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            if (rep > 0) tot += ms;  // first repetition warms up
        }
        if (verbose)
            std::fprintf(stderr,
                         "[bolt autotune] block=%d smem_shift=%d warp_agg=%d load_shift=%d smem_fill=%d/8 staged=%d "
                         "part=%d -> %s%.4f ms\n",
                         c.block, c.smem_shift, c.warp_agg, c.load_shift, c.smem_fill, c.staged, c.part,
                         ok ? "" : "(not eligible) ", tot / 2);
        if (ok && tot / 2 < best.ms) {
            best = c;
            best.ms = tot / 2;
        }
    }
    if (best.ms < 1e29) ctx->tune[shape] = best;
    if (best_ms) *best_ms = best.ms;
    // Leave `out` holding the result of the tuned configuration.
    return gb_single(ctx, desc, out, 0, nrows, 0, s, nullptr, nullptr, "GROUP BY autotune");
}

extern "C" bolt_status bolt_ctx_tuning_save(const bolt_ctx* ctx, const char* path) {
    if (!ctx || !path) return BOLT_ERR_INVALID;
    FILE* fp = std::fopen(path, "w");
    if (!fp) return BOLT_ERR_INVALID;
    for (const auto& kv : ctx->tune)
        std::fprintf(fp, "%llx %d %d %d %d %d %d %.6f %d\n", (unsigned long long)kv.first, kv.second.block,
                     kv.second.smem_shift, kv.second.warp_agg, kv.second.load_shift, kv.second.smem_fill,
                     kv.second.staged, kv.second.ms, kv.second.part);
    std::fclose(fp);
    return BOLT_OK;
}

extern "C" bolt_status bolt_ctx_tuning_load(bolt_ctx* ctx, const char* path) {
    if (!ctx || !path) return BOLT_ERR_INVALID;
    FILE* fp = std::fopen(path, "r");
    if (!fp) return fail(ctx, BOLT_ERR_INVALID, "tuning file %s not readable", path);
    unsigned long long key;
    char line[256];
    // One shape per line; the tier column (part) is optional (older files).
    while (std::fgets(line, sizeof line, fp)) {
        bolt_ctx::GbTune t{};
        const int got = std::sscanf(line, "%llx %d %d %d %d %d %d %lf %d", &key, &t.block, &t.smem_shift, &t.warp_agg,
                                    &t.load_shift, &t.smem_fill, &t.staged, &t.ms, &t.part);
        if (got < 8) continue;
        if (got == 8) t.part = 0;
        const bool valid = (t.part == 0 || t.part == 1) && (t.block == 256 || t.block == 512) && t.smem_shift >= 0 &&
                           t.smem_shift <= 8 && (t.warp_agg == 0 || t.warp_agg == 1) && t.load_shift >= 0 &&
                           t.load_shift <= 3 && t.smem_fill >= 1 && t.smem_fill <= 8 &&
                           (t.staged == 0 || t.staged == 1 || t.staged == 2 || t.staged == 4);
        if (valid) ctx->tune[(uint64_t)key] = t;
    }
    std::fclose(fp);
    return BOLT_OK;
}

