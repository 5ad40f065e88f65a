// groupby_part.cu — the hash-partitioned tier of GROUP BY for sm_100a.
//
// Serves the queries whose groups far outnumber a CTA's shared-memory table
// (the reference's Tier-2: partition -> scatter -> per-partition
// shared-memory reduce, groupby_tier2_orchestrator.rs:214-534,
// partition_kernel.rs:86, partition_reduce_kernel.rs:241; there the
// partition counts make a host round trip and a spilling partition
// recomputes the query). Five launches, no host round trip:
//
//  A  gb_spill_kernel        streams the columns once through bulk copies into
//                            shared memory (producer warp), evaluates WHERE and
//                            folds every surviving row whose key is in the
//                            CTA's shared table (the frequent keys under skew).
//                            A row whose key is not there is appended to the
//                            CTA's own spill segment (key + raw value words,
//                            column-wise, coalesced stores): the streaming
//                            kernel never waits on a global-memory round trip.
//                            At exit the shared table is written out as
//                            partial-state records with their partition counts.
//  B1 gb_part_count_kernel   per segment, the rows of every hash partition.
//  S  gb_part_scan_kernel    per partition, the offsets of every segment's
//                            records (exclusive prefix over segments); the
//                            last CTA scans the partition totals.
//  B2 gb_part_scatter_kernel each CTA moves its segment's rows to their
//                            partitions' ranges as aligned 32-byte records (one
//                            whole DRAM sector each) and its partial records.
//  C  gb_part_reduce_kernel  one partition at a time per CTA: folds its
//                            partial records and rows into a shared-memory
//                            table, then writes each group once, densely, into
//                            the compact group array with its sort key. A
//                            partition with more groups than the table flags a
//                            spill and the host re-plans with more partitions.
//
// The finalize (radix sort of the group keys + typed output columns) is the
// one of the global-table path. Every aggregate state is integer-exact or a
// max, so the order in which rows reach a group does not change any result.
#include "groupby_part.cuh"
#include "gb_device.cuh"
#include "bulk.cuh"

#include <algorithm>

namespace bolt {
namespace {

constexpr ull HASH_P = HASH_G;  // partition hash (HASH_S indexes the tables)
constexpr int PART_MAX_STAGES = 6;
constexpr int REC_WORDS = 4;    // a spilled row in partition order: key + 3 value words

__device__ __forceinline__ uint32_t part_of(ull stored, int pbits) {
    return (uint32_t)((stored * HASH_P) >> (64 - pbits));
}

// Column bases of one tile: in shared memory for a staged tile, in global
// memory for the tail rows. Computed once per tile, not per row.
struct TileCols {
    const unsigned char* pc;  // WHERE column (Int32)
    const unsigned char* k0;
    const unsigned char* k1;
    const unsigned char* f[GB_PART_MAX_FIELDS];
};

__device__ __forceinline__ TileCols tile_cols(const GbParams& p, const GbPart& q, const unsigned char* stage,
                                              bool staged, uint64_t tile_row0) {
    auto col = [&](int c) -> const unsigned char* {
        if (c < 0) return nullptr;
        return staged ? stage + p.sc_off[c]
                      : static_cast<const unsigned char*>(p.sc_col[c]) + (p.row_begin + tile_row0) * (uint64_t)p.sc_w[c];
    };
    TileCols t;
    t.pc = q.has_pred ? col(p.pr_sc[0]) : nullptr;
    t.k0 = col(p.k_sc[0]);
    t.k1 = p.n_keys > 1 ? col(p.k_sc[1]) : nullptr;
#pragma unroll
    for (int f = 0; f < GB_PART_MAX_FIELDS; ++f) t.f[f] = f < q.n_fields ? col(q.field_sc[f]) : nullptr;
    return t;
}

// Packed, complemented key of row i (compile-time key layout).
template <int KP>
__device__ __forceinline__ ull stored_key(const TileCols& t, uint32_t i) {
    if constexpr (KP == GB_KP_I32X2) {
        const uint32_t a = reinterpret_cast<const uint32_t*>(t.k0)[i];
        const uint32_t b = reinterpret_cast<const uint32_t*>(t.k1)[i];
        return ~(((ull)a << 32) | (ull)b);
    } else if constexpr (KP == GB_KP_I32) {
        return ~(ull)(ll)reinterpret_cast<const int32_t*>(t.k0)[i];
    } else {
        return ~reinterpret_cast<const ull*>(t.k0)[i];
    }
}

// Raw 64-bit image of value field f of row i: 64-bit values as they are,
// Int32 sign-extended, Float32 widened to a float64 bit pattern (raw_at).
__device__ __forceinline__ ull field_val(const GbPart& q, const TileCols& t, int f, uint32_t i) {
    if (q.field_w[f] == 8) return reinterpret_cast<const ull*>(t.f[f])[i];
    const int32_t v = reinterpret_cast<const int32_t*>(t.f[f])[i];
    return q.field_float[f] ? (ull)__double_as_longlong((double)__int_as_float(v)) : (ull)(ll)v;
}

// Contribution (c0, c1) of one value to a state of kind K (contribution()
// with the dtype test resolved to a flag; dense columns). K is a constant
// after the state loop is unrolled, so the switch folds away.
__device__ __forceinline__ void contrib_of(const GbParams& p, int K, ull raw, bool fl, ull& c0, ull& c1,
                                           uint32_t& absbits) {
    c0 = 0;
    c1 = 0;
    switch (K) {
    case K_COUNT: c0 = 1; break;
    case K_SUM_I32: c0 = raw; break;
    case K_SUM_I64: {
        c0 = raw & 0xFFFFFFFFull;
        c1 = (ull)((ll)raw >> 32);
        const ll v = (ll)raw;
        const ull a = v < 0 ? (ull)(-(v + 1)) + 1ull : (ull)v;
        const uint32_t b = a ? 64u - (uint32_t)__clzll((ll)a) : 0u;
        absbits = b > absbits ? b : absbits;
        break;
    }
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
    case K_MAX_ORD: c0 = fl ? f64_order_key(__longlong_as_double((ll)raw)) : raw ^ 0x8000000000000000ull; break;
    case K_MIN_ORD: c0 = ~(fl ? f64_order_key(__longlong_as_double((ll)raw)) : raw ^ 0x8000000000000000ull); break;
    default: break;
    }
}

// All states of one row, from its field words.
template <class SP>
__device__ __forceinline__ void row_contrib(const GbParams& p, const GbPart& q, const ull* fw, ull* c0, ull* c1,
                                            uint32_t& absbits) {
#pragma unroll
    for (int s = 0; s < SP::n; ++s) {
        // (selected by comparison: a runtime index would put fw in local memory)
        const int f = q.field_of_state[s];
        const ull raw = f == 0 ? fw[0] : f == 1 ? fw[1] : f == 2 ? fw[2] : 0ull;
        contrib_of(p, SP::kind(s), raw, q.state_float[s] != 0, c0[s], c1[s], absbits);
    }
}

// What the streaming kernel does with a surviving row whose key is not in
// the CTA's shared table.
constexpr int MISS_SPILL = 0;   // append it to the CTA's spill segment (partitioned tier)
constexpr int MISS_GLOBAL = 1;  // fold it into the global hash table (global-table tier)

// Absent-key filter: one bit per hash of every key admitted to the CTA's
// shared table. Once the table admits no more keys, a row whose bit is clear
// is a miss without a probe (most misses under skew). A bit set after a
// concurrent lookup read it clear only sends that row down the miss path,
// which is correct for every row.
constexpr int FILT_WORDS = 2048;  // 65,536 bits, 8 KB

// Per-warp state of the streaming consumer.
struct LeanWarp {
    uint32_t absbits;  // largest |v| bit length fed to an Int64 SUM
    uint32_t inserts;  // new global-table keys (MISS_GLOBAL), not yet counted
    uint32_t pending;  // ... counted per warp, not yet published
    // Survivors carried to the next tile so that every fold step has 32
    // rows: lanes below npend hold a row (key + value words, loaded).
    uint32_t npend;
    ull pstored;
    ull pfw[GB_PART_MAX_FIELDS];
};

// Key and value words of row i.
template <int KP>
__device__ __forceinline__ void load_row(const GbPart& q, const TileCols& t, uint32_t i, ull& stored,
                                         ull (&fw)[GB_PART_MAX_FIELDS]) {
    stored = stored_key<KP>(t, i);
#pragma unroll
    for (int f = 0; f < GB_PART_MAX_FIELDS; ++f) fw[f] = f < q.n_fields ? field_val(q, t, f, i) : 0ull;
}

// Shared-table find-or-insert from a precomputed home slot; an admitted key
// sets its filter bit. -1 when the key is absent and the table admits no
// more keys (or the probe window ends).
__device__ __forceinline__ int hot_find_insert(ull* sk, uint32_t mask, uint32_t h, ull stored, uint32_t* fill,
                                               uint32_t limit, uint32_t* filt, uint32_t fb) {
    volatile ull* vk = sk;
    for (int i = 0; i < SMEM_PROBES; ++i) {
        const ull k = vk[h];
        if (k == stored) return (int)h;
        if (k == 0) {
            if (*reinterpret_cast<volatile uint32_t*>(fill) >= limit) return -1;
            const ull old = atomicCAS(&sk[h], 0ull, stored);
            if (old == 0) {
                atomicAdd(fill, 1u);
                atomicOr(&filt[fb >> 5], 1u << (fb & 31));
                return (int)h;
            }
            if (old == stored) return (int)h;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

// One warp step: up to 32 rows (lane's row valid when has) folded into the
// CTA's shared table, the misses handled per MISS.
template <class SP, int MISS>
__device__ __forceinline__ void fold_step(const GbParams& p, const GbPart& q, ull* sk, ull* sw, uint32_t* fill,
                                          uint32_t* filt, uint32_t* s_nspill, uint32_t* s_stop, bool has, ull stored,
                                          const ull (&fw)[GB_PART_MAX_FIELDS], LeanWarp& lw) {
    const uint32_t lane = lane_id();
    const int SW = p.sslot_words - 1;
    // The key whose complement is 0 keeps its own slot of the group table.
    if (has && stored == 0) {
        ull c0[SP::n], c1[SP::n];
        row_contrib<SP>(p, q, fw, c0, c1, lw.absbits);
        ull* w = p.gtab + (1ull << p.log2cap) * (ull)p.slot_words;
        if (ld_volatile(w) == 0) *reinterpret_cast<volatile ull*>(w) = 1ull;
#pragma unroll
        for (int s = 0; s < SP::n; ++s) merge_words(w + p.st[s].word, SP::kind(s), c0[s], c1[s]);
        has = false;
    }
    int sl = -1;
    if (has) {
        const ull hp = stored * HASH_S;
        const uint32_t fb = (uint32_t)hp >> 16;
        const bool maybe = (filt[fb >> 5] >> (fb & 31)) & 1u;
        if (maybe || *reinterpret_cast<volatile uint32_t*>(fill) < p.smem_fill)
            sl = hot_find_insert(sk, (1u << p.smem_log2) - 1, (uint32_t)(hp >> (64 - p.smem_log2)), stored, fill,
                                 p.smem_fill, filt, fb);
    }
    if (sl >= 0) {
        ull c0[SP::n], c1[SP::n];
        row_contrib<SP>(p, q, fw, c0, c1, lw.absbits);
        ull* w = sw + (ull)sl * SW - 1;
#pragma unroll
        for (int s = 0; s < SP::n; ++s) merge_words_smem(w + p.st[s].sword, SP::kind(s), c0[s], c1[s], true);
    }
    const bool miss = has && sl < 0;
    if constexpr (MISS == MISS_GLOBAL) {
        if (miss) {
            const int64_t g = g_find_insert(p, stored, lw.inserts);
            if (g >= 0) {
                ull c0[SP::n], c1[SP::n];
                row_contrib<SP>(p, q, fw, c0, c1, lw.absbits);
                ull* w = p.gtab + (ull)g * p.slot_words;
#pragma unroll
                for (int s = 0; s < SP::n; ++s) merge_words(w + p.st[s].word, SP::kind(s), c0[s], c1[s]);
            }
        }
    } else {
        const uint32_t mm = __ballot_sync(0xffffffffu, miss);
        if (mm == 0) return;
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(s_nspill, (uint32_t)__popc(mm));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (!miss) return;
        const uint64_t pos = (uint64_t)base + __popc(mm & lanemask_lt());
        if (pos >= q.seg_stride) {  // the segment is full: the host re-plans
            atomicOr(p.status, ST_FLAG_SPILL);
            *reinterpret_cast<volatile uint32_t*>(s_stop) = 1u;
            return;
        }
        const uint64_t at = (uint64_t)blockIdx.x * q.seg_stride + pos;
        q.skey[at] = stored;
#pragma unroll
        for (int f = 0; f < GB_PART_MAX_FIELDS; ++f)
            if (f < q.n_fields) q.sfield[f][at] = fw[f];
    }
}

// Filters the rows [first, first + 32 * nchunks) of a tile (tile-relative,
// below `limit`) into the warp's list with a range test on the WHERE column,
// then folds the survivors in steps of 32: the rows carried from earlier
// tiles fill the first step, and the survivors that would leave the last
// step part-empty are carried on (loaded into registers, so the stage can
// be released).
template <int KP, class SP, int MISS>
__device__ __forceinline__ void lean_rows(const GbParams& p, const GbPart& q, ull* sk, ull* sw, uint32_t* fill,
                                          uint32_t* filt, uint32_t* s_nspill, uint32_t* s_stop, const TileCols& t,
                                          uint32_t first, int nchunks, uint32_t limit, uint16_t* list, LeanWarp& lw) {
    const uint32_t lane = lane_id();
    uint32_t cnt = 0;
    const int32_t* pc = reinterpret_cast<const int32_t*>(t.pc);
    for (int c = 0; c < nchunks; ++c) {
        const uint32_t i = first + (uint32_t)c * 32u + lane;
        bool ok = i < limit;
        if (pc && ok) {
            const int32_t v = pc[i];
            ok = ((v >= q.pred_lo) & (v <= q.pred_hi)) != (q.pred_neg != 0);
        }
        const uint32_t m = __ballot_sync(0xffffffffu, ok);
        if (ok) list[cnt + __popc(m & lanemask_lt())] = (uint16_t)(i - first);
        cnt += __popc(m);
    }
    __syncwarp();
    uint32_t b = 0;  // survivors of this tile already taken
    while (lw.npend + (cnt - b) >= 32) {
        ull stored, fw[GB_PART_MAX_FIELDS];
        if (lane < lw.npend) {
            stored = lw.pstored;
#pragma unroll
            for (int f = 0; f < GB_PART_MAX_FIELDS; ++f) fw[f] = lw.pfw[f];
        } else {
            load_row<KP>(q, t, first + list[b + lane - lw.npend], stored, fw);
        }
        fold_step<SP, MISS>(p, q, sk, sw, fill, filt, s_nspill, s_stop, true, stored, fw, lw);
        b += 32 - lw.npend;
        lw.npend = 0;
    }
    const uint32_t left = cnt - b;
    if (lane >= lw.npend && lane < lw.npend + left)
        load_row<KP>(q, t, first + list[b + lane - lw.npend], lw.pstored, lw.pfw);
    lw.npend += left;
    __syncwarp();
}

// The streaming kernel (pass A of the partitioned tier with MISS_SPILL; the
// global-table tier's aggregation with MISS_GLOBAL). Warp 0's lane 0
// streams tiles of every staged column into a ring of stages (bulk copies
// completing on the stage's `full` mbarrier); the other warps filter, fold
// and handle misses, and release stages on `empty`. All waits are bounded.
// Shared memory: stages | table keys | table states | filter | per-warp
// survivor lists; with MISS_SPILL the stages hold the partial records'
// partition histogram after the ring has drained.
template <int KP, class SP, int MISS>
__global__ void __launch_bounds__(1024, 1) gb_lean_kernel(const __grid_constant__ GbParams p,
                                                          const __grid_constant__ GbPart q) {
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ __align__(8) uint64_t full[PART_MAX_STAGES], empty[PART_MAX_STAGES];
    __shared__ uint32_t s_fill, s_nspill, s_npart, s_stop;
    const int S = p.n_stages;
    const int NW = (int)(blockDim.x >> 5) - 1;
    const int warp = (int)(threadIdx.x >> 5);
    const uint32_t lane = lane_id();
    const int SW = p.sslot_words - 1;
    const int C = 1 << p.smem_log2;
    unsigned char* stages = dsm;
    ull* sk = reinterpret_cast<ull*>(dsm + (size_t)S * p.stage_bytes);
    ull* sw = sk + C;
    uint32_t* filt = reinterpret_cast<uint32_t*>(sw + (size_t)C * SW);
    uint16_t* lists = reinterpret_cast<uint16_t*>(filt + FILT_WORDS);
    const uint32_t T = p.tile_rows;
    const uint64_t ntiles = p.n_rows / T;

    for (int i = threadIdx.x; i < C * (SW + 1); i += blockDim.x) sk[i] = 0;
    for (int i = threadIdx.x; i < FILT_WORDS; i += blockDim.x) filt[i] = 0;
    if (threadIdx.x == 0) {
        s_fill = 0;
        s_nspill = 0;
        s_npart = 0;
        s_stop = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], (uint32_t)NW);
        }
        mbar_init_fence();
    }
    __syncthreads();

    LeanWarp lw{};
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
                if (*reinterpret_cast<volatile uint32_t*>(&s_stop)) {
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
            // Copies of the last (up to S) tiles may still be landing if a
            // consumer gave up early: wait for them before the CTA can exit.
            const uint32_t issued = j;
            for (uint32_t k = issued > (uint32_t)S ? issued - (uint32_t)S : 0u; k < issued; ++k)
                if (!mbar_wait(&full[k % (uint32_t)S], (k / (uint32_t)S) & 1u)) ok = false;
            if (!ok) {
                atomicOr(p.status, ST_FLAG_TIMEOUT);
                s_stop = 1u;
            }
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
                if (lane == 0) {
                    atomicOr(p.status, ST_FLAG_TIMEOUT);
                    *reinterpret_cast<volatile uint32_t*>(&s_stop) = 1u;
                }
                break;
            }
            const bool stop = *reinterpret_cast<volatile uint32_t*>(&s_stop) != 0;
            if (!stop) {
                const TileCols tc = tile_cols(p, q, stages + (size_t)st * p.stage_bytes, true, t * T);
                lean_rows<KP, SP, MISS>(p, q, sk, sw, &s_fill, filt, &s_nspill, &s_stop, tc,
                                        (uint32_t)cw * 32u * (uint32_t)p.chunks, p.chunks, T, list, lw);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[st]);
            if constexpr (MISS == MISS_GLOBAL) {
                // Occupancy of the global table; growth or a spill stops the CTA.
                if (gb_warp_epilogue(p, lw.inserts, lw.pending) && lane == 0)
                    *reinterpret_cast<volatile uint32_t*>(&s_stop) = 1u;
            }
        }
        // Rows after the last whole tile, 32 per consumer warp, from global memory.
        const uint64_t rem0 = ntiles * T;
        const uint32_t rem = (uint32_t)(p.n_rows - rem0);
        if (rem) {
            const TileCols tc = tile_cols(p, q, nullptr, false, rem0);
            for (uint32_t c = (uint32_t)(blockIdx.x * NW + cw) * 32u; c < rem; c += gridDim.x * (uint32_t)NW * 32u)
                lean_rows<KP, SP, MISS>(p, q, sk, sw, &s_fill, filt, &s_nspill, &s_stop, tc, c, 1, rem, list, lw);
        }
        // The rows still carried.
        if (lw.npend)
            fold_step<SP, MISS>(p, q, sk, sw, &s_fill, filt, &s_nspill, &s_stop, lane < lw.npend, lw.pstored,
                                lw.pfw, lw);
        if constexpr (MISS == MISS_GLOBAL) {
            lw.pending += __reduce_add_sync(0xffffffffu, lw.inserts);
            gb_warp_flush_pending(p, lw.pending);
        }
    }
    gb_flush_absbits(p, lw.absbits);
    __syncthreads();
    if constexpr (MISS == MISS_GLOBAL) {
        gb_flush_shared(p, sk, sw, C);
    } else {
        const uint32_t P = 1u << q.pbits;
        const uint32_t g = blockIdx.x;
        if (threadIdx.x == 0) q.n_spill[g] = (uint64_t)s_nspill < q.seg_stride ? s_nspill : (uint32_t)q.seg_stride;
        // The shared table as partial-state records (shared-table slot
        // layout), counted per partition in the (drained) stage memory.
        uint32_t* hist = reinterpret_cast<uint32_t*>(stages);
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) hist[i] = 0;
        __syncthreads();
        const int W = SW + 1;
        for (int i = threadIdx.x; i < C; i += blockDim.x) {
            const ull key = sk[i];
            if (key == 0) continue;
            const uint32_t pos = atomicAdd(&s_npart, 1u);  // pos < C
            ull* dst = q.ppart + ((uint64_t)g * q.hot_cap + pos) * (uint64_t)W;
            dst[0] = key;
            const ull* src = sw + (ull)i * SW;
            for (int k = 0; k < SW; ++k) dst[1 + k] = src[k];
            atomicAdd(&hist[part_of(key, q.pbits)], 1u);
        }
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) q.cnt_par[(uint64_t)g * P + i] = hist[i];
        if (threadIdx.x == 0) q.n_part[g] = s_npart;
    }
}

// Pass B1. CTA g counts segment g's rows per partition.
__global__ void __launch_bounds__(1024) gb_part_count_kernel(const __grid_constant__ GbPart q) {
    extern __shared__ uint32_t hist[];
    const uint32_t P = 1u << q.pbits;
    const uint32_t g = blockIdx.x;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) hist[i] = 0;
    __syncthreads();
    const uint32_t n = q.n_spill[g];
    const ull* keys = q.skey + (uint64_t)g * q.seg_stride;
    constexpr int U = 4;
    for (uint32_t b = threadIdx.x; b < n; b += blockDim.x * U) {
        ull k[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = b + (uint32_t)u * blockDim.x;
            k[u] = i < n ? __ldcg(keys + i) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            if (b + (uint32_t)u * blockDim.x < n) atomicAdd(&hist[part_of(k[u], q.pbits)], 1u);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) q.cnt_raw[(uint64_t)g * P + i] = hist[i];
}

// Scan S. Thread p: exclusive prefix over segments of partition p's counts;
// the last CTA to finish turns the partition totals into range starts.
__global__ void __launch_bounds__(256) gb_part_scan_kernel(const __grid_constant__ GbPart q) {
    __shared__ uint32_t s_last;
    __shared__ uint32_t s_warp[2][8];
    const uint32_t P = 1u << q.pbits;
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < P) {
        uint32_t ar = 0, ap = 0;
        for (int g = 0; g < q.grid_a; ++g) {
            const uint64_t i = (uint64_t)g * P + p;
            const uint32_t cr = q.cnt_raw[i], cp = q.cnt_par[i];
            q.rel_raw[i] = ar;
            q.rel_par[i] = ap;
            ar += cr;
            ap += cp;
        }
        q.base_raw[p] = ar;  // totals for now
        q.base_par[p] = ap;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(q.done, 1u) == gridDim.x - 1 ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // Exclusive scan of the P totals (two arrays) by this CTA, 256 threads,
    // P / 256 consecutive entries per thread.
    const uint32_t per = (P + blockDim.x - 1) / blockDim.x;
    const uint32_t b0 = threadIdx.x * per, b1 = min(P, b0 + per);
    uint32_t sr = 0, sp = 0;
    for (uint32_t i = b0; i < b1; ++i) {
        sr += __ldcg(q.base_raw + i);
        sp += __ldcg(q.base_par + i);
    }
    const uint32_t lane = lane_id(), w = threadIdx.x >> 5;
    uint32_t ir = sr, ip = sp;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t xr = __shfl_up_sync(0xffffffffu, ir, d), xp = __shfl_up_sync(0xffffffffu, ip, d);
        if (lane >= (uint32_t)d) {
            ir += xr;
            ip += xp;
        }
    }
    if (lane == 31) {
        s_warp[0][w] = ir;
        s_warp[1][w] = ip;
    }
    __syncthreads();
    uint32_t or_ = 0, op = 0;
    for (uint32_t k = 0; k < w; ++k) {
        or_ += s_warp[0][k];
        op += s_warp[1][k];
    }
    uint32_t er = or_ + ir - sr, ep = op + ip - sp;  // exclusive start of this thread's run
    for (uint32_t i = b0; i < b1; ++i) {
        const uint32_t tr = __ldcg(q.base_raw + i), tp = __ldcg(q.base_par + i);
        q.base_raw[i] = er;
        q.base_par[i] = ep;
        er += tr;
        ep += tp;
    }
    if (threadIdx.x == blockDim.x - 1) {
        q.base_raw[P] = er;
        q.base_par[P] = ep;
    }
}

// Pass B2. CTA g moves segment g's rows to their partitions' ranges as
// 32-byte records {key, field 0, field 1, field 2} (each one whole, aligned
// DRAM sector), and its partial records. Each thread loads U rows before it
// stores any, so U loads per thread are in flight.
__global__ void __launch_bounds__(1024) gb_part_scatter_kernel(const __grid_constant__ GbPart q, int words) {
    extern __shared__ uint32_t cur[];  // [2 * P]: row cursors, partial cursors
    const uint32_t P = 1u << q.pbits;
    const uint32_t g = blockIdx.x;
    for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) {
        cur[i] = q.base_raw[i] + q.rel_raw[(uint64_t)g * P + i];
        cur[P + i] = q.base_par[i] + q.rel_par[(uint64_t)g * P + i];
    }
    __syncthreads();
    const uint32_t n = q.n_spill[g];
    const uint64_t seg = (uint64_t)g * q.seg_stride;
    constexpr int U = 4;
    for (uint32_t b = threadIdx.x; b < n; b += blockDim.x * U) {
        ull key[U], f0[U], f1[U], f2[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = b + (uint32_t)u * blockDim.x;
            const bool in = i < n;
            key[u] = in ? __ldcs(q.skey + seg + i) : 0ull;
            f0[u] = in && q.n_fields > 0 ? __ldcs(q.sfield[0] + seg + i) : 0ull;
            f1[u] = in && q.n_fields > 1 ? __ldcs(q.sfield[1] + seg + i) : 0ull;
            f2[u] = in && q.n_fields > 2 ? __ldcs(q.sfield[2] + seg + i) : 0ull;
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (b + (uint32_t)u * blockDim.x >= n) continue;
            const uint32_t pos = atomicAdd(&cur[part_of(key[u], q.pbits)], 1u);
            ulonglong2* dst = reinterpret_cast<ulonglong2*>(q.drec + (uint64_t)pos * REC_WORDS);
            dst[0] = make_ulonglong2(key[u], f0[u]);
            dst[1] = make_ulonglong2(f1[u], f2[u]);
        }
    }
    const uint32_t np = q.n_part[g];
    for (uint32_t i = threadIdx.x; i < np; i += blockDim.x) {
        const ull* src = q.ppart + ((uint64_t)g * q.hot_cap + i) * (uint64_t)words;
        const uint32_t pos = atomicAdd(&cur[P + part_of(src[0], q.pbits)], 1u);
        ull* dst = q.dpar + (uint64_t)pos * words;
        for (int k = 0; k < words; ++k) dst[k] = src[k];
    }
}

// Shared-table find-or-insert without an admission limit: a partition's
// table must hold all of its groups. -1 when `limit` keys are already in
// (the partition has more groups than planned: spill).
__device__ __forceinline__ int r_find_insert(ull* sk, int log2, ull stored, uint32_t* fill, uint32_t limit) {
    const uint32_t mask = (1u << log2) - 1;
    uint32_t h = (uint32_t)((stored * HASH_S) >> (64 - log2));
    volatile ull* vk = sk;
    for (uint32_t i = 0; i <= mask; ++i) {
        const ull k = vk[h];
        if (k == stored) return (int)h;
        if (k == 0) {
            if (atomicAdd(fill, 1u) >= limit) return -1;
            const ull old = atomicCAS(&sk[h], 0ull, stored);
            if (old == 0) return (int)h;
            atomicSub(fill, 1u);
            if (old == stored) return (int)h;
        }
        h = (h + 1) & mask;
    }
    return -1;
}

// Pass C. Each CTA reduces partitions blockIdx.x, + gridDim.x, ... in a
// shared table (keys | states, the shared slot layout), then writes every
// group once into the compact group array (global slot layout) at an index
// inside a range the partition claims with one atomic, with its sort key.
// The table is left zeroed for the next partition.
template <class SP>
__global__ void __launch_bounds__(512) gb_part_reduce_kernel(const __grid_constant__ GbParams p,
                                                              const __grid_constant__ GbPart q, ull* n_groups,
                                                              ull* order_keys, uint32_t* slots) {
    extern __shared__ __align__(16) ull rsm[];
    __shared__ uint32_t s_fill;
    __shared__ ull s_base;
    const int SW = p.sslot_words - 1;
    const int W = SW + 1;
    const int C = 1 << q.red_log2;
    const uint32_t P = 1u << q.pbits;
    const ull gcap = 1ull << p.log2cap;
    const uint32_t lane = lane_id();
    ull* sk = rsm;
    ull* sw = rsm + C;
    for (int i = threadIdx.x; i < C * W; i += blockDim.x) rsm[i] = 0;
    if (threadIdx.x == 0) s_fill = 0;
    // The group whose key complement is 0 sits in its own slot (gcap).
    if (blockIdx.x == 0 && threadIdx.x == 0 && ld_volatile(p.gtab + gcap * (ull)p.slot_words) != 0) {
        const ull at = atomicAdd(n_groups, 1ull);
        if (at < gcap) {
            order_keys[at] = ~0ull ^ 0x8000000000000000ull;
            slots[at] = (uint32_t)gcap;
        } else {
            atomicOr(p.status, ST_FLAG_GROW);
        }
    }
    __syncthreads();
    uint32_t absbits = 0;
    // The first partition's rows into L2 (the others are prefetched one
    // partition ahead, below).
    if (threadIdx.x == 0 && blockIdx.x < P) {
        const uint32_t rb = q.base_raw[blockIdx.x], re = q.base_raw[blockIdx.x + 1];
        if (re > rb) bulk_prefetch_l2(q.drec + (uint64_t)rb * REC_WORDS, (re - rb) * REC_WORDS * 8u);
    }
    for (uint32_t part = blockIdx.x; part < P; part += gridDim.x) {
        if (threadIdx.x == 0 && part + gridDim.x < P) {
            const uint32_t nb = q.base_raw[part + gridDim.x], ne = q.base_raw[part + gridDim.x + 1];
            if (ne > nb) bulk_prefetch_l2(q.drec + (uint64_t)nb * REC_WORDS, (ne - nb) * REC_WORDS * 8u);
        }
        // Partial states of the pass-A shared tables.
        const uint32_t pb = q.base_par[part], pe = q.base_par[part + 1];
        for (uint32_t j = pb + threadIdx.x; j < pe; j += blockDim.x) {
            const ull* rec = q.dpar + (uint64_t)j * W;
            const int sl = r_find_insert(sk, q.red_log2, rec[0], &s_fill, q.red_fill);
            if (sl < 0) {
                atomicOr(p.status, ST_FLAG_SPILL);
                continue;
            }
            ull* w = sw + (ull)sl * SW - 1;
#pragma unroll
            for (int s = 0; s < SP::n; ++s) {
                const int at = p.st[s].sword;
                const int k = SP::kind(s);
                const bool two = k == K_SUM_I64 || k == K_SUM_FX;
                merge_words_smem(w + at, k, rec[at], two ? rec[at + 1] : 0ull, true);
            }
        }
        // Spilled rows, RU per thread loaded before any is folded.
        constexpr int RU = 4;
        const uint32_t rb = q.base_raw[part], re = q.base_raw[part + 1];
        for (uint32_t j0 = rb + threadIdx.x; j0 < re; j0 += blockDim.x * RU) {
            ulonglong2 r0[RU], r1[RU];
#pragma unroll
            for (int u = 0; u < RU; ++u) {
                const uint32_t j = j0 + (uint32_t)u * blockDim.x;
                const ulonglong2* rec = reinterpret_cast<const ulonglong2*>(q.drec + (uint64_t)j * REC_WORDS);
                r0[u] = j < re ? __ldcs(rec) : make_ulonglong2(0, 0);
                r1[u] = j < re ? __ldcs(rec + 1) : make_ulonglong2(0, 0);
            }
#pragma unroll
            for (int u = 0; u < RU; ++u) {
                if (j0 + (uint32_t)u * blockDim.x >= re) break;
                const ull fw[GB_PART_MAX_FIELDS] = {r0[u].y, r1[u].x, r1[u].y};
                const int sl = r_find_insert(sk, q.red_log2, r0[u].x, &s_fill, q.red_fill);
                if (sl < 0) {
                    atomicOr(p.status, ST_FLAG_SPILL);
                    continue;
                }
                ull c0[SP::n], c1[SP::n];
                row_contrib<SP>(p, q, fw, c0, c1, absbits);
                ull* w = sw + (ull)sl * SW - 1;
#pragma unroll
                for (int s = 0; s < SP::n; ++s)
                    merge_words_smem(w + p.st[s].sword, SP::kind(s), c0[s], c1[s], true);
            }
        }
        __syncthreads();
        // Drain: every occupied slot becomes one group of the compact array,
        // at an index inside the range the partition claims with one atomic
        // once its occupied slots are counted.
        if (threadIdx.x == 0) s_fill = 0;
        __syncthreads();
        for (int i0 = 0; i0 < C; i0 += blockDim.x) {
            const int i = i0 + (int)threadIdx.x;
            const uint32_t m = __ballot_sync(0xffffffffu, i < C && sk[i] != 0);
            if (lane == 0 && m) atomicAdd(&s_fill, (uint32_t)__popc(m));
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_base = s_fill ? atomicAdd(n_groups, (ull)s_fill) : 0ull;
            s_fill = 0;
        }
        __syncthreads();
        for (int i0 = 0; i0 < C; i0 += blockDim.x) {
            const int i = i0 + (int)threadIdx.x;
            const ull key = i < C ? sk[i] : 0ull;
            const bool occ = key != 0;
            const uint32_t m = __ballot_sync(0xffffffffu, occ);
            uint32_t at0 = 0;
            if (lane == 0 && m) at0 = atomicAdd(&s_fill, (uint32_t)__popc(m));
            at0 = __shfl_sync(0xffffffffu, at0, 0);
            if (occ) {
                const ull at = s_base + at0 + __popc(m & lanemask_lt());
                if (at < gcap) {
                    ull* out = p.gtab + at * (ull)p.slot_words;
                    const ull* src = sw + (ull)i * SW - 1;
                    out[0] = key;
#pragma unroll
                    for (int s = 0; s < SP::n; ++s) {
                        const int k = SP::kind(s);
                        const int gw = p.st[s].word, swd = p.st[s].sword;
                        if (k == K_SUM_FX) {  // shared (lo, hi) -> global (bits 0-31, bits 32-63, hi)
                            const ull lo = src[swd];
                            out[gw] = lo & 0xFFFFFFFFull;
                            out[gw + 1] = lo >> 32;
                            out[gw + 2] = src[swd + 1];
                        } else if (k == K_SUM_I64) {
                            out[gw] = src[swd];
                            out[gw + 1] = src[swd + 1];
                        } else {
                            out[gw] = src[swd];
                        }
                    }
                    order_keys[at] = ~key ^ 0x8000000000000000ull;
                    slots[at] = (uint32_t)at;
                } else {
                    atomicOr(p.status, ST_FLAG_GROW);
                }
                ull* z = sw + (ull)i * SW;
                for (int k = 0; k < SW; ++k) z[k] = 0;
                sk[i] = 0;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) s_fill = 0;
        __syncthreads();
    }
    gb_flush_absbits(p, absbits);
}

using LeanKernel = void (*)(GbParams, GbPart);
using ReduceKernel = void (*)(GbParams, GbPart, ull*, ull*, uint32_t*);

template <int KP, int MISS>
LeanKernel lean_for_spec(int spec) {
    switch (spec) {
    case 1: return gb_lean_kernel<KP, Spec1, MISS>;
    case 2: return gb_lean_kernel<KP, Spec2, MISS>;
    case 4: return gb_lean_kernel<KP, Spec4, MISS>;
    case 5: return gb_lean_kernel<KP, Spec5, MISS>;
    case 6: return gb_lean_kernel<KP, Spec6, MISS>;
    case 7: return gb_lean_kernel<KP, Spec7, MISS>;
    default: return nullptr;
    }
}

template <int MISS>
LeanKernel lean_kernel_for(int kp, int spec) {
    switch (kp) {
    case GB_KP_I32X2: return lean_for_spec<GB_KP_I32X2, MISS>(spec);
    case GB_KP_I32: return lean_for_spec<GB_KP_I32, MISS>(spec);
    default: return lean_for_spec<GB_KP_I64, MISS>(spec);
    }
}

ReduceKernel reduce_kernel_for(int spec) {
    switch (spec) {
    case 1: return gb_part_reduce_kernel<Spec1>;
    case 2: return gb_part_reduce_kernel<Spec2>;
    case 4: return gb_part_reduce_kernel<Spec4>;
    case 5: return gb_part_reduce_kernel<Spec5>;
    case 6: return gb_part_reduce_kernel<Spec6>;
    case 7: return gb_part_reduce_kernel<Spec7>;
    default: return nullptr;
    }
}

// The WHERE conjunct `v <cmp> lit` on an Int32 column as a range [lo, hi]
// (possibly empty), negated for <>.
void pred_range(int cmp, ll lit, int32_t& lo, int32_t& hi, int32_t& neg) {
    const ll MN = INT32_MIN, MX = INT32_MAX;
    lit = std::max(MN - 1, std::min(lit, MX + 1));  // (so lit - 1 and lit + 1 cannot overflow)
    ll l = MN, h = MX;
    neg = 0;
    switch (cmp) {
    case BOLT_CMP_LT: h = lit - 1; break;
    case BOLT_CMP_LE: h = lit; break;
    case BOLT_CMP_GT: l = lit + 1; break;
    case BOLT_CMP_GE: l = lit; break;
    case BOLT_CMP_EQ: l = h = lit; break;
    default: l = h = lit; neg = 1; break;  // NE
    }
    if (l > h || h < MN || l > MX) {  // no Int32 value is in range
        lo = INT32_MAX;
        hi = INT32_MIN;
        return;
    }
    lo = (int32_t)std::max(l, MN);
    hi = (int32_t)std::min(h, MX);
}

}  // namespace

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
bool gb_lean_applies(const GbPlan& pl, uint32_t flags) {
    const GbParams& p = pl.prm;
    if (flags & (BOLT_FLAG_FORCE_GLOBAL | BOLT_FLAG_FORCE_SHMEM | BOLT_FLAG_KERNEL_REGS)) return false;
    if (p.jslots || p.spec == 0 || p.spec == 3 || p.n_rows < GB_LEAN_MIN_ROWS || p.n_rows >= (1ull << 31)) return false;
    // Dense columns only; 32-bit integer keys (one or two) or one 64-bit
    // integer key; at most one WHERE conjunct, on a 32-bit integer column;
    // at most GB_PART_MAX_FIELDS distinct value columns.
    for (int k = 0; k < p.n_keys; ++k) {
        if (p.kvalid[k]) return false;
        const int dt = p.kdtype[k];
        if (p.n_keys == 2 ? dt != BOLT_I32 : (dt != BOLT_I32 && dt != BOLT_I64)) return false;
    }
    if (p.n_pred > 1) return false;
    if (p.n_pred == 1 && (p.pred[0].dtype != BOLT_I32 || p.pred[0].valid)) return false;
    for (int s = 0; s < p.n_st; ++s) {
        if (p.st[s].valid) return false;
        if (p.st[s].col && p.st[s].dtype == BOLT_DEC128) return false;
    }
    int nf = 0;
    for (int c = 0; c < p.n_sc; ++c) {
        bool is_value = true;
        for (int k = 0; k < p.n_keys; ++k)
            if (p.k_sc[k] == c) is_value = false;
        if (p.n_pred && p.pr_sc[0] == c) is_value = false;
        if (is_value) ++nf;
    }
    if (nf > GB_PART_MAX_FIELDS) return false;
    for (int c = 0; c < p.n_sc; ++c)  // bulk copies need 16-byte aligned tile starts
        if (((uintptr_t)p.sc_col[c] + p.row_begin * (uint64_t)p.sc_w[c]) % 16 != 0) return false;
    return true;
}

bool gb_part_applies(const bolt_ctx* ctx, const GbPlan& pl, uint32_t flags) {
    (void)ctx;
    if ((flags & BOLT_FLAG_NO_PART) || !gb_lean_applies(pl, flags)) return false;
    // Used when forced, or when the autotuner found it the faster tier for
    // this query shape (and the shape expects many groups).
    const bool forced = (flags & BOLT_FLAG_FORCE_PART) != 0;
    return forced || (pl.tune.part && pl.groups_hint >= GB_PART_MIN_GROUPS);
}

namespace {

// Launch shape of the streaming kernel, shared by both miss policies.
struct LeanShape {
    LeanKernel kernel;
    int block;
    size_t smem;
};

// Fills the value-field, predicate and staging parts of q and p for the
// streaming kernel: 1 producer + 31 consumer warps, tiles of 31 x 32 x
// chunks rows, as many stages (2..PART_MAX_STAGES) as fit beside the shared
// table, the absent-key filter and the survivor lists.
template <int MISS>
bolt_status lean_setup(bolt_ctx* ctx, GbPlan* pl, GbPart& q, LeanShape& out) {
    GbParams& p = pl->prm;
    q.n_fields = 0;
    int field_of_sc[GB_MAX_SC];
    for (int c = 0; c < GB_MAX_SC; ++c) field_of_sc[c] = -1;
    for (int s2 = 0; s2 < p.n_st; ++s2) {
        const int c = p.st_sc[s2];
        const int dt = p.st[s2].dtype;
        q.field_of_state[s2] = -1;
        q.state_float[s2] = (int8_t)(dt == BOLT_F32 || dt == BOLT_F64);
        if (c < 0) continue;
        if (field_of_sc[c] < 0) {
            if (q.n_fields == GB_PART_MAX_FIELDS)
                return fail(ctx, BOLT_DECLINE, "GROUP BY: more value columns than the streaming kernel carries");
            field_of_sc[c] = q.n_fields;
            q.field_sc[q.n_fields] = (int8_t)c;
            q.field_w[q.n_fields] = (int8_t)dtype_width(dt);
            q.field_float[q.n_fields] = (int8_t)(dt == BOLT_F32 || dt == BOLT_F64);
            q.n_fields++;
        }
        q.field_of_state[s2] = (int8_t)field_of_sc[c];
    }
    q.has_pred = p.n_pred == 1;
    if (q.has_pred) pred_range(p.pred[0].cmp, p.pred[0].lit_i, q.pred_lo, q.pred_hi, q.pred_neg);
    const int kp = p.n_keys == 2 ? GB_KP_I32X2 : (p.kdtype[0] == BOLT_I32 ? GB_KP_I32 : GB_KP_I64);
    out.kernel = lean_kernel_for<MISS>(kp, p.spec);
    if (!out.kernel) return fail(ctx, BOLT_DECLINE, "GROUP BY: no streaming kernel for this layout");

    const int chunks = std::max(1, std::min(pl->part_chunks, 2));
    const int block = 1024, nw = block / 32 - 1;
    const uint32_t T = (uint32_t)(nw * 32 * chunks);
    uint64_t row_w = 0;
    for (int c = 0; c < p.n_sc; ++c) row_w += (uint64_t)p.sc_w[c];
    const size_t stage = (size_t)T * row_w;
    const size_t lists = (size_t)nw * 32 * chunks * 2;
    const size_t filt = (size_t)FILT_WORDS * 4;
    const size_t budget = (size_t)std::max(ctx->max_smem_optin - 1024, 0);
    const size_t entry = 8ull * (size_t)p.sslot_words;
    int sl = pl->part_hot_log2 > 0 ? pl->part_hot_log2 : 11;
    int S = 0;
    for (;;) {
        const size_t table = ((size_t)1 << sl) * entry;
        if (table + filt + lists + 2 * stage <= budget) {
            S = (int)std::min<size_t>(PART_MAX_STAGES, (budget - table - filt - lists) / stage);
            break;
        }
        if (sl <= 8) return fail(ctx, BOLT_DECLINE, "GROUP BY: streaming kernel does not fit shared memory");
        --sl;
    }
    p.smem_log2 = sl;
    // Admission: a fraction of the table (eighths), so a key that is absent
    // meets an empty slot after a few probes.
    p.smem_fill = (uint32_t)(((1ull << sl) * (uint64_t)std::max(1, std::min(pl->tune.smem_fill, 6))) / 8);
    p.tile_rows = T;
    p.n_stages = S;
    p.stage_bytes = (uint32_t)stage;
    p.chunks = chunks;
    uint32_t off = 0;
    for (int c = 0; c < p.n_sc; ++c) {
        p.sc_off[c] = off;
        off += T * (uint32_t)p.sc_w[c];
    }
    q.grid_a = ctx->num_sms;
    q.hot_cap = 1 << sl;
    out.block = block;
    out.smem = (size_t)S * stage + ((size_t)1 << sl) * entry + filt + lists;
    return BOLT_OK;
}

}  // namespace

bool gb_lean_global(bolt_ctx* ctx, GbPlan* pl, cudaStream_t s, uint32_t flags, bolt_status* st) {
    if (!gb_lean_applies(*pl, flags)) return false;
    GbPart q{};
    LeanShape sh;
    *st = lean_setup<MISS_GLOBAL>(ctx, pl, q, sh);
    if (*st == BOLT_DECLINE) {
        ctx->last_error.clear();
        return false;  // the staged kernel serves the query
    }
    if (*st != BOLT_OK) return true;
    GbParams& p = pl->prm;
    if (cudaError_t e = smem_optin(sh.kernel, ctx); e != cudaSuccess) {
        *st = cuda_fail(ctx, e, "smem_optin");
        return true;
    }
    pl->grid = q.grid_a;
    kernel_mark_begin(ctx, flags, s);
    sh.kernel<<<q.grid_a, sh.block, sh.smem, s>>>(p, q);
    kernel_mark_end(ctx, flags, s);
    ctx->last_launches++;
    const cudaError_t e = cudaGetLastError();
    *st = e == cudaSuccess ? BOLT_OK : cuda_fail(ctx, e, "streaming GROUP BY launch");
    return true;
}

// Plans and launches passes A, B1, S, B2 and C for one query whose compact
// group array, words and finalize buffers are set up (see the header).
bolt_status gb_part_launch(bolt_ctx* ctx, GbPlan* pl, cudaStream_t s, uint32_t flags, int pbits_override) {
    GbParams& p = pl->prm;
    GbFinal& fin = pl->fin;
    GbPart q{};
    LeanShape sh;
    bolt_status st0 = lean_setup<MISS_SPILL>(ctx, pl, q, sh);
    if (st0 != BOLT_OK) return st0;
    const LeanKernel kA = sh.kernel;
    const ReduceKernel kC = reduce_kernel_for(p.spec);
    if (!kC) return fail(ctx, BOLT_DECLINE, "GROUP BY: no partitioned-tier kernel for this layout");
    const uint64_t groups = std::max<uint64_t>(pl->groups_hint, 1024);
    // Partitions: about RED_GROUPS expected groups each.
    int pbits = pbits_override > 0 ? pbits_override
                                   : ceil_log2_u64((groups + GB_PART_RED_GROUPS - 1) / GB_PART_RED_GROUPS);
    pbits = std::max(6, std::min(pbits, GB_PART_MAX_PBITS));
    q.pbits = pbits;
    const uint32_t P = 1u << pbits;
    // The drained stages hold the partial-record histogram (P words).
    if ((size_t)p.n_stages * p.stage_bytes < (size_t)P * 4)
        return fail(ctx, BOLT_DECLINE, "GROUP BY: partitioned tier stages smaller than the histogram");
    const int G = q.grid_a;
    const uint32_t T = p.tile_rows;
    const int nw = sh.block / 32 - 1;
    // Segment capacity: the most rows one CTA can see (its whole tiles plus
    // its share of the tail rows).
    const uint64_t ntiles = p.n_rows / T;
    const uint64_t rem = p.n_rows - ntiles * T;
    const uint64_t tail_step = (uint64_t)G * nw * 32;
    q.seg_stride = ((ntiles + G - 1) / G) * T + ((rem + tail_step - 1) / tail_step) * (uint64_t)nw * 32;
    q.seg_stride = (q.seg_stride + 31) & ~31ull;
    const int W = p.sslot_words;
    const size_t budget = (size_t)std::max(ctx->max_smem_optin - 1024, 0);
    const size_t entry = 8ull * (size_t)p.sslot_words;
    // Pass C table: 4x the expected groups per partition, at most the
    // shared memory; admission up to 7/8 of it.
    const uint64_t per_part = (groups + P - 1) / P;
    int rl = ceil_log2_u64(std::max<uint64_t>(per_part * 4, 256));
    while (((size_t)1 << rl) * entry > budget) --rl;
    q.red_log2 = rl;
    q.red_fill = (uint32_t)(((1ull << rl) * 7) / 8);

    // Scratch.
    const uint64_t nseg = (uint64_t)G * q.seg_stride;
    q.skey = (ull*)arena_alloc(ctx, nseg * 8);
    for (int fi = 0; fi < q.n_fields; ++fi) q.sfield[fi] = (ull*)arena_alloc(ctx, nseg * 8);
    q.drec = (ull*)arena_alloc(ctx, nseg * 8 * REC_WORDS);
    q.ppart = (ull*)arena_alloc(ctx, (uint64_t)G * q.hot_cap * W * 8);
    q.dpar = (ull*)arena_alloc(ctx, (uint64_t)G * q.hot_cap * W * 8);
    uint32_t* cnts = (uint32_t*)arena_alloc(ctx, 4ull * G * P * 4 + 2ull * (P + 1) * 4 + 2ull * G * 4 + 64);
    bool ok = q.skey && q.drec && q.ppart && q.dpar && cnts;
    for (int fi = 0; fi < q.n_fields; ++fi) ok = ok && q.sfield[fi];
    if (!ok) return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the partitioned tier");
    q.cnt_raw = cnts;
    q.cnt_par = q.cnt_raw + (uint64_t)G * P;
    q.rel_raw = q.cnt_par + (uint64_t)G * P;
    q.rel_par = q.rel_raw + (uint64_t)G * P;
    q.base_raw = q.rel_par + (uint64_t)G * P;
    q.base_par = q.base_raw + (P + 1);
    q.n_spill = q.base_par + (P + 1);
    q.n_part = q.n_spill + G;
    q.done = q.n_part + G;
    BOLT_CUDA(ctx, cudaMemsetAsync(q.done, 0, 4, s));

    // The profiled interval spans the aggregation kernels (A to C).
    BOLT_CUDA(ctx, smem_optin(kA, ctx));
    kernel_mark_begin(ctx, flags, s);
    kA<<<G, sh.block, sh.smem, s>>>(p, q);
    BOLT_CUDA(ctx, cudaGetLastError());
    BOLT_CUDA(ctx, smem_optin(gb_part_count_kernel, ctx));
    gb_part_count_kernel<<<G, 1024, (size_t)P * 4, s>>>(q);
    gb_part_scan_kernel<<<(P + 255) / 256, 256, 0, s>>>(q);
    BOLT_CUDA(ctx, smem_optin(gb_part_scatter_kernel, ctx));
    gb_part_scatter_kernel<<<G, 1024, 2ull * P * 4, s>>>(q, W);
    BOLT_CUDA(ctx, cudaGetLastError());
    const size_t smemC = ((size_t)1 << rl) * entry;
    BOLT_CUDA(ctx, smem_optin(kC, ctx));
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kC, 512, smemC) != cudaSuccess || per_sm < 1) per_sm = 1;
    const unsigned gC = (unsigned)std::min<uint64_t>(P, (uint64_t)per_sm * ctx->num_sms);
    kC<<<gC, 512, smemC, s>>>(p, q, fin.n_nonnull, fin.order_keys, fin.slots);
    BOLT_CUDA(ctx, cudaGetLastError());
    kernel_mark_end(ctx, flags, s);
    ctx->last_launches += 5;
    pl->part_pbits = pbits;
    return BOLT_OK;
}

}  // namespace bolt
