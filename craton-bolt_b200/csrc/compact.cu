// compact.cu — single-pass filter compaction with decoupled look-back.
//
// Replaces gpu_compact::compact_columns_on_gpu / prefix_scan_mask
// (src/exec/gpu_compact.rs:415,1005) and its kernels (prefix_scan.rs:175,
// 430,834,1227; scan_kernel.rs:265): a predicate kernel writing a u8 mask,
// a per-block scan, block sums scanned on the host (or a look-back with a
// 2-bit status / 30-bit value word) and one gather launch per column.
//
// Here one kernel per call: each CTA takes the next tile in arrival order,
// evaluates the WHERE conjunction (or reads the mask), ranks the kept rows
// with warp ballots in row order, obtains the tile's output offset by
// decoupled look-back over 64-bit (status, value) words, and writes every
// output column. Kept rows of one warp round land on consecutive output
// positions, so the writes are coalesced without staging.
//
// Two kernels share that structure. compact_bulk_kernel (columns that start
// on 16-byte boundaries, the usual case) has one thread stage every column's
// tile into shared memory with bulk copies (cp.async.bulk) completing on an
// mbarrier, and evaluates the WHERE conjuncts on the staged values.
// compact_kernel handles everything else (unaligned columns, wide rows, the
// row-id-only form ORDER BY uses for its NULL split) with per-element
// asynchronous copies or direct loads.
//
// Large bulk-staged inputs take a two-pass form instead: in one pass a CTA
// waits for its predecessors' counts, and while warp 0 looks back the other
// warps and the tile's memory traffic stand still. compact_count_kernel
// counts each tile's kept rows from the WHERE columns (or the mask) alone,
// compact_scan_kernel turns the counts into tile offsets, and
// compact_bulk_kernel<.., true> stages, ranks and writes every tile with no
// wait on another CTA. The cost is a second read of the WHERE columns
// (4 of the 28 bytes per row of a five-column filter).
#include "compact.cuh"

#include "bulk.cuh"

#include <algorithm>

namespace bolt {
namespace {

constexpr int CP_BLOCK = 256;
constexpr int CP_NW = CP_BLOCK / 32;
// Rows per thread: 8 when columns are read straight from global memory, 4
// when they are staged (smaller tiles keep more CTAs resident per SM).
constexpr int CP_ITEMS_DIRECT = 8;
constexpr int CP_ITEMS_STAGED = 4;
// Largest staged tile (bytes of shared memory per CTA).
constexpr uint32_t CP_STAGE_MAX = 48u << 10;
constexpr ull LB_AGG = 1ull << 62;
constexpr ull LB_INC = 2ull << 62;
constexpr ull LB_VAL = (1ull << 62) - 1;
constexpr uint32_t SPIN_LIMIT = 1u << 22;
constexpr int LB_WINDOW = 8;  // look-back words read per round trip
// Bulk-staged kernels: rows per thread by row width (bytes), and the largest
// stage. Small tiles keep many CTAs (and their copies) in flight per SM.
constexpr int CB_ITEMS_NARROW = 4;  // row_w <= 64: 1,024-row tiles (the vectorised count assumes 4)
constexpr int CB_ITEMS_WIDE = 2;    // row_w <= 128: 512-row tiles
constexpr uint32_t CB_STAGE_MAX = 64u << 10;
// Inputs from this many rows up take the two-pass form.
constexpr uint64_t CB_TWO_PASS_ROWS = 1ull << 22;

struct CpArgs {
    CompactSpec sp;
    ull* lookback;
    uint32_t* tile_ctr;
    uint32_t* status;
    uint32_t soff[CP_MAX_COLS];  // staged kernels: byte offset of each column's tile in shared memory
    uint32_t row_w;              // bytes per row over all columns
    uint32_t* tile_cnt;          // two-pass form: kept rows per tile (pass 1)
    ull* tile_off;               // two-pass form: output offset of each tile
};

// Asynchronous global -> shared copy of one element (4, 8 or 16 bytes; both
// addresses aligned to the size), cached in L1 so the predicate's loads of
// the same rows hit.
__device__ __forceinline__ void cp_async_elem(void* dst, const void* src, int width) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    switch (width) {
    case 4: asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory"); break;
    case 8: asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory"); break;
    default: asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory"); break;
    }
}

__device__ __forceinline__ bool cp_cmp_f(double v, int cmp, double lit) {
    switch (cmp) {
    case BOLT_CMP_LT: return v < lit;
    case BOLT_CMP_LE: return v <= lit;
    case BOLT_CMP_GT: return v > lit;
    case BOLT_CMP_GE: return v >= lit;
    case BOLT_CMP_EQ: return v == lit;
    default: return v != lit;
    }
}

__device__ __forceinline__ bool cp_cmp_i(ll v, int cmp, ll lit) {
    switch (cmp) {
    case BOLT_CMP_LT: return v < lit;
    case BOLT_CMP_LE: return v <= lit;
    case BOLT_CMP_GT: return v > lit;
    case BOLT_CMP_GE: return v >= lit;
    case BOLT_CMP_EQ: return v == lit;
    default: return v != lit;
    }
}

__device__ __forceinline__ bool cp_pred(const CompactPred& d, uint64_t r) {
    if (!bit_valid(d.valid, r)) return false;
    if (d.dtype == BOLT_F64 || d.dtype == BOLT_F32) {
        double v = d.dtype == BOLT_F64 ? __ldg((const double*)d.col + r) : (double)__ldg((const float*)d.col + r);
        return cp_cmp_f(v, d.cmp, d.lit_f);
    }
    ll v = d.dtype == BOLT_I32 ? (ll)__ldg((const int32_t*)d.col + r) : __ldg((const ll*)d.col + r);
    return cp_cmp_i(v, d.cmp, d.lit_i);
}

// The same conjunct on a value staged in shared memory (element i of the
// column's tile starting at `st`); the validity bit is read at row r.
__device__ __forceinline__ bool cp_pred_staged(const CompactPred& d, const unsigned char* st, uint32_t i, uint64_t r) {
    if (!bit_valid(d.valid, r)) return false;
    switch (d.dtype) {
    case BOLT_F64: return cp_cmp_f(reinterpret_cast<const double*>(st)[i], d.cmp, d.lit_f);
    case BOLT_F32: return cp_cmp_f((double)reinterpret_cast<const float*>(st)[i], d.cmp, d.lit_f);
    case BOLT_I64: return cp_cmp_i(reinterpret_cast<const ll*>(st)[i], d.cmp, d.lit_i);
    default: return cp_cmp_i((ll)reinterpret_cast<const int32_t*>(st)[i], d.cmp, d.lit_i);
    }
}

// A conjunct split in two so a thread can issue all of its loads before
// the first comparison: the raw 64-bit image of row r's value (integers
// sign-extended, floats as f64 bits), then the comparison on it.
__device__ __forceinline__ ull cp_raw(const CompactPred& d, uint64_t r) {
    switch (d.dtype) {
    case BOLT_F64: return (ull)__ldg((const ll*)d.col + r);
    case BOLT_F32: return (ull)__double_as_longlong((double)__ldg((const float*)d.col + r));
    case BOLT_I64: return (ull)__ldg((const ll*)d.col + r);
    default: return (ull)(ll)__ldg((const int32_t*)d.col + r);
    }
}
__device__ __forceinline__ bool cp_test_raw(const CompactPred& d, ull raw) {
    if (d.dtype == BOLT_F64 || d.dtype == BOLT_F32) return cp_cmp_f(__longlong_as_double((ll)raw), d.cmp, d.lit_f);
    return cp_cmp_i((ll)raw, d.cmp, d.lit_i);
}

// Run by warp 0 once the per-(round, warp) kept counts of the tile are in
// cnt: turns them into row-major exclusive offsets within the tile and
// returns the tile's kept count.
template <int ITEMS>
__device__ __forceinline__ uint32_t cp_tile_scan(uint32_t (*cnt)[CP_NW]) {
    const int lane = threadIdx.x & 31;
    uint32_t local = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t v = lane < CP_NW ? cnt[j][lane] : 0;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, x, 31);
        if (lane < CP_NW) cnt[j][lane] = local + x - v;
        local += tot;
    }
    return local;
}

// Run by warp 0 after the tile's counts are in cnt: cp_tile_scan, then lane
// 0 publishes the tile's count and looks back over the earlier tiles'
// (status, value) words for the tile's output offset, left in *s_base.
// The last tile stores the total kept count.
template <int ITEMS>
__device__ __forceinline__ void cp_tile_offsets(const CpArgs& a, uint32_t tile, uint32_t ntiles,
                                                uint32_t (*cnt)[CP_NW], ull* s_base) {
    const uint32_t local = cp_tile_scan<ITEMS>(cnt);
    if ((threadIdx.x & 31) != 0) return;
    ull* my = a.lookback + tile;
    ull excl = 0;
    if (tile == 0) {
        *reinterpret_cast<volatile ull*>(my) = LB_INC | local;
    } else {
        *reinterpret_cast<volatile ull*>(my) = LB_AGG | local;
        // Look back LB_WINDOW words per round trip: sum aggregates until an
        // inclusive prefix.
        int64_t t = (int64_t)tile - 1;
        uint32_t spins = 0;
        while (t >= 0) {
            const int cnt_w = (t + 1) < LB_WINDOW ? (int)(t + 1) : LB_WINDOW;
            ull v[LB_WINDOW];
#pragma unroll
            for (int i = 0; i < LB_WINDOW; ++i) v[i] = i < cnt_w ? ld_volatile(a.lookback + (t - i)) : 0ull;
            int used = 0;
            bool done = false, stalled = false;
#pragma unroll
            for (int i = 0; i < LB_WINDOW; ++i) {
                if (done || stalled || i >= cnt_w) continue;
                const ull st = v[i] >> 62;
                if (st == 0) {
                    stalled = true;
                    continue;
                }
                excl += v[i] & LB_VAL;
                ++used;
                if (st == 2) done = true;
            }
            if (done) break;
            t -= used;
            if (stalled) {
                if (++spins > SPIN_LIMIT) {
                    atomicOr(a.status, ST_FLAG_TIMEOUT);
                    break;
                }
                if (spins > 4) __nanosleep(64);
            }
        }
        *reinterpret_cast<volatile ull*>(my) = LB_INC | (excl + local);
    }
    *s_base = excl;
    if (tile == ntiles - 1) {
        const ull total = excl + local;
        *a.sp.n_out_dev = total;
        if (total > a.sp.out_cap) atomicOr(a.status, ST_FLAG_CAPACITY);
    }
}

// STAGED: every thread first issues asynchronous copies of its rows of every
// output column into shared memory, so the column reads are in flight while
// the predicate is evaluated and the tile's offset is looked back; the
// scatter then reads them back (each thread only its own rows).
template <bool STAGED>
__global__ void __launch_bounds__(CP_BLOCK) compact_kernel(const __grid_constant__ CpArgs a) {
    constexpr int CP_ITEMS = STAGED ? CP_ITEMS_STAGED : CP_ITEMS_DIRECT;
    constexpr int CP_TILE = CP_BLOCK * CP_ITEMS;
    extern __shared__ __align__(16) unsigned char cp_stage[];
    __shared__ uint32_t s_tile;
    __shared__ uint32_t cnt[CP_ITEMS][CP_NW];
    __shared__ ull s_base;
    const CompactSpec& sp = a.sp;
    const uint64_t n = sp.n;
    const uint32_t ntiles = (uint32_t)((n + CP_TILE - 1) / CP_TILE);
    if (threadIdx.x == 0) s_tile = atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t base = (uint64_t)tile * CP_TILE;
    if (STAGED) {
#pragma unroll
        for (int j = 0; j < CP_ITEMS; ++j) {
            const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
            if (e >= n) continue;
            const uint32_t slot = (uint32_t)j * CP_BLOCK + threadIdx.x;
            for (int c = 0; c < sp.n_cols; ++c) {
                const int wd = sp.col[c].width;
                cp_async_elem(cp_stage + a.soff[c] + slot * (uint32_t)wd,
                              static_cast<const unsigned char*>(sp.col[c].in) + e * (uint64_t)wd, wd);
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }

    uint32_t keep = 0;  // bit j: element base + j*BLOCK + tid is kept
#pragma unroll
    for (int j = 0; j < CP_ITEMS; ++j) {
        const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
        bool k = e < n;
        if (k) {
            if (sp.mask) k = sp.mask[e] != 0;
            if (sp.keep_valid_of) k = k && bit_valid(sp.keep_valid_of, sp.ids_in ? (uint64_t)sp.ids_in[e] : e);
            for (int q = 0; q < sp.n_pred; ++q) k = k && cp_pred(sp.pred[q], e);
            if (sp.invert) k = !k;
        }
        const uint32_t b = __ballot_sync(0xffffffffu, k && e < n);
        if (lane == 0) cnt[j][w] = __popc(b);
        if (k && e < n) keep |= 1u << j;
    }
    __syncthreads();
    if (w == 0) cp_tile_offsets<CP_ITEMS>(a, tile, ntiles, cnt, &s_base);
    __syncthreads();
    if (STAGED) asm volatile("cp.async.wait_all;" ::: "memory");
    const ull tbase = s_base;
    // Output row of each of this thread's kept rows (~0 when not kept or
    // beyond the output capacity).
    ull pos[CP_ITEMS];
#pragma unroll
    for (int j = 0; j < CP_ITEMS; ++j) {
        const uint32_t b = __ballot_sync(0xffffffffu, (keep >> j) & 1u);
        pos[j] = ~0ull;
        if ((keep >> j) & 1u) {
            const ull at = tbase + cnt[j][w] + __popc(b & lanemask_lt());
            if (at < sp.out_cap) pos[j] = at;
        }
    }
    // Column by column, so the width dispatch runs once per column.
    for (int c = 0; c < sp.n_cols; ++c) {
        const CompactCol& col = sp.col[c];
        const int wd = col.width;
#pragma unroll
        for (int j = 0; j < CP_ITEMS; ++j) {
            if (pos[j] == ~0ull) continue;
            const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
            const uint32_t slot = (uint32_t)j * CP_BLOCK + threadIdx.x;
            const unsigned char* src = STAGED ? cp_stage + a.soff[c] + slot * (uint32_t)wd
                                              : static_cast<const unsigned char*>(col.in) + e * (uint64_t)wd;
            if (wd == 4) {
                ((uint32_t*)col.out)[pos[j]] = STAGED ? *reinterpret_cast<const uint32_t*>(src)
                                                      : __ldg(reinterpret_cast<const uint32_t*>(src));
            } else if (wd == 8) {
                ((ull*)col.out)[pos[j]] = STAGED ? *reinterpret_cast<const ull*>(src)
                                                 : __ldg(reinterpret_cast<const ull*>(src));
            } else {
                ((ulonglong2*)col.out)[pos[j]] = STAGED ? *reinterpret_cast<const ulonglong2*>(src)
                                                        : __ldg(reinterpret_cast<const ulonglong2*>(src));
            }
            if (col.out_valid && bit_valid(col.in_valid, e)) set_bit_atomic(col.out_valid, pos[j], true);
        }
    }
    if (sp.row_ids) {
#pragma unroll
        for (int j = 0; j < CP_ITEMS; ++j) {
            if (pos[j] == ~0ull) continue;
            const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
            sp.row_ids[pos[j]] = (sp.ids_in ? sp.ids_in[e] : (uint32_t)e) + sp.row_id_base;
        }
    }
}

// Bulk-staged compaction (every column starts on a 16-byte boundary; no
// ids_in / keep_valid_of selection). Thread 0 issues one bulk copy per
// column of the tile's TILE rows (TILE * width bytes, a multiple of 16) into
// shared memory, completing on one mbarrier; the last, partial tile is
// copied element by element instead. Ranking, look-back and scatter follow
// compact_kernel, reading the staged values. TWO: the two-pass form's second
// pass (CTA i takes tile i; its offset comes from compact_scan_kernel).
template <int ITEMS, bool TWO>
__global__ void __launch_bounds__(CP_BLOCK) compact_bulk_kernel(const __grid_constant__ CpArgs a) {
    constexpr int TILE = CP_BLOCK * ITEMS;
    extern __shared__ __align__(128) unsigned char stg[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t s_tile;
    __shared__ uint32_t cnt[ITEMS][CP_NW];
    __shared__ ull s_base;
    const CompactSpec& sp = a.sp;
    const uint64_t n = sp.n;
    const uint32_t ntiles = (uint32_t)((n + TILE - 1) / TILE);
    if (threadIdx.x == 0) {
        s_tile = TWO ? blockIdx.x : atomicAdd(a.tile_ctr, 1u);
        mbar_init(&bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t base = (uint64_t)tile * TILE;
    const uint32_t rows = (n - base) < (uint64_t)TILE ? (uint32_t)(n - base) : (uint32_t)TILE;
    const bool whole = rows == (uint32_t)TILE;
    bool ok = true;
    if (whole) {
        if (threadIdx.x == 0) {
            mbar_arrive_expect_tx(&bar, (uint32_t)TILE * a.row_w);
            const uint64_t pol = l2_evict_first_policy();
            for (int c = 0; c < sp.n_cols; ++c) {
                const uint32_t wd = (uint32_t)sp.col[c].width;
                bulk_load(stg + a.soff[c], static_cast<const unsigned char*>(sp.col[c].in) + base * wd,
                          (uint32_t)TILE * wd, &bar, pol);
            }
        }
        ok = mbar_wait(&bar, 0);
    } else {
        for (int c = 0; c < sp.n_cols; ++c) {
            const int wd = sp.col[c].width;
            const unsigned char* src = static_cast<const unsigned char*>(sp.col[c].in) + base * (uint64_t)wd;
            unsigned char* dst = stg + a.soff[c];
            for (uint32_t i = threadIdx.x; i < rows; i += CP_BLOCK) {
                if (wd == 4) reinterpret_cast<uint32_t*>(dst)[i] = __ldg(reinterpret_cast<const uint32_t*>(src) + i);
                else if (wd == 8) reinterpret_cast<ull*>(dst)[i] = __ldg(reinterpret_cast<const ull*>(src) + i);
                else reinterpret_cast<ulonglong2*>(dst)[i] = __ldg(reinterpret_cast<const ulonglong2*>(src) + i);
            }
        }
        __syncthreads();
    }
    if (!ok && threadIdx.x == 0) atomicOr(a.status, ST_FLAG_TIMEOUT);

    // A tile whose copy did not complete keeps no rows (the call reports
    // TIMEOUT) but still publishes its count, so later tiles finish.
    uint32_t keep = 0;
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t i = (uint32_t)j * CP_BLOCK + threadIdx.x;
        const uint64_t e = base + i;
        bool k = ok && i < rows;
        if (k) {
            if (sp.mask) k = sp.mask[e] != 0;
            for (int q = 0; q < sp.n_pred; ++q) k = k && cp_pred_staged(sp.pred[q], stg + a.soff[sp.pred[q].col_idx], i, e);
            if (sp.invert) k = !k;
        }
        k = k && ok && i < rows;
        const uint32_t b = __ballot_sync(0xffffffffu, k);
        if (lane == 0) cnt[j][w] = __popc(b);
        if (k) keep |= 1u << j;
    }
    __syncthreads();
    if (w == 0) {
        if (TWO) {
            cp_tile_scan<ITEMS>(cnt);
            if (lane == 0) s_base = a.tile_off[tile];
        } else {
            cp_tile_offsets<ITEMS>(a, tile, ntiles, cnt, &s_base);
        }
    }
    __syncthreads();
    const ull tbase = s_base;
    ull pos[ITEMS];
#pragma unroll
    for (int j = 0; j < ITEMS; ++j) {
        const uint32_t b = __ballot_sync(0xffffffffu, (keep >> j) & 1u);
        pos[j] = ~0ull;
        if ((keep >> j) & 1u) {
            const ull at = tbase + cnt[j][w] + __popc(b & lanemask_lt());
            if (at < sp.out_cap) pos[j] = at;
        }
    }
    for (int c = 0; c < sp.n_cols; ++c) {
        const CompactCol& col = sp.col[c];
        const int wd = col.width;
        const unsigned char* st = stg + a.soff[c];
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (pos[j] == ~0ull) continue;
            const uint32_t i = (uint32_t)j * CP_BLOCK + threadIdx.x;
            if (wd == 4) ((uint32_t*)col.out)[pos[j]] = reinterpret_cast<const uint32_t*>(st)[i];
            else if (wd == 8) ((ull*)col.out)[pos[j]] = reinterpret_cast<const ull*>(st)[i];
            else ((ulonglong2*)col.out)[pos[j]] = reinterpret_cast<const ulonglong2*>(st)[i];
            if (col.out_valid && bit_valid(col.in_valid, base + i)) set_bit_atomic(col.out_valid, pos[j], true);
        }
    }
    if (sp.row_ids) {
#pragma unroll
        for (int j = 0; j < ITEMS; ++j) {
            if (pos[j] == ~0ull) continue;
            sp.row_ids[pos[j]] = (uint32_t)(base + (uint32_t)j * CP_BLOCK + threadIdx.x) + sp.row_id_base;
        }
    }
    // A copy that missed its wait may still be landing: wait for it (again
    // bounded) before the CTA's shared memory can be handed to another CTA.
    if (!ok && threadIdx.x == 0) mbar_wait(&bar, 0);
}

// Two-pass form, pass 1: kept rows of each tile of CP_BLOCK * ITEMS rows,
// from the mask or the WHERE columns alone. A CTA takes CC_GROUP tiles at a
// time (grid-stride) and issues every load of a conjunct before comparing.
// VEC: the selection is a byte mask or one Int32 conjunct without a
// validity bitmap, on a 16-byte aligned column: each thread then reads 16
// consecutive rows with 16-byte loads (counts need no row order).
constexpr int CC_GROUP = 4;
template <int ITEMS, bool VEC>
__global__ void __launch_bounds__(CP_BLOCK) compact_count_kernel(const __grid_constant__ CpArgs a) {
    constexpr int TILE = CP_BLOCK * ITEMS;
    constexpr int R = ITEMS * CC_GROUP;  // rows per thread per step
    static_assert(!VEC || CP_BLOCK * 16 == CC_GROUP * TILE, "vectorised count: 16 rows per thread cover the group");
    __shared__ uint32_t wcnt[CC_GROUP][CP_NW];
    const CompactSpec& sp = a.sp;
    const uint64_t n = sp.n;
    const uint32_t ntiles = (uint32_t)((n + TILE - 1) / TILE);
    const uint32_t ngroups = (ntiles + CC_GROUP - 1) / CC_GROUP;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (uint32_t grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        const uint64_t base = (uint64_t)grp * CC_GROUP * TILE;
        uint32_t c[CC_GROUP];
#pragma unroll
        for (int g = 0; g < CC_GROUP; ++g) c[g] = 0;
        if (VEC) {
            // Thread t: rows base + 16t .. base + 16t + 15, all inside tile
            // (16t) / TILE of the group.
            const uint64_t r0 = base + (uint64_t)threadIdx.x * 16;
            uint32_t k = 0;
            if (r0 + 16 <= n) {
                if (sp.mask) {
                    const uint4 m = __ldg(reinterpret_cast<const uint4*>(sp.mask + r0));
                    const uint32_t wv[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                    for (int q = 0; q < 4; ++q)
#pragma unroll
                        for (int b = 0; b < 4; ++b) k += ((wv[q] >> (8 * b)) & 0xFFu) != 0;
                } else {
                    const CompactPred& d = sp.pred[0];
                    const int4* src = reinterpret_cast<const int4*>((const int32_t*)d.col + r0);
                    int4 v[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) v[q] = __ldg(src + q);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        k += cp_cmp_i(v[q].x, d.cmp, d.lit_i);
                        k += cp_cmp_i(v[q].y, d.cmp, d.lit_i);
                        k += cp_cmp_i(v[q].z, d.cmp, d.lit_i);
                        k += cp_cmp_i(v[q].w, d.cmp, d.lit_i);
                    }
                }
            } else {
                for (uint64_t r = r0; r < n && r < r0 + 16; ++r)
                    k += sp.mask ? (sp.mask[r] != 0) : cp_cmp_i(((const int32_t*)sp.pred[0].col)[r], sp.pred[0].cmp,
                                                              sp.pred[0].lit_i);
            }
            // Warps w = 2g, 2g + 1 cover tile g of the group (TILE = 1024
            // rows = 64 threads x 16) when ITEMS == 4.
            k = __reduce_add_sync(0xffffffffu, k);
            if (lane == 0) wcnt[0][w] = k;
            __syncthreads();
            if (threadIdx.x < CC_GROUP) {
                const uint32_t tile = grp * CC_GROUP + threadIdx.x;
                constexpr int WPT = CP_NW / CC_GROUP;  // warps per tile
                uint32_t t = 0;
#pragma unroll
                for (int i = 0; i < WPT; ++i) t += wcnt[0][threadIdx.x * WPT + i];
                if (tile < ntiles) a.tile_cnt[tile] = t;
            }
            __syncthreads();
            continue;
        }
        uint32_t keep = 0;  // bit j: row base + j*BLOCK + tid
#pragma unroll
        for (int j = 0; j < R; ++j)
            if (base + (uint64_t)j * CP_BLOCK + threadIdx.x < n) keep |= 1u << j;
        if (sp.mask) {
            uint8_t m[R];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
                m[j] = ((keep >> j) & 1u) ? __ldg(sp.mask + e) : (uint8_t)0;
            }
#pragma unroll
            for (int j = 0; j < R; ++j)
                if (!m[j]) keep &= ~(1u << j);
        }
        for (int q = 0; q < sp.n_pred; ++q) {
            const CompactPred& d = sp.pred[q];
            ull raw[R];
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
                raw[j] = ((keep >> j) & 1u) ? cp_raw(d, e) : 0ull;
            }
#pragma unroll
            for (int j = 0; j < R; ++j) {
                const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
                if (((keep >> j) & 1u) && !(bit_valid(d.valid, e) && cp_test_raw(d, raw[j]))) keep &= ~(1u << j);
            }
        }
#pragma unroll
        for (int j = 0; j < R; ++j) {
            const uint64_t e = base + (uint64_t)j * CP_BLOCK + threadIdx.x;
            bool k = (keep >> j) & 1u;
            if (sp.invert && e < n) k = !k;
            c[j / ITEMS] += __popc(__ballot_sync(0xffffffffu, k));
        }
        if (lane == 0) {
#pragma unroll
            for (int g = 0; g < CC_GROUP; ++g) wcnt[g][w] = c[g];
        }
        __syncthreads();
        if (threadIdx.x < CC_GROUP) {
            const uint32_t tile = grp * CC_GROUP + threadIdx.x;
            uint32_t t = 0;
#pragma unroll
            for (int i = 0; i < CP_NW; ++i) t += wcnt[threadIdx.x][i];
            if (tile < ntiles) a.tile_cnt[tile] = t;
        }
        __syncthreads();
    }
}

// Two-pass form: one CTA turns the tile counts into exclusive output
// offsets (SCAN_ITEMS consecutive counts per thread per round), stores the
// total and flags a total beyond the output capacity.
constexpr int SCAN_ITEMS = 16;
__global__ void __launch_bounds__(1024) compact_scan_kernel(const __grid_constant__ CpArgs a, uint32_t ntiles) {
    __shared__ ull wsum[32];
    __shared__ ull carry;
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    if (t == 0) carry = 0;
    __syncthreads();
    for (uint64_t b = 0; b < ntiles; b += 1024 * SCAN_ITEMS) {
        const uint64_t i0 = b + (uint64_t)t * SCAN_ITEMS;
        uint32_t v[SCAN_ITEMS];
        ull mine = 0;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; ++k) {
            v[k] = i0 + k < ntiles ? a.tile_cnt[i0 + k] : 0u;
            mine += v[k];
        }
        ull x = mine;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const ull y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            ull ws = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const ull y = __shfl_up_sync(0xffffffffu, ws, o);
                if (lane >= o) ws += y;
            }
            wsum[lane] = ws;  // inclusive over warps
        }
        __syncthreads();
        ull run = carry + (w ? wsum[w - 1] : 0ull) + x - mine;
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; ++k) {
            if (i0 + k < ntiles) a.tile_off[i0 + k] = run;
            run += v[k];
        }
        __syncthreads();
        if (t == 0) carry += wsum[31];
        __syncthreads();
    }
    if (t == 0) {
        *a.sp.n_out_dev = carry;
        if (carry > a.sp.out_cap) atomicOr(a.status, ST_FLAG_CAPACITY);
    }
}

}  // namespace

bolt_status compact_enqueue(bolt_ctx* ctx, cudaStream_t s, const CompactSpec& spec, uint32_t flags) {
    CpArgs a{};
    a.sp = spec;
    uint32_t row_w = 0;
    bool aligned = spec.n_cols > 0, al16 = spec.n_cols > 0;
    for (int c = 0; c < spec.n_cols; ++c) {
        const int wd = spec.col[c].width;
        const uintptr_t addr = reinterpret_cast<uintptr_t>(spec.col[c].in);
        aligned = aligned && (wd == 4 || wd == 8 || wd == 16) && addr % (uintptr_t)wd == 0;
        al16 = al16 && addr % 16 == 0;
        row_w += (uint32_t)wd;
    }
    a.row_w = row_w;
    // Bulk-staged tiles: columns on 16-byte boundaries, a tile of them within
    // the stage budget, and a plain selection (no ids_in / keep_valid_of).
    int bulk_items = 0;
    if (aligned && al16 && !spec.ids_in && !spec.keep_valid_of && !(flags & BOLT_FLAG_KERNEL_REGS)) {
        if (row_w * (uint32_t)(CP_BLOCK * CB_ITEMS_NARROW) <= CB_STAGE_MAX) bulk_items = CB_ITEMS_NARROW;
        else if (row_w * (uint32_t)(CP_BLOCK * CB_ITEMS_WIDE) <= CB_STAGE_MAX) bulk_items = CB_ITEMS_WIDE;
    }
    // Otherwise per-element asynchronous copies when a tile fits the budget
    // and every input is aligned to its width, else direct loads.
    const bool staged = !bulk_items && aligned && row_w * (uint32_t)(CP_BLOCK * CP_ITEMS_STAGED) <= CP_STAGE_MAX;
    const uint32_t items = bulk_items ? (uint32_t)bulk_items : staged ? (uint32_t)CP_ITEMS_STAGED : (uint32_t)CP_ITEMS_DIRECT;
    uint32_t off = 0;
    for (int c = 0; c < spec.n_cols; ++c) {
        a.soff[c] = off;
        off += (uint32_t)spec.col[c].width * (uint32_t)CP_BLOCK * items;
    }
    const uint32_t stage_bytes = row_w * (uint32_t)CP_BLOCK * items;
    const uint64_t tile_rows = (uint64_t)CP_BLOCK * items;
    const uint64_t ntiles = (spec.n + tile_rows - 1) / tile_rows;
    // Large bulk-staged inputs run the two-pass form (no CTA waits on
    // another); the rest run one pass with decoupled look-back.
    const bool two = bulk_items && spec.n >= CB_TWO_PASS_ROWS;
    a.tile_ctr = (uint32_t*)arena_alloc(ctx, 64);
    if (two) {
        a.tile_cnt = (uint32_t*)arena_alloc(ctx, ntiles * 4);
        a.tile_off = (ull*)arena_alloc(ctx, ntiles * 8);
        if (!a.tile_cnt || !a.tile_off || !a.tile_ctr) return fail(ctx, BOLT_ERR_CAPACITY, "compaction: scratch arena too small");
    } else {
        a.lookback = (ull*)arena_alloc(ctx, (ntiles + 1) * 8);
        if (!a.lookback || !a.tile_ctr) return fail(ctx, BOLT_ERR_CAPACITY, "compaction: scratch arena too small");
        BOLT_CUDA(ctx, cudaMemsetAsync(a.lookback, 0, (ntiles + 1) * 8, s));
    }
    a.status = ctx->d_status;
    BOLT_CUDA(ctx, cudaMemsetAsync(a.tile_ctr, 0, 64, s));
    if (spec.n == 0) {
        BOLT_CUDA(ctx, cudaMemsetAsync(spec.n_out_dev, 0, 8, s));
        return BOLT_OK;
    }
    for (int c = 0; c < spec.n_cols; ++c) {
        const uint64_t rows = spec.out_cap < spec.n ? spec.out_cap : spec.n;
        if (spec.col[c].out_valid) BOLT_CUDA(ctx, cudaMemsetAsync(spec.col[c].out_valid, 0, (rows + 7) / 8, s));
    }
    kernel_mark_begin(ctx, flags, s);
    if (two) {
        const uint64_t ngroups = (ntiles + CC_GROUP - 1) / CC_GROUP;
        const unsigned cg = (unsigned)std::min<uint64_t>(ngroups, (uint64_t)ctx->num_sms * 8);
        // Vectorised count: a byte mask or one Int32 conjunct without a
        // validity bitmap, on 16-byte boundaries (1,024-row tiles only).
        const bool vec = bulk_items == 4 && !spec.invert &&
                         ((spec.mask && spec.n_pred == 0 && reinterpret_cast<uintptr_t>(spec.mask) % 16 == 0) ||
                          (!spec.mask && spec.n_pred == 1 && spec.pred[0].dtype == BOLT_I32 && !spec.pred[0].valid &&
                           reinterpret_cast<uintptr_t>(spec.pred[0].col) % 16 == 0));
        if (bulk_items == CB_ITEMS_NARROW) {
            if (vec) compact_count_kernel<CB_ITEMS_NARROW, true><<<cg, CP_BLOCK, 0, s>>>(a);
            else compact_count_kernel<CB_ITEMS_NARROW, false><<<cg, CP_BLOCK, 0, s>>>(a);
            compact_scan_kernel<<<1, 1024, 0, s>>>(a, (uint32_t)ntiles);
            BOLT_CUDA(ctx, smem_optin(compact_bulk_kernel<CB_ITEMS_NARROW, true>, ctx));
            compact_bulk_kernel<CB_ITEMS_NARROW, true><<<(unsigned)ntiles, CP_BLOCK, stage_bytes, s>>>(a);
        } else {
            compact_count_kernel<CB_ITEMS_WIDE, false><<<cg, CP_BLOCK, 0, s>>>(a);
            compact_scan_kernel<<<1, 1024, 0, s>>>(a, (uint32_t)ntiles);
            BOLT_CUDA(ctx, smem_optin(compact_bulk_kernel<CB_ITEMS_WIDE, true>, ctx));
            compact_bulk_kernel<CB_ITEMS_WIDE, true><<<(unsigned)ntiles, CP_BLOCK, stage_bytes, s>>>(a);
        }
        ctx->last_launches += 2;
    } else if (bulk_items == CB_ITEMS_NARROW) {
        BOLT_CUDA(ctx, smem_optin(compact_bulk_kernel<CB_ITEMS_NARROW, false>, ctx));
        compact_bulk_kernel<CB_ITEMS_NARROW, false><<<(unsigned)ntiles, CP_BLOCK, stage_bytes, s>>>(a);
    } else if (bulk_items == CB_ITEMS_WIDE) {
        BOLT_CUDA(ctx, smem_optin(compact_bulk_kernel<CB_ITEMS_WIDE, false>, ctx));
        compact_bulk_kernel<CB_ITEMS_WIDE, false><<<(unsigned)ntiles, CP_BLOCK, stage_bytes, s>>>(a);
    } else if (staged) {
        BOLT_CUDA(ctx, smem_optin(compact_kernel<true>, ctx));
        compact_kernel<true><<<(unsigned)ntiles, CP_BLOCK, stage_bytes, s>>>(a);
    } else {
        compact_kernel<false><<<(unsigned)ntiles, CP_BLOCK, 0, s>>>(a);
    }
    kernel_mark_end(ctx, flags, s);
    ctx->last_launches++;
    BOLT_CUDA(ctx, cudaGetLastError());
    return BOLT_OK;
}

}  // namespace bolt

using namespace bolt;

namespace {

int width_of(int dt) {
    switch (dt) {
    case BOLT_I32: case BOLT_F32: case BOLT_U32: return 4;
    case BOLT_I64: case BOLT_F64: return 8;
    case BOLT_DEC128: return 16;
    }
    return 0;
}

bolt_status compact_common(bolt_ctx* ctx, const bolt_col_view* cols, int32_t n_cols, const bolt_pred* preds,
                           int32_t n_preds, const uint8_t* mask, bolt_col_mut* out, bolt_col_mut* row_ids,
                           uint64_t* n_out, uint32_t flags, bolt_stream stream) {
    if (!ctx || !n_out || n_cols < 0 || n_cols > CP_MAX_COLS || n_preds < 0 || n_preds > CP_MAX_PREDS)
        return ctx ? fail(ctx, BOLT_ERR_INVALID, "compaction: bad arguments") : BOLT_ERR_INVALID;
    if (n_cols == 0 && !row_ids) return fail(ctx, BOLT_ERR_INVALID, "compaction: nothing to output");
    cudaStream_t s = (cudaStream_t)stream;
    bolt_status st = call_begin(ctx, flags, s);
    if (st != BOLT_OK) return st;
    CompactSpec sp;
    uint64_t n = n_cols > 0 ? cols[0].len : 0;
    if (n_cols == 0 && n_preds > 0) return fail(ctx, BOLT_ERR_INVALID, "compaction: predicates need columns");
    for (int c = 0; c < n_cols; ++c) {
        if (cols[c].len != n) return fail(ctx, BOLT_ERR_INVALID, "compaction: column lengths differ");
        const int wd = width_of(cols[c].dtype);
        if (!wd || !out || out[c].dtype != cols[c].dtype)
            return fail(ctx, BOLT_ERR_INVALID, "compaction: column %d dtype mismatch", c);
        if (!col_aligned(cols[c].data, cols[c].dtype) || !col_aligned(out[c].data, cols[c].dtype))
            return fail(ctx, BOLT_ERR_INVALID, "compaction: column %d is not aligned to its element width", c);
        sp.col[c] = CompactCol{cols[c].data, cols[c].validity, out[c].data, cols[c].validity ? out[c].validity : nullptr, wd};
        sp.out_cap = sp.out_cap < out[c].cap ? sp.out_cap : out[c].cap;
    }
    if (row_ids) {
        if (row_ids->dtype != BOLT_U32) return fail(ctx, BOLT_ERR_INVALID, "compaction: row ids must be U32");
        sp.row_ids = (uint32_t*)row_ids->data;
        sp.out_cap = sp.out_cap < row_ids->cap ? sp.out_cap : row_ids->cap;
    }
    if (n >= (1ull << 32) && row_ids) return fail(ctx, BOLT_DECLINE, "compaction: row ids need n < 2^32");
    sp.n_cols = n_cols;
    sp.n = n;
    sp.mask = mask;
    for (int q = 0; q < n_preds; ++q) {
        if (preds[q].col < 0 || preds[q].col >= n_cols) return fail(ctx, BOLT_ERR_INVALID, "compaction: WHERE column out of range");
        const bolt_col_view& c = cols[preds[q].col];
        if (c.dtype == BOLT_DEC128 || c.dtype == BOLT_U32) return fail(ctx, BOLT_DECLINE, "compaction: WHERE on dtype %d", c.dtype);
        sp.pred[q] = CompactPred{c.data, c.validity, c.dtype, preds[q].cmp, preds[q].lit_i, preds[q].lit_f, preds[q].col};
    }
    sp.n_pred = n_preds;
    ull* cnt = (ull*)arena_alloc(ctx, 256);
    if (!cnt) return fail(ctx, BOLT_ERR_CAPACITY, "compaction: scratch arena too small");
    sp.n_out_dev = cnt;
    st = compact_enqueue(ctx, s, sp, flags);
    if (st != BOLT_OK) return st;
    st = call_end(ctx, flags, s);
    if (st != BOLT_OK) return st;
    if (flags & BOLT_FLAG_ASYNC) return BOLT_OK;
    uint32_t f = 0;
    st = read_status(ctx, s, 0, &f);
    if (st != BOLT_OK) return st;
    ull v = 0;
    BOLT_CUDA(ctx, cudaMemcpy(&v, cnt, 8, cudaMemcpyDeviceToHost));
    *n_out = v;
    return flags_to_status(ctx, f, "compaction");
}

}  // namespace

extern "C" bolt_status bolt_compact(bolt_ctx* ctx, const bolt_col_view* cols, int32_t n_cols, const bolt_pred* preds,
                                    int32_t n_preds, bolt_col_mut* out, bolt_col_mut* row_ids, uint64_t* n_out,
                                    uint32_t flags, bolt_stream stream) {
    return compact_common(ctx, cols, n_cols, preds, n_preds, nullptr, out, row_ids, n_out, flags, stream);
}

extern "C" bolt_status bolt_compact_mask(bolt_ctx* ctx, const bolt_col_view* cols, int32_t n_cols, const uint8_t* mask,
                                         bolt_col_mut* out, bolt_col_mut* row_ids, uint64_t* n_out, uint32_t flags,
                                         bolt_stream stream) {
    if (!mask) return ctx ? fail(ctx, BOLT_ERR_INVALID, "compaction: no mask") : BOLT_ERR_INVALID;
    return compact_common(ctx, cols, n_cols, nullptr, 0, mask, out, row_ids, n_out, flags, stream);
}
