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
#include "compact.cuh"

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

struct CpArgs {
    CompactSpec sp;
    ull* lookback;
    uint32_t* tile_ctr;
    uint32_t* status;
    uint32_t soff[CP_MAX_COLS];  // staged kernel: byte offset of each column's tile in shared memory
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

__device__ __forceinline__ bool cp_pred(const CompactPred& d, uint64_t r) {
    if (!bit_valid(d.valid, r)) return false;
    if (d.dtype == BOLT_F64 || d.dtype == BOLT_F32) {
        double v = d.dtype == BOLT_F64 ? __ldg((const double*)d.col + r) : (double)__ldg((const float*)d.col + r);
        switch (d.cmp) {
        case BOLT_CMP_LT: return v < d.lit_f;
        case BOLT_CMP_LE: return v <= d.lit_f;
        case BOLT_CMP_GT: return v > d.lit_f;
        case BOLT_CMP_GE: return v >= d.lit_f;
        case BOLT_CMP_EQ: return v == d.lit_f;
        default: return v != d.lit_f;
        }
    }
    ll v = d.dtype == BOLT_I32 ? (ll)__ldg((const int32_t*)d.col + r) : __ldg((const ll*)d.col + r);
    switch (d.cmp) {
    case BOLT_CMP_LT: return v < d.lit_i;
    case BOLT_CMP_LE: return v <= d.lit_i;
    case BOLT_CMP_GT: return v > d.lit_i;
    case BOLT_CMP_GE: return v >= d.lit_i;
    case BOLT_CMP_EQ: return v == d.lit_i;
    default: return v != d.lit_i;
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
    // Row-major exclusive scan of the (round, warp) counts by warp 0.
    if (w == 0) {
        uint32_t v[CP_ITEMS];
        uint32_t local = 0;
#pragma unroll
        for (int j = 0; j < CP_ITEMS; ++j) {
            v[j] = lane < CP_NW ? cnt[j][lane] : 0;
            uint32_t x = v[j];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            const uint32_t tot = __shfl_sync(0xffffffffu, x, 31);
            if (lane < CP_NW) cnt[j][lane] = local + x - v[j];
            local += tot;
        }
        if (lane == 0) {
            // Decoupled look-back over tiles.
            ull* my = a.lookback + tile;
            ull excl = 0;
            if (tile == 0) {
                *reinterpret_cast<volatile ull*>(my) = LB_INC | local;
            } else {
                *reinterpret_cast<volatile ull*>(my) = LB_AGG | local;
                // Look back LB_WINDOW words per round trip: sum aggregates
                // until an inclusive prefix.
                int64_t t = (int64_t)tile - 1;
                uint32_t spins = 0;
                while (t >= 0) {
                    const int cnt = (t + 1) < LB_WINDOW ? (int)(t + 1) : LB_WINDOW;
                    ull v[LB_WINDOW];
#pragma unroll
                    for (int i = 0; i < LB_WINDOW; ++i) v[i] = i < cnt ? ld_volatile(a.lookback + (t - i)) : 0ull;
                    int used = 0;
                    bool done = false, stalled = false;
#pragma unroll
                    for (int i = 0; i < LB_WINDOW; ++i) {
                        if (done || stalled || i >= cnt) continue;
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
            s_base = excl;
            if (tile == ntiles - 1) {
                const ull total = excl + local;
                *sp.n_out_dev = total;
                if (total > sp.out_cap) atomicOr(a.status, ST_FLAG_CAPACITY);
            }
        }
    }
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

}  // namespace

bolt_status compact_enqueue(bolt_ctx* ctx, cudaStream_t s, const CompactSpec& spec, uint32_t flags) {
    CpArgs a{};
    a.sp = spec;
    // Stage the columns when a tile of them fits the budget and every input
    // is aligned to its width (the asynchronous copies need both).
    uint32_t row_w = 0;
    bool staged = spec.n_cols > 0;
    for (int c = 0; c < spec.n_cols; ++c) {
        const int wd = spec.col[c].width;
        staged = staged && (wd == 4 || wd == 8 || wd == 16) &&
                 reinterpret_cast<uintptr_t>(spec.col[c].in) % (uintptr_t)wd == 0;
        a.soff[c] = row_w * (uint32_t)(CP_BLOCK * CP_ITEMS_STAGED);
        row_w += (uint32_t)wd;
    }
    const uint32_t stage_bytes = row_w * (uint32_t)(CP_BLOCK * CP_ITEMS_STAGED);
    staged = staged && stage_bytes <= CP_STAGE_MAX;
    const uint64_t tile_rows = (uint64_t)CP_BLOCK * (staged ? CP_ITEMS_STAGED : CP_ITEMS_DIRECT);
    const uint64_t ntiles = (spec.n + tile_rows - 1) / tile_rows;
    a.lookback = (ull*)arena_alloc(ctx, (ntiles + 1) * 8);
    a.tile_ctr = (uint32_t*)arena_alloc(ctx, 64);
    if (!a.lookback || !a.tile_ctr) return fail(ctx, BOLT_ERR_CAPACITY, "compaction: scratch arena too small");
    a.status = ctx->d_status;
    BOLT_CUDA(ctx, cudaMemsetAsync(a.lookback, 0, (ntiles + 1) * 8, s));
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
    if (staged) {
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
        sp.pred[q] = CompactPred{c.data, c.validity, c.dtype, preds[q].cmp, preds[q].lit_i, preds[q].lit_f};
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
