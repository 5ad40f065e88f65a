// join.cu — INNER equi-join build and probe for sm_100a.
//
// Replaces gpu_join::hash_join_indices_on_gpu{,_aos} (src/exec/gpu_join.rs:
// 1295,1403) and its kernels (src/jit/hash_join_kernel.rs:484,711,1765,1949):
// an open-addressing table of cap = next_pow2(2 * n_build) slots
// (gpu_join.rs:577-606), 64-bit CAS build, linear-probe lookups, and pairs
// emitted through one global atomic counter, i.e. in no particular order.
//
// Here the table is a 16-byte array-of-structs slot per key (one sector
// read per probe at the default load factor), kept in the context arena
// between build and probe. The probe kernel takes probe tiles in arrival
// order, looks every key up, and writes the (probe_row, build_row) pairs of
// its tile at an offset found by decoupled look-back, so the output is in
// probe-row order and identical on every run.
#include "join.cuh"

#include <algorithm>

#include "compact.cuh"
#include "radix_sort.cuh"

namespace bolt {
namespace {

constexpr int JP_BLOCK = 256;
constexpr int JP_ITEMS = 8;
constexpr int JP_TILE = JP_BLOCK * JP_ITEMS;
constexpr int JP_NW = JP_BLOCK / 32;
constexpr ull LB_AGG = 1ull << 62;
constexpr ull LB_INC = 2ull << 62;
constexpr ull LB_VAL = (1ull << 62) - 1;
constexpr uint32_t SPIN_LIMIT = 1u << 22;

__device__ __forceinline__ bool load_join_key(const void* col, int dt, const uint8_t* valid, uint64_t i, ull& key) {
    if (!bit_valid(valid, i)) return false;
    key = dt == BOLT_I32 ? (ull)(ll)__ldg((const int32_t*)col + i) : (ull)__ldg((const ll*)col + i);
    return true;
}

__global__ void __launch_bounds__(256) join_build_kernel(ull* slots, int log2cap, const void* key, int kdt,
                                                          const uint8_t* kvalid, const int32_t* payload,
                                                          uint64_t n, uint32_t* status) {
    const ull cap = 1ull << log2cap;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        ull k;
        if (!load_join_key(key, kdt, kvalid, i, k)) continue;  // NULL keys never match
        const ull stored = ~k;
        const ull w1 = ((ull)i << 32) | (uint32_t)(payload ? __ldg(payload + i) : 0);
        if (stored == 0) {
            ull* sp = slots + 2 * cap;
            if (atomicCAS(sp, 0ull, 1ull) != 0) atomicOr(status, ST_FLAG_DUPKEY);
            else sp[1] = w1;
            continue;
        }
        ull h = (stored * JOIN_HASH) >> (64 - log2cap);
        bool placed = false;
        for (ull t = 0; t < cap; ++t) {
            ull* sp = slots + 2 * h;
            const ull old = atomicCAS(sp, 0ull, stored);
            if (old == 0) {
                sp[1] = w1;
                placed = true;
                break;
            }
            if (old == stored) {
                atomicOr(status, ST_FLAG_DUPKEY);
                placed = true;
                break;
            }
            h = (h + 1) & (cap - 1);
        }
        if (!placed) atomicOr(status, ST_FLAG_SPILL);
    }
}

struct ProbeArgs {
    const ull* slots;
    int32_t log2cap;
    int32_t kdt;
    const void* key;
    const uint8_t* kvalid;
    uint64_t n;
    uint32_t* out_probe;
    uint32_t* out_build;
    uint64_t out_cap;
    ull* lookback;
    uint32_t* tile_ctr;
    ull* n_out;
    uint32_t* status;
    const uint32_t* sorted_rows;  // multi-match tables only
};

// MULTI: the table maps a key to a run of sorted_rows (duplicate build keys):
// a probe row emits one pair per build row of its run, in build-row order, at
// a position from the tile's prefix of match counts.
template <bool MULTI>
__global__ void __launch_bounds__(JP_BLOCK) join_probe_kernel(const __grid_constant__ ProbeArgs a) {
    __shared__ uint32_t s_tile;
    __shared__ ull cnt[JP_ITEMS][JP_NW];
    __shared__ ull s_base;
    const uint32_t ntiles = (uint32_t)((a.n + JP_TILE - 1) / JP_TILE);
    if (threadIdx.x == 0) s_tile = atomicAdd(a.tile_ctr, 1u);
    __syncthreads();
    const uint32_t tile = s_tile;
    if (tile >= ntiles) return;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t base = (uint64_t)tile * JP_TILE;
    uint32_t brow[JP_ITEMS];  // build row, or (MULTI) first position of the run
    uint32_t nm[JP_ITEMS];    // (MULTI) build rows matched
    ull wex[JP_ITEMS];        // (MULTI) matches of the warp's earlier lanes
    uint32_t hit = 0;
#pragma unroll
    for (int j = 0; j < JP_ITEMS; ++j) {
        const uint64_t e = base + (uint64_t)j * JP_BLOCK + threadIdx.x;
        ull k;
        bool m = false;
        brow[j] = 0;
        nm[j] = 0;
        wex[j] = 0;
        if (e < a.n && load_join_key(a.key, a.kdt, a.kvalid, e, k)) {
            const ull w1 = join_lookup(a.slots, a.log2cap, k);
            if (w1 != ~0ull) {
                m = true;
                brow[j] = (uint32_t)(w1 >> 32);
                nm[j] = MULTI ? (uint32_t)w1 : 1u;
            }
        }
        if (MULTI) {
            ull x = nm[j];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const ull y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            wex[j] = x - nm[j];
            const ull tot = __shfl_sync(0xffffffffu, x, 31);
            if (lane == 0) cnt[j][w] = tot;
        } else {
            const uint32_t b = __ballot_sync(0xffffffffu, m);
            if (lane == 0) cnt[j][w] = __popc(b);
        }
        if (m) hit |= 1u << j;
    }
    __syncthreads();
    if (w == 0) {
        ull local = 0;
#pragma unroll
        for (int j = 0; j < JP_ITEMS; ++j) {
            const ull v = lane < JP_NW ? cnt[j][lane] : 0ull;
            ull x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const ull y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            const ull tot = __shfl_sync(0xffffffffu, x, 31);
            if (lane < JP_NW) cnt[j][lane] = local + x - v;
            local += tot;
        }
        if (lane == 0) {
            ull* my = a.lookback + tile;
            ull excl = 0;
            if (tile == 0) {
                *reinterpret_cast<volatile ull*>(my) = LB_INC | local;
            } else {
                *reinterpret_cast<volatile ull*>(my) = LB_AGG | local;
                int64_t t = (int64_t)tile - 1;
                uint32_t spins = 0;
                while (t >= 0) {
                    const ull v2 = ld_volatile(a.lookback + t);
                    const ull st = v2 >> 62;
                    if (st == 0) {
                        if (++spins > SPIN_LIMIT) {
                            atomicOr(a.status, ST_FLAG_TIMEOUT);
                            break;
                        }
                        if (spins > 4) __nanosleep(64);
                        continue;
                    }
                    excl += v2 & LB_VAL;
                    if (st == 2) break;
                    --t;
                }
                *reinterpret_cast<volatile ull*>(my) = LB_INC | (excl + local);
            }
            s_base = excl;
            if (tile == ntiles - 1) {
                *a.n_out = excl + local;
                if (excl + local > a.out_cap) atomicOr(a.status, ST_FLAG_CAPACITY);
            }
        }
    }
    __syncthreads();
    const ull tbase = s_base;
#pragma unroll
    for (int j = 0; j < JP_ITEMS; ++j) {
        const uint64_t e = base + (uint64_t)j * JP_BLOCK + threadIdx.x;
        if (MULTI) {
            const ull pos = tbase + cnt[j][w] + wex[j];
            for (uint32_t t = 0; t < nm[j] && pos + t < a.out_cap; ++t) {
                a.out_probe[pos + t] = (uint32_t)e;
                a.out_build[pos + t] = a.sorted_rows[(uint64_t)brow[j] + t];
            }
            continue;
        }
        const uint32_t b = __ballot_sync(0xffffffffu, (hit >> j) & 1u);
        if (!((hit >> j) & 1u)) continue;
        const ull pos = tbase + cnt[j][w] + __popc(b & lanemask_lt());
        if (pos >= a.out_cap) continue;
        a.out_probe[pos] = (uint32_t)e;
        a.out_build[pos] = brow[j];
    }
}

// Multi-match build, step 1: flag[i] = 1 where sorted position i starts a run
// of equal keys (the rows are the non-NULL build rows stably sorted by key).
__global__ void __launch_bounds__(256) jm_mark_kernel(const void* key, int kdt, const uint32_t* sorted, uint64_t nv,
                                                       uint8_t* flag) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nv; i += (uint64_t)gridDim.x * blockDim.x) {
        const ull k = kdt == BOLT_I32 ? (ull)(ll)__ldg((const int32_t*)key + sorted[i]) : (ull)__ldg((const ll*)key + sorted[i]);
        bool start = i == 0;
        if (!start) {
            const ull kp = kdt == BOLT_I32 ? (ull)(ll)__ldg((const int32_t*)key + sorted[i - 1])
                                           : (ull)__ldg((const ll*)key + sorted[i - 1]);
            start = k != kp;
        }
        flag[i] = start ? 1 : 0;
    }
}

// Multi-match build, step 2: one table entry per run: word 1 = (first sorted
// position << 32) | run length. The keys are distinct now, so a CAS that
// finds the key already present cannot happen.
__global__ void __launch_bounds__(256) jm_insert_kernel(ull* slots, int log2cap, const void* key, int kdt,
                                                         const uint32_t* sorted, const uint32_t* starts, uint64_t nruns,
                                                         uint64_t nv, uint32_t* status) {
    const ull cap = 1ull << log2cap;
    for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < nruns; r += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t start = starts[r];
        const uint64_t end = r + 1 < nruns ? starts[r + 1] : nv;
        const uint32_t row = sorted[start];
        const ull k = kdt == BOLT_I32 ? (ull)(ll)__ldg((const int32_t*)key + row) : (ull)__ldg((const ll*)key + row);
        const ull stored = ~k;
        const ull w1 = ((ull)start << 32) | (ull)(end - start);
        if (stored == 0) {
            ull* sp = slots + 2 * cap;
            sp[1] = w1;
            sp[0] = 1ull;
            continue;
        }
        ull h = (stored * JOIN_HASH) >> (64 - log2cap);
        bool placed = false;
        for (ull t = 0; t < cap; ++t) {
            ull* sp = slots + 2 * h;
            if (atomicCAS(sp, 0ull, stored) == 0) {
                sp[1] = w1;
                placed = true;
                break;
            }
            h = (h + 1) & (cap - 1);
        }
        if (!placed) atomicOr(status, ST_FLAG_SPILL);
    }
}

// Rebuilds table t as a multi-match table (the unique-key build found a
// duplicate key): the non-NULL build rows are stably sorted by key (so each
// key's rows stay in ascending order, as in the reference's host join map,
// src/exec/join.rs:843-855), runs of equal keys are marked and compacted, and
// each key maps to its run. The sorted rows stay pinned above the table.
bolt_status join_build_multi(bolt_ctx* ctx, cudaStream_t s, bolt_join_table* t, const bolt_col_view* bk) {
    const uint64_t n = bk->len;
    const uint64_t bytes = ((1ull << t->log2cap) + 1) * 16;
    ctx->arena_used = ctx->arena_pinned;
    uint32_t* sorted = (uint32_t*)arena_alloc(ctx, (n ? n : 1) * 4);
    if (!sorted) return fail(ctx, BOLT_ERR_CAPACITY, "hash join build: no room for the sorted build rows");
    ctx->arena_pinned = ctx->arena_used;
    ull* cnt = (ull*)arena_alloc(ctx, 64);
    uint32_t* valid_ids = bk->validity ? (uint32_t*)arena_alloc(ctx, (n ? n : 1) * 4) : nullptr;
    uint8_t* flag = (uint8_t*)arena_alloc(ctx, n ? n : 1);
    uint32_t* starts = (uint32_t*)arena_alloc(ctx, (n ? n : 1) * 4);
    if (!cnt || !flag || !starts || (bk->validity && !valid_ids))
        return fail(ctx, BOLT_ERR_CAPACITY, "hash join build: scratch arena too small for duplicate keys");
    BOLT_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, 16, s));
    BOLT_CUDA(ctx, cudaMemsetAsync(t->slots, 0, bytes, s));
    uint64_t nv = n;
    if (bk->validity) {  // NULL keys never match: sort only the valid rows
        CompactSpec cv;
        cv.n = n;
        cv.keep_valid_of = bk->validity;
        cv.row_ids = valid_ids;
        cv.n_out_dev = cnt;
        bolt_status st = compact_enqueue(ctx, s, cv);
        if (st != BOLT_OK) return st;
        BOLT_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, cnt, 8, cudaMemcpyDeviceToHost, s));
        BOLT_CUDA(ctx, cudaStreamSynchronize(s));
        nv = ctx->h_words[0];
    }
    t->multi = 1;
    t->sorted_rows = sorted;
    if (nv == 0) return BOLT_OK;
    SortSpec sp;
    sp.src = bk->dtype == BOLT_I32 ? SRC_I32 : SRC_I64;
    sp.indirect = valid_ids ? 1 : 0;
    SortSegment seg;
    seg.keys = bk->data;
    seg.payload_in = valid_ids;
    seg.payload_out = sorted;
    seg.n = nv;
    sp.segs.push_back(seg);
    bolt_status st = radix_sort(ctx, s, sp);
    if (st != BOLT_OK) return st;
    const unsigned g = grid_for(nv, 256, ctx->num_sms * 16);
    jm_mark_kernel<<<g, 256, 0, s>>>(bk->data, bk->dtype, sorted, nv, flag);
    CompactSpec cr;
    cr.n = nv;
    cr.mask = flag;
    cr.row_ids = starts;
    cr.n_out_dev = cnt;
    st = compact_enqueue(ctx, s, cr);
    if (st != BOLT_OK) return st;
    BOLT_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, cnt, 8, cudaMemcpyDeviceToHost, s));
    BOLT_CUDA(ctx, cudaStreamSynchronize(s));
    const uint64_t nruns = ctx->h_words[0];
    jm_insert_kernel<<<grid_for(nruns, 256, ctx->num_sms * 16), 256, 0, s>>>(
        t->slots, t->log2cap, bk->data, bk->dtype, sorted, starts, nruns, nv, ctx->d_status);
    BOLT_CUDA(ctx, cudaGetLastError());
    ctx->last_launches += 2;
    return BOLT_OK;
}

}  // namespace
}  // namespace bolt

using namespace bolt;

extern "C" bolt_status bolt_hash_join_build(bolt_ctx* ctx, const bolt_col_view* build_key, const bolt_col_view* payload,
                                            uint32_t flags, bolt_stream stream, bolt_join_table** table_out) {
    if (!ctx) return BOLT_ERR_INVALID;
    if (!build_key || !table_out) return fail(ctx, BOLT_ERR_INVALID, "hash join build: bad arguments");
    *table_out = nullptr;
    if (build_key->dtype != BOLT_I32 && build_key->dtype != BOLT_I64)
        return fail(ctx, BOLT_DECLINE, "hash join build: key dtype %d (Int32/Int64 supported)", build_key->dtype);
    if (payload && (payload->dtype != BOLT_I32 || payload->len != build_key->len))
        return fail(ctx, BOLT_ERR_INVALID, "hash join build: payload must be an Int32 column of the build length");
    if (!col_aligned(build_key->data, build_key->dtype) || (payload && !col_aligned(payload->data, BOLT_I32)))
        return fail(ctx, BOLT_ERR_INVALID, "hash join build: columns must be aligned to their element width");
    const uint64_t n = build_key->len;
    if (n >= 0xFFFFFFFFull) return fail(ctx, BOLT_DECLINE, "hash join build: %llu rows exceed u32 row ids", (ull)n);
    cudaStream_t s = (cudaStream_t)stream;
    bolt_status st = call_begin(ctx, flags, s);
    if (st != BOLT_OK) return st;
    const int log2cap = ceil_log2_u64(std::max<uint64_t>(2 * n, 64));
    const uint64_t bytes = ((1ull << log2cap) + 1) * 16;
    // The table lives at the bottom of the arena until it is released.
    ctx->arena_pinned = 0;
    ctx->arena_used = 0;
    ull* slots = (ull*)arena_alloc(ctx, bytes);
    if (!slots) return fail(ctx, BOLT_ERR_CAPACITY, "hash join build: %llu-byte table exceeds the scratch arena", (ull)bytes);
    ctx->arena_pinned = ctx->arena_used;
    BOLT_CUDA(ctx, cudaMemsetAsync(slots, 0, bytes, s));
    kernel_mark_begin(ctx, flags, s);
    join_build_kernel<<<grid_for(n, 256, ctx->num_sms * 16), 256, 0, s>>>(
        slots, log2cap, build_key->data, build_key->dtype, build_key->validity,
        payload ? (const int32_t*)payload->data : nullptr, n, ctx->d_status);
    kernel_mark_end(ctx, flags, s);
    ctx->last_launches = 1;
    st = call_end(ctx, flags, s);
    if (st != BOLT_OK) return st;
    bolt_join_table* t = new bolt_join_table();
    t->slots = slots;
    t->log2cap = log2cap;
    t->key_dtype = build_key->dtype;
    t->has_payload = payload != nullptr;
    t->n_build = n;
    t->pinned_mark = 0;
    t->owner = ctx;
    if (!(flags & BOLT_FLAG_ASYNC)) {
        uint32_t f = 0;
        st = read_status(ctx, s, 0, &f);
        if (st == BOLT_OK && f == ST_FLAG_DUPKEY) {
            // Duplicate build keys: rebuild as a multi-match table.
            st = join_build_multi(ctx, s, t, build_key);
            if (st == BOLT_OK) st = read_status(ctx, s, 0, &f);
        }
        if (st == BOLT_OK) st = flags_to_status(ctx, f, "hash join build");
        if (st != BOLT_OK) {
            ctx->arena_pinned = 0;
            delete t;
            return st;
        }
    }
    *table_out = t;
    return BOLT_OK;
}

extern "C" void bolt_hash_join_release(bolt_ctx* ctx, bolt_join_table* t) {
    if (!t) return;
    if (ctx && t->owner == ctx) ctx->arena_pinned = t->pinned_mark;
    delete t;
}

extern "C" bolt_status bolt_hash_join_probe(bolt_ctx* ctx, const bolt_join_table* t, const bolt_col_view* probe_key,
                                            bolt_col_mut* probe_idx, bolt_col_mut* build_idx, uint64_t* n_out,
                                            uint32_t flags, bolt_stream stream) {
    if (!ctx) return BOLT_ERR_INVALID;
    if (!t || !probe_key || !probe_idx || !build_idx || !n_out)
        return fail(ctx, BOLT_ERR_INVALID, "hash join probe: bad arguments");
    if (probe_key->dtype != BOLT_I32 && probe_key->dtype != BOLT_I64)
        return fail(ctx, BOLT_DECLINE, "hash join probe: key dtype %d", probe_key->dtype);
    if (probe_idx->dtype != BOLT_U32 || build_idx->dtype != BOLT_U32)
        return fail(ctx, BOLT_ERR_INVALID, "hash join probe: index outputs must be U32");
    if (probe_key->len >= 0xFFFFFFFFull) return fail(ctx, BOLT_DECLINE, "hash join probe: too many probe rows");
    if (!col_aligned(probe_key->data, probe_key->dtype) || !col_aligned(probe_idx->data, BOLT_U32) ||
        !col_aligned(build_idx->data, BOLT_U32))
        return fail(ctx, BOLT_ERR_INVALID, "hash join probe: columns must be aligned to their element width");
    cudaStream_t s = (cudaStream_t)stream;
    bolt_status st = call_begin(ctx, flags, s);
    if (st != BOLT_OK) return st;
    ProbeArgs a{};
    a.slots = t->slots;
    a.log2cap = t->log2cap;
    a.kdt = probe_key->dtype;
    a.key = probe_key->data;
    a.kvalid = probe_key->validity;
    a.n = probe_key->len;
    a.out_probe = (uint32_t*)probe_idx->data;
    a.out_build = (uint32_t*)build_idx->data;
    a.out_cap = std::min(probe_idx->cap, build_idx->cap);
    a.sorted_rows = t->sorted_rows;
    const uint64_t ntiles = (a.n + JP_TILE - 1) / JP_TILE;
    a.lookback = (ull*)arena_alloc(ctx, (ntiles + 1) * 8);
    a.tile_ctr = (uint32_t*)arena_alloc(ctx, 64);
    a.n_out = (ull*)arena_alloc(ctx, 64);
    if (!a.lookback || !a.tile_ctr || !a.n_out) return fail(ctx, BOLT_ERR_CAPACITY, "hash join probe: scratch arena too small");
    a.status = ctx->d_status;
    BOLT_CUDA(ctx, cudaMemsetAsync(a.lookback, 0, (ntiles + 1) * 8, s));
    BOLT_CUDA(ctx, cudaMemsetAsync(a.tile_ctr, 0, 64, s));
    BOLT_CUDA(ctx, cudaMemsetAsync(a.n_out, 0, 64, s));
    if (ntiles) {
        kernel_mark_begin(ctx, flags, s);
        if (t->multi) join_probe_kernel<true><<<(unsigned)ntiles, JP_BLOCK, 0, s>>>(a);
        else join_probe_kernel<false><<<(unsigned)ntiles, JP_BLOCK, 0, s>>>(a);
        kernel_mark_end(ctx, flags, s);
        ctx->last_launches = 1;
    }
    st = call_end(ctx, flags, s);
    if (st != BOLT_OK) return st;
    if (flags & BOLT_FLAG_ASYNC) return BOLT_OK;
    uint32_t f = 0;
    st = read_status(ctx, s, 0, &f);
    if (st != BOLT_OK) return st;
    ull v = 0;
    BOLT_CUDA(ctx, cudaMemcpy(&v, a.n_out, 8, cudaMemcpyDeviceToHost));
    *n_out = v;
    return flags_to_status(ctx, f, "hash join probe");
}
