// groupby_wide.cu — GROUP BY over two integer key columns that together do
// not pack into 64 bits (at least one of them Int64).
//
// Replaces the reference's host wide-key reduction, execute_groupby_wide
// (src/exec/groupby_wide.rs:85-262), for integer keys without a WHERE. The
// reference folds every row into a BTreeMap keyed by the key tuple; here the
// rows are sorted instead and each group is one run of the sorted order:
//
//   1. rows with a NULL in either key are dropped (groupby_wide.rs:153-158):
//      a byte mask and one order-preserving compaction give the kept row ids;
//   2. two stable LSD radix sorts (by key1, then by key0) order the kept rows
//      by (key0, key1) as signed integers, rows of one key in row order
//      (cmp_tuple, groupby_wide.rs:410);
//   3. run starts are marked and compacted: start g is group g's first
//      position, and the number of starts is the group count;
//   4. one warp per group folds each aggregate over the group's rows in row
//      order, so every result equals the reference's sequential fold bit for
//      bit: SUM over integers wraps in i64 (groupby_wide.rs:695-705), SUM and
//      AVG over floats add in f64, MIN / MAX keep the first valid value and
//      replace it only when x < v / x > v (a NaN never replaces a value, a
//      leading NaN stays), COUNT(col) counts valid inputs.
//
// The one difference from the reference: an aggregate whose group saw no
// valid input is NULL here (data 0, validity bit clear), as on every other
// GROUP BY path of this library; the reference emits the accumulator's
// initial value (0 for SUM and AVG, the type's extreme for MIN / MAX).
#include <algorithm>
#include <climits>

#include "compact.cuh"
#include "groupby.cuh"
#include "radix_sort.cuh"

namespace bolt {
namespace {

struct WideAgg {
    const void* in;
    const uint8_t* in_valid;
    void* out;
    uint8_t* out_valid;
    int32_t op;
    int32_t in_dtype;
    int32_t out_dtype;
    int32_t fold_f;  // fold in f64 (float inputs, and AVG of any input)
};

struct WideArgs {
    const void* key[2];
    int32_t kdt[2];
    void* out_key[2];
    uint8_t* out_key_valid[2];
    const uint32_t* perm;     // kept rows sorted by (key0, key1, row)
    const uint32_t* starts;   // first sorted position of each group
    uint64_t n_groups;
    uint64_t n_kept;
    uint64_t n_write;         // groups written: min(n_groups, output capacity)
    int32_t n_aggs;
    WideAgg agg[GB_MAX_AGGS];
};

__device__ __forceinline__ ll wide_load_i(const void* p, int dt, uint32_t r) {
    return dt == BOLT_I32 ? (ll)__ldg((const int32_t*)p + r) : __ldg((const ll*)p + r);
}

__device__ __forceinline__ double wide_load_f(const void* p, int dt, uint32_t r) {
    switch (dt) {
    case BOLT_I32: return (double)__ldg((const int32_t*)p + r);
    case BOLT_I64: return (double)__ldg((const ll*)p + r);
    case BOLT_F32: return (double)__ldg((const float*)p + r);
    default: return __ldg((const double*)p + r);
    }
}

// flag[i] = 1 when neither key of row i is NULL.
__global__ void __launch_bounds__(256) wide_valid_kernel(const uint8_t* v0, const uint8_t* v1, uint64_t n,
                                                          uint8_t* flag) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = (bit_valid(v0, i) && bit_valid(v1, i)) ? 1 : 0;
}

// flag[i] = 1 when sorted position i starts a run of equal (key0, key1).
__global__ void __launch_bounds__(256) wide_mark_kernel(const void* k0, int dt0, const void* k1, int dt1,
                                                         const uint32_t* perm, uint64_t n, uint8_t* flag) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        bool start = i == 0;
        if (!start) {
            const uint32_t r = perm[i];
            const uint32_t p = perm[i - 1];
            start = wide_load_i(k0, dt0, r) != wide_load_i(k0, dt0, p) ||
                    wide_load_i(k1, dt1, r) != wide_load_i(k1, dt1, p);
        }
        flag[i] = start ? 1 : 0;
    }
}

constexpr int WIDE_PF = 4;  // 32-row chunks of a fold in flight per warp

// One lane's element of a 32-row chunk of a group: validity and value.
struct WideElem {
    bool v;
    ll xi;
    double xf;
};

__device__ __forceinline__ WideElem wide_elem(const WideArgs& a, const WideAgg& w, uint64_t j, uint64_t end) {
    WideElem e = {false, 0, 0.0};
    if (j < end) {
        const uint32_t r = a.perm[j];
        e.v = bit_valid(w.in_valid, r);
        if (e.v && w.op != BOLT_AGG_COUNT) {
            if (w.fold_f) e.xf = wide_load_f(w.in, w.in_dtype, r);
            else e.xi = wide_load_i(w.in, w.in_dtype, r);
        }
    }
    return e;
}

// One warp per group: the group's keys from its first row, then every
// aggregate over the group's rows. Integer aggregates (wrapping SUM, COUNT,
// MIN / MAX) do not depend on the order: each lane folds its own rows
// (WIDE_PF chunks loaded at a time) and the warp reduces at the end. Float
// aggregates fold in row order: each 32-row chunk is loaded by the lanes
// together (WIDE_PF chunks ahead of the fold), then every lane walks the
// chunk's 32 values in order through shuffles, keeping the same accumulator.
__global__ void __launch_bounds__(256) wide_fold_kernel(const __grid_constant__ WideArgs a) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t g = warp; g < a.n_write; g += n_warps) {
        const uint64_t beg = a.starts[g];
        const uint64_t end = g + 1 < a.n_groups ? a.starts[g + 1] : a.n_kept;
        if (lane < 2) {
            const ll kv = wide_load_i(a.key[lane], a.kdt[lane], a.perm[beg]);
            if (a.kdt[lane] == BOLT_I32) ((int32_t*)a.out_key[lane])[g] = (int32_t)kv;
            else ((ll*)a.out_key[lane])[g] = kv;
            if (a.out_key_valid[lane]) set_bit_atomic(a.out_key_valid[lane], g, true);
        }
        for (int q = 0; q < a.n_aggs; ++q) {
            const WideAgg& w = a.agg[q];
            uint64_t cnt = 0;
            ull si = 0;       // integer SUM (wrapping)
            ll mi = 0;        // integer MIN / MAX
            double f = 0.0;   // float SUM, AVG numerator, float MIN / MAX
            bool seen = false;
            if (w.op == BOLT_AGG_COUNT_STAR) {
                cnt = end - beg;
            } else if (!w.fold_f) {
                const bool is_min = w.op == BOLT_AGG_MIN;
                ll lm = is_min ? LLONG_MAX : LLONG_MIN;
                bool lseen = false;
                for (uint64_t c = beg; c < end; c += 32 * WIDE_PF) {
                    WideElem e[WIDE_PF];  // every load of WIDE_PF chunks issued before any is used
#pragma unroll
                    for (int p = 0; p < WIDE_PF; ++p) e[p] = wide_elem(a, w, c + (uint64_t)p * 32 + lane, end);
#pragma unroll
                    for (int p = 0; p < WIDE_PF; ++p) {
                        cnt += (uint64_t)__popc(__ballot_sync(0xffffffffu, e[p].v));
                        if (e[p].v) {
                            si += (ull)e[p].xi;
                            lm = is_min ? (e[p].xi < lm ? e[p].xi : lm) : (e[p].xi > lm ? e[p].xi : lm);
                            lseen = true;
                        }
                    }
                }
                seen = __any_sync(0xffffffffu, lseen);
                for (int o = 16; o > 0; o >>= 1) {
                    si += __shfl_xor_sync(0xffffffffu, si, o);
                    const ll y = __shfl_xor_sync(0xffffffffu, lm, o);
                    lm = is_min ? (y < lm ? y : lm) : (y > lm ? y : lm);
                }
                mi = lm;
            } else {
                const int kind = (w.op == BOLT_AGG_SUM || w.op == BOLT_AGG_AVG) ? 0 : (w.op == BOLT_AGG_MIN ? 1 : 2);
                // WIDE_PF chunks in flight: chunk i + WIDE_PF is loaded
                // before chunk i is folded. Lanes past the group's end load
                // nothing and hold no valid value.
                WideElem buf[WIDE_PF];
#pragma unroll
                for (int p = 0; p < WIDE_PF; ++p) buf[p] = wide_elem(a, w, beg + (uint64_t)p * 32 + lane, end);
                for (uint64_t c = beg; c < end; c += 32 * WIDE_PF) {
#pragma unroll
                    for (int p = 0; p < WIDE_PF; ++p) {
                        const WideElem e = buf[p];
                        buf[p] = wide_elem(a, w, c + (uint64_t)(p + WIDE_PF) * 32 + lane, end);
                        const unsigned m = __ballot_sync(0xffffffffu, e.v);
                        if (m == 0) continue;  // warp-uniform
                        cnt += (uint64_t)__popc(m);
                        if (kind == 0) {
#pragma unroll
                            for (int t = 0; t < 32; ++t) {
                                const double x = __shfl_sync(0xffffffffu, e.xf, t);
                                f = ((m >> t) & 1) ? f + x : f;
                            }
                        } else {
#pragma unroll
                            for (int t = 0; t < 32; ++t) {
                                const double x = __shfl_sync(0xffffffffu, e.xf, t);
                                const bool on = (m >> t) & 1;
                                const bool take = on && (!seen || (kind == 1 ? x < f : x > f));
                                f = take ? x : f;
                                seen = seen || on;
                            }
                        }
                    }
                }
                if (kind == 0) seen = cnt > 0;
            }
            if (lane != 0) continue;
            bool valid = true;
            switch (w.op) {
            case BOLT_AGG_COUNT_STAR:
            case BOLT_AGG_COUNT:
                ((ll*)w.out)[g] = (ll)cnt;
                break;
            case BOLT_AGG_AVG:
                valid = cnt > 0;
                ((double*)w.out)[g] = valid ? f / (double)cnt : 0.0;
                break;
            default:  // SUM, MIN, MAX
                valid = seen;
                if (w.out_dtype == BOLT_F64) ((double*)w.out)[g] = valid ? f : 0.0;
                else if (w.out_dtype == BOLT_F32) ((float*)w.out)[g] = valid ? (float)f : 0.0f;
                else if (w.out_dtype == BOLT_I32) ((int32_t*)w.out)[g] = valid ? (int32_t)mi : 0;
                else ((ll*)w.out)[g] = valid ? (w.op == BOLT_AGG_SUM ? (ll)si : mi) : 0;
                break;
            }
            if (w.out_valid) set_bit_atomic(w.out_valid, g, valid);
        }
    }
}

}  // namespace

bool gb_wide_applies(const bolt_groupby_desc* d) {
    if (!d || !d->cols || !d->key_cols || d->n_keys != 2 || d->n_preds != 0) return false;
    int dt[2];
    for (int k = 0; k < 2; ++k) {
        const int c = d->key_cols[k];
        if (c < 0 || c >= d->n_cols) return false;
        dt[k] = d->cols[c].dtype;
        if (dt[k] != BOLT_I32 && dt[k] != BOLT_I64) return false;
    }
    return dt[0] == BOLT_I64 || dt[1] == BOLT_I64;
}

bolt_status gb_wide(bolt_ctx* ctx, const bolt_groupby_desc* d, bolt_groupby_out* out, uint32_t flags,
                    cudaStream_t s) {
    if (!out || !out->keys) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: missing output");
    if (flags & BOLT_FLAG_ASYNC)
        return fail(ctx, BOLT_DECLINE, "GROUP BY: keys wider than 64 bits need a synchronous call");
    if (d->n_aggs < 1 || d->n_aggs > GB_MAX_AGGS || !d->aggs)
        return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: %d aggregates", d->n_aggs);
    WideArgs wa = {};
    const bolt_col_view* kc[2] = {&d->cols[d->key_cols[0]], &d->cols[d->key_cols[1]]};
    const uint64_t n = kc[0]->len;
    uint64_t out_cap = UINT64_MAX;
    for (int k = 0; k < 2; ++k) {
        if (kc[k]->len != n) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: key columns differ in length");
        if (!col_aligned(kc[k]->data, kc[k]->dtype))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: key column %d is not aligned to its element width", k);
        if (out->keys[k].dtype != kc[k]->dtype)
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output key column %d dtype mismatch", k);
        if (!col_aligned(out->keys[k].data, kc[k]->dtype))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output key column %d is not aligned", k);
        wa.key[k] = kc[k]->data;
        wa.kdt[k] = kc[k]->dtype;
        wa.out_key[k] = out->keys[k].data;
        wa.out_key_valid[k] = out->keys[k].validity;
        out_cap = std::min<uint64_t>(out_cap, out->keys[k].cap);
    }
    if (n >= (1ull << 30)) return fail(ctx, BOLT_DECLINE, "GROUP BY: wide keys over %llu rows exceed 2^30", (ull)n);
    wa.n_aggs = d->n_aggs;
    for (int q = 0; q < d->n_aggs; ++q) {
        const bolt_agg_spec& sp = d->aggs[q];
        WideAgg& w = wa.agg[q];
        w.op = sp.op;
        const bool star = sp.op == BOLT_AGG_COUNT_STAR;
        const bolt_col_view* c = nullptr;
        if (!star) {
            if (sp.input_col < 0 || sp.input_col >= d->n_cols)
                return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: aggregate %d input column out of range", q);
            c = &d->cols[sp.input_col];
            if (c->len < n) return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: value column shorter than the rows");
            if (!col_aligned(c->data, c->dtype))
                return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: aggregate %d input is not aligned to its element width", q);
        }
        const int dt = c ? c->dtype : BOLT_I64;
        w.in = c ? c->data : nullptr;
        w.in_valid = c ? c->validity : nullptr;
        w.in_dtype = dt;
        switch (sp.op) {
        case BOLT_AGG_COUNT_STAR:
        case BOLT_AGG_COUNT:
            w.out_dtype = BOLT_I64;
            break;
        case BOLT_AGG_SUM:
            if (dt != BOLT_I32 && dt != BOLT_I64 && dt != BOLT_F64)
                return fail(ctx, BOLT_DECLINE, "GROUP BY: SUM over dtype %d with wide keys", dt);
            w.out_dtype = dt == BOLT_F64 ? BOLT_F64 : BOLT_I64;
            w.fold_f = dt == BOLT_F64;
            break;
        case BOLT_AGG_AVG:
            if (dt != BOLT_I32 && dt != BOLT_I64 && dt != BOLT_F64)
                return fail(ctx, BOLT_DECLINE, "GROUP BY: AVG over dtype %d with wide keys", dt);
            w.out_dtype = BOLT_F64;
            w.fold_f = 1;
            break;
        case BOLT_AGG_MIN:
        case BOLT_AGG_MAX:
            if (dt != BOLT_I32 && dt != BOLT_I64 && dt != BOLT_F32 && dt != BOLT_F64)
                return fail(ctx, BOLT_DECLINE, "GROUP BY: MIN/MAX over dtype %d with wide keys", dt);
            w.out_dtype = dt;
            w.fold_f = dt == BOLT_F32 || dt == BOLT_F64;
            break;
        default:
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: unknown aggregate op %d", sp.op);
        }
        if (!out->aggs || out->aggs[q].dtype != w.out_dtype)
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output column %d must have dtype %d", q, w.out_dtype);
        if (!col_aligned(out->aggs[q].data, w.out_dtype))
            return fail(ctx, BOLT_ERR_INVALID, "GROUP BY: output column %d is not aligned to its element width", q);
        w.out = out->aggs[q].data;
        w.out_valid = out->aggs[q].validity;
        out_cap = std::min<uint64_t>(out_cap, out->aggs[q].cap);
    }

    bolt_status st = call_begin(ctx, flags, s);
    if (st != BOLT_OK) return st;
    ctx->last_tier = 3;
    const uint64_t nb = n ? n : 1;
    ull* cnt = (ull*)arena_alloc(ctx, 256);
    const bool key_nulls = kc[0]->validity || kc[1]->validity;
    uint32_t* kept = key_nulls ? (uint32_t*)arena_alloc(ctx, nb * 4) : nullptr;
    uint8_t* flag = (uint8_t*)arena_alloc(ctx, nb);
    uint32_t* by_k1 = (uint32_t*)arena_alloc(ctx, nb * 4);
    uint32_t* perm = (uint32_t*)arena_alloc(ctx, nb * 4);
    uint32_t* starts = (uint32_t*)arena_alloc(ctx, nb * 4);
    if (!cnt || !flag || !by_k1 || !perm || !starts || (key_nulls && !kept))
        return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: scratch arena too small for the wide-key sort");
    const unsigned grid = grid_for(n, 256, ctx->num_sms * 16);
    uint32_t launches = 0;
    kernel_mark_begin(ctx, flags, s);
    uint64_t n_kept = n;
    if (key_nulls && n) {
        wide_valid_kernel<<<grid, 256, 0, s>>>(kc[0]->validity, kc[1]->validity, n, flag);
        CompactSpec cv;
        cv.n = n;
        cv.mask = flag;
        cv.row_ids = kept;
        cv.n_out_dev = cnt;
        st = compact_enqueue(ctx, s, cv);
        if (st != BOLT_OK) return st;
        BOLT_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, cnt, 8, cudaMemcpyDeviceToHost, s));
        BOLT_CUDA(ctx, cudaStreamSynchronize(s));
        n_kept = ctx->h_words[0];
        launches += 1;
    }
    uint64_t n_groups = 0;
    if (n_kept) {
        for (int k = 1; k >= 0; --k) {  // LSD over the key columns: key1 first
            SortSpec sp;
            sp.src = kc[k]->dtype == BOLT_I32 ? SRC_I32 : SRC_I64;
            SortSegment seg;
            seg.keys = kc[k]->data;
            seg.payload_in = k == 1 ? kept : by_k1;
            seg.payload_out = k == 1 ? by_k1 : perm;
            seg.n = n_kept;
            sp.indirect = seg.payload_in != nullptr;
            sp.segs.push_back(seg);
            st = radix_sort(ctx, s, sp);
            if (st != BOLT_OK) return st;
        }
        wide_mark_kernel<<<grid_for(n_kept, 256, ctx->num_sms * 16), 256, 0, s>>>(
            kc[0]->data, kc[0]->dtype, kc[1]->data, kc[1]->dtype, perm, n_kept, flag);
        CompactSpec cr;
        cr.n = n_kept;
        cr.mask = flag;
        cr.row_ids = starts;
        cr.n_out_dev = cnt;
        st = compact_enqueue(ctx, s, cr);
        if (st != BOLT_OK) return st;
        BOLT_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, cnt, 8, cudaMemcpyDeviceToHost, s));
        BOLT_CUDA(ctx, cudaStreamSynchronize(s));
        n_groups = ctx->h_words[0];
        launches += 1;
    }
    wa.perm = perm;
    wa.starts = starts;
    wa.n_groups = n_groups;
    wa.n_kept = n_kept;
    wa.n_write = std::min<uint64_t>(n_groups, out_cap);
    if (wa.n_write) {
        const unsigned blocks = (unsigned)std::min<uint64_t>((wa.n_write + 7) / 8, (uint64_t)ctx->num_sms * 8);
        wide_fold_kernel<<<blocks, 256, 0, s>>>(wa);
        BOLT_CUDA(ctx, cudaGetLastError());
        launches += 1;
    }
    kernel_mark_end(ctx, flags, s);
    ctx->last_launches += launches;  // the sorts and compactions count their own
    st = call_end(ctx, flags, s);
    if (st != BOLT_OK) return st;
    out->n_groups = n_groups;
    uint32_t f = 0;
    st = read_status(ctx, s, 0, &f);
    if (st != BOLT_OK) return st;
    st = flags_to_status(ctx, f, "GROUP BY");
    if (st != BOLT_OK) return st;
    if (n_groups > out_cap)
        return fail(ctx, BOLT_ERR_CAPACITY, "GROUP BY: %llu groups exceed the output capacity %llu", (ull)n_groups,
                    (ull)out_cap);
    return BOLT_OK;
}

}  // namespace bolt
