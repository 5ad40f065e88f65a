/*
 * bolt_oracle.c — CPU restatement of the reference's relational hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker and the timed CPU baseline.
 * Nothing in the product library links, loads or calls this file.
 *
 * Reference files restated (Craton Bolt, Rust; paths inside its project):
 *   key packing ........ src/exec/groupby_common.rs:302-514 (pack_keys,
 *                        canonicalise_f64/_f32, decode_key)
 *   GROUP BY ........... src/exec/groupby.rs:295-833 (execute_groupby: NULL
 *                        group at i64::MAX sorted last, output sorted by the
 *                        packed key, :789-800), groupby.rs:1775-1798
 *                        (checked_group_sum: per-group checked i64 add in
 *                        row order), logical_plan.rs:2191-2215
 *                        (sum_output_dtype), groupby.rs:2877-2885 (AVG)
 *   host reduction ..... src/exec/engine.rs:380-620 (host_multi_agg_groupby)
 *   float MIN/MAX ...... tests/semantics_e2e.rs:359-440 (NaN is the largest)
 *   decimal SUM ........ src/exec/aggregate.rs:1220 (checked i128 add)
 *   join ............... src/exec/join.rs:843-858 (build_hash_map + probe),
 *                        join.rs:1-60 (NULL keys never match)
 *   sort keys .......... src/exec/gpu_sort.rs:1089-1163
 *   compaction ......... src/exec/compact.rs:61-146
 *   fixtures ........... tests/common/mod.rs:46-111
 */
#include "bolt_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef __int128 i128;

static int g_threads = 1;
void orc_set_threads(int32_t n) { g_threads = n < 1 ? 1 : n; }

static inline int is_valid(const uint8_t* v, uint64_t i) {
    return v == NULL || ((v[i >> 3] >> (i & 7)) & 1);
}

/* ---- column reads -------------------------------------------------------- */
static inline int64_t col_i64(const orc_col* c, uint64_t i) {
    switch (c->dtype) {
    case ORC_I32: return (int64_t)((const int32_t*)c->data)[i];
    case ORC_I64: return ((const int64_t*)c->data)[i];
    case ORC_U32: return (int64_t)((const uint32_t*)c->data)[i];
    case ORC_DEC128: return ((const int64_t*)c->data)[2 * i];
    default: return 0;
    }
}
static inline double col_f64(const orc_col* c, uint64_t i) {
    switch (c->dtype) {
    case ORC_F32: return (double)((const float*)c->data)[i];
    case ORC_F64: return ((const double*)c->data)[i];
    default: return (double)col_i64(c, i);
    }
}
static inline i128 col_i128(const orc_col* c, uint64_t i) {
    if (c->dtype == ORC_DEC128) {
        const uint64_t* p = (const uint64_t*)c->data;
        uint64_t lo = p[2 * i], hi = p[2 * i + 1];
        return (i128)(((unsigned __int128)hi << 64) | lo);
    }
    return (i128)col_i64(c, i);
}
static inline int is_float(int dt) { return dt == ORC_F32 || dt == ORC_F64; }

/* canonicalise_f64 / _f32 (groupby_common.rs:302-330). */
static inline uint64_t canon_f64_bits(double x) {
    if (isnan(x)) return 0x7FF8000000000000ull;
    if (x == 0.0) return 0;
    uint64_t b; memcpy(&b, &x, 8); return b;
}
static inline uint32_t canon_f32_bits(float x) {
    if (isnan(x)) return 0x7FC00000u;
    if (x == 0.0f) return 0;
    uint32_t b; memcpy(&b, &x, 4); return b;
}

/* pack_keys (groupby_common.rs:352): lossless i64 packing. */
static inline uint32_t key_bits32(const orc_col* c, uint64_t i) {
    if (c->dtype == ORC_F32) return canon_f32_bits(((const float*)c->data)[i]);
    return (uint32_t)((const int32_t*)c->data)[i];
}
int64_t orc_pack_key(const orc_col* cols, const int32_t* key_cols, int32_t n_keys, uint64_t row) {
    const orc_col* a = &cols[key_cols[0]];
    if (n_keys == 1) {
        switch (a->dtype) {
        case ORC_I32: return (int64_t)((const int32_t*)a->data)[row];
        case ORC_I64: return ((const int64_t*)a->data)[row];
        case ORC_F32: return (int64_t)(uint64_t)canon_f32_bits(((const float*)a->data)[row]);
        case ORC_F64: return (int64_t)canon_f64_bits(((const double*)a->data)[row]);
        default: return 0;
        }
    }
    const orc_col* b = &cols[key_cols[1]];
    uint64_t hi = key_bits32(a, row), lo = key_bits32(b, row);
    return (int64_t)((hi << 32) | lo);
}

int orc_row_passes(const orc_col* cols, const orc_pred* preds, int32_t n_preds, uint64_t row) {
    for (int32_t p = 0; p < n_preds; ++p) {
        const orc_col* c = &cols[preds[p].col];
        if (!is_valid(c->validity, row)) return 0;
        int r;
        if (is_float(c->dtype)) {
            double v = col_f64(c, row), l = preds[p].lit_f;
            switch (preds[p].cmp) {
            case ORC_LT: r = v < l; break;
            case ORC_LE: r = v <= l; break;
            case ORC_GT: r = v > l; break;
            case ORC_GE: r = v >= l; break;
            case ORC_EQ: r = v == l; break;
            default: r = v != l; break;
            }
        } else {
            int64_t v = col_i64(c, row), l = preds[p].lit_i;
            switch (preds[p].cmp) {
            case ORC_LT: r = v < l; break;
            case ORC_LE: r = v <= l; break;
            case ORC_GT: r = v > l; break;
            case ORC_GE: r = v >= l; break;
            case ORC_EQ: r = v == l; break;
            default: r = v != l; break;
            }
        }
        if (!r) return 0;
    }
    return 1;
}

/* ---- open-addressing map u64 -> group index ------------------------------ */
typedef struct { uint64_t* keys; uint32_t* idx; uint64_t cap; } omap;
static inline uint64_t mix64(uint64_t x) {
    x ^= x >> 33; x *= 0xff51afd7ed558ccdull; x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull; x ^= x >> 33; return x;
}
static int omap_init(omap* m, uint64_t expect) {
    uint64_t cap = 64;
    while (cap < expect * 2) cap <<= 1;
    m->cap = cap;
    m->keys = (uint64_t*)malloc(cap * 8);
    m->idx = (uint32_t*)malloc(cap * 4);
    if (!m->keys || !m->idx) return -1;
    memset(m->idx, 0xFF, cap * 4);
    return 0;
}
static void omap_free(omap* m) { free(m->keys); free(m->idx); }
static int omap_grow(omap* m) {
    omap n;
    n.cap = m->cap * 2;
    n.keys = (uint64_t*)malloc(n.cap * 8);
    n.idx = (uint32_t*)malloc(n.cap * 4);
    if (!n.keys || !n.idx) return -1;
    memset(n.idx, 0xFF, n.cap * 4);
    for (uint64_t i = 0; i < m->cap; ++i) {
        if (m->idx[i] == 0xFFFFFFFFu) continue;
        uint64_t h = mix64(m->keys[i]) & (n.cap - 1);
        while (n.idx[h] != 0xFFFFFFFFu) h = (h + 1) & (n.cap - 1);
        n.keys[h] = m->keys[i]; n.idx[h] = m->idx[i];
    }
    omap_free(m);
    *m = n;
    return 0;
}
/* Returns the group index of key, inserting next_idx when absent. */
static inline uint32_t omap_get(omap* m, uint64_t key, uint32_t next_idx, int* inserted) {
    uint64_t h = mix64(key) & (m->cap - 1);
    for (;;) {
        uint32_t ix = m->idx[h];
        if (ix == 0xFFFFFFFFu) {
            m->keys[h] = key; m->idx[h] = next_idx; *inserted = 1; return next_idx;
        }
        if (m->keys[h] == key) { *inserted = 0; return ix; }
        h = (h + 1) & (m->cap - 1);
    }
}
static inline int64_t omap_find(const omap* m, uint64_t key) {
    uint64_t h = mix64(key) & (m->cap - 1);
    for (;;) {
        uint32_t ix = m->idx[h];
        if (ix == 0xFFFFFFFFu) return -1;
        if (m->keys[h] == key) return ix;
        h = (h + 1) & (m->cap - 1);
    }
}

/* ---- GROUP BY ------------------------------------------------------------ */
typedef struct {
    int64_t key;
    int is_null;
    uint32_t row_first;
} grp_t;

/* Per group, per aggregate accumulator. */
typedef struct {
    i128 isum;        /* integer / decimal SUM (checked in row order)   */
    double fsum;      /* sequential f64 SUM (row order)                  */
    double csum, comp;/* Neumaier compensated sum                        */
    int64_t cnt;      /* COUNT(col) / COUNT(*)                           */
    uint64_t mnk, mxk;/* MIN/MAX order keys (valid when cnt > 0)         */
} acc_t;

/* Order-preserving u64 key used for MIN/MAX (NaN largest, -0 == +0). */
static inline uint64_t mm_key(const orc_col* c, uint64_t i) {
    if (is_float(c->dtype)) {
        uint64_t b = canon_f64_bits(col_f64(c, i));
        uint64_t mask = (uint64_t)(((int64_t)b) >> 63) | 0x8000000000000000ull;
        return b ^ mask;
    }
    return (uint64_t)col_i64(c, i) ^ 0x8000000000000000ull;
}
static inline double mm_key_to_f64(uint64_t k) {
    uint64_t b = (k & 0x8000000000000000ull) ? (k ^ 0x8000000000000000ull) : ~k;
    double d; memcpy(&d, &b, 8); return d;
}

static int cmp_grp(const void* x, const void* y) {
    const grp_t* a = (const grp_t*)x; const grp_t* b = (const grp_t*)y;
    if (a->is_null != b->is_null) return a->is_null - b->is_null;
    if (a->key < b->key) return -1;
    if (a->key > b->key) return 1;
    return 0;
}

/* One GROUP BY fold in progress: the key map, the groups in first-seen
 * order and their accumulators. */
typedef struct {
    const orc_col* cols;
    const int32_t* key_cols;
    int32_t n_keys;
    const orc_agg* aggs;
    int32_t n_aggs;
    omap m;
    uint64_t ng, gcap;
    grp_t* groups;
    acc_t* acc;
    int64_t null_group;
    int status;
    char err[256];
} gb_state;

static int gbs_init(gb_state* s, const orc_col* cols, const int32_t* key_cols, int32_t n_keys,
                    const orc_agg* aggs, int32_t n_aggs, uint64_t expect) {
    memset(s, 0, sizeof *s);
    s->cols = cols; s->key_cols = key_cols; s->n_keys = n_keys; s->aggs = aggs; s->n_aggs = n_aggs;
    s->null_group = -1;
    s->gcap = expect < 1024 ? 1024 : expect;
    if (omap_init(&s->m, s->gcap)) return -1;
    s->groups = (grp_t*)malloc(s->gcap * sizeof(grp_t));
    s->acc = (acc_t*)calloc(s->gcap * (uint64_t)n_aggs, sizeof(acc_t));
    return (s->groups && s->acc) ? 0 : -1;
}

static void gbs_free(gb_state* s) {
    omap_free(&s->m);
    free(s->groups);
    free(s->acc);
}

/* Folds row r (it passed the WHERE conjunction; a multi-column key with a
 * NULL part was already dropped, groupby.rs:600-615) into its group. The
 * accumulators follow the reference's host fold in row order: checked i64
 * SUM (checked_group_sum, groupby.rs:1775-1798), sequential f64 SUM,
 * checked i128 Decimal SUM (aggregate.rs:1220). */
static void gbs_fold_row(gb_state* st, uint64_t r, int key_null) {
    const orc_col* cols = st->cols;
    uint32_t g;
    if (key_null) {
        if (st->null_group < 0) {
            st->null_group = (int64_t)st->ng;
            goto new_group;
        }
        g = (uint32_t)st->null_group;
    } else {
        int ins;
        int64_t key = orc_pack_key(cols, st->key_cols, st->n_keys, r);
        if (st->ng * 2 >= st->m.cap && omap_grow(&st->m)) { st->status = ORC_CAPACITY; return; }
        g = omap_get(&st->m, (uint64_t)key, (uint32_t)st->ng, &ins);
        if (ins) goto new_group;
    }
    goto have_group;
new_group:
    if (st->ng == st->gcap) {
        uint64_t nc = st->gcap * 2;
        st->groups = (grp_t*)realloc(st->groups, nc * sizeof(grp_t));
        st->acc = (acc_t*)realloc(st->acc, nc * (uint64_t)st->n_aggs * sizeof(acc_t));
        memset(st->acc + st->gcap * (uint64_t)st->n_aggs, 0, (nc - st->gcap) * (uint64_t)st->n_aggs * sizeof(acc_t));
        st->gcap = nc;
    }
    g = (uint32_t)st->ng++;
    st->groups[g].is_null = key_null;
    st->groups[g].key = key_null ? INT64_MAX : orc_pack_key(cols, st->key_cols, st->n_keys, r);
    st->groups[g].row_first = (uint32_t)r;
have_group:
    for (int32_t a = 0; a < st->n_aggs; ++a) {
        acc_t* s = &st->acc[(uint64_t)g * st->n_aggs + a];
        int op = st->aggs[a].op;
        if (op == ORC_COUNT_STAR) { s->cnt++; continue; }
        const orc_col* c = &cols[st->aggs[a].input_col];
        if (!is_valid(c->validity, r)) continue;
        if (op == ORC_COUNT) { s->cnt++; continue; }
        if (op == ORC_MIN || op == ORC_MAX) {
            uint64_t k = mm_key(c, r);
            if (s->cnt == 0) { s->mnk = s->mxk = k; }
            else { if (k < s->mnk) s->mnk = k; if (k > s->mxk) s->mxk = k; }
            s->cnt++;
            continue;
        }
        /* SUM / AVG */
        s->cnt++;
        if (is_float(c->dtype)) {
            double v = col_f64(c, r);
            s->fsum += v;
            double t = s->csum + v;
            if (fabs(s->csum) >= fabs(v)) s->comp += (s->csum - t) + v;
            else s->comp += (v - t) + s->csum;
            s->csum = t;
        } else if (c->dtype == ORC_DEC128) {
            i128 v = col_i128(c, r), out;
            if (__builtin_add_overflow(s->isum, v, &out)) {
                if (st->status == ORC_OK) {
                    snprintf(st->err, sizeof st->err,
                             "SUM(Decimal128) precision overflow: accumulator exceeds i128 range");
                    st->status = ORC_OVERFLOW;
                }
            } else s->isum = out;
        } else {
            int64_t v = col_i64(c, r);
            if (c->dtype == ORC_I64 && op == ORC_SUM) {
                /* checked_group_sum (groupby.rs:1775): checked i64 add in row order */
                int64_t cur = (int64_t)s->isum, out;
                if (__builtin_add_overflow(cur, v, &out)) {
                    if (st->status == ORC_OK) {
                        snprintf(st->err, sizeof st->err, "SUM(integer) overflow: accumulator exceeds i64 range");
                        st->status = ORC_OVERFLOW;
                    }
                } else s->isum = out;
            } else {
                s->isum += v;
            }
        }
    }
}

/* Group indices in output order: packed key ascending as i64, NULL group
 * last (groupby.rs:789-800). */
static uint32_t* gbs_order(const gb_state* st) {
    const uint64_t ng = st->ng;
    uint32_t* order = (uint32_t*)malloc((ng ? ng : 1) * sizeof(uint32_t));
    grp_t* sorted = (grp_t*)malloc((ng ? ng : 1) * sizeof(grp_t));
    for (uint64_t g = 0; g < ng; ++g) { sorted[g] = st->groups[g]; sorted[g].row_first = (uint32_t)g; }
    qsort(sorted, ng, sizeof(grp_t), cmp_grp);
    for (uint64_t g = 0; g < ng; ++g) order[g] = sorted[g].row_first;
    free(sorted);
    return order;
}

/* Writes the groups of `order` to output rows [o_base, o_base + ng). */
static void gbs_emit(const gb_state* st, const uint32_t* order, uint64_t o_base,
                     int64_t* out_keys, uint8_t* out_key_null,
                     void** out_vals, uint8_t** out_valid, double** out_accurate) {
    const orc_col* cols = st->cols;
    for (uint64_t i = 0; i < st->ng; ++i) {
        const uint64_t o = o_base + i;
        uint32_t g = order[i];
        out_keys[o] = st->groups[g].is_null ? 0 : st->groups[g].key;
        out_key_null[o] = (uint8_t)st->groups[g].is_null;
        for (int32_t a = 0; a < st->n_aggs; ++a) {
            const acc_t* s = &st->acc[(uint64_t)g * st->n_aggs + a];
            int op = st->aggs[a].op;
            uint8_t valid = 1;
            const orc_col* c = op == ORC_COUNT_STAR ? NULL : &cols[st->aggs[a].input_col];
            if (op == ORC_COUNT_STAR || op == ORC_COUNT) {
                ((int64_t*)out_vals[a])[o] = s->cnt;
            } else if (op == ORC_MIN || op == ORC_MAX) {
                valid = s->cnt > 0;
                uint64_t k = op == ORC_MIN ? s->mnk : s->mxk;
                if (is_float(c->dtype)) ((double*)out_vals[a])[o] = valid ? mm_key_to_f64(k) : 0.0;
                else ((int64_t*)out_vals[a])[o] = valid ? (int64_t)(k ^ 0x8000000000000000ull) : 0;
            } else if (op == ORC_SUM) {
                valid = s->cnt > 0;
                if (is_float(c->dtype)) {
                    ((double*)out_vals[a])[o] = valid ? s->fsum : 0.0;
                    if (out_accurate && out_accurate[a]) out_accurate[a][o] = s->csum + s->comp;
                } else if (c->dtype == ORC_DEC128) {
                    i128 v = valid ? s->isum : 0;
                    ((uint64_t*)out_vals[a])[2 * o] = (uint64_t)v;
                    ((uint64_t*)out_vals[a])[2 * o + 1] = (uint64_t)((unsigned __int128)v >> 64);
                } else {
                    ((int64_t*)out_vals[a])[o] = valid ? (int64_t)s->isum : 0;
                }
            } else { /* AVG = (sum f64) / count (groupby.rs:2877-2885) */
                valid = s->cnt > 0;
                double sum = is_float(c->dtype) ? s->fsum : (double)s->isum;
                ((double*)out_vals[a])[o] = valid ? sum / (double)s->cnt : 0.0;
                if (out_accurate && out_accurate[a])
                    out_accurate[a][o] = valid ? (is_float(c->dtype) ? (s->csum + s->comp) : (double)s->isum) / (double)s->cnt : 0.0;
            }
            if (out_valid && out_valid[a]) out_valid[a][o] = valid;
        }
    }
}

static int gb_check_aggs(const orc_col* cols, const orc_agg* aggs, int32_t n_aggs) {
    for (int32_t a = 0; a < n_aggs; ++a) {
        int op = aggs[a].op;
        if (op == ORC_COUNT_STAR) continue;
        const orc_col* c = &cols[aggs[a].input_col];
        if ((op == ORC_SUM || op == ORC_AVG) && c->dtype == ORC_F32) return ORC_DECLINE;
        if ((op == ORC_MIN || op == ORC_MAX || op == ORC_AVG) && c->dtype == ORC_DEC128)
            return ORC_DECLINE;
    }
    return ORC_OK;
}

/* Key NULL-ness of row r; -1 when the row is dropped (multi-column key with a
 * NULL part). */
static inline int gb_key_null(const orc_col* cols, const int32_t* key_cols, int32_t n_keys, uint64_t r) {
    int key_null = 0;
    for (int32_t k = 0; k < n_keys; ++k)
        if (!is_valid(cols[key_cols[k]].validity, r)) key_null = 1;
    return (key_null && n_keys > 1) ? -1 : key_null;
}

int orc_groupby(uint64_t n, const orc_col* cols, int32_t n_cols,
                const int32_t* key_cols, int32_t n_keys,
                const orc_pred* preds, int32_t n_preds,
                const orc_agg* aggs, int32_t n_aggs,
                int64_t* out_keys, uint8_t* out_key_null,
                void** out_vals, uint8_t** out_valid, double** out_accurate,
                uint64_t cap, uint64_t* n_groups, char* err, int32_t err_cap) {
    (void)n_cols;
    if (n_keys < 1 || n_keys > 2 || n_aggs < 1) return ORC_INVALID;
    int st0 = gb_check_aggs(cols, aggs, n_aggs);
    if (st0 != ORC_OK) return st0;
    gb_state st;
    if (gbs_init(&st, cols, key_cols, n_keys, aggs, n_aggs, 1024)) { gbs_free(&st); return ORC_CAPACITY; }
    for (uint64_t r = 0; r < n && st.status != ORC_CAPACITY; ++r) {
        if (!orc_row_passes(cols, preds, n_preds, r)) continue;
        const int key_null = gb_key_null(cols, key_cols, n_keys, r);
        if (key_null < 0) continue;
        gbs_fold_row(&st, r, key_null);
    }
    int status = st.status;
    if (status == ORC_OVERFLOW) snprintf(err, err_cap, "%s", st.err);
    if (status == ORC_OK && st.ng > cap) { *n_groups = st.ng; status = ORC_CAPACITY; }
    if (status == ORC_OK) {
        uint32_t* order = gbs_order(&st);
        gbs_emit(&st, order, 0, out_keys, out_key_null, out_vals, out_valid, out_accurate);
        free(order);
        *n_groups = st.ng;
    }
    gbs_free(&st);
    return status;
}

/* ---- GROUP BY on every host thread --------------------------------------- */
/* The same fold run on T threads, with results identical to orc_groupby:
 * rows are range-partitioned by their packed key (splitters from a sample of
 * the keys), each partition is folded by one thread in row order (so every
 * group sees its rows in the order the sequential fold does), sorted, and
 * the partitions' outputs are concatenated in key order. The NULL group has
 * a partition of its own, emitted last. */
typedef struct {
    uint64_t n;
    const orc_col* cols;
    const int32_t* key_cols;
    int32_t n_keys;
    const orc_pred* preds;
    int32_t n_preds;
    const orc_agg* aggs;
    int32_t n_aggs;
    int T;        /* threads */
    int P;        /* key-range partitions (the NULL partition is P) */
    const int64_t* splitters;  /* P - 1 ascending */
    uint16_t* part;            /* per row: partition or 0xFFFF */
    uint64_t* count;           /* [T][P + 1] */
    uint64_t* off;             /* [T][P + 1] */
    uint64_t* pbeg;            /* [P + 2] */
    uint32_t* rows;            /* rows grouped by partition, row order inside */
    gb_state* st;              /* [P + 1] */
    uint32_t** order;          /* [P + 1] */
    uint64_t* gbeg;            /* [P + 2] */
    int64_t* out_keys;
    uint8_t* out_key_null;
    void** out_vals;
    uint8_t** out_valid;
    double** out_accurate;
    int phase;
    int next;                  /* dynamic partition counter */
} gb_par;

typedef struct { gb_par* g; int t; } gb_par_arg;

static int upper_bound_i64(const int64_t* a, int n, int64_t k) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] <= k) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static void* gb_par_worker(void* vp) {
    gb_par_arg* arg = (gb_par_arg*)vp;
    gb_par* g = arg->g;
    const int t = arg->t, P1 = g->P + 1;
    const uint64_t r0 = g->n * (uint64_t)t / (uint64_t)g->T, r1 = g->n * (uint64_t)(t + 1) / (uint64_t)g->T;
    if (g->phase == 0) {          /* classify rows of this thread's range */
        uint64_t* cnt = g->count + (uint64_t)t * P1;
        for (uint64_t r = r0; r < r1; ++r) {
            uint16_t p = 0xFFFF;
            if (orc_row_passes(g->cols, g->preds, g->n_preds, r)) {
                const int kn = gb_key_null(g->cols, g->key_cols, g->n_keys, r);
                if (kn == 1) p = (uint16_t)g->P;
                else if (kn == 0)
                    p = (uint16_t)upper_bound_i64(g->splitters, g->P - 1,
                                                  orc_pack_key(g->cols, g->key_cols, g->n_keys, r));
            }
            g->part[r] = p;
            if (p != 0xFFFF) cnt[p]++;
        }
    } else if (g->phase == 1) {   /* scatter row numbers by partition */
        uint64_t* off = g->off + (uint64_t)t * P1;
        for (uint64_t r = r0; r < r1; ++r) {
            const uint16_t p = g->part[r];
            if (p != 0xFFFF) g->rows[off[p]++] = (uint32_t)r;
        }
    } else if (g->phase == 2) {   /* fold and order whole partitions */
        for (;;) {
            const int p = __atomic_fetch_add(&g->next, 1, __ATOMIC_RELAXED);
            if (p >= P1) break;
            gb_state* s = &g->st[p];
            const uint64_t b = g->pbeg[p], e = g->pbeg[p + 1];
            if (gbs_init(s, g->cols, g->key_cols, g->n_keys, g->aggs, g->n_aggs, (e - b) / 64 + 1024)) {
                s->status = ORC_CAPACITY;
                continue;
            }
            for (uint64_t i = b; i < e && s->status != ORC_CAPACITY; ++i) gbs_fold_row(s, g->rows[i], p == g->P);
            g->order[p] = gbs_order(s);
        }
    } else {                      /* emit whole partitions at their offsets */
        for (;;) {
            const int p = __atomic_fetch_add(&g->next, 1, __ATOMIC_RELAXED);
            if (p >= P1) break;
            gbs_emit(&g->st[p], g->order[p], g->gbeg[p], g->out_keys, g->out_key_null, g->out_vals,
                     g->out_valid, g->out_accurate);
        }
    }
    return NULL;
}

static void gb_par_run(gb_par* g, int phase) {
    pthread_t th[256];
    gb_par_arg args[256];
    g->phase = phase;
    g->next = 0;
    for (int t = 0; t < g->T; ++t) {
        args[t].g = g;
        args[t].t = t;
        if (t > 0) pthread_create(&th[t], NULL, gb_par_worker, &args[t]);
    }
    gb_par_worker(&args[0]);
    for (int t = 1; t < g->T; ++t) pthread_join(th[t], NULL);
}

static int cmp_i64(const void* x, const void* y) {
    const int64_t a = *(const int64_t*)x, b = *(const int64_t*)y;
    return (a > b) - (a < b);
}

int orc_groupby_par(uint64_t n, const orc_col* cols, int32_t n_cols,
                    const int32_t* key_cols, int32_t n_keys,
                    const orc_pred* preds, int32_t n_preds,
                    const orc_agg* aggs, int32_t n_aggs,
                    int64_t* out_keys, uint8_t* out_key_null,
                    void** out_vals, uint8_t** out_valid, double** out_accurate,
                    uint64_t cap, uint64_t* n_groups, char* err, int32_t err_cap, int32_t threads) {
    if (threads > 256) threads = 256;
    if (threads <= 1 || n < 4096 || n >= 0xFFFFFFFFull)
        return orc_groupby(n, cols, n_cols, key_cols, n_keys, preds, n_preds, aggs, n_aggs, out_keys,
                           out_key_null, out_vals, out_valid, out_accurate, cap, n_groups, err, err_cap);
    if (n_keys < 1 || n_keys > 2 || n_aggs < 1) return ORC_INVALID;
    int st0 = gb_check_aggs(cols, aggs, n_aggs);
    if (st0 != ORC_OK) return st0;
    gb_par g;
    memset(&g, 0, sizeof g);
    g.n = n; g.cols = cols; g.key_cols = key_cols; g.n_keys = n_keys; g.preds = preds; g.n_preds = n_preds;
    g.aggs = aggs; g.n_aggs = n_aggs; g.T = threads; g.P = threads * 8;
    g.out_keys = out_keys; g.out_key_null = out_key_null; g.out_vals = out_vals; g.out_valid = out_valid;
    g.out_accurate = out_accurate;
    const int P1 = g.P + 1;
    /* Splitters: row quantiles of a strided sample of the non-NULL keys. */
    const uint64_t stride = n / 65536 + 1;
    int64_t* sample = (int64_t*)malloc((n / stride + 1) * sizeof(int64_t));
    uint64_t ns = 0;
    for (uint64_t r = 0; r < n; r += stride)
        if (orc_row_passes(cols, preds, n_preds, r) && gb_key_null(cols, key_cols, n_keys, r) == 0)
            sample[ns++] = orc_pack_key(cols, key_cols, n_keys, r);
    qsort(sample, ns, sizeof(int64_t), cmp_i64);
    int64_t* spl = (int64_t*)malloc((size_t)g.P * sizeof(int64_t));
    for (int i = 0; i + 1 < g.P; ++i) spl[i] = ns ? sample[(uint64_t)(i + 1) * ns / (uint64_t)g.P] : 0;
    free(sample);
    g.splitters = spl;
    g.part = (uint16_t*)malloc(n * sizeof(uint16_t));
    g.count = (uint64_t*)calloc((size_t)g.T * P1, sizeof(uint64_t));
    g.off = (uint64_t*)calloc((size_t)g.T * P1, sizeof(uint64_t));
    g.pbeg = (uint64_t*)calloc((size_t)P1 + 1, sizeof(uint64_t));
    g.gbeg = (uint64_t*)calloc((size_t)P1 + 1, sizeof(uint64_t));
    g.st = (gb_state*)calloc((size_t)P1, sizeof(gb_state));
    g.order = (uint32_t**)calloc((size_t)P1, sizeof(uint32_t*));
    int status = ORC_OK;
    if (!g.part || !g.count || !g.off || !g.pbeg || !g.gbeg || !g.st || !g.order) { status = ORC_CAPACITY; goto out; }
    gb_par_run(&g, 0);
    {
        uint64_t tot = 0;
        for (int p = 0; p < P1; ++p) {
            g.pbeg[p] = tot;
            for (int t = 0; t < g.T; ++t) {
                g.off[(uint64_t)t * P1 + p] = tot;
                tot += g.count[(uint64_t)t * P1 + p];
            }
        }
        g.pbeg[P1] = tot;
        g.rows = (uint32_t*)malloc((tot ? tot : 1) * sizeof(uint32_t));
        if (!g.rows) { status = ORC_CAPACITY; goto out; }
    }
    gb_par_run(&g, 1);
    gb_par_run(&g, 2);
    /* The first failing partition in key order names the error. */
    for (int p = 0; p < P1 && status == ORC_OK; ++p) {
        status = g.st[p].status;
        if (status == ORC_OVERFLOW) snprintf(err, err_cap, "%s", g.st[p].err);
    }
    if (status == ORC_OK) {
        uint64_t ng = 0;
        for (int p = 0; p < P1; ++p) { g.gbeg[p] = ng; ng += g.st[p].ng; }
        *n_groups = ng;
        if (ng > cap) status = ORC_CAPACITY;
        else gb_par_run(&g, 3);
    }
out:
    if (g.st)
        for (int p = 0; p < P1; ++p) {
            if (g.st[p].groups || g.st[p].acc || g.st[p].m.keys) gbs_free(&g.st[p]);
            if (g.order) free(g.order[p]);
        }
    free(spl); free(g.part); free(g.count); free(g.off); free(g.pbeg); free(g.gbeg); free(g.st);
    free(g.order); free(g.rows);
    return status;
}

/* ---- hash join ----------------------------------------------------------- */
static inline int join_key(const orc_col* c, uint64_t i, uint64_t* out) {
    if (!is_valid(c->validity, i)) return 0;
    if (c->dtype == ORC_I32) *out = (uint64_t)(int64_t)((const int32_t*)c->data)[i];
    else *out = (uint64_t)((const int64_t*)c->data)[i];
    return 1;
}

int orc_hash_join(uint64_t n_build, const orc_col* build_key,
                  uint64_t n_probe, const orc_col* probe_key,
                  uint32_t* out_probe, uint32_t* out_build, uint64_t cap, uint64_t* n_out) {
    omap m;
    if (omap_init(&m, n_build + 16)) return ORC_CAPACITY;
    for (uint64_t i = 0; i < n_build; ++i) {
        uint64_t k; int ins;
        if (!join_key(build_key, i, &k)) continue;
        omap_get(&m, k, (uint32_t)i, &ins);
        if (!ins) { omap_free(&m); return ORC_DECLINE; }
    }
    uint64_t cnt = 0;
    for (uint64_t p = 0; p < n_probe; ++p) {
        uint64_t k;
        if (!join_key(probe_key, p, &k)) continue;
        int64_t b = omap_find(&m, k);
        if (b < 0) continue;
        if (cnt < cap) { out_probe[cnt] = (uint32_t)p; out_build[cnt] = (uint32_t)b; }
        cnt++;
    }
    omap_free(&m);
    *n_out = cnt;
    return cnt > cap ? ORC_CAPACITY : ORC_OK;
}

typedef struct { int64_t k0, k1; uint64_t row; } wrow_t;
static int cmp_wrow(const void* x, const void* y) {
    const wrow_t* a = (const wrow_t*)x;
    const wrow_t* b = (const wrow_t*)y;
    if (a->k0 != b->k0) return a->k0 < b->k0 ? -1 : 1;
    if (a->k1 != b->k1) return a->k1 < b->k1 ? -1 : 1;
    return (a->row > b->row) - (a->row < b->row);
}

static inline int64_t wide_key(const orc_col* c, uint64_t i) {
    return c->dtype == ORC_I32 ? (int64_t)((const int32_t*)c->data)[i] : ((const int64_t*)c->data)[i];
}

static inline double num_f64(const orc_col* c, uint64_t i) {
    switch (c->dtype) {
    case ORC_I32: return (double)((const int32_t*)c->data)[i];
    case ORC_I64: return (double)((const int64_t*)c->data)[i];
    case ORC_F32: return (double)((const float*)c->data)[i];
    default: return ((const double*)c->data)[i];
    }
}

/* The groups are the runs of the rows sorted by (key0, key1, row): equal to
 * the reference's hash map of tuples sorted by tuple afterwards, and each
 * run is folded in row order as the reference's row loop folds it. */
int orc_groupby_wide(uint64_t n, const orc_col* key0, const orc_col* key1, int32_t n_aggs, const int32_t* ops,
                     const orc_col* inputs, int64_t* out_k0, int64_t* out_k1, int64_t* out_i, double* out_f,
                     uint8_t* out_valid, uint64_t cap, uint64_t* n_groups) {
    wrow_t* w = (wrow_t*)malloc(sizeof(wrow_t) * (n ? n : 1));
    if (!w) return ORC_CAPACITY;
    uint64_t m = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (!is_valid(key0->validity, i) || !is_valid(key1->validity, i)) continue;
        w[m].k0 = wide_key(key0, i);
        w[m].k1 = wide_key(key1, i);
        w[m].row = i;
        ++m;
    }
    qsort(w, m, sizeof(wrow_t), cmp_wrow);
    uint64_t g = 0;
    for (uint64_t s = 0; s < m;) {
        uint64_t e = s + 1;
        while (e < m && w[e].k0 == w[s].k0 && w[e].k1 == w[s].k1) ++e;
        if (g < cap) {
            out_k0[g] = w[s].k0;
            out_k1[g] = w[s].k1;
            for (int a = 0; a < n_aggs; ++a) {
                const orc_col* in = &inputs[a];
                int64_t ti = 0;
                double tf = 0.0;
                uint64_t cnt = 0;
                int seen = 0;
                const int is_f = in->data && (in->dtype == ORC_F32 || in->dtype == ORC_F64);
                for (uint64_t j = s; j < e; ++j) {
                    const uint64_t r = w[j].row;
                    if (ops[a] == ORC_COUNT_STAR) { ++cnt; continue; }
                    if (!is_valid(in->validity, r)) continue;
                    ++cnt;
                    if (ops[a] == ORC_SUM) {
                        if (is_f) tf += num_f64(in, r);
                        else ti = (int64_t)((uint64_t)ti + (uint64_t)wide_key(in, r));
                    } else if (ops[a] == ORC_AVG) {
                        tf += num_f64(in, r);
                    } else if (ops[a] == ORC_MIN || ops[a] == ORC_MAX) {
                        if (is_f) {
                            const double x = num_f64(in, r);
                            if (!seen || (ops[a] == ORC_MIN ? x < tf : x > tf)) tf = x;
                        } else {
                            const int64_t x = wide_key(in, r);
                            if (!seen || (ops[a] == ORC_MIN ? x < ti : x > ti)) ti = x;
                        }
                    }
                    seen = 1;
                }
                uint8_t valid = 1;
                if (ops[a] == ORC_COUNT_STAR || ops[a] == ORC_COUNT) ti = (int64_t)cnt;
                else if (ops[a] == ORC_AVG) { valid = cnt > 0; tf = cnt ? tf / (double)cnt : 0.0; }
                else valid = (uint8_t)seen;
                if (!valid) { ti = 0; tf = 0.0; }
                out_i[(uint64_t)a * cap + g] = ti;
                out_f[(uint64_t)a * cap + g] = tf;
                out_valid[(uint64_t)a * cap + g] = valid;
            }
        }
        ++g;
        s = e;
    }
    free(w);
    *n_groups = g;
    return g > cap ? ORC_CAPACITY : ORC_OK;
}

typedef struct { uint64_t k; uint32_t row; } krow_t;
static int cmp_krow(const void* x, const void* y) {
    const krow_t* a = (const krow_t*)x;
    const krow_t* b = (const krow_t*)y;
    if (a->k != b->k) return a->k < b->k ? -1 : 1;
    return (a->row > b->row) - (a->row < b->row);
}

/* The map from a key to its build rows in ascending row order is kept as the
 * valid (key, row) pairs sorted by key then row; a probe key's rows are the
 * run that a binary search finds. */
int orc_hash_join_multi(uint64_t n_build, const orc_col* build_key,
                        uint64_t n_probe, const orc_col* probe_key,
                        uint32_t* out_probe, uint32_t* out_build, uint64_t cap, uint64_t* n_out) {
    krow_t* kr = (krow_t*)malloc(sizeof(krow_t) * (n_build ? n_build : 1));
    if (!kr) return ORC_CAPACITY;
    uint64_t m = 0;
    for (uint64_t i = 0; i < n_build; ++i) {
        uint64_t k;
        if (!join_key(build_key, i, &k)) continue;  /* NULL keys never match */
        kr[m].k = k;
        kr[m].row = (uint32_t)i;
        ++m;
    }
    qsort(kr, m, sizeof(krow_t), cmp_krow);
    uint64_t cnt = 0;
    for (uint64_t p = 0; p < n_probe; ++p) {
        uint64_t k;
        if (!join_key(probe_key, p, &k)) continue;
        uint64_t lo = 0, hi = m;  /* first entry with key >= k */
        while (lo < hi) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (kr[mid].k < k) lo = mid + 1;
            else hi = mid;
        }
        for (uint64_t j = lo; j < m && kr[j].k == k; ++j) {
            if (cnt < cap) {
                out_probe[cnt] = (uint32_t)p;
                out_build[cnt] = kr[j].row;
            }
            cnt++;
        }
    }
    free(kr);
    *n_out = cnt;
    return cnt > cap ? ORC_CAPACITY : ORC_OK;
}

typedef struct { int32_t g; uint32_t slot; } gslot_t;
static int cmp_gslot(const void* x, const void* y) {
    int32_t a = ((const gslot_t*)x)->g, b = ((const gslot_t*)y)->g;
    return (a > b) - (a < b);
}

int orc_join_groupby(uint64_t n_build, const orc_col* build_key, const int32_t* build_payload,
                     uint64_t n_probe, const orc_col* probe_key, const orc_col* value,
                     int32_t* out_group, int64_t* out_sum_lo, int64_t* out_sum_hi,
                     int64_t* out_count, uint64_t cap, uint64_t* n_groups,
                     char* err, int32_t err_cap) {
    omap m, gm;
    if (omap_init(&m, n_build + 16)) return ORC_CAPACITY;
    for (uint64_t i = 0; i < n_build; ++i) {
        uint64_t k; int ins;
        if (!join_key(build_key, i, &k)) continue;
        omap_get(&m, k, (uint32_t)i, &ins);
        if (!ins) { omap_free(&m); return ORC_DECLINE; }
    }
    if (omap_init(&gm, 1024)) { omap_free(&m); return ORC_CAPACITY; }
    uint64_t ng = 0, gcap = 1024;
    int32_t* gkey = (int32_t*)malloc(gcap * 4);
    i128* sums = (i128*)calloc(gcap, sizeof(i128));
    int64_t* cnts = (int64_t*)calloc(gcap, 8);
    int status = ORC_OK;
    for (uint64_t p = 0; p < n_probe; ++p) {
        uint64_t k;
        if (!join_key(probe_key, p, &k)) continue;
        int64_t b = omap_find(&m, k);
        if (b < 0) continue;
        int32_t g = build_payload[b];
        int ins;
        if (ng * 2 >= gm.cap) omap_grow(&gm);
        uint32_t gi = omap_get(&gm, (uint64_t)(int64_t)g, (uint32_t)ng, &ins);
        if (ins) {
            if (ng == gcap) {
                gcap *= 2;
                gkey = (int32_t*)realloc(gkey, gcap * 4);
                sums = (i128*)realloc(sums, gcap * sizeof(i128));
                cnts = (int64_t*)realloc(cnts, gcap * 8);
                memset(sums + gcap / 2, 0, gcap / 2 * sizeof(i128));
                memset(cnts + gcap / 2, 0, gcap / 2 * 8);
            }
            gkey[ng] = g;
            ng++;
        }
        cnts[gi]++;
        if (value && is_valid(value->validity, p)) {
            i128 v = col_i128(value, p), out;
            if (__builtin_add_overflow(sums[gi], v, &out)) {
                if (status == ORC_OK) {
                    snprintf(err, err_cap, "SUM(Decimal128) precision overflow: accumulator exceeds i128 range");
                    status = ORC_OVERFLOW;
                }
            } else sums[gi] = out;
        }
    }
    if (status == ORC_OK && ng > cap) status = ORC_CAPACITY;
    if (status == ORC_OK) {
        gslot_t* order = (gslot_t*)malloc((ng ? ng : 1) * sizeof(gslot_t));
        for (uint64_t i = 0; i < ng; ++i) { order[i].g = gkey[i]; order[i].slot = (uint32_t)i; }
        qsort(order, ng, sizeof(gslot_t), cmp_gslot);
        for (uint64_t o = 0; o < ng; ++o) {
            uint32_t i = order[o].slot;
            out_group[o] = gkey[i];
            out_sum_lo[o] = (int64_t)(uint64_t)sums[i];
            out_sum_hi[o] = (int64_t)(uint64_t)((unsigned __int128)sums[i] >> 64);
            out_count[o] = cnts[i];
        }
        free(order);
    }
    *n_groups = ng;
    omap_free(&m); omap_free(&gm);
    free(gkey); free(sums); free(cnts);
    return status;
}

/* ---- sort ---------------------------------------------------------------- */
uint64_t orc_sort_key(const orc_col* key, uint64_t row, int32_t descending) {
    uint64_t k;
    switch (key->dtype) {
    case ORC_I32: {
        /* radix_pre_transform_i32: val ^ i32::MIN, widened to the top of a u64 */
        uint32_t v = (uint32_t)((const int32_t*)key->data)[row] ^ 0x80000000u;
        k = (uint64_t)v;
        if (descending) k = (uint64_t)(~v);
        return k;
    }
    case ORC_I64:
        k = (uint64_t)((const int64_t*)key->data)[row] ^ 0x8000000000000000ull;
        return descending ? ~k : k;
    case ORC_U32:
        k = (uint64_t)((const uint32_t*)key->data)[row];
        return descending ? (uint64_t)(~(uint32_t)k) : k;
    case ORC_F32: {
        /* radix_float_key_f32 (gpu_sort.rs:1143) */
        uint32_t b = canon_f32_bits(((const float*)key->data)[row]);
        uint32_t mask = (uint32_t)(((int32_t)b) >> 31) | 0x80000000u;
        uint32_t asc = b ^ mask;
        return descending ? (uint64_t)(~asc) : (uint64_t)asc;
    }
    case ORC_F64: {
        uint64_t b = canon_f64_bits(((const double*)key->data)[row]);
        uint64_t mask = (uint64_t)(((int64_t)b) >> 63) | 0x8000000000000000ull;
        uint64_t asc = b ^ mask;
        return descending ? ~asc : asc;
    }
    default: return 0;
    }
}

/* Stable LSD radix sort of (key, row) by key, 16-bit digits. */
static void lsd_sort_u64(uint64_t* keys, uint32_t* rows, uint64_t n, int nbits) {
    uint64_t* k2 = (uint64_t*)malloc((n ? n : 1) * 8);
    uint32_t* r2 = (uint32_t*)malloc((n ? n : 1) * 4);
    uint64_t* cnt = (uint64_t*)malloc(65536 * 8);
    for (int shift = 0; shift < nbits; shift += 16) {
        memset(cnt, 0, 65536 * 8);
        for (uint64_t i = 0; i < n; ++i) cnt[(keys[i] >> shift) & 0xFFFF]++;
        uint64_t s = 0;
        for (int d = 0; d < 65536; ++d) { uint64_t c = cnt[d]; cnt[d] = s; s += c; }
        for (uint64_t i = 0; i < n; ++i) {
            uint64_t d = (keys[i] >> shift) & 0xFFFF;
            uint64_t o = cnt[d]++;
            k2[o] = keys[i]; r2[o] = rows[i];
        }
        memcpy(keys, k2, n * 8); memcpy(rows, r2, n * 4);
    }
    free(k2); free(r2); free(cnt);
}

static int key_bits(int dtype) {
    return (dtype == ORC_I32 || dtype == ORC_F32 || dtype == ORC_U32) ? 32 : 64;
}

int orc_sort_perm_multi(uint64_t n, const orc_col* keys, int32_t n_keys,
                        const int32_t* descending, const int32_t* nulls_first, uint32_t* perm) {
    uint64_t* k = (uint64_t*)malloc((n ? n : 1) * 8);
    uint32_t* cur = (uint32_t*)malloc((n ? n : 1) * 4);
    for (uint64_t i = 0; i < n; ++i) perm[i] = (uint32_t)i;
    /* LSD over the keys from last to first; each key's pass is stable. */
    for (int32_t kk = n_keys - 1; kk >= 0; --kk) {
        const orc_col* c = &keys[kk];
        uint64_t nn = 0;
        /* NULL rows: placed first/last as a block, input order kept. */
        for (uint64_t i = 0; i < n; ++i) {
            uint32_t r = perm[i];
            cur[i] = r;
            k[i] = orc_sort_key(c, r, descending[kk]);
        }
        lsd_sort_u64(k, cur, n, key_bits(c->dtype));
        if (c->validity) {
            uint32_t* tmp = (uint32_t*)malloc((n ? n : 1) * 4);
            /* valid rows in sorted order, nulls in the previous (stable) order */
            uint64_t nv = 0;
            uint32_t* valid_rows = (uint32_t*)malloc((n ? n : 1) * 4);
            for (uint64_t i = 0; i < n; ++i) if (is_valid(c->validity, cur[i])) valid_rows[nv++] = cur[i];
            uint64_t o = 0;
            if (nulls_first[kk])
                for (uint64_t i = 0; i < n; ++i) if (!is_valid(c->validity, perm[i])) tmp[o++] = perm[i];
            for (uint64_t i = 0; i < nv; ++i) tmp[o++] = valid_rows[i];
            if (!nulls_first[kk])
                for (uint64_t i = 0; i < n; ++i) if (!is_valid(c->validity, perm[i])) tmp[o++] = perm[i];
            memcpy(perm, tmp, n * 4);
            free(tmp); free(valid_rows);
        } else {
            memcpy(perm, cur, n * 4);
        }
        nn++;
        (void)nn;
    }
    free(k); free(cur);
    return ORC_OK;
}

int orc_sort_perm(uint64_t n, const orc_col* key, int32_t descending, int32_t nulls_first,
                  uint32_t* perm) {
    return orc_sort_perm_multi(n, key, 1, &descending, &nulls_first, perm);
}

/* ---- compaction ---------------------------------------------------------- */
int orc_compact(uint64_t n, const orc_col* cols, const orc_pred* preds, int32_t n_preds,
                uint32_t* out_rows, uint64_t* n_out) {
    uint64_t c = 0;
    for (uint64_t i = 0; i < n; ++i)
        if (orc_row_passes(cols, preds, n_preds, i)) out_rows[c++] = (uint32_t)i;
    *n_out = c;
    return ORC_OK;
}

/* ---- fixtures ------------------------------------------------------------ */
void orc_xorshift64star_fill(uint64_t seed, uint64_t* out, uint64_t n) {
    uint64_t s = seed + 0x9E3779B97F4A7C15ull;
    if (s == 0) s = 0xDEADBEEFCAFEBABEull;
    for (uint64_t i = 0; i < n; ++i) {
        s ^= s >> 12; s ^= s << 25; s ^= s >> 27;
        out[i] = s * 0x2545F4914F6CDD1Dull;
    }
}

void orc_shuffle_deterministic_u32(uint32_t* xs, uint64_t n, uint64_t seed) {
    uint64_t s = seed;
    for (uint64_t i = n; i-- > 1;) {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        uint64_t j = s % (i + 1);
        uint32_t t = xs[i]; xs[i] = xs[j]; xs[j] = t;
    }
}
