// radix_sort.cu — onesweep LSD radix sort producing stable permutations for
// one or many independent segments at once.
//
// Replaces the reference's 4-bit LSD radix with a host scan per pass
// (src/exec/gpu_sort.rs:995-1230, src/jit/sort_kernel_radix.rs:489-991):
//   * one histogram kernel reads the keys once and counts all digit
//     positions of every segment (8-bit digits: 4 passes for 32-bit keys,
//     8 for 64-bit);
//   * one kernel per digit: tiles of 4096 (64-bit) or 5120 (32-bit) keys are
//     taken in arrival order from a flattened (segment, tile) list; each
//     tile's digit counts (per-warp shared atomics) are published first and
//     chained across the segment's tiles with decoupled look-back (Merrill &
//     Garland 2016); the keys are ranked per warp (stable: element order
//     within a warp's part of the tile, warps in order; the lanes holding one
//     digit find each other through a shared mask word), staged digit-sorted
//     in shared memory and written out in coalesced runs;
//   * a digit where all of a segment's keys fall in one bucket is skipped
//     for that segment on the device;
//   * the first pass applies the key transform of gpu_sort.rs:1089-1163 to
//     the raw column and generates the row-index payload; the last pass
//     writes only the payload (the permutation) to its destination.
// Many GROUP BY queries finalised together sort as many segments in the
// same handful of launches.
#include "radix_sort.cuh"

#include <algorithm>

namespace bolt {
namespace {

constexpr int SORT_BLOCK = 256;
// Keys per thread in a pass: 32-bit keys leave registers and shared memory
// for larger tiles (fewer tiles to chain, more independent loads per thread).
constexpr int SORT_ITEMS_32 = 20;
constexpr int SORT_ITEMS_64 = 16;
constexpr int SORT_TILE_MIN = SORT_BLOCK * SORT_ITEMS_64;
constexpr int HIST_CHUNK = 16384;
constexpr uint32_t LB_AGG = 1u << 30;
constexpr uint32_t LB_INC = 2u << 30;
constexpr uint32_t LB_VAL = (1u << 30) - 1;
constexpr uint32_t LB_SPIN_LIMIT = 1u << 22;
constexpr int LB_WINDOW = 8;  // look-back words read per round trip

template <typename K> struct KeyTraits;
template <> struct KeyTraits<uint32_t> {
    static constexpr int NPASS = 4;
    static constexpr int ITEMS = SORT_ITEMS_32;
    static constexpr int TILE = SORT_BLOCK * ITEMS;
};
template <> struct KeyTraits<ull> {
    static constexpr int NPASS = 8;
    static constexpr int ITEMS = SORT_ITEMS_64;
    static constexpr int TILE = SORT_BLOCK * ITEMS;
};

struct SegDesc {
    const void* keys;
    const uint32_t* payload_in;
    uint32_t* payload_out;
    const ull* n_dev;
    ull n;
    ull buf_off;
    uint32_t item_begin;
    uint32_t hist_begin;
};

struct SortArgs {
    int32_t src;
    int32_t desc;
    int32_t indirect;
    int32_t nseg;
    const SegDesc* segs;
    const uint32_t* item_begins;  // nseg + 1
    const uint32_t* hist_begins;  // nseg + 1
    void* kA;
    void* kB;
    uint32_t* pA;
    uint32_t* pB;
    uint32_t* hist;        // nseg * NPASS * 256
    uint32_t* digit_base;  // nseg * NPASS * 256
    uint32_t* active;      // nseg
    uint32_t* lookback;    // 2 * lb_stride
    uint64_t lb_stride;    // total_items * 256
    uint32_t total_items;
    uint32_t total_hist_items;
    uint32_t* tile_ctr;    // NPASS
    uint32_t* status;
};

// Order-preserving unsigned image of a key's raw bits: one load serves
// every source type, the transform follows (so unrolled loads stay in flight
// together).
__device__ __forceinline__ uint32_t order_key(int src, uint32_t b, int desc) {
    uint32_t k = b;
    if (src == SRC_I32) {
        k = b ^ 0x80000000u;
    } else if (src == SRC_F32) {
        const uint32_t c = canon_f32_bits(__uint_as_float(b));
        k = c ^ ((uint32_t)(((int32_t)c) >> 31) | 0x80000000u);
    }
    return desc ? ~k : k;
}
__device__ __forceinline__ ull order_key(int src, ull b, int desc) {
    ull k = b;
    if (src == SRC_I64) k = b ^ 0x8000000000000000ull;
    else if (src == SRC_F64) k = f64_order_key(__longlong_as_double((long long)b));
    return desc ? ~k : k;
}

template <typename K>
__device__ __forceinline__ K raw_key(const void* p, uint64_t r) {
    return __ldg(reinterpret_cast<const K*>(p) + r);
}

// Digit of a key at bit offset `shift` (a multiple of 8): a digit never
// straddles the two 32-bit halves of a 64-bit key, so it is taken from the
// half that holds it.
template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) {
    if constexpr (sizeof(K) == 8) {
        const uint32_t h = shift >= 32 ? (uint32_t)(k >> 32) : (uint32_t)k;
        return (h >> (shift & 31)) & 0xFFu;
    } else {
        return ((uint32_t)k >> shift) & 0xFFu;
    }
}

__device__ __forceinline__ void st_volatile_u32(uint32_t* p, uint32_t v) {
    *reinterpret_cast<volatile uint32_t*>(p) = v;
}
__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t* p) {
    return *reinterpret_cast<const volatile uint32_t*>(p);
}

// Index of the segment owning flattened item `item` (begins is nondecreasing).
__device__ __forceinline__ int seg_of(const uint32_t* begins, int nseg, uint32_t item) {
    int lo = 0, hi = nseg;  // answer in [0, nseg)
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(begins + mid) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Rows of a segment: the device count when given, never more than the
// segment's buffers hold (a producer that ran out of room may count past it).
__device__ __forceinline__ uint64_t seg_n(const SegDesc& d) {
    if (!d.n_dev) return d.n;
    const uint64_t n = *d.n_dev;
    return n < d.n ? n : d.n;
}

template <typename K>
__global__ void __launch_bounds__(256) sort_hist_kernel(SortArgs a) {
    constexpr int NP = KeyTraits<K>::NPASS;
    __shared__ uint32_t h[NP * 256];
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // Clear the first look-back buffer and the pass tile counters.
    for (uint64_t i = tid; i < a.lb_stride; i += stride) a.lookback[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x < NP) a.tile_ctr[threadIdx.x] = 0;
    for (uint32_t item = blockIdx.x; item < a.total_hist_items; item += gridDim.x) {
        const int sg = seg_of(a.hist_begins, a.nseg, item);
        const SegDesc& d = a.segs[sg];
        const uint64_t n = seg_n(d);
        const uint64_t c0 = (uint64_t)(item - d.hist_begin) * HIST_CHUNK;
        for (int i = threadIdx.x; i < NP * 256; i += blockDim.x) h[i] = 0;
        __syncthreads();
        const uint64_t c1 = c0 + HIST_CHUNK < n ? c0 + HIST_CHUNK : n;
        for (uint64_t i0 = c0 + threadIdx.x; i0 < c1; i0 += 4 * blockDim.x) {
            K raw[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const uint64_t i = i0 + (uint64_t)u * blockDim.x;
                raw[u] = 0;
                if (i < c1) raw[u] = raw_key<K>(d.keys, a.indirect ? d.payload_in[i] : i);
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (i0 + (uint64_t)u * blockDim.x >= c1) continue;
                const K k = order_key(a.src, raw[u], a.desc);
#pragma unroll
                for (int p = 0; p < NP; ++p) atomicAdd(&h[p * 256 + digit_of<K>(k, 8 * p)], 1u);
            }
        }
        __syncthreads();
        uint32_t* gh = a.hist + (uint64_t)sg * NP * 256;
        for (int i = threadIdx.x; i < NP * 256; i += blockDim.x)
            if (h[i]) atomicAdd(&gh[i], h[i]);
        __syncthreads();
    }
}

// One CTA per segment: exclusive scan of each digit histogram; marks the
// passes whose digit is not constant over the segment's keys.
template <int NP>
__global__ void __launch_bounds__(256) sort_scan_kernel(SortArgs a) {
    __shared__ uint32_t wsum[8];
    __shared__ uint32_t trivial;
    const int sg = blockIdx.x;
    const uint64_t n = seg_n(a.segs[sg]);
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const uint32_t* hist = a.hist + (uint64_t)sg * NP * 256;
    uint32_t* base = a.digit_base + (uint64_t)sg * NP * 256;
    uint32_t act = 0;
    for (int p = 0; p < NP; ++p) {
        if (t == 0) trivial = 0;
        __syncthreads();
        const uint32_t v = hist[p * 256 + t];
        if ((uint64_t)v == n) trivial = 1;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        uint32_t wp = 0;
        for (int i = 0; i < w; ++i) wp += wsum[i];
        base[p * 256 + t] = wp + x - v;
        __syncthreads();
        if (!trivial) act |= 1u << p;
        __syncthreads();
    }
    if (t == 0) a.active[sg] = act ? act : 1u;
}

template <typename K>
__global__ void __launch_bounds__(SORT_BLOCK, 3) sort_pass_kernel(SortArgs a, int p) {
    constexpr int NW = SORT_BLOCK / 32;
    constexpr int SORT_ITEMS = KeyTraits<K>::ITEMS;
    constexpr int SORT_TILE = KeyTraits<K>::TILE;
    __shared__ uint32_t s_item;
    __shared__ uint32_t warp_pos[NW][256];  // per-warp digit counts, then each warp's next staged position
    __shared__ uint32_t peer_bits[NW][256];  // per-warp lane masks of the lanes holding a digit
    __shared__ uint32_t gdelta[256];         // global position of staged position 0, per digit
    __shared__ uint32_t wsum[NW];
    // Staged tile: keys (or, in the last pass, the digit of every position)
    // and payloads (3 CTAs of 256 threads per SM).
    extern __shared__ __align__(16) unsigned char dyn[];
    K* stage_key = reinterpret_cast<K*>(dyn);
    uint32_t* stage_pay = reinterpret_cast<uint32_t*>(dyn + sizeof(K) * SORT_TILE);
    uint8_t* stage_dig = dyn + (sizeof(K) + 4) * SORT_TILE;

    if (threadIdx.x == 0) s_item = atomicAdd(&a.tile_ctr[p], 1u);
    for (int i = threadIdx.x; i < NW * 256; i += SORT_BLOCK) {
        (&warp_pos[0][0])[i] = 0;
        (&peer_bits[0][0])[i] = 0;
    }
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= a.total_items) return;
    const int sg = seg_of(a.item_begins, a.nseg, item);
    const SegDesc& d = a.segs[sg];
    const uint32_t active = a.active[sg];
    if (!((active >> p) & 1u)) return;
    const uint64_t n = seg_n(d);
    const uint32_t tile = item - d.item_begin;
    if ((uint64_t)tile * SORT_TILE >= n) return;

    const uint32_t before = active & ((1u << p) - 1u);
    const bool first = before == 0;
    const bool last = (active >> (p + 1)) == 0;
    const int kidx = __popc(before);
    const K* kin = ((kidx & 1) ? (const K*)a.kA : (const K*)a.kB) + d.buf_off;
    const uint32_t* pin = ((kidx & 1) ? a.pA : a.pB) + d.buf_off;
    K* kout = last ? nullptr : ((kidx & 1) ? (K*)a.kB : (K*)a.kA) + d.buf_off;
    uint32_t* pout = last ? d.payload_out : ((kidx & 1) ? a.pB : a.pA) + d.buf_off;
    uint32_t* lb = a.lookback + (uint64_t)(kidx & 1) * a.lb_stride;
    uint32_t* lb_next = a.lookback + (uint64_t)((kidx + 1) & 1) * a.lb_stride;

    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* peers_w = peer_bits[w];
    const uint64_t seg0 = (uint64_t)tile * SORT_TILE + (uint64_t)w * 32 * SORT_ITEMS;
    const int shift = 8 * p;
    const bool full = (uint64_t)(tile + 1) * SORT_TILE <= n;
    K key[SORT_ITEMS];
    uint32_t pay[SORT_ITEMS];
    if (first) {
        // Raw key bits first (all loads in flight), then the transform.
        if (a.indirect) {
#pragma unroll
            for (int j = 0; j < SORT_ITEMS; ++j) {
                const uint64_t e = seg0 + (uint64_t)j * 32 + lane;
                pay[j] = (full || e < n) ? d.payload_in[e] : 0u;
            }
#pragma unroll
            for (int j = 0; j < SORT_ITEMS; ++j) {
                const uint64_t e = seg0 + (uint64_t)j * 32 + lane;
                key[j] = (full || e < n) ? raw_key<K>(d.keys, pay[j]) : (K)0;
            }
        } else {
#pragma unroll
            for (int j = 0; j < SORT_ITEMS; ++j) {
                const uint64_t e = seg0 + (uint64_t)j * 32 + lane;
                key[j] = 0;
                pay[j] = 0;
                if (full || e < n) {
                    pay[j] = d.payload_in ? d.payload_in[e] : (uint32_t)e;
                    key[j] = raw_key<K>(d.keys, e);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < SORT_ITEMS; ++j) key[j] = order_key(a.src, key[j], a.desc);
    } else {
#pragma unroll
        for (int j = 0; j < SORT_ITEMS; ++j) {
            const uint64_t e = seg0 + (uint64_t)j * 32 + lane;
            key[j] = 0;
            pay[j] = 0;
            if (full || e < n) {
                key[j] = kin[e];
                pay[j] = pin[e];
            }
        }
    }
    // Early counts: per-warp digit histograms from shared atomics, so the
    // tile's counts are published before the (longer) ranking and later
    // tiles' look-backs find them sooner.
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; ++j) {
        const uint64_t e = seg0 + (uint64_t)j * 32 + lane;
        if (full || e < n) atomicAdd(&warp_pos[w][digit_of<K>(key[j], shift)], 1u);
    }
    __syncthreads();
    const uint32_t dg_me = threadIdx.x;  // SORT_BLOCK == 256: one digit per thread
    uint32_t cnt[NW];
    uint32_t run = 0;
#pragma unroll
    for (int ww = 0; ww < NW; ++ww) {
        cnt[ww] = warp_pos[ww][dg_me];
        run += cnt[ww];
    }
    st_volatile_u32(lb + (uint64_t)item * 256 + dg_me, (tile == 0 ? LB_INC : LB_AGG) | run);
    // Exclusive scan of the tile's digit counts; each warp's first staged
    // position per digit follows.
    uint32_t x = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t tile_off = x - run;
    for (int i = 0; i < w; ++i) tile_off += wsum[i];
    {
        uint32_t off = tile_off;
#pragma unroll
        for (int ww = 0; ww < NW; ++ww) {
            warp_pos[ww][dg_me] = off;
            off += cnt[ww];
        }
    }
    __syncthreads();

    // Stable ranking in element order (items in order, lanes in order within
    // an item), straight to the staged position. The lanes holding the same
    // digit find each other through one shared mask word per (warp, digit);
    // the highest of them advances the warp's position for that digit.
#pragma unroll
    for (int j = 0; j < SORT_ITEMS; ++j) {
        const uint64_t e = seg0 + (uint64_t)j * 32 + lane;
        const bool valid = full || e < n;
        const uint32_t dg = digit_of<K>(key[j], shift);
        if (valid) atomicOr(&peers_w[dg], 1u << lane);
        __syncwarp();
        const uint32_t peers = valid ? peers_w[dg] : (1u << lane);
        __syncwarp();
        const int leader = 31 - __clz(peers);
        uint32_t b = 0;
        if (valid && lane == leader) {
            peers_w[dg] = 0;
            b = warp_pos[w][dg];
            warp_pos[w][dg] = b + __popc(peers);
        }
        b = __shfl_sync(0xffffffffu, b, leader);
        if (valid) {
            const uint32_t pos = b + __popc(peers & lanemask_lt());
            if (kout) stage_key[pos] = key[j];
            else stage_dig[pos] = (uint8_t)dg;  // the last pass stages no keys
            stage_pay[pos] = pay[j];
        }
        __syncwarp();
    }

    // Look back over the segment's earlier tiles, LB_WINDOW words in flight
    // at a time: sum aggregates until an inclusive prefix.
    {
        uint32_t excl = 0;
        if (tile != 0) {
            int64_t t = (int64_t)item - 1;
            const int64_t t_end = (int64_t)d.item_begin;
            uint32_t spins = 0;
            while (t >= t_end) {
                const int cnt_w = (t - t_end + 1) < LB_WINDOW ? (int)(t - t_end + 1) : LB_WINDOW;
                uint32_t v[LB_WINDOW];
#pragma unroll
                for (int i = 0; i < LB_WINDOW; ++i)
                    v[i] = i < cnt_w ? ld_volatile_u32(lb + (uint64_t)(t - i) * 256 + dg_me) : 0u;
                int used = 0;
                bool done = false, stalled = false;
#pragma unroll
                for (int i = 0; i < LB_WINDOW; ++i) {
                    if (done || stalled || i >= cnt_w) continue;
                    const uint32_t st = v[i] >> 30;
                    if (st == 0) {
                        stalled = true;  // not published yet: poll again from here
                        continue;
                    }
                    excl += v[i] & LB_VAL;
                    ++used;
                    if (st == 2) done = true;
                }
                if (done) break;
                t -= used;
                if (stalled) {
                    if (++spins > LB_SPIN_LIMIT) {
                        atomicOr(a.status, ST_FLAG_TIMEOUT);
                        break;
                    }
                    if (spins > 4) __nanosleep(64);
                }
            }
            st_volatile_u32(lb + (uint64_t)item * 256 + dg_me, LB_INC | ((excl + run) & LB_VAL));
        }
        lb_next[(uint64_t)item * 256 + dg_me] = 0;
        // Positions fit in 32 bits (n < 2^30), so the difference wraps safely.
        gdelta[dg_me] = a.digit_base[((uint64_t)sg * KeyTraits<K>::NPASS + p) * 256 + dg_me] + excl - tile_off;
    }
    __syncthreads();

    // Coalesced runs out of the staged tile.
    const uint64_t tb = (uint64_t)tile * SORT_TILE;
    const uint32_t tile_n = (uint32_t)((n - tb) < (uint64_t)SORT_TILE ? (n - tb) : (uint64_t)SORT_TILE);
    const uint32_t n32 = (uint32_t)n;  // n < 2^30
    if (kout) {
        for (uint32_t i = threadIdx.x; i < tile_n; i += SORT_BLOCK) {
            const K k = stage_key[i];
            const uint32_t g = gdelta[digit_of<K>(k, shift)] + i;
            if (g >= n32) {  // only reachable after a look-back timeout
                atomicOr(a.status, ST_FLAG_TIMEOUT);
                continue;
            }
            kout[g] = k;
            pout[g] = stage_pay[i];
        }
    } else {
        for (uint32_t i = threadIdx.x; i < tile_n; i += SORT_BLOCK) {
            const uint32_t g = gdelta[stage_dig[i]] + i;
            if (g >= n32) {
                atomicOr(a.status, ST_FLAG_TIMEOUT);
                continue;
            }
            pout[g] = stage_pay[i];
        }
    }
}

template <typename K>
bolt_status run_sort(bolt_ctx* ctx, cudaStream_t s, const SortSpec& sp) {
    constexpr int NP = KeyTraits<K>::NPASS;
    constexpr int SORT_TILE = KeyTraits<K>::TILE;
    const int nseg = (int)sp.segs.size();
    if (nseg == 0) return BOLT_OK;
    std::vector<SegDesc> segs(nseg);
    std::vector<uint32_t> begins(2 * (nseg + 1));
    uint64_t total_n = 0, items = 0, hitems = 0;
    for (int i = 0; i < nseg; ++i) {
        const SortSegment& g = sp.segs[i];
        if (g.n >= (1ull << 30))
            return fail(ctx, BOLT_DECLINE, "radix sort: %llu rows exceed the 2^30 row limit", (ull)g.n);
        if (!g.payload_out && g.n) return fail(ctx, BOLT_ERR_INVALID, "radix sort: no payload output");
        segs[i] = SegDesc{g.keys, g.payload_in, g.payload_out, g.n_dev, g.n, total_n, (uint32_t)items, (uint32_t)hitems};
        begins[i] = (uint32_t)items;
        begins[nseg + 1 + i] = (uint32_t)hitems;
        total_n += g.n;
        items += (g.n + SORT_TILE - 1) / SORT_TILE;
        hitems += (g.n + HIST_CHUNK - 1) / HIST_CHUNK;
    }
    begins[nseg] = (uint32_t)items;
    begins[2 * nseg + 1] = (uint32_t)hitems;
    if (items >= (1ull << 31)) return fail(ctx, BOLT_DECLINE, "radix sort: too many tiles");
    if (items == 0) return BOLT_OK;

    SortArgs a{};
    a.src = sp.src;
    a.desc = sp.descending;
    a.indirect = sp.indirect;
    a.nseg = nseg;
    a.total_items = (uint32_t)items;
    a.total_hist_items = (uint32_t)hitems;
    a.lb_stride = items * 256;
    const uint64_t nb = total_n ? total_n : 1;
    SegDesc* d_segs = (SegDesc*)arena_alloc(ctx, sizeof(SegDesc) * nseg);
    uint32_t* d_begins = (uint32_t*)arena_alloc(ctx, 4 * begins.size());
    a.kA = arena_alloc(ctx, nb * sizeof(K));
    a.kB = arena_alloc(ctx, nb * sizeof(K));
    a.pA = (uint32_t*)arena_alloc(ctx, nb * 4);
    a.pB = (uint32_t*)arena_alloc(ctx, nb * 4);
    a.hist = (uint32_t*)arena_alloc(ctx, (uint64_t)nseg * NP * 256 * 4);
    a.digit_base = (uint32_t*)arena_alloc(ctx, (uint64_t)nseg * NP * 256 * 4);
    a.active = (uint32_t*)arena_alloc(ctx, (uint64_t)nseg * 4);
    a.lookback = (uint32_t*)arena_alloc(ctx, 2 * a.lb_stride * 4);
    a.tile_ctr = (uint32_t*)arena_alloc(ctx, 64);
    a.status = ctx->d_status;
    if (!d_segs || !d_begins || !a.kA || !a.kB || !a.pA || !a.pB || !a.hist || !a.digit_base || !a.active ||
        !a.lookback || !a.tile_ctr)
        return fail(ctx, BOLT_ERR_CAPACITY, "radix sort: scratch arena too small for %llu rows", (ull)total_n);
    a.segs = d_segs;
    a.item_begins = d_begins;
    a.hist_begins = d_begins + nseg + 1;
    bolt_status st = stage_upload(ctx, s, d_segs, segs.data(), sizeof(SegDesc) * nseg);
    if (st != BOLT_OK) return st;
    st = stage_upload(ctx, s, d_begins, begins.data(), 4 * begins.size());
    if (st != BOLT_OK) return st;
    BOLT_CUDA(ctx, cudaMemsetAsync(a.hist, 0, (uint64_t)nseg * NP * 256 * 4, s));
    const unsigned hb = (unsigned)std::min<uint64_t>(hitems, (uint64_t)ctx->num_sms * 8);
    sort_hist_kernel<K><<<hb, 256, 0, s>>>(a);
    sort_scan_kernel<NP><<<nseg, 256, 0, s>>>(a);
    ctx->last_launches += 2;
    const size_t dyn = (sizeof(K) + 5) * SORT_TILE;
    BOLT_CUDA(ctx, smem_optin(sort_pass_kernel<K>, ctx));
    for (int p = 0; p < NP; ++p) {
        sort_pass_kernel<K><<<(unsigned)items, SORT_BLOCK, dyn, s>>>(a, p);
        ctx->last_launches++;
    }
    BOLT_CUDA(ctx, cudaGetLastError());
    return BOLT_OK;
}

}  // namespace

uint64_t radix_sort_scratch(uint64_t total_n, uint64_t nseg, int32_t src) {
    const uint64_t ksz = (src == SRC_I32 || src == SRC_F32 || src == SRC_U32) ? 4 : 8;
    const uint64_t items = total_n / SORT_TILE_MIN + nseg + 1;
    return 2 * total_n * (ksz + 4) + 2 * items * 256 * 4 + nseg * (2 * 8 * 256 * 4 + 96) + 64 * 1024;
}

bolt_status radix_sort(bolt_ctx* ctx, cudaStream_t s, const SortSpec& sp) {
    switch (sp.src) {
    case SRC_I32:
    case SRC_F32:
    case SRC_U32:
        return run_sort<uint32_t>(ctx, s, sp);
    case SRC_I64:
    case SRC_F64:
    case SRC_U64_KEYS:
        return run_sort<ull>(ctx, s, sp);
    }
    return fail(ctx, BOLT_ERR_INVALID, "radix sort: unknown key source %d", sp.src);
}

}  // namespace bolt

// ---------------------------------------------------------------------------
// ORDER BY entry points
// ---------------------------------------------------------------------------
#include "compact.cuh"

using namespace bolt;

namespace {

int sort_src_of(int dt) {
    switch (dt) {
    case BOLT_I32: return SRC_I32;
    case BOLT_I64: return SRC_I64;
    case BOLT_F32: return SRC_F32;
    case BOLT_F64: return SRC_F64;
    case BOLT_U32: return SRC_U32;
    }
    return -1;
}

}  // namespace

extern "C" bolt_status bolt_radix_sort_perm_multi(bolt_ctx* ctx, const bolt_col_view* keys, int32_t n_keys,
                                                  const int32_t* descending, const int32_t* nulls_first,
                                                  bolt_col_mut* perm, uint32_t flags, bolt_stream stream) {
    if (!ctx) return BOLT_ERR_INVALID;
    if (!keys || n_keys < 1 || !perm || !descending || !nulls_first)
        return fail(ctx, BOLT_ERR_INVALID, "ORDER BY: bad arguments");
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t n = keys[0].len;
    for (int k = 0; k < n_keys; ++k) {
        if (keys[k].len != n) return fail(ctx, BOLT_ERR_INVALID, "ORDER BY: key lengths differ");
        if (sort_src_of(keys[k].dtype) < 0) return fail(ctx, BOLT_DECLINE, "ORDER BY: key dtype %d", keys[k].dtype);
        if (!col_aligned(keys[k].data, keys[k].dtype))
            return fail(ctx, BOLT_ERR_INVALID, "ORDER BY: key %d is not aligned to its element width", k);
    }
    if (perm->dtype != BOLT_U32 || perm->cap < n) return fail(ctx, BOLT_ERR_CAPACITY, "ORDER BY: permutation output too small");
    if (n >= (1ull << 30)) return fail(ctx, BOLT_DECLINE, "ORDER BY: %llu rows exceed 2^30", (ull)n);
    bolt_status st = call_begin(ctx, flags, s);
    if (st != BOLT_OK) return st;
    uint32_t* out = (uint32_t*)perm->data;
    // Ping-pong between the caller's output and one scratch array so the
    // last (most significant) key writes the caller's buffer.
    uint32_t* tmp = n_keys > 1 ? (uint32_t*)arena_alloc(ctx, (n ? n : 1) * 4) : nullptr;
    ull* cnt = (ull*)arena_alloc(ctx, 256);
    if ((n_keys > 1 && !tmp) || !cnt) return fail(ctx, BOLT_ERR_CAPACITY, "ORDER BY: scratch arena too small");
    const uint32_t* cur = nullptr;  // nullptr = identity order
    kernel_mark_begin(ctx, flags, s);
    for (int k = n_keys - 1; k >= 0; --k) {
        uint32_t* dst = ((n_keys - 1 - k) % 2 == (n_keys - 1) % 2) ? out : tmp;
        const uint64_t mark = ctx->arena_used;
        const bolt_col_view& key = keys[k];
        SortSpec sp;
        sp.src = sort_src_of(key.dtype);
        sp.descending = descending[k];
        SortSegment seg;
        seg.keys = key.data;
        if (!key.validity) {
            seg.payload_in = cur;
            sp.indirect = cur != nullptr;
            seg.n = n;
            seg.payload_out = dst;
            sp.segs.push_back(seg);
            st = radix_sort(ctx, s, sp);
            if (st != BOLT_OK) return st;
        } else {
            // Stable NULL partition: valid rows are sorted, NULL rows keep
            // their current relative order and go first or last.
            uint32_t* valid_ids = (uint32_t*)arena_alloc(ctx, (n ? n : 1) * 4);
            if (!valid_ids) return fail(ctx, BOLT_ERR_CAPACITY, "ORDER BY: scratch arena too small");
            CompactSpec cv;
            cv.n = n;
            cv.keep_valid_of = key.validity;
            cv.ids_in = cur;
            cv.row_ids = valid_ids;
            cv.n_out_dev = cnt;
            st = compact_enqueue(ctx, s, cv);
            if (st != BOLT_OK) return st;
            BOLT_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, cnt, 8, cudaMemcpyDeviceToHost, s));
            BOLT_CUDA(ctx, cudaStreamSynchronize(s));
            const ull nv = ctx->h_words[0];
            const uint64_t nn = n - nv;
            CompactSpec cn = cv;
            cn.invert = 1;
            cn.row_ids = dst + (nulls_first[k] ? 0 : nv);
            st = compact_enqueue(ctx, s, cn);
            if (st != BOLT_OK) return st;
            seg.payload_in = valid_ids;
            sp.indirect = 1;
            seg.n = nv;
            seg.payload_out = dst + (nulls_first[k] ? nn : 0);
            sp.segs.push_back(seg);
            st = radix_sort(ctx, s, sp);
            if (st != BOLT_OK) return st;
        }
        ctx->arena_used = mark;
        cur = dst;
    }
    kernel_mark_end(ctx, flags, s);
    st = call_end(ctx, flags, s);
    if (st != BOLT_OK) return st;
    if (flags & BOLT_FLAG_ASYNC) return BOLT_OK;
    uint32_t f = 0;
    st = read_status(ctx, s, 0, &f);
    if (st != BOLT_OK) return st;
    return flags_to_status(ctx, f, "ORDER BY");
}

extern "C" bolt_status bolt_radix_sort_perm(bolt_ctx* ctx, const bolt_col_view* key, int32_t descending,
                                            int32_t nulls_first, bolt_col_mut* perm, uint32_t flags,
                                            bolt_stream stream) {
    return bolt_radix_sort_perm_multi(ctx, key, 1, &descending, &nulls_first, perm, flags, stream);
}
