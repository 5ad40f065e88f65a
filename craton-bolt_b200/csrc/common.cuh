// common.cuh — shared device/host helpers of the bolt-b200 library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "bolt_b200.h"

typedef unsigned long long ull;
typedef long long ll;

namespace bolt {

// ---- device status word bits (read back by the host after a call) --------
enum : uint32_t {
    ST_FLAG_SPILL = 1u << 0,     // global hash table probe limit reached
    ST_FLAG_OVERFLOW = 1u << 1,  // integer / decimal SUM out of range
    ST_FLAG_RANGE = 1u << 2,     // f64 SUM value outside the fixed-point window
    ST_FLAG_TIMEOUT = 1u << 3,   // bounded spin gave up
    ST_FLAG_DUPKEY = 1u << 4,    // duplicate join build key
    ST_FLAG_GROW = 1u << 5,      // table occupancy over the load limit
    ST_FLAG_DECRANGE = 1u << 6,  // decimal value does not fit the 64-bit fast path
    ST_FLAG_CAPACITY = 1u << 7,  // output capacity exceeded
    ST_FLAG_DECOVERFLOW = 1u << 8,  // SUM(Decimal128) outside the i128 range
    ST_FLAG_INTERNAL = 1u << 9,     // a finalize index outside its table (never expected)
};

// Bytes per row of a column dtype (0 for an unknown dtype).
__host__ __device__ __forceinline__ int dtype_width(int dt) {
    switch (dt) {
    case BOLT_I32: case BOLT_F32: case BOLT_U32: return 4;
    case BOLT_I64: case BOLT_F64: return 8;
    case BOLT_DEC128: return 16;
    }
    return 0;
}

// A column's data pointer must be aligned to its element width (kernels use
// native-width and 16-byte vector accesses); checked on the host.
inline bool col_aligned(const void* p, int dt) {
    const int w = dtype_width(dt);
    return w != 0 && (reinterpret_cast<uintptr_t>(p) % (uintptr_t)w) == 0;
}

// ---- bit-level helpers ----------------------------------------------------
__host__ __device__ __forceinline__ int ceil_log2_u64(uint64_t x) {
    int r = 0;
    while ((1ull << r) < x && r < 63) ++r;
    return r;
}

__device__ __forceinline__ bool bit_valid(const uint8_t* v, uint64_t i) {
    return v == nullptr || ((__ldg(v + (i >> 3)) >> (i & 7)) & 1);
}

__device__ __forceinline__ void set_bit_atomic(uint8_t* bm, uint64_t i, bool on) {
    // Byte-granular bitmap writes from different threads need atomics on the
    // containing 32-bit word.
    uint32_t* w = reinterpret_cast<uint32_t*>(reinterpret_cast<uintptr_t>(bm + (i >> 3)) & ~uintptr_t(3));
    uint32_t shift = ((reinterpret_cast<uintptr_t>(bm + (i >> 3)) & 3) * 8) + (i & 7);
    if (on) atomicOr(w, 1u << shift);
    else atomicAnd(w, ~(1u << shift));
}

// Canonicalised float bit patterns (-0.0 -> +0.0, any NaN -> one quiet NaN),
// the GROUP BY / JOIN / ORDER BY float key equivalence of the reference.
__device__ __forceinline__ uint64_t canon_f64_bits(double x) {
    if (x != x) return 0x7FF8000000000000ull;
    if (x == 0.0) return 0ull;
    return (uint64_t)__double_as_longlong(x);
}
__device__ __forceinline__ uint32_t canon_f32_bits(float x) {
    if (x != x) return 0x7FC00000u;
    if (x == 0.0f) return 0u;
    return (uint32_t)__float_as_uint(x);
}

// Order-preserving u64 image of a float64 (NaN largest, -0 == +0).
__device__ __forceinline__ uint64_t f64_order_key(double x) {
    uint64_t b = canon_f64_bits(x);
    uint64_t mask = (uint64_t)(((int64_t)b) >> 63) | 0x8000000000000000ull;
    return b ^ mask;
}
__device__ __forceinline__ double f64_from_order_key(uint64_t k) {
    uint64_t b = (k & 0x8000000000000000ull) ? (k ^ 0x8000000000000000ull) : ~k;
    return __longlong_as_double((long long)b);
}

// Streaming loads: evict-first so the hash tables keep L2.
template <typename T>
__device__ __forceinline__ T ld_stream(const T* p) { return __ldcs(p); }

// Volatile (L2-coherent) 64-bit read of a word other threads update atomically.
__device__ __forceinline__ ull ld_volatile(const ull* p) {
    return *reinterpret_cast<const volatile ull*>(p);
}

// Lane helpers.
__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Signed 128-bit fixed-point -> correctly rounded double, times 2^-e.
// Round-to-nearest-even on the 128-bit magnitude, then an exact power-of-two
// scale. (Values here stay in the normal range of double.)
__device__ __forceinline__ double i128_to_double_scaled(ull lo, ll hi, int e) {
    bool neg = hi < 0;
    unsigned __int128 mag = ((unsigned __int128)(ull)hi << 64) | lo;
    if (neg) mag = (unsigned __int128)0 - mag;
    if (mag == 0) return 0.0;
    ull mhi = (ull)(mag >> 64), mlo = (ull)mag;
    int top = mhi ? 127 - __clzll((ll)mhi) : 63 - __clzll((ll)mlo);
    double d;
    int shift = 0;
    if (top <= 52) {
        d = (double)mlo;  // exact
    } else {
        shift = top - 52;
        unsigned __int128 mant = mag >> shift;
        unsigned __int128 rem = mag - (mant << shift);
        unsigned __int128 half = (unsigned __int128)1 << (shift - 1);
        if (rem > half || (rem == half && ((ull)mant & 1ull))) mant += 1;
        d = (double)(ull)mant;  // <= 2^53, exact
    }
    // d * 2^(shift - e) by one multiply with the exact power of two: the
    // callers' scales (0 <= e <= 94, shift <= 75) keep it a normal double.
    d *= __longlong_as_double((long long)(1023 + shift - e) << 52);
    return neg ? -d : d;
}

// float64 -> 128-bit fixed point with e fractional bits (0 <= e <= 1000),
// rounded to nearest-even at bit -e. Returns false for non-finite values or
// |v| >= 2^32 (the window the scale was chosen for).
//
// Done in float64 arithmetic, which is exact here: t = |v| * 2^e is a
// power-of-two scaling; h = floor(t / 2^64) is exact; r = t - h * 2^64 lies in
// [0, 2^64) and is a multiple of ulp(t), so it has at most 53 significant bits
// (when t >= 2^64, ulp(t) >= 2^12) and the fused multiply-add yields it
// exactly. Only the final conversion of r rounds.
__device__ __forceinline__ bool f64_to_fixed(double v, int e, ull& lo, ll& hi) {
    const double a = fabs(v);
    if (!(a < 4294967296.0)) return false;  // also NaN and infinities
    const double scale = __longlong_as_double((ll)(1023 + e) << 52);
    const double t = a * scale;
    const double h = floor(t * 0x1p-64);
    const double r = fma(-h, 0x1p64, t);
    ull l = __double2ull_rn(r);
    ull u = (ull)__double2ll_rz(h);
    if (__double_as_longlong(v) < 0) {  // negate the 128-bit magnitude
        l = ~l + 1ull;
        u = ~u + (l == 0 ? 1ull : 0ull);
    }
    lo = l;
    hi = (ll)u;
    return true;
}

}  // namespace bolt
