// ctx.cuh — bolt_ctx: device, scratch arena, status word, timing.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <unordered_map>

#include "common.cuh"

struct bolt_ctx {
    int device = 0;
    int num_sms = 148;
    int max_smem_optin = 0;
    // Scratch arena: a bump allocator reset at the start of every call. All
    // kernels of one call are ordered on one stream, so reuse across calls is
    // safe without frees.
    char* arena = nullptr;
    uint64_t arena_bytes = 0;
    uint64_t arena_used = 0;
    uint64_t arena_pinned = 0;   // bytes at the arena's start kept across calls (join tables)
    // Device status block: [0] status flags (u32), [2..] per-call counters.
    uint32_t* d_status = nullptr;
    ull* d_words = nullptr;      // 64 general device words (counts, reductions)
    ull* h_words = nullptr;      // pinned host mirror
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // Ring of event pairs around the dominant kernel of profiled calls.
    static constexpr uint32_t KRING = 256;
    cudaEvent_t kev[2 * KRING] = {};
    uint32_t kcount = 0;
    double last_ms = 0.0;
    uint32_t last_launches = 0;
    int32_t last_tier = 0;       // GROUP BY tier of the last bolt_groupby (1 global table, 2 partitioned, 3 wide keys)
    uint32_t async_pending = 0;
    std::string last_error;
    // Pinned staging ring for descriptor uploads: each upload copies into the
    // next free chunk and records an event; a chunk is reused only after its
    // event completed, so asynchronous calls never see their descriptors
    // overwritten.
    static constexpr uint32_t STAGE_SLOTS = 64;
    char* stage = nullptr;
    uint64_t stage_bytes = 0;
    uint64_t stage_head = 0;
    struct StageUse { uint64_t off, len; cudaEvent_t ev; bool live; };
    StageUse stage_use[STAGE_SLOTS] = {};
    uint32_t stage_next = 0;
    // Autotuned GROUP BY launch choices per query shape (see gb_shape_key).
    // GROUP BY launch choices: block size, shared-table shrink (8 = no shared
    // tier), warp pre-aggregation, table load (1 << load_shift - 1 headroom),
    // shared-table admission in eighths, the staged kernel's 32-row chunks
    // per consumer warp (0 = the register kernel), and whether the
    // hash-partitioned tier serves the shape (part = 1).
    struct GbTune {
        int32_t block, smem_shift, warp_agg, load_shift, smem_fill, staged;
        double ms;
        int32_t part = 0;
    };
    std::unordered_map<uint64_t, GbTune> tune;
    // Host-column GROUP BY (bolt_groupby_host): a copy stream and, per
    // staging slot, "copied" / "consumed" events; created on first use.
    static constexpr int HOST_SLOTS = 3;
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t host_ev[2 * HOST_SLOTS + 1] = {};
};

namespace bolt {

// Records a failure message and returns the status.
bolt_status fail(bolt_ctx* ctx, bolt_status s, const char* fmt, ...);

// Maps a CUDA error to BOLT_ERR_CUDA with its message.
bolt_status cuda_fail(bolt_ctx* ctx, cudaError_t e, const char* where);

#define BOLT_CUDA(ctx, call)                                   \
    do {                                                       \
        cudaError_t _e = (call);                               \
        if (_e != cudaSuccess) return bolt::cuda_fail(ctx, _e, #call); \
    } while (0)

// Raises a kernel's dynamic shared-memory limit to the device's opt-in
// maximum, once per (kernel, device). The attribute is process-wide, so
// per-call values would race between host threads that launch the same
// kernel with different sizes; one maximal value never does.
cudaError_t ensure_smem_optin(const void* kernel, int device, int max_optin);
template <class F>
inline cudaError_t smem_optin(F* kernel, const bolt_ctx* ctx) {
    return ensure_smem_optin(reinterpret_cast<const void*>(kernel), ctx->device, ctx->max_smem_optin);
}

// Arena allocation (256-byte aligned); returns nullptr when exhausted.
void* arena_alloc(bolt_ctx* ctx, uint64_t bytes);
inline void arena_reset(bolt_ctx* ctx) { ctx->arena_used = ctx->arena_pinned; }

// Copies `bytes` of host data to device memory `dst` in stream order through
// the pinned staging ring (the host buffer may be reused on return).
bolt_status stage_upload(bolt_ctx* ctx, cudaStream_t s, void* dst, const void* src, uint64_t bytes);

// Begins / ends a call: resets the arena, clears the status word, records the
// profiling event.
bolt_status call_begin(bolt_ctx* ctx, uint32_t flags, cudaStream_t s);
bolt_status call_end(bolt_ctx* ctx, uint32_t flags, cudaStream_t s);

// Event pair around the dominant kernel of a profiled call.
inline void kernel_mark_begin(bolt_ctx* ctx, uint32_t flags, cudaStream_t s) {
    if ((flags & (BOLT_FLAG_PROFILE | BOLT_FLAG_KERNEL_TIMES)) && ctx->kcount < bolt_ctx::KRING)
        cudaEventRecord(ctx->kev[2 * ctx->kcount], s);
}
inline void kernel_mark_end(bolt_ctx* ctx, uint32_t flags, cudaStream_t s) {
    if ((flags & (BOLT_FLAG_PROFILE | BOLT_FLAG_KERNEL_TIMES)) && ctx->kcount < bolt_ctx::KRING) {
        cudaEventRecord(ctx->kev[2 * ctx->kcount + 1], s);
        ctx->kcount++;
    }
}

// Reads the status word + n device words into ctx->h_words (synchronises s).
bolt_status read_status(bolt_ctx* ctx, cudaStream_t s, int n_words, uint32_t* flags);

// Translates device status flags into a bolt_status + message.
bolt_status flags_to_status(bolt_ctx* ctx, uint32_t flags, const char* op);

inline unsigned grid_for(uint64_t n, unsigned block, unsigned max_blocks) {
    uint64_t g = (n + block - 1) / block;
    if (g < 1) g = 1;
    if (g > max_blocks) g = max_blocks;
    return (unsigned)g;
}

}  // namespace bolt
