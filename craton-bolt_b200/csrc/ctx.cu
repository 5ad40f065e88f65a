// ctx.cu — context lifecycle, arena, status plumbing and small ABI helpers.
#include "ctx.cuh"

#include <mutex>
#include <set>
#include <utility>

#include <cstring>

namespace bolt {

bolt_status fail(bolt_ctx* ctx, bolt_status s, const char* fmt, ...) {
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return s;
}

bolt_status cuda_fail(bolt_ctx* ctx, cudaError_t e, const char* where) {
    return fail(ctx, BOLT_ERR_CUDA, "CUDA error %d (%s) at %s", (int)e, cudaGetErrorString(e), where);
}

void* arena_alloc(bolt_ctx* ctx, uint64_t bytes) {
    uint64_t off = (ctx->arena_used + 255) & ~uint64_t(255);
    if (off + bytes > ctx->arena_bytes) return nullptr;
    ctx->arena_used = off + bytes;
    return ctx->arena + off;
}

bolt_status stage_upload(bolt_ctx* ctx, cudaStream_t s, void* dst, const void* src, uint64_t bytes) {
    if (bytes == 0) return BOLT_OK;
    if (bytes > ctx->stage_bytes)
        return fail(ctx, BOLT_ERR_CAPACITY, "descriptor upload of %llu bytes exceeds the staging ring", (ull)bytes);
    uint64_t off = (ctx->stage_head + 255) & ~uint64_t(255);
    if (off + bytes > ctx->stage_bytes) off = 0;
    // Wait for every earlier upload that overlaps [off, off + bytes).
    for (uint32_t i = 0; i < bolt_ctx::STAGE_SLOTS; ++i) {
        auto& u = ctx->stage_use[i];
        if (u.live && u.off < off + bytes && off < u.off + u.len) {
            BOLT_CUDA(ctx, cudaEventSynchronize(u.ev));
            u.live = false;
        }
    }
    auto& slot = ctx->stage_use[ctx->stage_next];
    if (slot.live) {
        BOLT_CUDA(ctx, cudaEventSynchronize(slot.ev));
        slot.live = false;
    }
    std::memcpy(ctx->stage + off, src, bytes);
    BOLT_CUDA(ctx, cudaMemcpyAsync(dst, ctx->stage + off, bytes, cudaMemcpyHostToDevice, s));
    BOLT_CUDA(ctx, cudaEventRecord(slot.ev, s));
    slot.off = off;
    slot.len = bytes;
    slot.live = true;
    ctx->stage_next = (ctx->stage_next + 1) % bolt_ctx::STAGE_SLOTS;
    ctx->stage_head = off + bytes;
    return BOLT_OK;
}

bolt_status call_begin(bolt_ctx* ctx, uint32_t flags, cudaStream_t s) {
    arena_reset(ctx);
    ctx->last_error.clear();
    ctx->last_launches = 0;
    BOLT_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!(flags & BOLT_FLAG_ASYNC) || ctx->async_pending == 0)
        BOLT_CUDA(ctx, cudaMemsetAsync(ctx->d_status, 0, 16, s));
    if (flags & BOLT_FLAG_PROFILE) BOLT_CUDA(ctx, cudaEventRecord(ctx->ev0, s));
    return BOLT_OK;
}

bolt_status call_end(bolt_ctx* ctx, uint32_t flags, cudaStream_t s) {
    BOLT_CUDA(ctx, cudaGetLastError());
    if (flags & BOLT_FLAG_PROFILE) {
        BOLT_CUDA(ctx, cudaEventRecord(ctx->ev1, s));
        if (!(flags & BOLT_FLAG_ASYNC)) {
            BOLT_CUDA(ctx, cudaEventSynchronize(ctx->ev1));
            float ms = 0.f;
            BOLT_CUDA(ctx, cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
            ctx->last_ms = ms;
        }
    }
    if (flags & BOLT_FLAG_ASYNC) ctx->async_pending++;
    return BOLT_OK;
}

cudaError_t ensure_smem_optin(const void* kernel, int device, int max_optin) {
    static std::mutex mu;
    static std::set<std::pair<const void*, int>> done;
    std::lock_guard<std::mutex> lk(mu);
    if (done.count({kernel, device})) return cudaSuccess;
    // The limit covers dynamic memory only: leave room for the static part.
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    const int dyn = max_optin - (int)fa.sharedSizeBytes;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn > 0 ? dyn : 0);
    if (e == cudaSuccess) done.insert({kernel, device});
    return e;
}

bolt_status read_status(bolt_ctx* ctx, cudaStream_t s, int n_words, uint32_t* flags) {
    BOLT_CUDA(ctx, cudaMemcpyAsync(ctx->h_words, ctx->d_status, 16, cudaMemcpyDeviceToHost, s));
    if (n_words > 0)
        BOLT_CUDA(ctx, cudaMemcpyAsync(ctx->h_words + 2, ctx->d_words, n_words * sizeof(ull),
                                       cudaMemcpyDeviceToHost, s));
    BOLT_CUDA(ctx, cudaStreamSynchronize(s));
    *flags = (uint32_t)(ctx->h_words[0] & 0xFFFFFFFFu);
    return BOLT_OK;
}

bolt_status flags_to_status(bolt_ctx* ctx, uint32_t f, const char* op) {
    if (f & ST_FLAG_OVERFLOW)
        return fail(ctx, BOLT_ERR_OVERFLOW, "%s: SUM(integer) overflow: accumulator exceeds i64 range", op);
    if (f & ST_FLAG_TIMEOUT) return fail(ctx, BOLT_ERR_TIMEOUT, "%s: bounded device wait expired", op);
    if (f & ST_FLAG_SPILL) return fail(ctx, BOLT_ERR_SPILL, "partition_reduce spill: %s hash table probe limit reached", op);
    if (f & ST_FLAG_DUPKEY) return fail(ctx, BOLT_DECLINE, "%s: duplicate build keys", op);
    if (f & ST_FLAG_CAPACITY) return fail(ctx, BOLT_ERR_CAPACITY, "%s: output capacity exceeded", op);
    if (f & ST_FLAG_INTERNAL) return fail(ctx, BOLT_ERR_CUDA, "%s: internal error (group index outside its table)", op);
    return BOLT_OK;
}

}  // namespace bolt

using namespace bolt;

extern "C" {

const char* bolt_version(void) { return "bolt-b200 0.1.0 sm_100a"; }

const char* bolt_status_str(bolt_status s) {
    switch (s) {
    case BOLT_OK: return "ok";
    case BOLT_DECLINE: return "decline";
    case BOLT_ERR_SPILL: return "spill";
    case BOLT_ERR_OVERFLOW: return "overflow";
    case BOLT_ERR_CAPACITY: return "capacity";
    case BOLT_ERR_TIMEOUT: return "timeout";
    case BOLT_ERR_CUDA: return "cuda";
    case BOLT_ERR_INVALID: return "invalid";
    }
    return "unknown";
}

bolt_status bolt_ctx_create(int device, uint64_t scratch_bytes, bolt_ctx** out) {
    if (!out) return BOLT_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BOLT_ERR_CUDA;
    if (device < 0 || device >= ndev) return BOLT_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) return BOLT_ERR_CUDA;
    bolt_ctx* ctx = new bolt_ctx();
    ctx->device = device;
    cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&ctx->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
    if (scratch_bytes == 0) {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        scratch_bytes = (uint64_t)fr / 4;
    }
    scratch_bytes = (scratch_bytes + 255) & ~uint64_t(255);
    if (cudaMalloc(&ctx->arena, scratch_bytes) != cudaSuccess ||
        cudaMalloc(&ctx->d_status, 16) != cudaSuccess ||
        cudaMalloc(&ctx->d_words, 64 * sizeof(ull)) != cudaSuccess ||
        cudaHostAlloc(&ctx->h_words, 72 * sizeof(ull), cudaHostAllocDefault) != cudaSuccess ||
        cudaEventCreate(&ctx->ev0) != cudaSuccess || cudaEventCreate(&ctx->ev1) != cudaSuccess ||
        [&] {
            for (uint32_t i = 0; i < 2 * bolt_ctx::KRING; ++i)
                if (cudaEventCreate(&ctx->kev[i]) != cudaSuccess) return true;
            for (uint32_t i = 0; i < bolt_ctx::STAGE_SLOTS; ++i)
                if (cudaEventCreateWithFlags(&ctx->stage_use[i].ev, cudaEventDisableTiming) != cudaSuccess) return true;
            return false;
        }() ||
        cudaHostAlloc(&ctx->stage, 32ull << 20, cudaHostAllocDefault) != cudaSuccess) {
        bolt_ctx_destroy(ctx);
        cudaGetLastError();
        return BOLT_ERR_CAPACITY;
    }
    ctx->arena_bytes = scratch_bytes;
    ctx->stage_bytes = 32ull << 20;
    cudaMemset(ctx->d_status, 0, 16);
    cudaMemset(ctx->d_words, 0, 64 * sizeof(ull));
    cudaDeviceSynchronize();
    *out = ctx;
    return BOLT_OK;
}

void bolt_ctx_destroy(bolt_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->arena) cudaFree(ctx->arena);
    if (ctx->d_status) cudaFree(ctx->d_status);
    if (ctx->d_words) cudaFree(ctx->d_words);
    if (ctx->h_words) cudaFreeHost(ctx->h_words);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    for (uint32_t i = 0; i < 2 * bolt_ctx::KRING; ++i)
        if (ctx->kev[i]) cudaEventDestroy(ctx->kev[i]);
    for (uint32_t i = 0; i < bolt_ctx::STAGE_SLOTS; ++i)
        if (ctx->stage_use[i].ev) cudaEventDestroy(ctx->stage_use[i].ev);
    if (ctx->stage) cudaFreeHost(ctx->stage);
    for (int i = 0; i < 2 * bolt_ctx::HOST_SLOTS + 1; ++i)
        if (ctx->host_ev[i]) cudaEventDestroy(ctx->host_ev[i]);
    if (ctx->copy_stream) cudaStreamDestroy(ctx->copy_stream);
    delete ctx;
}

uint32_t bolt_ctx_kernel_times(bolt_ctx* ctx, double* ms, uint32_t max) {
    if (!ctx) return 0;
    uint32_t n = ctx->kcount < max ? ctx->kcount : max;
    for (uint32_t i = 0; i < n; ++i) {
        float t = 0.f;
        cudaEventSynchronize(ctx->kev[2 * i + 1]);
        if (cudaEventElapsedTime(&t, ctx->kev[2 * i], ctx->kev[2 * i + 1]) != cudaSuccess) t = -1.f;
        if (ms) ms[i] = t;
    }
    cudaGetLastError();
    ctx->kcount = 0;
    return n;
}

const char* bolt_ctx_last_error(const bolt_ctx* ctx) { return ctx ? ctx->last_error.c_str() : ""; }
double bolt_ctx_last_device_ms(const bolt_ctx* ctx) { return ctx ? ctx->last_ms : 0.0; }
uint32_t bolt_ctx_last_launches(const bolt_ctx* ctx) { return ctx ? ctx->last_launches : 0; }
int32_t bolt_ctx_last_groupby_tier(const bolt_ctx* ctx) { return ctx ? ctx->last_tier : 0; }
uint64_t bolt_ctx_scratch_bytes(const bolt_ctx* ctx) { return ctx ? ctx->arena_bytes : 0; }

bolt_status bolt_ctx_sync_status(bolt_ctx* ctx, bolt_stream stream) {
    if (!ctx) return BOLT_ERR_INVALID;
    uint32_t f = 0;
    bolt_status st = read_status(ctx, (cudaStream_t)stream, 0, &f);
    if (st != BOLT_OK) return st;
    ctx->async_pending = 0;
    if (ctx->last_ms == 0.0) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1) == cudaSuccess) ctx->last_ms = ms;
        cudaGetLastError();
    }
    cudaMemsetAsync(ctx->d_status, 0, 16, (cudaStream_t)stream);
    return flags_to_status(ctx, f, "async call");
}

}  // extern "C"
