// graph.cu — a batch of GROUP BY queries captured once as a CUDA graph.
//
// The whole batched enqueue (table memsets, descriptor uploads, the
// persistent aggregation launch, the batched finalize with its segmented
// sort) is recorded with stream capture into one graph and replayed with a
// single cudaGraphLaunch. The graph owns a private bolt_ctx (arena + pinned
// descriptor staging) so nothing another call does can overwrite the
// buffers the graph's nodes point to.
#include <vector>

#include "groupby.cuh"

struct bolt_graph {
    bolt_ctx* ctx = nullptr;
    cudaStream_t cap_stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<bolt::GbPlan> plans;
    std::vector<ull> words;  // host copy of the per-query device words
    int nq = 0;
};

using namespace bolt;

extern "C" void bolt_graph_destroy(bolt_graph* g) {
    if (!g) return;
    if (g->ctx) cudaSetDevice(g->ctx->device);
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (g->cap_stream) cudaStreamDestroy(g->cap_stream);
    if (g->ctx) bolt_ctx_destroy(g->ctx);
    delete g;
}

extern "C" bolt_status bolt_batch_graph_create(int device, bolt_query* qs, int32_t n, bolt_graph** out) {
    if (!qs || n <= 0 || !out) return BOLT_ERR_INVALID;
    *out = nullptr;
    bolt_graph* g = new bolt_graph();
    g->nq = n;
    g->plans.resize(n);
    // Size the private arena from the plans (a scratch-free probe context
    // only reads device attributes).
    bolt_ctx* probe = nullptr;
    bolt_status st = bolt_ctx_create(device, 1 << 20, &probe);
    if (st != BOLT_OK) {
        delete g;
        return st;
    }
    uint64_t need = 64ull << 20;
    for (int i = 0; i < n; ++i) {
        st = gb_plan(probe, &qs[i].desc, &qs[i].out, qs[i].row_begin, qs[i].row_end, BOLT_FLAG_ASYNC, 0, 0,
                     &g->plans[i]);
        qs[i].status = st;
        if (st != BOLT_OK) {
            bolt_ctx_destroy(probe);
            delete g;
            return st;
        }
        need += gb_plan_scratch(g->plans[i]) + (64ull << 10);
    }
    bolt_ctx_destroy(probe);
    st = bolt_ctx_create(device, need, &g->ctx);
    if (st != BOLT_OK) {
        delete g;
        return st;
    }
    bolt_ctx* ctx = g->ctx;
    if (cudaStreamCreateWithFlags(&g->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
        bolt_graph_destroy(g);
        return BOLT_ERR_CUDA;
    }
    std::vector<GbPlan*> run(n);
    for (int i = 0; i < n; ++i) {
        g->plans[i].prm.status = ctx->d_status;
        g->plans[i].fin.status = ctx->d_status;
        g->plans[i].fin.n_groups_user = (ull*)qs[i].out.n_groups_dev;
        run[i] = &g->plans[i];
    }
    arena_reset(ctx);
    if (cudaStreamBeginCapture(g->cap_stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        bolt_graph_destroy(g);
        return BOLT_ERR_CUDA;
    }
    cudaMemsetAsync(ctx->d_status, 0, 16, g->cap_stream);
    st = gb_run(ctx, run.data(), n, g->cap_stream, 0, true);
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(g->cap_stream, &graph);
    if (st != BOLT_OK || ce != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        bolt_graph_destroy(g);
        return st != BOLT_OK ? st : BOLT_ERR_CUDA;
    }
    g->graph = graph;
    if (cudaGraphInstantiate(&g->exec, graph, 0) != cudaSuccess) {
        bolt_graph_destroy(g);
        return BOLT_ERR_CUDA;
    }
    g->words.resize((size_t)n * 8);
    *out = g;
    return BOLT_OK;
}

extern "C" bolt_status bolt_graph_launch(bolt_graph* g, bolt_stream stream) {
    if (!g || !g->exec) return BOLT_ERR_INVALID;
    cudaSetDevice(g->ctx->device);
    return cudaGraphLaunch(g->exec, (cudaStream_t)stream) == cudaSuccess ? BOLT_OK : BOLT_ERR_CUDA;
}

extern "C" bolt_status bolt_graph_sync_status(bolt_graph* g, bolt_stream stream, int32_t* statuses,
                                              uint64_t* n_groups) {
    if (!g) return BOLT_ERR_INVALID;
    bolt_ctx* ctx = g->ctx;
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t gf = 0;
    bolt_status st = read_status(ctx, s, 0, &gf);
    if (st != BOLT_OK) return st;
    BOLT_CUDA(ctx, cudaMemcpy(g->words.data(), g->plans[0].words, (size_t)g->nq * 64, cudaMemcpyDeviceToHost));
    bolt_status first = BOLT_OK;
    for (int i = 0; i < g->nq; ++i) {
        const uint32_t f = (uint32_t)g->words[(size_t)i * 8 + 3];
        bolt_status q = BOLT_OK;
        if (f & (ST_FLAG_GROW | ST_FLAG_SPILL | ST_FLAG_RANGE | ST_FLAG_DECRANGE)) q = BOLT_ERR_SPILL;
        else if (f & (ST_FLAG_OVERFLOW | ST_FLAG_DECOVERFLOW)) q = BOLT_ERR_OVERFLOW;
        else if (f & ST_FLAG_CAPACITY) q = BOLT_ERR_CAPACITY;
        if (gf & ST_FLAG_TIMEOUT) q = BOLT_ERR_TIMEOUT;
        if (statuses) statuses[i] = q;
        if (n_groups) n_groups[i] = g->words[(size_t)i * 8 + 2];
        if (q != BOLT_OK && first == BOLT_OK) first = q;
    }
    return first;
}
