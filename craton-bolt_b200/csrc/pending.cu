// pending.cu — entry points whose kernels are not in this build yet. Each
// declines loudly with a message so callers take their next path.
#include "ctx.cuh"

using namespace bolt;

extern "C" {

bolt_status bolt_batch_groupby(bolt_ctx* ctx, bolt_query*, int32_t, uint32_t, bolt_stream) {
    return fail(ctx, BOLT_DECLINE, "batched GROUP BY is not available in this build");
}

bolt_status bolt_hash_join_build(bolt_ctx* ctx, const bolt_col_view*, const bolt_col_view*, uint32_t, bolt_stream,
                                 bolt_join_table** t) {
    if (t) *t = nullptr;
    return fail(ctx, BOLT_DECLINE, "hash join is not available in this build");
}
bolt_status bolt_hash_join_probe(bolt_ctx* ctx, const bolt_join_table*, const bolt_col_view*, bolt_col_mut*,
                                 bolt_col_mut*, uint64_t*, uint32_t, bolt_stream) {
    return fail(ctx, BOLT_DECLINE, "hash join is not available in this build");
}
void bolt_hash_join_release(bolt_ctx*, bolt_join_table*) {}
bolt_status bolt_join_groupby(bolt_ctx* ctx, const bolt_join_table*, const bolt_col_view*, const bolt_col_view*,
                              bolt_col_mut*, bolt_col_mut*, bolt_col_mut*, uint64_t*, uint32_t, bolt_stream) {
    return fail(ctx, BOLT_DECLINE, "hash join is not available in this build");
}

bolt_status bolt_server_create(const bolt_server_config*, bolt_server** out) {
    if (out) *out = nullptr;
    return BOLT_DECLINE;
}
bolt_status bolt_server_submit(bolt_server*, bolt_query*, uint64_t*) { return BOLT_DECLINE; }
bolt_status bolt_server_wait(bolt_server*, uint64_t, double*) { return BOLT_DECLINE; }
void bolt_server_destroy(bolt_server*) {}

}  // extern "C"
