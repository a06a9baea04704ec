// k_train_simt.cu -- training step (placeholder until the kernels land).
#include "context.hpp"

namespace nrrs {
size_t train_scratch_bytes(const nrrs_config&, uint32_t, int) { return 256; }
int train_step_impl(nrrs_ctx* ctx, const VertexPtrs&, const float*, uint32_t, double*, cudaStream_t) {
    ctx->last_error = "training not built yet";
    return NRRS_ERR_UNSUPPORTED;
}
}  // namespace nrrs
