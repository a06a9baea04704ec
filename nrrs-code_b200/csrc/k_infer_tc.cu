// k_infer_tc.cu -- tcgen05 inference (placeholder until the kernel lands).
#include "kernels.hpp"
namespace nrrs {
size_t infer_tc_smem_bytes(int, int, int, int) { return 0; }
cudaError_t launch_infer_tc(const InferArgs&, int, int, int, int, int, int, int, cudaStream_t) {
    return cudaErrorNotSupported;
}
}  // namespace nrrs
