// context.hpp -- the nrrs_ctx object behind the C-ABI (internal to libnrrs_b200).
//
// One context replaces the reference's NRRSNetwork (src/render/nrrs/net/network.h:22-214): it
// owns the FP32 master parameters [table | StatNet | RRSNet], their gradients and Adam
// moments, the derived FP16 table and packed MLP images, and the scratch of the decision and
// training kernels. All device memory is allocated once in nrrs_create (NRRSNetwork::resize
// allocates per frame size; capacities here are max_queue / max_train).
#pragma once
#include <string>

#include "kernels.hpp"

struct nrrs_ctx {
    nrrs_config cfg{};
    int device = 0;
    int sm_count = 148;
    nrrs::EncodeParams enc{};
    uint64_t table_rows = 0;
    uint64_t n_table = 0, n_stat = 0, n_rrs = 0, n_params = 0;

    float* params = nullptr;   // FP32 master [n_params]
    float* grads = nullptr;    // [n_params]
    float* adam_m = nullptr;   // [n_params]
    float* adam_v = nullptr;   // [n_params]
    uint64_t adam_t = 0;

    __half* table_h = nullptr; // FP16 table copy (mixed precision)
    float* wt = nullptr;       // transposed FP32 MLP weights
    void* wpack = nullptr;     // UMMA-packed FP16/BF16 MLP weights
    size_t wt_floats = 0, wpack_bytes = 0;
    size_t wt_rrs_offset = 0;  // floats from wt to the RRSNet part

    nrrs::DecideScratch* scr = nullptr;
    unsigned long long* states = nullptr;
    uint32_t max_chunks = 0;

    // training scratch
    void* train_scratch = nullptr;
    size_t train_scratch_bytes = 0;
    double* loss_dev = nullptr;  // [2] last losses

    int tc_ctas_per_sm = 0;      // autotuned occupancy of the tcgen05 kernel (0 = default)
    std::string last_error;
};

namespace nrrs {
int train_step_impl(nrrs_ctx* ctx, const VertexPtrs& v, const float* target, uint32_t n,
                    double* loss_dev, cudaStream_t s);
size_t train_scratch_bytes(const nrrs_config& cfg, uint32_t n, int sm_count);
}  // namespace nrrs
