// context.hpp -- the nrrs_ctx object behind the C-ABI (internal to libnrrs_b200).
//
// One context replaces the reference's NRRSNetwork (src/render/nrrs/net/network.h:22-214): it
// owns the FP32 master parameters [table | StatNet | RRSNet], their gradients and Adam
// moments, the derived FP16 table and packed MLP images, and the scratch of the decision and
// training kernels. All device memory is allocated once in nrrs_create (NRRSNetwork::resize
// allocates per frame size; capacities here are max_queue / max_train).
#pragma once
#include <string>
#include <vector>

#include "kernels.hpp"

namespace nrrs {
// launch counters and optional per-launch CUDA-event timing (nrrs_profile_*)
struct Profiler {
    bool enabled = false;
    uint64_t launches[NRRS_KERNEL_KINDS] = {};
    uint64_t total_launches = 0;
    std::vector<cudaEvent_t> pool;                    // event pairs, reused
    std::vector<std::pair<int, int>> pending[NRRS_KERNEL_KINDS];
    size_t next = 0;
    uint64_t timed_launches[NRRS_KERNEL_KINDS] = {};
    double timed_ms[NRRS_KERNEL_KINDS] = {};
};
}  // namespace nrrs

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
    uint4* cells = nullptr;    // cell image of the FP16 table's dense levels (EncodeParams::cells)
    uint32_t n_cells = 0;
    // moving average of the weights (ema_decay > 0): the raw average, its debiased copy and the
    // inference images derived from that copy (the training images above stay on params)
    float* ema = nullptr;          // [n_params]
    float* params_inf = nullptr;   // [n_params] ema / (1 - d^t)
    float* wt_inf = nullptr;       // transposed FP32 MLP weights of params_inf
    __half* table_h_inf = nullptr; // FP16 table of params_inf (mixed precision)
    uint4* cells_inf = nullptr;    // its cell image
    uint64_t ema_t = 0;
    float* wt = nullptr;       // transposed FP32 MLP weights
    float* wrow = nullptr;     // aligned row-major copy of the FP32 MLP weights
    void* wpack = nullptr;     // UMMA-packed FP16/BF16 MLP weights
    void* tpack = nullptr;     // training image: forward layers, FP16 StatNet / BF16 RRSNet
    size_t wt_floats = 0, wpack_bytes = 0;
    size_t wt_rrs_offset = 0;  // floats from wt to the RRSNet part

    nrrs::DecideScratch* scr = nullptr;
    unsigned long long* states = nullptr;
    uint32_t max_chunks = 0;
    // split counts of the two-pass decision when the caller passes no split array
    uint8_t* split_tmp = nullptr;
    // the split training step runs the table-gradient scatter on this stream, forked from and
    // joined back into the caller's stream with the two events
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // segment tables resolved on the device from device-resident queue sizes: [0] in inference
    // tiles, [1] in decision chunks (the *_dev entry points)
    nrrs::SegmentTable* segs_dev = nullptr;

    // training scratch
    void* train_scratch = nullptr;
    size_t train_scratch_bytes = 0;
    double* loss_dev = nullptr;  // [2] last losses
    double* loss_sums = nullptr; // [4] batch sums of the loss weights (nrrs_train_step_batch)

    int last_infer_grid = 0;
    int tc_ctas_per_sm = 0;      // autotuned occupancy of the tcgen05 kernel (0 = default)
    int tc_wgs = 1;              // autotuned warpgroups per CTA of the tcgen05 kernel (1 or 2)
    int simt_ctas_per_sm = 0;    // autotuned occupancy of the FP32 kernel (0 = default)
    int tc_split = 0;            // inference mode of the tcgen05 path: 0 fused, 1 split
    int train_split = 1;         // training mode of the tcgen05 path: 0 fused, 1 split
    uint8_t* enc_tiles = nullptr;  // split mode: hash-feature tiles (kEncTileBytes each)
    uint32_t enc_tiles_cap = 0;
    uint8_t* x1_tiles = nullptr;   // split mode 2: RRSNet input tiles (kX1TileBytes each)
    nrrs::Profiler prof;
    std::string last_error;
};

namespace nrrs {
// RAII scope around one kernel launch: counts it and, when profiling is on, records an event
// pair on the launch stream.
struct ProfScope {
    nrrs_ctx* ctx;
    int kind;
    cudaStream_t s;
    int ev = -1;
    ProfScope(nrrs_ctx* c, int k, cudaStream_t st) : ctx(c), kind(k), s(st) {
        ++ctx->prof.launches[kind];
        ++ctx->prof.total_launches;
        Profiler& p = ctx->prof;
        if (p.enabled && p.next + 2 <= p.pool.size()) {
            ev = (int)p.next;
            p.next += 2;
            cudaEventRecord(p.pool[ev], s);
        }
    }
    ~ProfScope() {
        if (ev >= 0) {
            cudaEventRecord(ctx->prof.pool[ev + 1], s);
            ctx->prof.pending[kind].push_back({ev, ev + 1});
        }
    }
};
}  // namespace nrrs

namespace nrrs {
// gradients of one step; with apply, the Adam update too
// (lw: per-sample loss weights of nrrs_train_step_batch; NULL = plain means)
int train_step_impl(nrrs_ctx* ctx, const VertexPtrs& v, const float* target, uint32_t n,
                    double* loss_dev, cudaStream_t s, bool apply = true,
                    const LossWeights* lw = nullptr);
// batch sums of the loss weights into out[3] (sum s, sum w, mean pixel error)
cudaError_t launch_loss_sums(const LossWeights& w, uint32_t n, const float* error_sum,
                             uint32_t n_pixels, double* out, cudaStream_t s);
// Adam on ctx->grads scaled by `scale` (copied in from grads_dev first when it is not ctx->grads)
cudaError_t launch_adam_step(nrrs_ctx* ctx, bool train_rrs, cudaStream_t s, float scale = 1.0f);
size_t train_scratch_bytes(const nrrs_config& cfg, uint32_t n, int sm_count);
// the tensor-core training step covers 64-wide networks in mixed precision
bool train_tc_supported(const nrrs_config& cfg);
}  // namespace nrrs
