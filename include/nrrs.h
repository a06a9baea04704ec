/*
 * nrrs.h -- C-ABI of the B200 (sm_100a) neural Russian-roulette-and-splitting step.
 *
 * One library (libnrrs_b200.so) exports the per-path-vertex NRRS hot path:
 *   1. inference on a SoA wavefront queue: hash-grid + spherical-harmonics encoding,
 *      StatNet MLP, glue, RRSNet MLP, activation, clamp           (nrrs_infer)
 *   2. RRS normalisation and the stochastic kill/split decision,
 *      compaction of survivors into the next-bounce queue         (nrrs_decide_emit)
 *   3. both fused (nrrs_step) and batched over uneven depths      (nrrs_step_batched)
 *   4. one training step of StatNet and RRSNet on a sample batch  (nrrs_train_step)
 *   5. the training frame's path-node records, their radiance and the training batch built
 *      from them                                   (nrrs_record_nodes ... nrrs_sample_weights)
 *   6. the per-pixel error of the RRSNet loss      (nrrs_count_patch_samples ...
 *                                                   nrrs_calculate_error)
 *   7. the per-depth strategy search and the training schedule (host; nrrs_ubs_*,
 *      nrrs_train_schedule_*)
 *
 * Everything is asynchronous on the caller's CUDA stream (passed as void*; NULL = legacy
 * default stream). Input and output buffers are device pointers owned by the caller. The
 * context owns the weights, optimizer state and scratch. No entry point synchronises the
 * stream except the ones documented as synchronous (nrrs_get_device_status, parameter
 * copies to host, nrrs_save/nrrs_load).
 *
 * Reference interfaces replaced (paths inside banbao990/NRRS-Code):
 *   NRRSNetwork class                    src/render/nrrs/net/network.h:22-214
 *   NRRSPathTracer::generateRRSNumber    src/render/nrrs/integrator.cpp:1057-1483
 *   NRRSPathTracer::trainStep            src/render/nrrs/integrator.cpp:2337-2657
 *   calcSum2PassAsync<true>              src/render/common/commoncudautilshost.cpp:6-22
 *   TidQueue::push / pushCheck           src/render/common/commonworkqueue.h:19-42
 *   NRRSPathNodesBuffer                  src/render/nrrs/workqueue.h:108-188
 *   nrrs_generate_training_data          src/render/nrrs/train.cu:432-570
 *   nrrs_calculate_sample_weight         src/render/nrrs/train.cu:572-592
 *   nrrs_update_weighted_L, nrrs_calculate_error   src/render/nrrs/train.cu:344-430
 */
#ifndef NRRS_B200_H
#define NRRS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NRRS_ABI_VERSION 2

/* ---- status codes (the reference has none: Log(Fatal) aborts, overflow only printf's) ---- */
typedef enum {
    NRRS_OK = 0,
    NRRS_ERR_INVALID_ARG = -1,      /* bad pointer / size / config value                     */
    NRRS_ERR_CAPACITY_OVERFLOW = -2,/* next queue too small; *next_size still holds the need */
    NRRS_ERR_NAN = -3,              /* a NaN/Inf factor or loss was seen on the device       */
    NRRS_ERR_TIMEOUT = -4,          /* a bounded device wait gave up                         */
    NRRS_ERR_CUDA = -5,             /* a CUDA runtime call failed (see nrrs_last_error)      */
    NRRS_ERR_NO_DEVICE = -6,        /* no sm_100 device / library built without kernels      */
    NRRS_ERR_UNSUPPORTED = -7,      /* configuration outside what the kernels implement     */
    NRRS_ERR_IO = -8                /* nrrs_save / nrrs_load file error                       */
} nrrs_status;

/* device status bits accumulated by the kernels (nrrs_get_device_status) */
#define NRRS_DEV_OVERFLOW   0x1u    /* a queue write past capacity was dropped  */
#define NRRS_DEV_NAN        0x2u    /* non-finite factor or loss                */
#define NRRS_DEV_TIMEOUT    0x4u    /* look-back / barrier wait ran out         */
#define NRRS_DEV_SATURATED  0x8u    /* a split count above 255 was clamped      */
#define NRRS_DEV_BAD_INDEX  0x10u   /* a pixel or parent index out of range was skipped */

typedef enum {
    NRRS_PREC_FP32 = 0,   /* plain path: FP32 table, FP32 SIMT MLP                         */
    NRRS_PREC_FP16 = 1,   /* mixed: FP16 table, FP16 tcgen05 MLP, FP32 accumulate          */
    NRRS_PREC_BF16 = 2    /* mixed: FP16 table, BF16 tcgen05 MLP, FP32 accumulate          */
} nrrs_precision;

typedef enum {
    NRRS_FACTOR_ADRRS = 2,   /* step 2: mean(clamp(L,1e-4,1e4)*thp/(ref+0.01)) (integrator.cpp:1244-1254) */
    NRRS_FACTOR_RRSNET = 3   /* step 3: activationSigma(RRSNet raw)              (integrator.cpp:1188-1243) */
} nrrs_factor_source;

/* Network, encoding, optimizer and loss hyper-parameters.
 * Replaces the JSON config of common/configs/nrrs/nrrs/2net-simple.json + NRRSNetwork::reset
 * (src/render/nrrs/net/network.cpp:443-576). Fill with nrrs_config_default(). */
typedef struct {
    /* multiresolution hash grid (Instant-NGP); level l has floor(base_resolution*scale^l) cells */
    int32_t n_levels;              /* 16                                  */
    int32_t n_features_per_level;  /* 2 (only 2 is implemented)           */
    int32_t log2_hashmap_size;     /* 19                                  */
    int32_t base_resolution;       /* 16                                  */
    float per_level_scale;         /* 1.5                                 */
    int32_t sh_degree;             /* 4 -> 16 coefficients (only 4)       */
    /* networks: bias-free MLPs (a constant-1 input lane carries the bias, as in the reference) */
    int32_t statnet_width;         /* 64 or 128                           */
    int32_t statnet_hidden;        /* hidden layers: 2 or 3               */
    int32_t rrsnet_width;          /* 64 or 128                           */
    int32_t rrsnet_hidden;         /* 2 or 3                              */
    int32_t precision;             /* nrrs_precision                      */
    /* initialisation */
    uint64_t seed;                 /* Xavier-uniform weights + table init */
    float table_init_scale;        /* table ~ U(-s, s); 1e-4 as tcnn      */
    /* Adam (FP32 master weights and moments) */
    float lr, beta1, beta2, eps, l2_reg;
    /* losses */
    float stat_eps;                /* 0.01: StatNet target is log(L + stat_eps) */
    float ref_eps;                 /* 0.01: pixel estimate offset (integrator.cpp:1249) */
    float loss_clamp_max;          /* 10: per-sample relative contribution clamp (2net-simple.json clamp_max) */
    float cost_offset;             /* 1: path cost of a vertex = cost_offset + q */
    /* scene AABB for position normalisation (nrctrain.h:111-115); normalize_pos=0 feeds pos as-is */
    int32_t normalize_pos;
    float aabb_min[3], aabb_max[3];
    /* capacities (NRRSNetwork::resize, network.cpp:351) */
    uint32_t max_queue;            /* largest n for infer/decide        */
    uint32_t max_train;            /* largest batch for nrrs_train_step */
    int32_t step;                  /* setStep: 0..3 (network.cpp:578-589) */
    /* network family (nrrs_network_family): NRRS_NET_WORKLOAD or NRRS_NET_REFERENCE; fill the
     * reference family with nrrs_config_reference_network */
    int32_t network;
    /* Exponential moving average of the weights for inference (the Ema optimizer that wraps
     * Adam in 2net-simple.json:17-20, decay 0.95 there): after every Adam step
     * e <- d e + (1 - d) w over all parameters (e starts at 0 when parameters are uploaded),
     * and the inference entry points use e / (1 - d^t), t the number of steps since; training
     * keeps using w. 0 (the default) = off: inference uses w. */
    float ema_decay;
    /* Adam learning rate of the RRSNet parameters; 0 (the default) = lr. The reference trains
     * its two networks with separate optimizers (2net-simple.json level0 lr 5e-3 for the
     * encoding and StatNet, level1 lr 5e-4 for RRSNet). */
    float lr_rrsnet;
    /* Contexts whose exact normalisation sums are added together (sharded queues:
     * nrrs_infer_accumulate on every rank, then an integer all-reduce). The fixed-point shift
     * leaves room for sum_shards x max_queue terms, so the added sum cannot overflow; give
     * every rank the same value. 0 or 1 = one context. */
    uint32_t sum_shards;
} nrrs_config;

/* The two network families.
 * NRRS_NET_WORKLOAD: the benchmark workload's network. StatNet input 64 lanes (16-level hash
 *   grid, SH degree 4 of wi, normal, albedo, warped roughness, a bias lane); ReLU MLPs 64 or 128
 *   wide; 3 log-statistics log(L + stat_eps); RRSNet input [bc(L) x3, bc(thp) x3, warped
 *   roughness, bc(ref_mean), depth / 8, 1, 0 x6].
 * NRRS_NET_REFERENCE: the network the reference ships (common/configs/nrrs/nrrs/2net-simple.json
 *   level0/level1, myNetworkLL2.h:86, train.cu:41-112). StatNet input 32 lanes: HashGrid 8 levels
 *   x 2 features, base 16, scale 2.0 (16 lanes), OneBlob 4 bins on each lat-long coordinate of wi
 *   (8 lanes), OneBlob 8 bins on the warped roughness (8 lanes); no bias lane. LeakyReLU (slope
 *   0.01) MLPs 32 wide x 3 hidden layers; 6 outputs L RGB and L^2 RGB (L2_OFFSET 3). RRSNet
 *   input [bc(max(L,0)) x3, bc(max(L^2,0)) x3, bc(thp) x3, warped roughness, bc(ref_mean), 1,
 *   0 x4]. The StatNet loss is the relative squared error of L and L^2 against the target L and
 *   its square, (y - T)^2 / (T^2 + 0.01), averaged over the 6 outputs (the reference's NRRS_LL2
 *   lives in its absent tiny-cuda-nn fork). */
typedef enum { NRRS_NET_WORKLOAD = 0, NRRS_NET_REFERENCE = 1 } nrrs_network_family;

/* Input record of one path vertex, SoA (NRRSInferenceWorkItem, src/render/nrrs/workitem.h:9-15,
 * extended with the fields of the synthetic benchmark record). vec3 fields are [n][3] float. */
typedef struct {
    const float* pos;              /* [n][3] world (normalize_pos=1) or normalised position */
    const float* wi;               /* [n][3] unit incoming direction                         */
    const float* normal;           /* [n][3] unit shading normal                             */
    const float* roughness;        /* [n]                                                    */
    const float* albedo;           /* [n][3]                                                 */
    const float* thp;              /* [n][3] path throughput before RRS                      */
    const uint32_t* depth;         /* [n] bounce depth                                       */
    const float* ref_mean;         /* [n] mean of the pixel estimate (MyFilm, train.cu:54-58); NULL = 0.5 */
    const uint32_t* scatter_index; /* [n] mScatterQueueIndex; NULL = identity                */
} nrrs_vertex_soa;

/* Decision parameters (NRRSPathTracer members, src/render/nrrs/integrator.h:265-275, 521-539). */
typedef struct {
    float clamp_min;               /* RRS_CLAMP_MIN  (kill threshold)              */
    float clamp_max;               /* RRS_CLAMP_MAX  (split cap)                   */
    float normalize_rate;          /* RRS_NORMALIZE_RATE (used when !use_ceil)     */
    int32_t use_ceil;              /* mRRSNormalizeUseCeil                         */
    int32_t scale_up;              /* !mDonnotNormalizeWhenLessThanOne             */
    int32_t use_weight_window;     /* mUseWeightWindow (RRSWeightWindow, size 5)   */
    float weight_window_size;      /* 5                                            */
    int32_t factor_source;         /* nrrs_factor_source                           */
} nrrs_decide_params;

/* One segment of the batched launch: one depth's queue inside a concatenated SoA. */
typedef struct {
    uint32_t offset;               /* first vertex of this depth in the SoA        */
    uint32_t count;                /* vertices of this depth                       */
    uint32_t budget;               /* normalisation budget B (pixel count)         */
    uint32_t n_specular;           /* specular vertices excluded from the budget   */
    uint32_t queue_offset;         /* where this depth's next queue starts         */
    uint32_t queue_capacity;       /* capacity of this depth's next queue          */
} nrrs_segment;

typedef struct nrrs_ctx nrrs_ctx;

/* ---- lifetime ---- */
void nrrs_config_default(nrrs_config* cfg);
/* the reference's shipped network (NRRS_NET_REFERENCE) with its grid, widths and optimizer
 * settings (2net-simple.json: HashGrid 8 x 2, 2^19, base 16, scale 2.0; 32 x 3; Adam lr 5e-3
 * (RRSNet 5e-4), beta 0.9 / 0.99, eps 1e-15, l2 3e-6, moving average 0.95); the other fields
 * keep nrrs_config_default's values */
void nrrs_config_reference_network(nrrs_config* cfg);
/* NRRSNetwork::NRRSNetwork + reset + resize (network.cpp:443-576, 351-441). */
int nrrs_create(const nrrs_config* cfg, nrrs_ctx** out);
void nrrs_destroy(nrrs_ctx* ctx);
/* NRRSNetwork::setStep (network.cpp:578-589): 0/1 train StatNet only, 2 ADRRS factors, 3 RRSNet. */
int nrrs_set_step(nrrs_ctx* ctx, int32_t step);
const char* nrrs_last_error(const nrrs_ctx* ctx);
const char* nrrs_status_string(int status);
/* 1 when the library carries sm_100a kernels and a device is present. */
int nrrs_device_available(void);
void nrrs_decide_params_default(nrrs_decide_params* p);

/* ---- inference: replaces prepareInferenceData + inference + "Gen RRS Number"
 *      (network.cpp:297-349, integrator.cpp:1184-1298). Writes the 3 log-statistics
 *      (may be NULL), the clamped factor rrs[n] and, when use_ceil, adds ceil(rrs) to the
 *      context's exact 64-bit normalisation accumulator instead of rrs. ---- */
int nrrs_infer(nrrs_ctx* ctx, const nrrs_vertex_soa* v, uint32_t n,
               const nrrs_decide_params* p, float* stats, float* rrs, void* stream);

/* ---- decision + emission on given factors: replaces calcSum2PassAsync<true> +
 *      "Gen Tids" + TidQueue::push (integrator.cpp:1301-1460, commonworkqueue.h:19-25).
 *      Sums rrs (or ceil(rrs)) exactly, forms nf = (budget - n_specular) / sum, scales,
 *      draws s = int(r) + (rnd <= r - int(r)) and writes s copies of scatter_index[i] (or i)
 *      to next_queue in vertex order. rrs_norm[stid] receives the normalised factor
 *      (mScatterRayQueue->mRRS). split[i] receives s (may be NULL). n_specular_dev, when not
 *      NULL, overrides n_specular from device memory. *next_size_dev receives the total;
 *      writes at or past capacity are dropped and flagged. ---- */
int nrrs_decide_emit(nrrs_ctx* ctx, const float* rrs, const float* rnd,
                     const uint32_t* scatter_index, uint32_t n, uint32_t budget,
                     uint32_t n_specular, const uint32_t* n_specular_dev,
                     const nrrs_decide_params* p, float* rrs_norm, uint8_t* split,
                     uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev,
                     void* stream);

/* ---- decision + emission without any device allocation. No counterpart in the reference:
 *      for callers that cannot call cudaMalloc (a plugin whose host framework owns all device
 *      memory, a fixed start-up memory budget, a frame loop that must not take cudaMalloc's
 *      implicit synchronisation). Needs no context; the same results as nrrs_decide_emit on a
 *      context whose max_queue is NRRS_NOALLOC_MAX_N, with one difference in the arguments:
 *      n_specular is a host value only (there is no n_specular_dev). Its scratch is a static
 *      device array of about 66 KB (NRRS_NOALLOC_MAX_N vertices), resident on every GPU that
 *      loads the library until exit; n above NRRS_NOALLOC_MAX_N returns NRRS_ERR_INVALID_ARG.
 *      The first call in a CUDA context looks up the array's device address
 *      (cudaGetSymbolAddress) with that context current, so make that first call before any
 *      stream capture; a context created again after cudaDeviceReset gets a new lookup. All
 *      calls share the array: calls that overlap on the GPU (other streams, other host threads)
 *      race and must be serialised by the caller. ---- */
#define NRRS_NOALLOC_MAX_N (1u << 24)
int nrrs_decide_emit_noalloc(const float* rrs, const float* rnd, const uint32_t* scatter_index,
                             uint32_t n, uint32_t budget, uint32_t n_specular,
                             const nrrs_decide_params* p, float* rrs_norm, uint8_t* split,
                             uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev,
                             void* stream);
/* Device status bits (NRRS_DEV_*) that nrrs_decide_emit_noalloc calls have raised since the last
 * read, from the same static array: synchronises the stream, returns and clears them. The return
 * code follows nrrs_get_device_status (TIMEOUT, then CAPACITY_OVERFLOW, then NAN, else OK).
 * No counterpart in the reference (its overflow and NaN checks only printf). */
int nrrs_noalloc_device_status(uint32_t* flags, void* stream);

/* ---- fused: infer + decide + emit for one depth (generateRRSNumber<false,*>) ---- */
int nrrs_step(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd, uint32_t n,
              uint32_t budget, uint32_t n_specular, const nrrs_decide_params* p,
              float* stats, float* rrs, float* rrs_norm, uint8_t* split,
              uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev, void* stream);

/* ---- batched uneven depths in one persistent launch sequence (graph-capturable).
 *      segs is a HOST array of n_segs segments; next_size_dev[n_segs]. ---- */
int nrrs_step_batched(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                      const nrrs_segment* segs, int32_t n_segs, const nrrs_decide_params* p,
                      float* stats, float* rrs, float* rrs_norm, uint8_t* split,
                      uint32_t* next_queue, uint32_t* next_size_dev, void* stream);

/* ---- device-resident queue sizes. The reference's inference queue size lives on the device:
 *      the closest-hit program pushes vertices with an atomic and the integrator reads the size
 *      back before each depth (integrator.cpp:1073-1085, 1533-1555). These forms take the size
 *      as a device word (*n_dev) and a host bound max_n, which sizes every grid and capacity,
 *      so a depth loop needs no host read between the trace and the step and can be captured
 *      whole in a CUDA graph. The kernels read the count on the device; a count above max_n is
 *      clamped to max_n and flags NRRS_DEV_OVERFLOW. Results equal the host-size forms on the
 *      same count, bit for bit. All other arguments are those of the host-size forms. ---- */
int nrrs_infer_dev(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const uint32_t* n_dev,
                   uint32_t max_n, const nrrs_decide_params* p, float* stats, float* rrs,
                   void* stream);
int nrrs_decide_emit_dev(nrrs_ctx* ctx, const float* rrs, const float* rnd,
                         const uint32_t* scatter_index, const uint32_t* n_dev, uint32_t max_n,
                         uint32_t budget, uint32_t n_specular, const uint32_t* n_specular_dev,
                         const nrrs_decide_params* p, float* rrs_norm, uint8_t* split,
                         uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev,
                         void* stream);
/* generateRRSNumber<false,*> (integrator.cpp:1057-1483) on a device-sized queue */
int nrrs_step_dev(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                  const uint32_t* n_dev, uint32_t max_n, uint32_t budget, uint32_t n_specular,
                  const uint32_t* n_specular_dev, const nrrs_decide_params* p, float* stats,
                  float* rrs, float* rrs_norm, uint8_t* split, uint32_t* next_queue,
                  uint32_t capacity, uint32_t* next_size_dev, void* stream);
/* batched depths with device-resident counts: segs[k].count is the largest count of depth k
 * (its SoA range and queue capacity are sized for it), counts_dev[k] the actual count */
int nrrs_step_batched_dev(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                          const nrrs_segment* segs, const uint32_t* counts_dev, int32_t n_segs,
                          const nrrs_decide_params* p, float* stats, float* rrs, float* rrs_norm,
                          uint8_t* split, uint32_t* next_queue, uint32_t* next_size_dev,
                          void* stream);

/* ---- sharded inference and decision across GPUs (no counterpart in the single-GPU
 *      reference; the reference's sum is calcSum2PassAsync, commoncudautilshost.cpp:6-22).
 *      The normalisation sum is an exact 64-bit fixed-point integer, so shards add it with an
 *      integer all-reduce (NCCL or any transport) and every shard decides bit-identically to a
 *      single GPU processing the concatenated queue:
 *        *sum = 0; nrrs_infer_accumulate(shard, sum); allreduce_sum_int64(sum);
 *        nrrs_decide_emit_with_sum(shard, global budget, global n_specular, sum)
 *      sum_acc_dev is a caller-owned int64 on the device; the shift is fixed by max_queue and
 *      sum_shards, so all ranks must use the same max_queue, sum_shards (at least the number of
 *      ranks) and decision parameters. ---- */
int nrrs_infer_accumulate(nrrs_ctx* ctx, const nrrs_vertex_soa* v, uint32_t n,
                          const nrrs_decide_params* p, float* stats, float* rrs,
                          int64_t* sum_acc_dev, void* stream);
int nrrs_decide_emit_with_sum(nrrs_ctx* ctx, const float* rrs, const float* rnd,
                              const uint32_t* scatter_index, uint32_t n, uint32_t budget,
                              uint32_t n_specular, const int64_t* sum_acc_dev,
                              const nrrs_decide_params* p, float* rrs_norm, uint8_t* split,
                              uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev,
                              void* stream);
/* exact-sum value of an accumulator: sum = acc * 2^-shift (host helper) */
double nrrs_sum_from_accumulator(const nrrs_ctx* ctx, const nrrs_decide_params* p, int64_t acc);

/* ---- data-parallel training: gradients without the update, then Adam on (all-reduced)
 *      gradients. nrrs_train_grads leaves this step's gradients in the context;
 *      nrrs_copy_grads copies them to a caller device buffer [nrrs_param_count] for the
 *      all-reduce; nrrs_adam_apply runs Adam on grads_dev * scale (scale = 1/ranks for a mean)
 *      and refreshes the derived weight images. nrrs_train_step == grads + apply(own, 1). ---- */
int nrrs_train_grads(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* target, uint32_t n,
                     double* loss_dev, void* stream);
int nrrs_copy_grads(nrrs_ctx* ctx, float* grads_dev, void* stream);
int nrrs_adam_apply(nrrs_ctx* ctx, const float* grads_dev, float scale, void* stream);

/* ---- training: replaces NRRSNetwork::train (network.cpp:196-295) with the two
 *      tcnn training_step calls it makes. target is [n][3] radiance. loss_dev (may be
 *      NULL) receives {statnet_loss, rrsnet_loss} as FP64 on the device. ---- */
int nrrs_train_step(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* target,
                    uint32_t n, double* loss_dev, void* stream);

/* ---- parameters: FP32 master copy. Layout: [table | statnet W0..Wk | rrsnet V0..Vk],
 *      each W row-major [out][in]. Pointers are HOST pointers (synchronous copies). ---- */
uint64_t nrrs_param_count(const nrrs_ctx* ctx);
int nrrs_param_layout(const nrrs_ctx* ctx, uint64_t* table_params, uint64_t* statnet_params,
                      uint64_t* rrsnet_params);
int nrrs_get_params(const nrrs_ctx* ctx, float* host_dst, uint64_t count);
int nrrs_set_params(nrrs_ctx* ctx, const float* host_src, uint64_t count);
/* the weights the inference entry points use: the debiased moving average when ema_decay > 0
 * (equal to the trained weights right after an upload), else the trained weights */
int nrrs_get_inference_params(const nrrs_ctx* ctx, float* host_dst, uint64_t count);
/* gradients of the last nrrs_train_step (before the Adam update); host copy */
int nrrs_get_grads(const nrrs_ctx* ctx, float* host_dst, uint64_t count);
/* Adam step count and moments (host copies, count each) */
int nrrs_get_adam_state(const nrrs_ctx* ctx, float* m, float* v, uint64_t count, uint64_t* t);
/* level table: per level {offset (entries), entries, resolution, dense} as 4 uint32 */
int nrrs_level_table(const nrrs_ctx* ctx, uint32_t* host_dst, int32_t max_levels);

/* checkpoint: FP32 master weights, Adam m/v and step (loadWeights/saveWeights are stubs in
 * the reference, network.cpp:157-194) */
int nrrs_save(const nrrs_ctx* ctx, const char* path);
int nrrs_load(nrrs_ctx* ctx, const char* path);

/* ---- status: synchronises the stream, returns and clears the device status bits ---- */
int nrrs_get_device_status(nrrs_ctx* ctx, uint32_t* flags, void* stream);

/* ---- launch shape and autotuning (no counterpart in the reference, whose launches come from
 *      the occupancy API, commoncudautilshost.cpp:10-21). The inference kernel's shape is
 *      CTAs per SM x warpgroups per CTA (tcgen05 path: 1, 2 or 4, one 128-vertex tile in
 *      flight each, as the shared memory allows; the FP32 path uses CTAs per SM only).
 *      nrrs_autotune times every admissible shape on n synthetic vertices, keeps the fastest in
 *      the context and, with a cache path, reuses or records the choice in a JSON file keyed by
 *      device name, network shape and precision. report (may be NULL) receives a JSON summary.
 *      Synchronous. ---- */
int nrrs_autotune(nrrs_ctx* ctx, uint32_t n, const char* cache_path, char* report,
                  size_t report_len);
int nrrs_set_launch_shape(nrrs_ctx* ctx, int32_t ctas_per_sm, int32_t warpgroups);
int nrrs_get_launch_shape(const nrrs_ctx* ctx, int32_t* ctas_per_sm, int32_t* warpgroups);
/* Inference mode of the tensor-core path (the autotuner's third knob): 0 = fused (the MLP kernel
 * gathers the hash-grid corners itself), 1 = split (a level-major encoding kernel writes every
 * tile's hash features to HBM, four levels at a time so that the table slices in use stay in
 * L2, and the MLP kernel bulk-loads them; for tables larger than L2), 2 = split with the MLP
 * in two kernels (StatNet, which writes each tile's RRSNet input to HBM, then RRSNet; each
 * holds only its own weights, so more tiles are in flight per SM; with ADRRS factors only the
 * StatNet kernel runs), 3 = as 2 with each hidden layer's activations kept in TMEM as the next
 * layer's A operand (tcgen05.mma reads only the weights from shared memory; 1 or 2 warpgroups).
 * All modes give bit-identical results. Selecting split allocates (max_queue/128 + 17) feature
 * tiles of 8 KB, and modes 2 and 3 as many RRSNet input tiles of 4 KB; not available for the
 * FP32 path. */
int nrrs_set_infer_split(nrrs_ctx* ctx, int32_t split);
int nrrs_get_infer_split(const nrrs_ctx* ctx, int32_t* split);
/* Cell image of the dense hash-grid levels (mixed-precision contexts with at least one dense
 * level): for every cell of a dense level, its 8 FP16 corner entries in one 32-byte block, rebuilt
 * after every table update (32 bytes x the dense cells: 7.1 MB for 16 levels at 2^19, 81 MB at
 * 2^22). With it on (the default) a dense level costs the gathers one 32-byte load instead of
 * four 16-byte row loads. The corner values and their summation order are the table's, so
 * results are bit-identical either way. Enabling it where there is none returns
 * NRRS_ERR_UNSUPPORTED. */
int nrrs_set_cell_image(nrrs_ctx* ctx, int32_t enable);
int nrrs_get_cell_image(const nrrs_ctx* ctx, int32_t* enable);
/* Training mode of the tensor-core path: 1 (the default) = split: a level-major encoding kernel
 * writes the hash features of the batch, the StatNet kernel trains on them and writes each
 * sample's hash-lane gradients, and a level-major scatter kernel adds those into the table
 * gradient; 0 = fused: the StatNet kernel gathers and scatters itself. The two modes differ only
 * in the order of the FP32 gradient additions. */
int nrrs_set_train_split(nrrs_ctx* ctx, int32_t split);
int nrrs_get_train_split(const nrrs_ctx* ctx, int32_t* split);

/* ---- CUDA graph of the batched step: captures nrrs_step_batched on a private stream and
 *      instantiates it; each nrrs_graph_launch replays the whole multi-depth step (inference
 *      over all depths, then the decision and emission of all depths) with one launch. The
 *      buffers and segment table are those given at capture. ---- */
typedef struct nrrs_graph nrrs_graph;
int nrrs_graph_capture_batched(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                               const nrrs_segment* segs, int32_t n_segs,
                               const nrrs_decide_params* p, float* stats, float* rrs,
                               float* rrs_norm, uint8_t* split, uint32_t* next_queue,
                               uint32_t* next_size_dev, nrrs_graph** out);
int nrrs_graph_launch(nrrs_graph* g, void* stream);
void nrrs_graph_destroy(nrrs_graph* g);

/* ---- instrumentation: launch counters and optional CUDA-event timing per kernel kind.
 *      The reference's equivalent is KiRaRay's PROFILE("...") scopes (integrator.cpp:1069,
 *      1151, 1158, 1302, 1346, 2638). Timing records one event pair per launch on the launch
 *      stream while enabled; nrrs_profile_read synchronises on those events. ---- */
typedef enum {
    NRRS_KERNEL_INFER_FP32 = 0, NRRS_KERNEL_INFER_TC = 1, NRRS_KERNEL_SUM = 2,
    NRRS_KERNEL_DECIDE = 3, NRRS_KERNEL_PACK = 4, NRRS_KERNEL_TABLE_HALF = 5,
    NRRS_KERNEL_TRAIN_STAT = 6, NRRS_KERNEL_TRAIN_RRS = 7, NRRS_KERNEL_TRAIN_WGRAD = 8,
    NRRS_KERNEL_TRAIN_REDUCE = 9, NRRS_KERNEL_ADAM = 10, NRRS_KERNEL_ENCODE = 11,
    NRRS_KERNEL_TRAIN_SCATTER = 12, NRRS_KERNEL_TRAIN_ENCODE = 13, NRRS_KERNEL_INFER_RRS = 14,
    NRRS_KERNEL_CELL_IMAGE = 15, NRRS_KERNEL_KINDS = 16
} nrrs_kernel_kind;
uint64_t nrrs_launch_count(const nrrs_ctx* ctx);
/* grid (CTAs) of the last inference launch: SMs x resident CTAs per SM */
int32_t nrrs_last_infer_grid(const nrrs_ctx* ctx);
const char* nrrs_kernel_name(int32_t kind);
int nrrs_profile_enable(nrrs_ctx* ctx, int32_t enable);
int nrrs_profile_read(nrrs_ctx* ctx, int32_t kind, uint64_t* launches, double* total_ms);

/* ==== path records and training data =========================================================
 * The training side of the path tracer, beside the hot path: the per-node records of the
 * training paths, their radiance, and the training batch built from them. No context: the
 * records live in one caller-owned device block. Replaces, in the reference:
 *   NRRSPathNodesBuffer (reset, recordNode, recordRadiance, size)  src/render/nrrs/workqueue.h:108-188
 *   nrrs_generate_training_data                                    src/render/nrrs/train.cu:432-570
 *   nrrs_calculate_sample_weight                                   src/render/nrrs/train.cu:572-592
 *   their call sites in NRRSPathTracer       integrator.cpp:704, 730, 824-831, 1430-1438, 2572-2605
 * Deterministic where the reference depends on atomic order:
 *   - the nodes of one nrrs_record_nodes call are numbered in vertex order (reference: atomicAdd);
 *   - radiance is summed as exact fixed-point integers, three signed 64-bit limbs per channel
 *     with the lowest bit worth 2^-64 (a contribution keeps every bit at or above 2^-64), so the
 *     node totals do not depend on the order of contributions (reference: FP32 atomicAdd);
 *   - the training batch is in node order (reference: atomic push order);
 *   - of the children of one node, the one with the lowest node index keeps its RRSNet target
 *     (reference: the first to reach an atomic counter, train.cu:462-466).
 * The entry points of one node block run in stream order on one stream; none synchronises
 * except nrrs_path_nodes_status. */
typedef struct {
    uint32_t capacity;      /* nodes (nAlloc)                                                   */
    uint32_t max_record;    /* largest n of one nrrs_record_nodes call                          */
    float* pos;             /* [capacity][3] world position (intr.p)                            */
    float* wi;              /* [capacity][3] unit direction, as nrrs_vertex_soa.wi (the reference
                               stores intr.wo as lat-long, workqueue.h:159)                     */
    float* normal;          /* [capacity][3] the network's normal lanes (not in the reference's
                               record; 0 when the vertex SoA has none)                          */
    float* albedo;          /* [capacity][3] the network's albedo lanes (likewise)              */
    float* roughness;       /* [capacity]                                                       */
    float* thp;             /* [capacity][3] throughput given at record time                    */
    int32_t* parent;        /* [capacity] mLastNodeIdx; -1 = first node of its path             */
    uint32_t* pixel;        /* [capacity]                                                       */
    float* rrs;             /* [capacity]                                                       */
    uint32_t* depth;        /* [capacity]                                                       */
    int64_t* radiance;      /* [capacity][3 channels][3 limbs]: channel value =
                               (limb0 + limb1 * 2^32 + limb2 * 2^64) * 2^-64                    */
    uint32_t* first_child;  /* [capacity] lowest index among the node's children, or ~0u        */
    uint32_t* children;     /* [capacity] children recorded                                     */
    uint32_t* arrived;      /* [capacity] children whose radiance the radiance pass has added   */
    uint32_t* node_flags;   /* [capacity] bit 0: a non-finite contribution reached this node    */
    uint32_t* header;       /* device words: size, dropped, status, scan state                  */
    uint64_t* scan_states;  /* device scratch of the order-preserving scans                     */
} nrrs_path_nodes;

/* Bytes of the device block for capacity nodes and record calls of up to max_record vertices. */
uint64_t nrrs_path_nodes_bytes(uint32_t capacity, uint32_t max_record);
/* Carves the arrays of *out from dev_mem (256-byte aligned, at least nrrs_path_nodes_bytes) and
 * clears the header and scan scratch on the stream (NRRSPathNodesBuffer(n, alloc)). */
int nrrs_path_nodes_init(void* dev_mem, uint64_t bytes, uint32_t capacity, uint32_t max_record,
                         nrrs_path_nodes* out, void* stream);
/* NRRSPathNodesBuffer::reset (workqueue.h:113-120): no nodes, no dropped records. */
int nrrs_path_nodes_reset(const nrrs_path_nodes* nodes, void* stream);
/* Synchronises the stream; *size = nodes recorded, *dropped = records refused at capacity
 * (mInvalidNode), *flags = NRRS_DEV_* bits since the last read (then cleared). Any may be NULL. */
int nrrs_path_nodes_status(const nrrs_path_nodes* nodes, uint32_t* size, uint32_t* dropped,
                           uint32_t* flags, void* stream);

/* NRRSPathNodesBuffer::recordNode (workqueue.h:142-170) for a wavefront: every vertex i with
 * record[i] != 0 (record NULL = all) becomes a node whose fields come from v (pos, wi, thp;
 * normal, albedo, roughness, depth: NULL = 0), parent[i], pixel[i] and rrs[i] (NULL = 1, the work item's
 * default, device.cu:83). Nodes are numbered after the existing ones in vertex order.
 * node_out[i] receives the vertex's node index, or parent[i] when it records nothing or the
 * buffer is full (the reference's fallback, integrator.cpp:828-830, 1436-1438); node_out may be
 * parent (in place). n <= max_record. */
int nrrs_record_nodes(const nrrs_path_nodes* nodes, const nrrs_vertex_soa* v,
                      const int32_t* parent, const uint32_t* pixel, const float* rrs,
                      const uint8_t* record, uint32_t n, int32_t* node_out, void* stream);

/* NRRSPathNodesBuffer::recordRadiance (workqueue.h:122-136) for a queue of contributions:
 * contrib[i] ([n][3]) is added to node[i] and every ancestor. node[i] = -1 or >= size is skipped,
 * as in the reference. The ancestors receive it in nrrs_generate_training_data's radiance pass
 * (one pass over the nodes, each node's total added once into its parent) or, after that pass,
 * here directly; the totals are the same integers either way. A non-finite contribution is not
 * added: it marks its node and ancestors, whose samples are then dropped (the reference's NaN
 * filter, train.cu:514), and sets NRRS_DEV_NAN. */
int nrrs_record_radiance(const nrrs_path_nodes* nodes, const int32_t* node, const float* contrib,
                         uint32_t n, void* stream);

/* Switches of nrrs_generate_training_data (NRRSPathTracer members, integrator.h). */
typedef struct {
    int32_t ignore_zero_l;      /* mNRRSParams.mIgnoreZeroL: drop samples with mean(L) == 0      */
    int32_t copy_rrs_node;      /* mCopyTheRRSNode: training throughput = thp * rrs             */
    int32_t dedupe_rrs_target;  /* mIgnoreSameTrainingDataForRRSNet: later siblings get -1      */
    float thp_eps;              /* L_c = radiance_c / thp_c only where thp_c > thp_eps
                                   (KiRaRay's M_EPSILON)                                         */
    /* the error image (see nrrs_calculate_error); all zero / NULL when not used */
    uint32_t frame_width;       /* frame width in pixels; needed when error_image_scale > 1    */
    uint32_t error_image_scale; /* 0 or 1: image and error arrays are per frame pixel; s > 1:
                                   per s x s patch (offsetFrame2Scaled, myFilm.h:6-15)          */
    const float* error_per_pixel;   /* [2][n_pixels] of nrrs_calculate_error, or NULL          */
    const float* samples_per_patch; /* [patches] of nrrs_count_patch_samples, or NULL          */
} nrrs_train_data_params;

/* The training batch: the arrays of nrrs_vertex_soa and nrrs_train_step's target, plus the
 * reference's per-sample side arrays. All [capacity] device arrays; any may be NULL to skip. */
typedef struct {
    float* pos;             /* [cap][3] node position (NRRSNetworkInput0::mPos before the AABB map) */
    float* wi;              /* [cap][3]                                                         */
    float* normal;          /* [cap][3]                                                         */
    float* albedo;          /* [cap][3]                                                         */
    float* roughness;       /* [cap] (unwarped; the network warps it)                           */
    float* thp;             /* [cap][3] thpForTraining                                          */
    uint32_t* depth;        /* [cap]                                                            */
    float* ref_mean;        /* [cap] refMeanForTraining: mean of the image's RGB at the pixel    */
    float* target;          /* [cap][3] NRRSNetworkOutputTraining0::mL = max(radiance/thp, 0)    */
    float* rrs_target;      /* [cap] NRRSNetworkOutputTraining1::mRRS: node rrs, or -1           */
    uint32_t* pixel;        /* [cap] rayPixelID                                                 */
    float* error;           /* [cap] errorForTraining = error_per_pixel[patch]     (train.cu:537-543) */
    float* error_for_avg;   /* [cap] errorForAvgForTraining = error_per_pixel[n_pixels + patch] */
    float* number_samples;  /* [cap] numSamples = samples_per_patch[patch]                      */
} nrrs_train_batch;

/* nrrs_generate_training_data (train.cu:432-570): one sample per node with finite radiance,
 * finite position and direction and (ignore_zero_l) mean(L) > 0, in node order; at most
 * capacity (further samples are dropped and flag NRRS_DEV_OVERFLOW). First completes the
 * radiance of every node (see nrrs_record_radiance), once per reset. image (may be NULL) is
 * the rendered film, [patches][image_channels] float, channels 3 or 4, read at the sample's
 * patch (MyFilm::getPixel; with error_image_scale <= 1 a patch is a pixel); pixel_samples (may be
 * NULL) is [n_pixels] and gains one per sample that keeps its RRSNet target (mTrainingSamples,
 * which the caller zeroes per frame, integrator.cpp:1041). A pixel >= n_pixels flags
 * NRRS_DEV_BAD_INDEX and reads and counts nothing. *size_dev receives the sample count. */
int nrrs_generate_training_data(const nrrs_path_nodes* nodes, const nrrs_train_data_params* p,
                                const float* image, int32_t image_channels, uint32_t n_pixels,
                                uint32_t* pixel_samples, const nrrs_train_batch* out,
                                uint32_t capacity, uint32_t* size_dev, void* stream);

/* nrrs_calculate_sample_weight (train.cu:572-592): weight[t] = 1 / pixel_samples[pixel[t]]
 * (0 where that count is 0 or the pixel is >= n_pixels) for t < *size_dev; max_n bounds the
 * grid (the reference's host copy of the size). */
int nrrs_sample_weights(const uint32_t* pixel, const uint32_t* pixel_samples, uint32_t n_pixels,
                        const uint32_t* size_dev, uint32_t max_n, float* weight, void* stream);

/* ---- training on the batch built from the path records, with the reference's per-sample loss
 *      inputs. Replaces NRRSNetwork::train (network.cpp:196-295) with the loss hyper-parameters
 *      and side arrays the reference passes to its NRRS_LL2 / NRRS_RRS losses
 *      (network.cpp:423-435, 532-557): sample_weight (nrrs_sample_weights, train.cu:572-592),
 *      the batch's error, error_for_avg and number_samples (train.cu:537-543), the RRSNet target
 *      whose -1 marks a duplicate sibling to skip (train.cu:520-523), its thp and ref_mean, the
 *      error sum (nrrs_calculate_error), gamma1..4 and clamp_on / clamp_max. The loss arithmetic
 *      of the reference lives in its absent tiny-cuda-nn fork; this library's definition (also
 *      restated in the oracle) is, per sample i with s = sample_weight (1 when NULL):
 *        w_i = s_i, or 0 where rrs_target[i] < 0;  e_mean = *error_sum_dev / n_pixels (1 when NULL)
 *        e_i = error[i] / e_mean,  a_i = error_for_avg[i] / e_mean  (1 when NULL; each clamped to
 *              clamp_max when clamp_on);  u_i = gamma1 + gamma2 e_i + gamma3 a_i
 *        k_i = max(number_samples[i], 1) (1 when NULL)
 *        loss_S = sum s_i sum_c (y_ic - log(L_ic + stat_eps))^2 / (3 sum s)
 *        V = sum w u r^2 / (k q) / sum w,  C = sum w (cost_offset + q) / sum w,
 *        R = sum w (ln q)^2 / sum w,  loss_R = V C + gamma4 R
 *      with q and r as in nrrs_train_step. With every side array NULL and the default
 *      parameters (gamma 1, 0, 0, 0) it is nrrs_train_step's loss. n is a host value (the
 *      reference reads the batch size back too, integrator.cpp:2619-2625). ---- */
typedef struct {
    float gamma1, gamma2, gamma3, gamma4; /* NRRS_RRS gammas (2net-simple.json level1.loss)    */
    int32_t clamp_on;                     /* clamp the error ratios at clamp_max               */
    float clamp_max;
    uint32_t n_pixels;                    /* pixels (patches) of the error image              */
} nrrs_loss_params;
void nrrs_loss_params_default(nrrs_loss_params* p);
int nrrs_train_step_batch(nrrs_ctx* ctx, const nrrs_train_batch* batch, uint32_t n,
                          const float* sample_weight, const float* error_sum_dev,
                          const nrrs_loss_params* lp, double* loss_dev, void* stream);


/* ==== per-pixel error of the RRSNet loss =========================================================
 * The image-space inputs of the RRSNet loss, computed once per training frame (trainStep,
 * integrator.cpp:2358-2471): a blended estimate of each patch's radiance, its relative error
 * against the rendered image, and the sum of the errors. A patch is a scale x scale block of
 * frame pixels (error_image_scale; 1, a single pixel, in the shipped configuration). Where the
 * reference adds a patch's pixels with FP32 atomics, these kernels add them in pixel order, so
 * every result is deterministic; all arithmetic is FP32 without contraction. Replaces:
 *   the patch sample counts        integrator.cpp:1027-1050, 803-808
 *   weighted L, first frame + STEP#1.1   integrator.cpp:2358-2395
 *   nrrs_update_weighted_L         train.cu:344-363
 *   nrrs_calculate_error           train.cu:365-430
 *   the error sum (calcSum2PassAsync<false>)   integrator.cpp:2466-2471
 * The optional denoiser between these steps (OptiX, integrator.cpp:2412-2462) is not part of this
 * library: a caller that denoises runs it between nrrs_update_weighted_l and
 * nrrs_calculate_error on its own buffers. */
typedef struct {
    uint32_t frame_width, frame_height;  /* the frame; both divisible by scale               */
    uint32_t scale;                      /* error_image_scale (integrator.h:549); 0 means 1  */
    float blend_weight;                  /* blend_weight_for_error, 0.5 (integrator.h:527)   */
    int32_t clamp;                       /* clamp_pixel_error, on (network.cpp:519): <= 100  */
    int32_t multiply_samples;            /* pixel_error_multiply_samples, off (network.cpp:520):
                                            error_for_avg = error * sqrt(samples of the patch) */
} nrrs_pixel_error_params;

/* Exact sum of the errors: caller-owned device struct, zeroed once (cudaMemset); every call
 * leaves acc and done at zero again and writes value. */
typedef struct {
    int64_t acc[3];                      /* fixed-point limbs, lowest bit 2^-64              */
    uint32_t done;                       /* CTAs finished                                    */
    float value;                         /* the sum, rounded to nearest; NaN if any error is
                                            not finite                                        */
} nrrs_error_sum;

/* Adds 1 to samples_per_patch[patch of pixel[i]] for every i (camera rays, integrator.cpp:1050;
 * scattered rays, :803-808). samples_per_patch is zeroed by the caller per frame. */
int nrrs_count_patch_samples(const nrrs_pixel_error_params* p, const uint32_t* pixel, uint32_t n,
                             float* samples_per_patch, void* stream);

/* The frame's radiance per patch: pixel_l is [frame pixels][3] (mPixelState->mL, the sum of
 * this frame's spp samples). weighted_l_current[patch] = sum of the patch's pixel_l in pixel
 * order and weighted_l_current_acc[patch] = spp x pixels per patch (STEP#1.1, replacing the
 * per-frame reset of integrator.cpp:1027-1028 and its atomics); with first_frame,
 * weighted_l[patch] = sum of pixel_l / spp as well (integrator.cpp:2358-2375). */
int nrrs_accumulate_weighted_l(const nrrs_pixel_error_params* p, const float* pixel_l,
                               uint32_t spp_this_frame, int32_t first_frame, float* weighted_l,
                               float* weighted_l_current, uint32_t* weighted_l_current_acc,
                               void* stream);

/* nrrs_update_weighted_L (train.cu:344-363): weighted_l = weighted_l * (1 - blend) +
 * (weighted_l_current / acc) * blend, per patch and channel. */
int nrrs_update_weighted_l(const nrrs_pixel_error_params* p, const float* weighted_l_current,
                           const uint32_t* weighted_l_current_acc, float* weighted_l,
                           void* stream);

/* nrrs_calculate_error (train.cu:365-430) and the error sum (integrator.cpp:2466-2471).
 * ref is the rendered film per patch, [patches][ref_channels] (3 or 4). For each patch:
 * err = mean_c (L_c - ref_c)^2 / (ref_c^2 + 0.01), min(err, 100) when clamp;
 * error[patch] = err; error[frame pixels + patch] = err x sqrt(samples_per_patch[patch]) when
 * multiply_samples, else err. error is [2][frame pixels]; sum (may be NULL) receives the exact
 * sum of the second half over the patches. */
int nrrs_calculate_error(const nrrs_pixel_error_params* p, const float* ref, int32_t ref_channels,
                         const float* weighted_l, const float* samples_per_patch, float* error,
                         nrrs_error_sum* sum, void* stream);

/* UBS per-pixel error (nrrs_UBS_calc_error, train.cu:594-608) and its sum (integrator.cpp:
 * 2875-2886): error[pixel] = mean_c (L_c - ref_c)^2 / (ref_c^2 + 0.01) with L = pixel_l / spp
 * and ref the film read at the pixel's patch; sum (may be NULL) receives the exact sum. */
int nrrs_ubs_error(const nrrs_pixel_error_params* p, const float* pixel_l, uint32_t spp,
                   const float* ref, int32_t ref_channels, float* error, nrrs_error_sum* sum,
                   void* stream);

/* ==== per-depth strategy search (UBS) and the training schedule =================================
 * Host-side control of which factor source the path uses per depth, and when training moves
 * through steps 0-3. No GPU work; all calls are synchronous. Replaces, in NRRSPathTracer:
 *   UBS ("use best strategy")       integrator.h:324-439, integrator.cpp:2787-2891, 1088-1090, 1610,
 *                                   1780-1783; isInferMode integrator.h:67-71
 *   autoTrainControl                integrator.cpp:2659-2736 */
typedef enum {
    NRRS_UBS_FIXED_RR = 0,          /* no inference at this depth (the tracer's own RR)          */
    NRRS_UBS_ADRRS = 1,             /* ADRRS factors (step 2)                                     */
    NRRS_UBS_NRRS = 2,              /* RRSNet factors (step 3)                                    */
    NRRS_UBS_COUNT = 3
} nrrs_ubs_strategy;

typedef struct nrrs_ubs nrrs_ubs;
/* max_depth: strategies searched per depth 0..max_depth-1 (mMaxDepth, at most 19 so that every
 * strategy string fits in 32 bits). error_eval_seconds: the cost of computing the error, taken off
 * each frame's time (0.17e-3, integrator.cpp:2856-2858). */
int nrrs_ubs_create(int32_t max_depth, double error_eval_seconds, nrrs_ubs** out);
void nrrs_ubs_destroy(nrrs_ubs* u);
/* UBSResetAndBeginSearch (integrator.h:376-389) */
int nrrs_ubs_begin_search(nrrs_ubs* u);
/* At the start of a frame while searching: UBSNextState (integrator.cpp:2798-2820); when the
 * enumeration is over, UBSEndSearch (integrator.h:391-405) makes the best strategy current and
 * this returns 0; 1 while the search goes on. */
int nrrs_ubs_next_state(nrrs_ubs* u);
/* At the end of a frame while searching: UBSAnalyseFrame's bookkeeping (integrator.cpp:
 * 2822-2877). now_seconds is the caller's clock at this call; frame_error_sum the exact sum of
 * nrrs_ubs_error over the frame just rendered, used at the next call as the reference uses its
 * asynchronous copy; resolution the frame's pixels. */
int nrrs_ubs_analyse_frame(nrrs_ubs* u, double now_seconds, double frame_error_sum,
                           uint32_t resolution);
/* The strategy of a depth: while searching, digit `depth` of the search state; with a best (or
 * set) strategy in use, its entry; -1 when neither (no strategy chooses). Depths at or beyond
 * max_depth (up to 63) are NRRS_UBS_FIXED_RR, as the reference's zero-filled array gives. */
int nrrs_ubs_get_strategy(const nrrs_ubs* u, int32_t depth);
/* Whether depth runs inference (isInferMode) and with which factor source: *factor_source is
 * NRRS_FACTOR_ADRRS or NRRS_FACTOR_RRSNET (may be NULL); without search or a best strategy the
 * source is use_net_output_rrs ? RRSNET : ADRRS (mLossUseNetworkOutputRRS). */
int nrrs_ubs_need_infer(const nrrs_ubs* u, int32_t depth, int32_t enable_rrs, float clamp_min,
                        float clamp_max, int32_t max_rrs_depth, int32_t use_net_output_rrs,
                        int32_t* factor_source);
/* The best strategy per depth ([max_depth]) and its efficiency (resolution / (time x error)). */
int nrrs_ubs_best(const nrrs_ubs* u, int32_t* strategy, float* efficiency);
/* mUBSArrayChar (UBSUpdateAccordingArrayChar, integrator.h:364-374): one digit 0-2 per depth;
 * other characters become 0. Sets the best strategy and uses it (mUseBestStrategy). */
int nrrs_ubs_set_best(nrrs_ubs* u, const char* digits);
/* searching (1) or not (0) */
int nrrs_ubs_searching(const nrrs_ubs* u);

/* autoTrainControl (integrator.cpp:2659-2736): the steps by elapsed time. durations: seconds of
 * states 0-3 (mAutoTrainStateTime). Each tick returns the state to apply this frame. */
typedef struct {
    int32_t state;                  /* 0..4                                                       */
    int32_t step;                   /* nrrs_set_step value                                        */
    int32_t enable_rrs;             /* mEnableRRS                                                 */
    int32_t use_net_output_rrs;     /* mLossUseNetworkOutputRRS                                   */
    int32_t stop_training;          /* mStopTraining                                              */
    int32_t request_exit;           /* mAutoTrainRequestExit                                      */
    double seconds_per_frame;       /* measured over 100 frames after training (0 before)         */
} nrrs_train_schedule_state;
typedef struct nrrs_train_schedule nrrs_train_schedule;
int nrrs_train_schedule_create(const double durations[4], nrrs_train_schedule** out);
void nrrs_train_schedule_destroy(nrrs_train_schedule* s);
/* elapsed: seconds since the schedule started (the reference's clock() difference); now_seconds:
 * a wall clock for the 100-frame timing. */
int nrrs_train_schedule_tick(nrrs_train_schedule* s, double elapsed, double now_seconds,
                             nrrs_train_schedule_state* out);

/* ==== the wavefront steps either side of the path: trace and scatter ============================
 * A CUDA ray tracer around the NRRS step, in place of the reference's OptiX programs and its
 * scatter step:
 *   trace (closest hit, shadow any-hit)      src/render/nrrs/device.cu:48-161 (OptiX programs)
 *   handleEmissiveHit / handleMiss           src/render/nrrs/integrator.cpp:688-735
 *   handleIntersections, generateScatteredRays   src/render/nrrs/integrator.cpp:737-887
 *   generateCameraRays                       src/render/nrrs/integrator.cpp:889-935
 * Scenes are triangle meshes with diffuse (Lambertian) materials; emissive triangles are area
 * lights, sampled uniformly by light then by area, and misses see a constant environment. Next-
 * event estimation and BSDF sampling are combined with the power heuristic (the reference's
 * evalMIS, KiRaRay). The BVH is built on the host when the scene is created; traversal runs on
 * the GPU. Random numbers are a counter-based hash of (seed, depth, ray slot, dimension), so a
 * frame is deterministic. Radiance goes to an exact fixed-point film: [pixels][3 channels][3
 * limbs] int64, as the path nodes' radiance (lowest bit 2^-64), resolved once per frame. */
typedef struct nrrs_scene nrrs_scene;
/* vertices [n_vertices][3], triangles [n_triangles][3] vertex indices, tri_material
 * [n_triangles], materials [n_materials][6] = albedo rgb, emission rgb, environment [3] (may be
 * NULL = black). HOST arrays; the scene's device copy and BVH belong to the handle. */
int nrrs_scene_create(const float* vertices, uint32_t n_vertices, const uint32_t* triangles,
                      uint32_t n_triangles, const uint32_t* tri_material, const float* materials,
                      uint32_t n_materials, const float* environment, nrrs_scene** out);
void nrrs_scene_destroy(nrrs_scene* s);
/* mEnableNEE (integrator.h:139, on by default): 0 turns next-event estimation off. Scatter then
 * writes no shadow contribution, and an emitter hit by a BSDF ray counts in full (no MIS
 * weight). Takes effect for the launches that follow. */
int nrrs_scene_set_nee(nrrs_scene* s, int32_t enable);
/* BVH nodes, emissive triangles and the BVH depth */
int nrrs_scene_info(const nrrs_scene* s, uint32_t* n_nodes, uint32_t* n_lights,
                    uint32_t* max_depth);

/* A queue of rays, [capacity] device arrays. pdf: the BSDF pdf (solid angle) the ray was sampled
 * with, 0 for camera rays (no MIS weight on what they hit); thp 0 marks an unused slot. */
typedef struct {
    float* origin;          /* [cap][3]  */
    float* dir;             /* [cap][3] unit */
    float* thp;             /* [cap][3]  */
    float* pdf;             /* [cap]     */
    uint32_t* pixel;        /* [cap]     */
    int32_t* node;          /* [cap] path node of the vertex the ray leaves (-1 = none) */
} nrrs_ray_soa;

/* Closest hits: prim = triangle index of the scene's input order, ~0u for a miss. */
typedef struct {
    uint32_t* prim;
    float* t;
    float* u;               /* barycentrics of the hit */
    float* v;
} nrrs_hit_soa;

/* Shadow rays of next-event estimation: contrib is the radiance the pixel gains if the light is
 * visible (thp x f x Le x cos / pdf x MIS weight); tmax the distance to the light sample. */
typedef struct {
    float* origin;          /* [cap][3]  */
    float* dir;             /* [cap][3]  */
    float* tmax;            /* [cap]     */
    float* contrib;         /* [cap][3]; 0 = no shadow ray in this slot */
    uint32_t* pixel;        /* [cap]     */
    int32_t* node;          /* [cap]     */
} nrrs_shadow_soa;

/* The path vertices of one depth, compacted in ray order: the fields of nrrs_vertex_soa (pos, wi
 * = -ray direction, normal facing the ray, albedo, roughness 1, thp, depth) plus the pixel, the
 * path node and the pdf of the ray that found the vertex. [cap] device arrays. */
typedef struct {
    float* pos;
    float* wi;
    float* normal;
    float* albedo;
    float* roughness;
    float* thp;
    uint32_t* depth;
    uint32_t* pixel;
    int32_t* node;
} nrrs_path_vertices;

typedef struct {
    float pos[3], forward[3], up[3];
    float tan_half_fov_y;   /* tan of half the vertical field of view */
    uint32_t width, height;
} nrrs_camera;

/* generateCameraRays: one ray per pixel (width x height), jittered inside the pixel by the hash
 * of (seed, sample, pixel); thp 1, pdf 0, node -1. */
int nrrs_camera_rays(const nrrs_camera* c, uint32_t sample, uint32_t seed,
                     const nrrs_ray_soa* rays, void* stream);

/* Closest hits of the first *n_dev rays (max_n bounds the grid). Ties in t go to the lower
 * triangle index, so the result does not depend on the BVH. */
int nrrs_trace(const nrrs_scene* s, const nrrs_ray_soa* rays, const uint32_t* n_dev,
               uint32_t max_n, const nrrs_hit_soa* hits, void* stream);

/* nrrs_trace with the rays walked in a spatial order: a counting sort of the ray indices by
 * (direction octant, 12-bit Morton code of the origin in the scene's box) runs first, so that a
 * warp's rays start close together and head the same way. Same hits as nrrs_trace, bit for bit
 * (each written at its ray's own index). scratch: nrrs_trace_scratch_bytes(max_n) bytes of
 * device memory, 4-byte aligned, not shared with a concurrent call. Below 65,536 rays (max_n)
 * the sort is skipped. */
uint64_t nrrs_trace_scratch_bytes(uint32_t max_n);
int nrrs_trace_sorted(const nrrs_scene* s, const nrrs_ray_soa* rays, const uint32_t* n_dev,
                      uint32_t max_n, const nrrs_hit_soa* hits, void* scratch, void* stream);

/* handleEmissiveHit / handleMiss and the vertex queue: for each of the first *n_dev rays, an
 * emissive hit adds Le x thp (MIS-weighted against light sampling when pdf > 0) and a miss adds
 * environment x thp to film[pixel] and contrib[ray] ([max_n][3], 0 otherwise; the ray's node
 * receives it through nrrs_record_radiance). Rays that hit a surface become the vertices
 * out[0 .. *n_out_dev) in ray order. scratch: nrrs_shade_scratch_bytes(max_n) bytes of device
 * memory. */
uint64_t nrrs_shade_scratch_bytes(uint32_t max_n);
int nrrs_shade(const nrrs_scene* s, const nrrs_ray_soa* rays, const nrrs_hit_soa* hits,
               const uint32_t* n_dev, uint32_t max_n, uint32_t depth, int64_t* film,
               float* contrib, const nrrs_path_vertices* out, uint32_t* n_out_dev,
               void* scratch, void* stream);
/* nrrs_shade with the closest-hit program's specular branch (device.cu:88-95): hits on mirror
 * or glass materials (nrrs_scene_set_specular) go, in ray order, to out_specular[0 ..
 * *n_specular_dev) (roughness 0 for a mirror, -1 for glass) instead of the inference queue `out`, as the reference pushes specular hits to
 * its emitted queue directly and excludes them from the budget (the decision's n_specular).
 * Same scratch as nrrs_shade. */
int nrrs_shade_split(const nrrs_scene* s, const nrrs_ray_soa* rays, const nrrs_hit_soa* hits,
                     const uint32_t* n_dev, uint32_t max_n, uint32_t depth, int64_t* film,
                     float* contrib, const nrrs_path_vertices* out, uint32_t* n_out_dev,
                     const nrrs_path_vertices* out_specular, uint32_t* n_specular_dev,
                     void* scratch, void* stream);
/* Specular materials ([n_materials] HOST array, n_materials as at creation): specular[m] = 1
 * makes material m a perfect mirror, 2 a thin glass sheet (index 1.5, air on both sides); the
 * albedo tints either. 0 keeps it diffuse; other values are rejected. */
int nrrs_scene_set_specular(nrrs_scene* s, const uint8_t* specular, uint32_t n_materials);

/* handleIntersections (the RRS branch) + generateScatteredRays for the first *queue_size_dev
 * entries of the emitted queue (nrrs_step's next_queue, each vertex once per split): the vertex's
 * thp is divided by its normalised factor rrs_norm[vertex] (integrator.cpp:787-791), then one
 * shadow ray (next-event estimation) and one BSDF ray go to slot j of shadow and rays. */
int nrrs_scatter(const nrrs_scene* s, const nrrs_path_vertices* v, const float* rrs_norm,
                 const uint32_t* queue, const uint32_t* queue_size_dev, uint32_t max_queue,
                 uint32_t depth, uint32_t seed, const nrrs_ray_soa* rays,
                 const nrrs_shadow_soa* shadow, void* stream);

/* handleIntersections, the fixed Russian-roulette branch (integrator.cpp:744-769), for depths
 * that run no inference (the strategy search's fixed-RR depths): vertex j of the first *n_dev
 * survives when dimension 31 of its slot's random hash is below rr, its thp divided by rr, and
 * scatters into slot j of rays and shadow as nrrs_scatter does. A killed vertex leaves slot j
 * empty (thp 0, contrib 0), which the next trace and shade skip, so the next ray count is *n_dev.
 * rr in (0, 1]; rr = 1 (the reference's training frames) keeps every vertex. */
int nrrs_scatter_fixed_rr(const nrrs_scene* s, const nrrs_path_vertices* v, const uint32_t* n_dev,
                          uint32_t max_n, float rr, uint32_t depth, uint32_t seed,
                          const nrrs_ray_soa* rays, const nrrs_shadow_soa* shadow, void* stream);

/* generateScatteredRays for the specular vertices (the emitted queue's specular entries, rrs 1):
 * the bounce of the first *n_dev vertices of v into ray slots *ray_offset_dev + j (after the
 * nrrs_scatter rays: pass its queue size). A mirror reflects; thin glass reflects with the
 * sheet's reflectance 2F/(1+F) (F: one face's unpolarised Fresnel reflectance), chosen by the
 * slot's random hash of (seed, depth), and otherwise passes straight through. thp x albedo,
 * pdf 0 (the emitter the ray hits counts without an MIS weight), no light sampling
 * (integrator.cpp:833: NEE needs a smooth BSDF). Slots at or past max_rays are dropped.
 * *n_rays_out_dev (not ray_offset_dev) receives min(*ray_offset_dev + *n_dev, max_rays), the
 * next bounce's ray count. */
int nrrs_scatter_specular(const nrrs_scene* s, const nrrs_path_vertices* v, const uint32_t* n_dev,
                          uint32_t max_n, const uint32_t* ray_offset_dev, uint32_t max_rays,
                          uint32_t depth, uint32_t seed, const nrrs_ray_soa* rays,
                          uint32_t* n_rays_out_dev, void* stream);

/* The shadow rays of the first *n_dev slots: a visible light adds the slot's contrib to
 * film[pixel] and leaves it in contrib_out ([max_n][3]); an occluded one leaves 0. */
int nrrs_trace_shadow(const nrrs_scene* s, const nrrs_shadow_soa* shadow, const uint32_t* n_dev,
                      uint32_t max_n, int64_t* film, float* contrib_out, void* stream);

/* film [n_pixels][9] limbs -> image [n_pixels][3] = radiance x scale, rounded once */
int nrrs_film_resolve(const int64_t* film, uint32_t n_pixels, float scale, float* image,
                      void* stream);

/* ---- synthetic inputs (host, deterministic): mt19937_64 + explicit transforms. Buffers are
 *      HOST arrays sized as in nrrs_vertex_soa; any may be NULL to skip. target [n][3]. ---- */
void nrrs_synth_vertices(uint64_t seed, uint64_t first, uint64_t n, float* pos, float* wi,
                         float* normal, float* roughness, float* albedo, float* thp,
                         uint32_t* depth, float* rnd, float* ref_mean, float* target);

#ifdef __cplusplus
}
#endif
#endif /* NRRS_B200_H */
