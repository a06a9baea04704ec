// k_train_simt.cu -- one training step of StatNet and RRSNet (replaces NRRSNetwork::train,
// src/render/nrrs/net/network.cpp:196-295, and the two tcnn Trainer::training_step calls it makes:
// myNetworkLL2.cpp:51 for StatNet, network.cpp:274 for RRSNet).
//
// Losses (the reference's NRRS_LL2 / NRRS_RRS live in the absent tiny-cuda-nn fork; these are
// the workload's written definitions):
//   StatNet: loss_S = mean over samples and RGB of (y_c - log(L_c + stat_eps))^2
//   RRSNet:  q = activationSigma(raw), r = min(mean_c(thp_c L_c)/(ref + ref_eps), clamp),
//            V = mean(r^2 / q), C = mean(cost_offset + q), loss_R = V * C
//   RRSNet inputs come from the detached StatNet forward of the same step (the reference trains
//   the networks separately and builds RRSNet's input after StatNet's step, train.cu:155-240).
//
// Pipeline (all on the caller's stream, no host synchronisation):
//   k_train_stat  per sample: encode, StatNet forward, loss gradient, backward to the input,
//                 hash-grid scatter-add (FP32 atomics), glue; RRSNet forward for the batch sums
//                 V and C (FP64 per-CTA partials). Activations and deltas go to feature-major
//                 scratch for the weight gradients.
//   k_train_rrs   per sample: RRSNet forward and backward with the final V and C.
//   k_wgrad       dW = sum_i delta_i (x) a_i for every layer, split over sample chunks.
//   k_wreduce     chunk partials -> gradients, in fixed order (deterministic).
//   k_adam        Adam on FP32 master weights/moments; writes the FP16 table copy in the same pass.
#include "context.hpp"
#include "simt_gemm.cuh"

namespace nrrs {

namespace {

constexpr int kTT = 128;           // threads per CTA of the training kernels
constexpr int kChunk = 2048;       // samples per weight-gradient partial
constexpr int kMaxJobs = 8;

struct TrainArgs {
    VertexPtrs v;
    const float* target;
    uint32_t n;
    uint32_t ld;                   // row stride of the feature-major scratch
    EncodeParams enc;
    FactorParams fp;
    float loss_clamp, cost_offset;
    int32_t train_rrs;
    const float* table;
    float* table_grad;
    const float* wt_stat;          // transposed [in][out4] (forward)
    const float* wt_rrs;
    const float* w_stat;           // row-major master [out][in] (backward)
    const float* w_rrs;
    float* act;                    // feature-major scratch
    uint32_t r_x0, r_hs, r_dhs, r_dy, r_x1, r_hr, r_dhr, r_draw;
    double* part;                  // [grid][4]: loss_S sum, V sum, C sum, R sum
    uint32_t part_n;               // CTAs of k_train_stat
    double* loss_out;              // [2]
    LossWeights lw;                // per-sample loss weights (inactive: plain means)
};

__device__ __forceinline__ double block_sum_d(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < kTT / 32; ++k) t += red[k];
    return t;  // valid on thread 0
}

// relative contribution used by the RRS loss
__device__ __forceinline__ float rel_contrib(const TrainArgs& a, uint32_t i) {
    const size_t i3 = 3 * (size_t)i;
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) acc += a.v.thp[i3 + c] * a.target[i3 + c];
    const float ref = (a.v.ref ? a.v.ref[i] : 0.5f) + a.fp.ref_eps;
    const float r = acc / 3.0f / ref;
    return r < a.loss_clamp ? r : a.loss_clamp;
}

using simt::kLd;
using simt::kTM;

// activation tile rows and weight-chunk floats of the training kernels
template <int W>
struct TrShape {
    static constexpr int kRows = simt::imax(stat_in_of(W), W);
    static constexpr int kChunk = simt::kKC * simt::imax(stat_in_of(W), W);
    static constexpr size_t kSmem = sizeof(float) * ((size_t)kRows * kLd + 2 * kChunk);
};

// forward layer: ReLU (LeakyReLU for the reference network, W = 32) in place, and the activations
// to scratch rows row0 + n (samples i0 ..)
template <int W>
__device__ __forceinline__ void fwd_layer(const float* __restrict__ wt, int k_rows, int k_eff,
                                          float* tile, float* wch, int tid, float* scr,
                                          uint32_t ld, uint32_t i0, uint32_t row0, bool store) {
    simt::tile_gemm<W>(wt, k_rows, k_eff, tile, wch, tid, [&](int n, int m0, const float* v) {
        float r[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) r[i] = W == 32 ? leaky(v[i]) : fmaxf(v[i], 0.f);
        simt::tile_store8(tile, n, m0, r);
        if (store) {
            float* g = scr + (size_t)(row0 + n) * ld + i0 + m0;
            *reinterpret_cast<float4*>(g) = make_float4(r[0], r[1], r[2], r[3]);
            *reinterpret_cast<float4*>(g + 4) = make_float4(r[4], r[5], r[6], r[7]);
        }
    });
}

// backward layer through row-major W [k_rows = outputs of the forward layer][W = its inputs]:
// delta_in[n][m] = (sum_k W[k][n] delta_out[k][m]) times the activation's slope at the forward
// activation stored in scratch rows mask0 + n (ReLU: 1 or 0; LeakyReLU: 1 or 0.01); in place, and
// to scratch rows out0 + n
template <int W>
__device__ __forceinline__ void bwd_layer(const float* __restrict__ w, int k_rows, float* tile,
                                          float* wch, int tid, float* scr, uint32_t ld, uint32_t i0,
                                          uint32_t mask0, uint32_t out0) {
    simt::tile_gemm<W>(w, k_rows, k_rows, tile, wch, tid, [&](int n, int m0, const float* v) {
        const float* h = scr + (size_t)(mask0 + n) * ld + i0 + m0;
        const float4 h0 = *reinterpret_cast<const float4*>(h);
        const float4 h1 = *reinterpret_cast<const float4*>(h + 4);
        const float hv[8] = {h0.x, h0.y, h0.z, h0.w, h1.x, h1.y, h1.z, h1.w};
        float r[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) r[i] = hv[i] > 0.f ? v[i] : (W == 32 ? 0.01f * v[i] : 0.f);
        simt::tile_store8(tile, n, m0, r);
        float* g = scr + (size_t)(out0 + n) * ld + i0 + m0;
        *reinterpret_cast<float4*>(g) = make_float4(r[0], r[1], r[2], r[3]);
        *reinterpret_cast<float4*>(g + 4) = make_float4(r[4], r[5], r[6], r[7]);
    });
}

// y[o] = sum_k wt[k][o] tile[k][m] for a narrow output layer (wt [W][4])
template <int W, int OUT>
__device__ __forceinline__ void narrow_out(const float* __restrict__ wt, const float* tile, int m,
                                           float* y) {
    constexpr int OP = (OUT + 3) / 4 * 4;   // wt is [W][OUT rounded up to 4]
    float acc[OUT];
#pragma unroll
    for (int o = 0; o < OUT; ++o) acc[o] = 0.f;
#pragma unroll 4
    for (int k = 0; k < W; ++k) {
        const float x = tile[k * kLd + m];
#pragma unroll
        for (int q = 0; q < OP / 4; ++q) {
            const float4 w = __ldg(reinterpret_cast<const float4*>(wt + OP * k + 4 * q));
            const float wv[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
            for (int e = 0; e < 4; ++e)
                if (4 * q + e < OUT) acc[4 * q + e] = fmaf(wv[e], x, acc[4 * q + e]);
        }
    }
#pragma unroll
    for (int o = 0; o < OUT; ++o) y[o] = acc[o];
}

// The StatNet step and the RRSNet forward sums on 64-sample tiles (128 threads): encoding (two
// threads per sample), the forward layers as tile GEMMs storing every activation, the loss
// gradient, the backward layers as tile GEMMs through the row-major weights (masks from the
// stored activations), the input gradient of the 32 hash lanes, the hash-grid scatter (two
// threads per sample, eight levels each), then the glue and the RRSNet forward for the sums.
template <int WS, int HS, int WR, int HR>
__global__ void __launch_bounds__(simt::kThr) k_train_stat(const __grid_constant__ TrainArgs a) {
    static_assert(WS == WR, "one tile shape for both networks");
    constexpr bool REF = WS == 32;             // the reference's shipped network
    constexpr int SIN = stat_in_of(WS), SOUT = stat_out_of(WS);
    constexpr int NLH = REF ? kRefLevels / 2 : 8;   // hash levels per thread (two per sample)
    constexpr int X1 = REF ? kRefRrsLanes : 10;     // live RRSNet input lanes
    using S = TrShape<WS>;
    extern __shared__ float4 smem4[];
    float* tile = reinterpret_cast<float*>(smem4);
    float* wch = tile + S::kRows * kLd;
    __shared__ double red[kTT / 32];
    const int tid = threadIdx.x;
    const int m = tid & (kTM - 1);
    const bool lead = tid < kTM;
    const int half = tid >> 6;
    const uint32_t ld = a.ld;
    float* scr = a.act;
    double lossS = 0.0, sumV = 0.0, sumC = 0.0, sumR = 0.0;
    const float2* table = reinterpret_cast<const float2*>(a.table);
    // forward (transposed) and backward (row-major) layer images
    const float* ts = a.wt_stat;
    const float* ts_out = ts + (size_t)SIN * WS + (size_t)(HS - 1) * WS * WS;
    const float* rs = a.w_stat;
    const float* rs_out = rs + (size_t)SIN * WS + (size_t)(HS - 1) * WS * WS;   // [SOUT][WS]
    const float* tr = a.wt_rrs;
    const float* tr_out = tr + (size_t)kRrsIn * WR + (size_t)(HR - 1) * WR * WR;
    const uint32_t items = (a.n + kTM - 1) / kTM;
#pragma unroll 1
    for (uint32_t u = blockIdx.x; u < items; u += gridDim.x) {
        const uint32_t i0 = u * kTM, i = i0 + m;
        const bool valid = i < a.n;
        __syncthreads();   // the previous tile's column reads are over
        // ---- encode: lanes 0..55 of this sample's column (half 0: levels 0-7 + SH, 1: 8-15 +
        //      misc), copied to the x0 scratch rows ----
        float p[3] = {0.f, 0.f, 0.f};
        if (valid) {
            norm_pos(a.enc, a.v.pos, i, p);
#pragma unroll 2
            for (int l = half * NLH; l < half * NLH + NLH; ++l) {
                const LevelDev L = a.enc.lv[l];
                const CellCoord c = cell_of(p, L.res);
                float f0 = 0.f, f1 = 0.f;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const uint32_t row = grid_row(L, a.enc.hash_mask, c.ix + (k & 1),
                                                  c.iy + ((k >> 1) & 1), c.iz + ((k >> 2) & 1));
                    const float2 tv = __ldg(table + row);
                    const float w = corner_weight(c, k);
                    f0 += w * tv.x;
                    f1 += w * tv.y;
                }
                tile[(2 * l) * kLd + m] = f0;
                tile[(2 * l + 1) * kLd + m] = f1;
            }
            if (REF) {
                // the reference network: direction blobs (half 0) or roughness blob (half 1)
                float blob[16];
                ref_blob_lanes(a.v, i, blob);
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    tile[(16 + 8 * half + k) * kLd + m] = half ? blob[8 + k] : blob[k];
            } else if (half == 0) {
                float sh[16];
                const size_t i3 = 3 * (size_t)i;
                sh16(a.v.wi[i3], a.v.wi[i3 + 1], a.v.wi[i3 + 2], sh);
#pragma unroll
                for (int k = 0; k < 16; ++k) tile[(32 + k) * kLd + m] = sh[k];
            } else {
                float mm[16];
                misc_lanes(a.v, i, mm);
#pragma unroll
                for (int k = 0; k < 8; ++k) tile[(48 + k) * kLd + m] = mm[k];
            }
            const int hl = 2 * NLH;                              // hash lanes of this half
            for (int k = half * hl; k < half * hl + hl; ++k)
                scr[(size_t)(a.r_x0 + k) * ld + i] = tile[k * kLd + m];
            const int q0 = REF ? 16 + 8 * half : (half ? 48 : 32);
            const int q1 = REF ? q0 + 8 : (half ? 56 : 48);      // the other lanes of this half
            for (int k = q0; k < q1; ++k) scr[(size_t)(a.r_x0 + k) * ld + i] = tile[k * kLd + m];
        } else {
            constexpr int LANES = REF ? 32 : 56;
            for (int k = half * LANES / 2; k < (half + 1) * LANES / 2; ++k) tile[k * kLd + m] = 0.f;
        }

        // ---- StatNet forward, every hidden activation to scratch ----
        fwd_layer<WS>(ts, SIN, REF ? 32 : 56, tile, wch, tid, scr, ld, i0, a.r_hs, true);
#pragma unroll 1
        for (int h = 1; h < HS; ++h)
            fwd_layer<WS>(ts + (size_t)SIN * WS + (size_t)(h - 1) * WS * WS, WS, WS, tile, wch,
                          tid, scr, ld, i0, a.r_hs + h * WS, true);

        // ---- output, loss gradient, and the delta of the last hidden layer (own column) ----
        float y[SOUT];
#pragma unroll
        for (int k = 0; k < SOUT; ++k) y[k] = 0.f;
        SampleMul mu{1.f, 1.f, 1.f, 0.f};
        if (lead) {
            narrow_out<WS, SOUT>(ts_out, tile, m, y);
            float g[SOUT];
#pragma unroll
            for (int k = 0; k < SOUT; ++k) g[k] = 0.f;
            if (valid) {
                const size_t i3 = 3 * (size_t)i;
                mu = sample_mul(a.lw, i, a.n);
                if (REF) {
                    // relative squared error of L and L^2 against the target L and its square
#pragma unroll
                    for (int c = 0; c < 6; ++c) {
                        const float L = a.target[i3 + (c % 3)];
                        const float T = c < 3 ? L : L * L;
                        const float den = T * T + 0.01f;
                        const float d = y[c] - T;
                        lossS += (double)mu.stat * (double)d * (double)d / (double)den;
                        g[c] = mu.stat * (2.0f * d) / (den * 6.0f * (float)a.n);
                        scr[(size_t)(a.r_dy + c) * ld + i] = g[c];
                    }
                } else {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const float d = y[c] - logf(a.target[i3 + c] + a.fp.stat_eps);
                        if (a.lw.active) {
                            lossS += (double)mu.stat * (double)d * (double)d;
                            g[c] = mu.stat * (2.0f * d) / (3.0f * (float)a.n);
                        } else {
                            lossS += (double)d * (double)d;
                            g[c] = 2.0f * d / (3.0f * (float)a.n);
                        }
                        scr[(size_t)(a.r_dy + c) * ld + i] = g[c];
                    }
                }
            }
            // d h_last = W_out^T g times the activation's slope at h_last (this column)
            float* dl = scr + (size_t)(a.r_dhs + (HS - 1) * WS) * ld + i;
#pragma unroll 4
            for (int k = 0; k < WS; ++k) {
                float acc = 0.f;
#pragma unroll
                for (int o = 0; o < SOUT; ++o) acc = fmaf(rs_out[o * WS + k], g[o], acc);
                const float dk = tile[k * kLd + m] > 0.f ? acc : (REF ? 0.01f * acc : 0.f);
                tile[k * kLd + m] = dk;
                if (valid) dl[(size_t)k * ld] = dk;
            }
        }

        // ---- backward through the hidden layers, then the hash-lane gradients ----
#pragma unroll 1
        for (int h = HS - 1; h >= 1; --h)
            bwd_layer<WS>(rs + (size_t)SIN * WS + (size_t)(h - 1) * WS * WS, WS, tile, wch,
                          tid, scr, ld, i0, a.r_hs + (h - 1) * WS, a.r_dhs + (h - 1) * WS);
        simt::tile_gemm<SIN>(rs, WS, WS, tile, wch, tid, [&](int n, int m0, const float* v) {
            simt::tile_store8(tile, n, m0, v);
        });

        // ---- hash-grid scatter: two threads per sample, half the levels each ----
        {
            const unsigned lanes = valid_lanes(i0 + (uint32_t)(m & ~31), a.n);
            if (valid) {
#pragma unroll 2
                for (int l = half * NLH; l < half * NLH + NLH; ++l) {
                    const LevelDev L = a.enc.lv[l];
                    const CellCoord c = cell_of(p, L.res);
                    warp_scatter_level(a.table_grad, L, a.enc.hash_mask, c, tile[(2 * l) * kLd + m],
                                       tile[(2 * l + 1) * kLd + m], lanes);
                }
            }
        }
        __syncthreads();

        // ---- glue and the RRSNet forward for the batch sums ----
        if (a.train_rrs) {
            if (lead) {
                float x1[16];
                if (REF) glue16_ref_aux(y, load_aux(a.v, valid ? i : 0u), x1);
                else glue16(a.fp, y, a.v, valid ? i : 0u, x1);
#pragma unroll
                for (int k = 0; k < X1; ++k) {
                    tile[k * kLd + m] = valid ? x1[k] : 0.f;
                    if (valid) scr[(size_t)(a.r_x1 + k) * ld + i] = x1[k];
                }
            }
            fwd_layer<WR>(tr, kRrsIn, X1, tile, wch, tid, scr, ld, i0, 0, false);
#pragma unroll 1
            for (int h = 1; h < HR; ++h)
                fwd_layer<WR>(tr + (size_t)kRrsIn * WR + (size_t)(h - 1) * WR * WR, WR, WR, tile,
                              wch, tid, scr, ld, i0, 0, false);
            if (lead && valid) {
                float raw;
                narrow_out<WR, 1>(tr_out, tile, m, &raw);
                const float q = act_sigma(raw);
                const float r = rel_contrib(a, i);
                if (a.lw.active) {
                    const float lq = logf(q);
                    sumV += (double)(mu.var * (r * r / q));
                    sumC += (double)(mu.cost * (a.cost_offset + q));
                    sumR += (double)(mu.reg * (lq * lq));
                } else {
                    sumV += (double)(r * r / q);
                    sumC += (double)(a.cost_offset + q);
                }
            }
        }
    }
    const double s0 = block_sum_d(lossS, red);
    const double s1 = block_sum_d(sumV, red);
    const double s2 = block_sum_d(sumC, red);
    const double s3 = block_sum_d(sumR, red);
    if (threadIdx.x == 0) {
        a.part[4 * blockIdx.x + 0] = s0;
        a.part[4 * blockIdx.x + 1] = s1;
        a.part[4 * blockIdx.x + 2] = s2;
        a.part[4 * blockIdx.x + 3] = s3;
    }
}

// The RRSNet step on 64-sample tiles: the forward layers again (activations to scratch), the
// loss gradient with the batch's V and C, and the backward layers.
template <int WR, int HR>
__global__ void __launch_bounds__(simt::kThr) k_train_rrs(const __grid_constant__ TrainArgs a) {
    constexpr bool REF = WR == 32;             // the reference's shipped network
    constexpr int X1 = REF ? kRefRrsLanes : 10;
    using S = TrShape<WR>;
    extern __shared__ float4 smem4[];
    float* tile = reinterpret_cast<float*>(smem4);
    float* wch = tile + S::kRows * kLd;
    __shared__ double s_tot[4];
    const int tid = threadIdx.x;
    const int m = tid & (kTM - 1);
    const bool lead = tid < kTM;
    const uint32_t ld = a.ld;
    float* scr = a.act;
    if (tid < 4) {
        double t = 0.0;
        for (uint32_t b = 0; b < a.part_n; ++b) t += a.part[4 * b + tid];
        s_tot[tid] = t;
    }
    __syncthreads();
    const double Vm = s_tot[1] / (double)a.n, Cm = s_tot[2] / (double)a.n;
    if (blockIdx.x == 0 && tid == 0) {
        a.loss_out[0] = s_tot[0] / ((REF ? 6.0 : 3.0) * (double)a.n);
        a.loss_out[1] = a.train_rrs ? (a.lw.active ? Vm * Cm + s_tot[3] / (double)a.n : Vm * Cm)
                                    : 0.0;
    }
    if (!a.train_rrs) return;
    const float Vf = (float)Vm, Cf = (float)Cm;
    const float* tr = a.wt_rrs;
    const float* tr_out = tr + (size_t)kRrsIn * WR + (size_t)(HR - 1) * WR * WR;
    const float* rr = a.w_rrs;
    const float* rr_out = rr + (size_t)kRrsIn * WR + (size_t)(HR - 1) * WR * WR;   // [1][WR]
    const uint32_t items = (a.n + kTM - 1) / kTM;
#pragma unroll 1
    for (uint32_t u = blockIdx.x; u < items; u += gridDim.x) {
        const uint32_t i0 = u * kTM, i = i0 + m;
        const bool valid = i < a.n;
        __syncthreads();
        if (lead) {
#pragma unroll
            for (int k = 0; k < X1; ++k)
                tile[k * kLd + m] = valid ? scr[(size_t)(a.r_x1 + k) * ld + i] : 0.f;
        }
        fwd_layer<WR>(tr, kRrsIn, X1, tile, wch, tid, scr, ld, i0, a.r_hr, true);
#pragma unroll 1
        for (int h = 1; h < HR; ++h)
            fwd_layer<WR>(tr + (size_t)kRrsIn * WR + (size_t)(h - 1) * WR * WR, WR, WR, tile, wch,
                          tid, scr, ld, i0, a.r_hr + h * WR, true);
        if (lead) {
            float draw = 0.f;
            if (valid) {
                float raw;
                narrow_out<WR, 1>(tr_out, tile, m, &raw);
                const float q = act_sigma(raw);
                const float r = rel_contrib(a, i);
                float dq;
                if (a.lw.active) {
                    const SampleMul mu = sample_mul(a.lw, i, a.n);
                    dq = (mu.var * (-(r * r) / (q * q)) * Cf + mu.cost * Vf +
                          mu.reg * (2.0f * logf(q) / q)) / (float)a.n;
                } else {
                    dq = (-(r * r) / (q * q) * Cf + Vf) / (float)a.n;
                }
                draw = dq * act_sigma_grad(raw);
                scr[(size_t)a.r_draw * ld + i] = draw;
            }
            // d g_last = V_out^T draw, masked by g_last (this column of the tile)
            float* dl = scr + (size_t)(a.r_dhr + (HR - 1) * WR) * ld + i;
#pragma unroll 4
            for (int k = 0; k < WR; ++k) {
                const float dk = tile[k * kLd + m] > 0.f ? rr_out[k] * draw
                                                         : (REF ? 0.01f * (rr_out[k] * draw) : 0.f);
                tile[k * kLd + m] = dk;
                if (valid) dl[(size_t)k * ld] = dk;
            }
        }
#pragma unroll 1
        for (int h = HR - 1; h >= 1; --h)
            bwd_layer<WR>(rr + (size_t)kRrsIn * WR + (size_t)(h - 1) * WR * WR, WR, tile, wch, tid,
                          scr, ld, i0, a.r_hr + (h - 1) * WR, a.r_dhr + (h - 1) * WR);
    }
}

// ---- batch sums of the loss weights (one block, fixed order: deterministic) ----
// out[0] = sum s_i, out[1] = sum w_i, out[2] = the mean pixel error error_sum / n_pixels (1 when
// no error sum is given)
__global__ void __launch_bounds__(1024) k_loss_sums(const __grid_constant__ LossWeights w,
                                                   uint32_t n, const float* error_sum,
                                                   uint32_t n_pixels, double* out) {
    __shared__ double red[2][32];
    double s = 0.0, ww = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) {
        s += (double)loss_w_stat(w, i);
        ww += (double)loss_w_rrs(w, i);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        ww += __shfl_xor_sync(0xffffffffu, ww, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = s;
        red[1][threadIdx.x >> 5] = ww;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double ts = 0.0, tw = 0.0;
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) ts += red[0][k], tw += red[1][k];
        out[0] = ts;
        out[1] = tw;
        double em = 1.0;
        if (error_sum && n_pixels) {
            em = (double)*error_sum / (double)n_pixels;
            if (!(em > 1e-30)) em = 1e-30;
        }
        out[2] = em;
    }
}

}  // namespace

cudaError_t launch_loss_sums(const LossWeights& w, uint32_t n, const float* error_sum,
                             uint32_t n_pixels, double* out, cudaStream_t s) {
    k_loss_sums<<<1, 1024, 0, s>>>(w, n, error_sum, n_pixels, out);
    return cudaGetLastError();
}

namespace {

// ---- weight gradients: dW[o][k] = sum_i D[o][i] * A[k][i] over the batch ----
struct WJob {
    uint32_t d_row, a_row;   // first scratch row of the deltas / activations
    uint32_t M, N;           // outputs x inputs actually stored
    uint32_t ldw;            // input width of the layer (row stride of W, >= N)
    uint32_t out;            // offset of the layer in the MLP gradient vector
};

struct WGradArgs {
    const float* act;
    uint32_t ld, n, chunks;
    float* partial;          // [chunks][total]
    uint32_t total;          // MLP gradient length
    int32_t njobs;
    WJob job[kMaxJobs];
};

// one CTA: one job x one 64x64 output tile x one sample chunk
__global__ void __launch_bounds__(256) k_wgrad(const __grid_constant__ WGradArgs a) {
    __shared__ float sD[32][65];
    __shared__ float sA[32][65];
    const WJob& j = a.job[blockIdx.z];
    const uint32_t tiles_n = (j.N + 63) / 64;
    const uint32_t tm = blockIdx.y / tiles_n, tn = blockIdx.y % tiles_n;
    if (tm * 64 >= j.M || tn * 64 >= j.N) return;
    const uint32_t m0 = tm * 64, n0 = tn * 64;
    const uint32_t i0 = blockIdx.x * kChunk;
    const uint32_t i1 = min(a.n, i0 + kChunk);
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    float acc[4][4] = {};
    for (uint32_t ib = i0; ib < i1; ib += 32) {
        // stage 32 samples of 64 delta rows and 64 activation rows (samples contiguous)
        for (int e = threadIdx.x; e < 32 * 64; e += 256) {
            const int r = e / 32, s = e % 32;
            const uint32_t i = ib + s;
            const bool ok_i = i < i1;
            sD[s][r] = (ok_i && m0 + r < j.M) ? a.act[(size_t)(j.d_row + m0 + r) * a.ld + i] : 0.f;
            sA[s][r] = (ok_i && n0 + r < j.N) ? a.act[(size_t)(j.a_row + n0 + r) * a.ld + i] : 0.f;
        }
        __syncthreads();
#pragma unroll 8
        for (int s = 0; s < 32; ++s) {
            float d[4], x[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) d[u] = sD[s][ty * 4 + u];
#pragma unroll
            for (int u = 0; u < 4; ++u) x[u] = sA[s][tx * 4 + u];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int w = 0; w < 4; ++w) acc[u][w] = fmaf(d[u], x[w], acc[u][w]);
        }
        __syncthreads();
    }
    float* out = a.partial + (size_t)blockIdx.x * a.total + j.out;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const uint32_t m = m0 + ty * 4 + u;
        if (m >= j.M) continue;
#pragma unroll
        for (int w = 0; w < 4; ++w) {
            const uint32_t k = n0 + tx * 4 + w;
            if (k < j.N) out[(size_t)m * j.ldw + k] = acc[u][w];
        }
    }
}

// gradients = sum of the chunk partials in chunk order; entries no job writes (zero input
// lanes) are zero in every partial, set once at creation
__global__ void k_wreduce(const float* partial, uint32_t chunks, uint32_t total, float* grad,
                          float scale) {
    for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (uint32_t c = 0; c < chunks; ++c) s += partial[(size_t)c * total + e];
        grad[e] = s * scale;
    }
}

struct AdamArgs {
    float* p;
    const float* g;
    float gscale;
    float* m;
    float* v;
    __half* table_h;       // FP16 copy of [0, n_table) refreshed in the same pass (may be null)
    uint64_t n_table;
    uint64_t first, count;
    uint64_t rrs_first;    // parameters from here on (the RRSNet) use lr_rrs
    float lr, lr_rrs, b1, b2, eps, l2, inv_c1, inv_c2;
};

// Adam on one parameter. The bias corrections are multiplications by 1/c1 and 1/c2 computed on
// the host, and the step is one fast division: IEEE divisions made this streaming kernel
// instruction-bound (69 % issue-active at 50 % of HBM bandwidth).
__device__ __forceinline__ float adam_one(const AdamArgs& a, uint64_t k, float w, float g0,
                                          float& m, float& v) {
    const float g = g0 * a.gscale + a.l2 * w;
    m = a.b1 * m + (1.0f - a.b1) * g;
    v = a.b2 * v + (1.0f - a.b2) * g * g;
    const float lr = k < a.rrs_first ? a.lr : a.lr_rrs;
    return w - __fdividef(lr * (m * a.inv_c1), sqrtf(v * a.inv_c2) + a.eps);
}

// HBM-bound (30 B per parameter): four parameters per thread with 16-byte loads and stores of
// the weights, gradients and both moments; the FP16 copy of the table is written in the same
// pass. first is a multiple of 4 and the arrays are 16-byte aligned; a scalar tail finishes.
__global__ void k_adam(const __grid_constant__ AdamArgs a) {
    const uint64_t quads = a.count / 4;
    for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q < quads;
         q += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = a.first + 4 * q;
        const float4 w = *reinterpret_cast<const float4*>(a.p + k);
        const float4 g = *reinterpret_cast<const float4*>(a.g + k);
        float4 m = *reinterpret_cast<const float4*>(a.m + k);
        float4 v = *reinterpret_cast<const float4*>(a.v + k);
        float4 nw;
        nw.x = adam_one(a, k, w.x, g.x, m.x, v.x);
        nw.y = adam_one(a, k + 1, w.y, g.y, m.y, v.y);
        nw.z = adam_one(a, k + 2, w.z, g.z, m.z, v.z);
        nw.w = adam_one(a, k + 3, w.w, g.w, m.w, v.w);
        *reinterpret_cast<float4*>(a.m + k) = m;
        *reinterpret_cast<float4*>(a.v + k) = v;
        *reinterpret_cast<float4*>(a.p + k) = nw;
        if (a.table_h && k + 4 <= a.n_table) {
            __half2 h0 = __floats2half2_rn(nw.x, nw.y), h1 = __floats2half2_rn(nw.z, nw.w);
            uint2 u;
            u.x = *reinterpret_cast<uint32_t*>(&h0);
            u.y = *reinterpret_cast<uint32_t*>(&h1);
            *reinterpret_cast<uint2*>(a.table_h + k) = u;
        } else if (a.table_h) {
            const float nv[4] = {nw.x, nw.y, nw.z, nw.w};
            for (int j = 0; j < 4; ++j)
                if (k + j < a.n_table) a.table_h[k + j] = __float2half_rn(nv[j]);
        }
    }
    for (uint64_t k = a.first + 4 * quads + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
         k < a.first + a.count; k += (uint64_t)gridDim.x * blockDim.x) {
        float m = a.m[k], v = a.v[k];
        const float nw = adam_one(a, k, a.p[k], a.g[k], m, v);
        a.m[k] = m;
        a.v[k] = v;
        a.p[k] = nw;
        if (a.table_h && k < a.n_table) a.table_h[k] = __float2half_rn(nw);
    }
}

struct EmaArgs {
    const float* p;
    float* e;
    float* pi;             // the debiased average
    __half* table_h;       // FP16 copy of pi over [0, n_table) (may be null)
    uint64_t n_table, count;
    float d, omd, inv;     // decay, 1 - decay, 1 / (1 - decay^t)
};

// the moving average after an Adam step: e = d e + (1 - d) w, pi = e / (1 - d^t), each product
// and the sum rounded separately (no contraction), so a float32 restatement gives the same bits
__global__ void k_ema(const __grid_constant__ EmaArgs a) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < a.count;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const float e = __fadd_rn(__fmul_rn(a.d, a.e[k]), __fmul_rn(a.omd, a.p[k]));
        const float pi = __fmul_rn(e, a.inv);
        a.e[k] = e;
        a.pi[k] = pi;
        if (a.table_h && k < a.n_table) a.table_h[k] = __float2half_rn(pi);
    }
}

template <int WS, int HS, int WR, int HR>
cudaError_t launch_train(nrrs_ctx* ctx, TrainArgs& a, cudaStream_t s) {
    const size_t smem = TrShape<WS>::kSmem;
    auto ks = k_train_stat<WS, HS, WR, HR>;
    auto kr = k_train_rrs<WR, HR>;
    cudaError_t e = cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const uint32_t tiles = (a.n + kTM - 1) / kTM;
    uint32_t grid = (uint32_t)(ctx->sm_count * resident_ctas((const void*)ks, simt::kThr, smem, 16));
    if (grid > tiles) grid = tiles;
    a.part_n = grid;
    {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_STAT, s);
        ks<<<grid, simt::kThr, smem, s>>>(a);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_RRS, s);
        kr<<<grid, simt::kThr, smem, s>>>(a);
    }
    return cudaGetLastError();
}

struct Layout {
    uint32_t r_x0, r_hs, r_dhs, r_dy, r_x1, r_hr, r_dhr, r_draw, rows;
};

Layout layout_of(const nrrs_config& c) {
    Layout L{};
    uint32_t r = 0;
    const bool ref = c.network == NRRS_NET_REFERENCE;
    L.r_x0 = r; r += ref ? kRefStatIn : 56;
    L.r_hs = r; r += c.statnet_hidden * c.statnet_width;
    L.r_dhs = r; r += c.statnet_hidden * c.statnet_width;
    L.r_dy = r; r += ref ? 8 : 4;
    L.r_x1 = r; r += 16;
    L.r_hr = r; r += c.rrsnet_hidden * c.rrsnet_width;
    L.r_dhr = r; r += c.rrsnet_hidden * c.rrsnet_width;
    L.r_draw = r; r += 4;
    L.rows = r;
    return L;
}

uint32_t ld_of(uint32_t n) { return (n + 127) / 128 * 128; }

}  // namespace

cudaError_t launch_wreduce(const float* partial, uint32_t chunks, uint32_t total, float* grad,
                           float scale, cudaStream_t s) {
    k_wreduce<<<(total + 255) / 256, 256, 0, s>>>(partial, chunks, total, grad, scale);
    return cudaGetLastError();
}

// Adam over the trained parameters: table + StatNet (+ RRSNet at step 3); refreshes the FP16 table
cudaError_t launch_adam_step(nrrs_ctx* ctx, bool train_rrs, cudaStream_t s, float scale) {
    const nrrs_config& c = ctx->cfg;
    ctx->adam_t += 1;
    AdamArgs ad{};
    ad.p = ctx->params;
    ad.g = ctx->grads;
    ad.gscale = scale;
    ad.m = ctx->adam_m;
    ad.v = ctx->adam_v;
    ad.table_h = ctx->table_h;
    ad.n_table = ctx->n_table;
    ad.first = 0;
    ad.count = ctx->n_table + ctx->n_stat + (train_rrs ? ctx->n_rrs : 0);
    ad.lr = c.lr;
    ad.rrs_first = ctx->n_table + ctx->n_stat;
    ad.lr_rrs = c.lr_rrsnet > 0.f ? c.lr_rrsnet : c.lr;
    ad.b1 = c.beta1;
    ad.b2 = c.beta2;
    ad.eps = c.eps;
    ad.l2 = c.l2_reg;
    ad.inv_c1 = 1.0f / (1.0f - powf(c.beta1, (float)ctx->adam_t));
    ad.inv_c2 = 1.0f / (1.0f - powf(c.beta2, (float)ctx->adam_t));
    {
        ProfScope ps(ctx, NRRS_KERNEL_ADAM, s);
        k_adam<<<(unsigned)ctx->sm_count * 8, 256, 0, s>>>(ad);
    }
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && ctx->cells) {
        ProfScope ps(ctx, NRRS_KERNEL_CELL_IMAGE, s);
        e = launch_cell_image(ctx->table_h, ctx->enc, ctx->cells, ctx->n_cells, ctx->sm_count, s);
    }
    if (e != cudaSuccess || !ctx->ema) return e;
    // the moving average of every parameter and the inference table derived from it
    ctx->ema_t += 1;
    EmaArgs ea{};
    ea.p = ctx->params;
    ea.e = ctx->ema;
    ea.pi = ctx->params_inf;
    ea.table_h = ctx->table_h_inf;
    ea.n_table = ctx->n_table;
    ea.count = ctx->n_params;
    ea.d = c.ema_decay;
    ea.omd = 1.0f - c.ema_decay;
    ea.inv = (float)(1.0 / (1.0 - std::pow((double)c.ema_decay, (double)ctx->ema_t)));
    {
        ProfScope ps(ctx, NRRS_KERNEL_ADAM, s);
        k_ema<<<(unsigned)ctx->sm_count * 8, 256, 0, s>>>(ea);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess || !ctx->cells_inf) return e;
    ProfScope ps(ctx, NRRS_KERNEL_CELL_IMAGE, s);
    return launch_cell_image(ctx->table_h_inf, ctx->enc, ctx->cells_inf, ctx->n_cells,
                             ctx->sm_count, s);
}

bool train_tc_supported(const nrrs_config& c);
size_t train_tc_scratch_bytes(const nrrs_config& c, uint32_t n, int sm_count);
int train_step_tc(nrrs_ctx* ctx, const VertexPtrs& v, const float* target, uint32_t n,
                  double* loss_dev, cudaStream_t s, bool apply, const LossWeights* lw);

size_t train_scratch_bytes(const nrrs_config& c, uint32_t n, int sm_count) {
    if (train_tc_supported(c)) return train_tc_scratch_bytes(c, n, sm_count);
    const Layout L = layout_of(c);
    const uint64_t mlp = (uint64_t)64 * c.statnet_width + (uint64_t)(c.statnet_hidden - 1) *
                         c.statnet_width * c.statnet_width + 3ull * c.statnet_width +
                         16ull * c.rrsnet_width + (uint64_t)(c.rrsnet_hidden - 1) * c.rrsnet_width *
                         c.rrsnet_width + (uint64_t)c.rrsnet_width;
    const uint64_t chunks = (n + kChunk - 1) / kChunk;
    return sizeof(float) * (uint64_t)L.rows * ld_of(n) + sizeof(double) * 4 * (uint64_t)sm_count * 16 +
           sizeof(float) * chunks * mlp + 1024;
}

int train_step_impl(nrrs_ctx* ctx, const VertexPtrs& v, const float* target, uint32_t n,
                    double* loss_dev, cudaStream_t s, bool apply, const LossWeights* lw) {
    if (train_tc_supported(ctx->cfg))
        return train_step_tc(ctx, v, target, n, loss_dev, s, apply, lw);
    const nrrs_config& c = ctx->cfg;
    const Layout L = layout_of(c);
    const uint32_t ld = ld_of(c.max_train);
    const uint64_t chunks = (n + kChunk - 1) / kChunk;
    const uint64_t mlp = ctx->n_stat + ctx->n_rrs;
    uint8_t* base = reinterpret_cast<uint8_t*>(ctx->train_scratch);
    float* act = reinterpret_cast<float*>(base);
    double* part = reinterpret_cast<double*>(base + sizeof(float) * (size_t)L.rows * ld);
    float* partial = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(part) +
                                              sizeof(double) * 4 * (size_t)ctx->sm_count * 16);
    const bool train_rrs = c.step >= 3;
    cudaError_t e;

    // gradients of this step only
    e = cudaMemsetAsync(ctx->grads, 0, sizeof(float) * ctx->n_params, s);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(partial, 0, sizeof(float) * chunks * mlp, s);
    if (e != cudaSuccess) {
        ctx->last_error = std::string("train memset: ") + cudaGetErrorString(e);
        return NRRS_ERR_CUDA;
    }

    TrainArgs a{};
    a.v = v;
    a.target = target;
    a.n = n;
    a.ld = ld;
    a.enc = ctx->enc;
    a.fp.stat_eps = c.stat_eps;
    a.fp.ref_eps = c.ref_eps;
    a.loss_clamp = c.loss_clamp_max;
    a.cost_offset = c.cost_offset;
    a.train_rrs = train_rrs;
    a.table = ctx->params;
    a.table_grad = ctx->grads;
    a.wt_stat = ctx->wt;
    a.wt_rrs = ctx->wt + ctx->wt_rrs_offset;
    a.w_stat = ctx->wrow;
    a.w_rrs = ctx->wrow + ctx->n_stat;
    a.act = act;
    a.r_x0 = L.r_x0; a.r_hs = L.r_hs; a.r_dhs = L.r_dhs; a.r_dy = L.r_dy;
    a.r_x1 = L.r_x1; a.r_hr = L.r_hr; a.r_dhr = L.r_dhr; a.r_draw = L.r_draw;
    a.part = part;
    a.loss_out = loss_dev ? loss_dev : ctx->loss_dev;
    if (lw) a.lw = *lw;

    if (c.statnet_width == 64 && c.statnet_hidden == 2)
        e = launch_train<64, 2, 64, 2>(ctx, a, s);
    else if (c.statnet_width == 64 && c.statnet_hidden == 3)
        e = launch_train<64, 3, 64, 3>(ctx, a, s);
    else if (c.statnet_width == 32)   // the reference network
        e = launch_train<32, 3, 32, 3>(ctx, a, s);
    else
        e = launch_train<128, 3, 128, 3>(ctx, a, s);
    if (e != cudaSuccess) {
        ctx->last_error = std::string("train launch: ") + cudaGetErrorString(e);
        return NRRS_ERR_CUDA;
    }

    // weight-gradient jobs: (delta rows, activation rows, M, N, layer input width, offset)
    WGradArgs w{};
    w.act = act;
    w.ld = ld;
    w.n = n;
    w.chunks = (uint32_t)chunks;
    w.partial = partial;
    w.total = (uint32_t)mlp;
    int nj = 0;
    uint32_t off = 0;
    const uint32_t WS = c.statnet_width, HS = c.statnet_hidden;
    const uint32_t WR = c.rrsnet_width, HR = c.rrsnet_hidden;
    const bool ref = c.network == NRRS_NET_REFERENCE;
    const uint32_t sin = stat_in_of((int)WS), sout = stat_out_of((int)WS);
    w.job[nj++] = WJob{L.r_dhs, L.r_x0, WS, ref ? (uint32_t)kRefStatIn : 56u, sin, off};
    off += WS * sin;
    for (uint32_t h = 1; h < HS; ++h) {
        w.job[nj++] = WJob{L.r_dhs + h * WS, L.r_hs + (h - 1) * WS, WS, WS, WS, off};
        off += WS * WS;
    }
    w.job[nj++] = WJob{L.r_dy, L.r_hs + (HS - 1) * WS, sout, WS, WS, off};
    off += sout * WS;
    if (train_rrs) {
        w.job[nj++] = WJob{L.r_dhr, L.r_x1, WR, ref ? (uint32_t)kRefRrsLanes : 10u, kRrsIn, off};
        off += WR * kRrsIn;
        for (uint32_t h = 1; h < HR; ++h) {
            w.job[nj++] = WJob{L.r_dhr + h * WR, L.r_hr + (h - 1) * WR, WR, WR, WR, off};
            off += WR * WR;
        }
        w.job[nj++] = WJob{L.r_draw, L.r_hr + (HR - 1) * WR, 1, WR, WR, off};
    }
    w.njobs = nj;
    const uint32_t tiles_y = ((128 + 63) / 64) * ((128 + 63) / 64);
    {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_WGRAD, s);
        k_wgrad<<<dim3((unsigned)chunks, tiles_y, (unsigned)nj), 256, 0, s>>>(w);
    }
    {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_REDUCE, s);
        e = launch_wreduce(partial, (uint32_t)chunks, (uint32_t)mlp, ctx->grads + ctx->n_table, 1.0f, s);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) {
        ctx->last_error = std::string("wgrad launch: ") + cudaGetErrorString(e);
        return NRRS_ERR_CUDA;
    }

    if (!apply) return NRRS_OK;
    e = launch_adam_step(ctx, train_rrs, s);
    if (e != cudaSuccess) {
        ctx->last_error = std::string("adam launch: ") + cudaGetErrorString(e);
        return NRRS_ERR_CUDA;
    }
    return NRRS_OK;
}

}  // namespace nrrs
