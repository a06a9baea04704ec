// k_infer_simt.cu -- plain FP32 inference: hash grid + SH encoding, StatNet, glue, RRSNet,
// activation, clamp and the exact normalisation sum, on the FP32 SIMT pipes.
//
// This is the "plain FP32 per-depth path" the mixed-precision tcgen05 path is measured
// against. It fuses what the reference runs as nrrs_generate_inference_data (train.cu:269-287),
// tcnn inference_mixed_precision x2 (myNetworkLL2.cpp:206, network.cpp:346),
// nrrs_generate_inference_data_from_0to1 (train.cu:41-112) and the "Gen RRS Number" lambda
// (integrator.cpp:1184-1298), so the AoS round trips of the reference disappear.
//
// A CTA of 128 threads works on 64 vertices at a time (half of a 128-vertex tile of the segment
// table). Their activations live in one shared-memory tile, K-major ([k][64 vertices + 4 pad]).
// Every hidden layer is a register-tiled FP32 GEMM: each thread owns an 8 x (W/16) block of outputs
// (8 vertices x 8 or 4 neurons), and per k it reads 8 activations and 8 (or 4) weights as
// float4 and issues 64 (or 32) FMAs. The layer's transposed weights ([in][out]) come from L2 in
// 32-row chunks, double-buffered with cp.async while the previous chunk is consumed. Every output
// is accumulated as fmaf(w_k, x_k, acc) over k ascending, the same sequence for any launch shape.
// The narrow layers (3 and 1 outputs), the glue, the factor and the exact-sum term run one thread
// per vertex on that vertex's column of the tile.
#include "simt_gemm.cuh"

namespace nrrs {

namespace {

using simt::kLd;
using simt::kThr;
using simt::kTM;

template <int W>
struct FpShape {
    static constexpr int kRows = simt::imax(stat_in_of(W), W);     // rows of the activation tile
    static constexpr int kActFloats = kRows * kLd;
    static constexpr int kChunkFloats = simt::kKC * W;
    static constexpr size_t kSmem = sizeof(float) * (kActFloats + 2 * kChunkFloats);
};

// out[n][m] = act(sum_k wt[k][n] act[k][m]) for k < k_eff, in place on the activation tile, with
// ReLU (the workload's network) or LeakyReLU (the reference network, W = 32); wt is [k_rows][W]
// in global memory; rows k_eff .. k_rows-1 are loaded but multiply zeros.
template <int W>
__device__ __forceinline__ void hidden_layer(const float* __restrict__ wt, int k_rows, int k_eff,
                                             float* act, float* wch, int tid) {
    simt::tile_gemm<W>(wt, k_rows, k_eff, act, wch, tid, [&](int n, int m0, const float* v) {
        float r[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) r[i] = W == 32 ? leaky(v[i]) : fmaxf(v[i], 0.f);
        simt::tile_store8(act, n, m0, r);
    });
}

// the network's narrow output layer for vertex column m: y[o] = sum_k wt[k][o] act[k][m], with
// wt [W][OUT rounded up to 4]
template <int W, int OUT>
__device__ __forceinline__ void output_layer(const float* __restrict__ wt, const float* act, int m,
                                             float* y) {
    constexpr int OP = (OUT + 3) / 4 * 4;
    float acc[OUT];
#pragma unroll
    for (int o = 0; o < OUT; ++o) acc[o] = 0.f;
#pragma unroll 4
    for (int k = 0; k < W; ++k) {
        const float x = act[k * kLd + m];
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

// hash-grid levels l0 .. l0+NL-1 of vertex i into its column of the tile (FP32 table)
template <int NL = 8>
__device__ __forceinline__ void encode_levels8(const InferArgs& a, const float* p, int l0, float* act,
                                               int m) {
    const float2* table = reinterpret_cast<const float2*>(a.table);
#pragma unroll 2
    for (int l = l0; l < l0 + NL; ++l) {
        const LevelDev L = a.enc.lv[l];
        const CellCoord c = cell_of(p, L.res);
        uint32_t rows[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            rows[k] = grid_row(L, a.enc.hash_mask, c.ix + (k & 1), c.iy + ((k >> 1) & 1),
                               c.iz + ((k >> 2) & 1));
        float2 t[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) t[k] = __ldg(table + rows[k]);
        float f0 = 0.f, f1 = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float w = corner_weight(c, k);
            f0 += w * t[k].x;
            f1 += w * t[k].y;
        }
        act[(2 * l) * kLd + m] = f0;
        act[(2 * l + 1) * kLd + m] = f1;
    }
}

template <int WS, int HS, int WR, int HR>
__global__ void __launch_bounds__(kThr) k_infer_fp32(const __grid_constant__ InferArgs a) {
    static_assert(WS == WR, "one tile shape for both networks");
    constexpr bool REF = WS == 32;             // the reference's shipped network
    constexpr int SIN = stat_in_of(WS), SOUT = stat_out_of(WS);
    using S = FpShape<WS>;
    extern __shared__ float4 smem4[];
    float* act = reinterpret_cast<float*>(smem4);
    float* wch = act + S::kActFloats;
    const int tid = threadIdx.x;
    const int m = tid & (kTM - 1);
    const bool lead = tid < kTM;               // the thread that owns vertex column m
    const SegmentTable& ST = seg_table(a.segs);
    const uint32_t items = 2u * ST.total_tiles;
    // transposed layer images: [in][out] (outputs padded to 4), StatNet then RRSNet
    const float* s0 = a.wt_stat;
    const float* s_out = s0 + (size_t)SIN * WS + (size_t)(HS - 1) * WS * WS;
    const float* r0 = a.wt_rrs;
    const float* r_out = r0 + (size_t)kRrsIn * WR + (size_t)(HR - 1) * WR * WR;

#pragma unroll 1
    for (uint32_t u = blockIdx.x; u < items; u += gridDim.x) {
        const uint32_t t = u >> 1;
        const int si = find_segment(ST, t);
        const Segment& sg = ST.s[si];
        const uint32_t i = sg.offset + (t - sg.tile_start) * kTile + (u & 1u) * kTM + m;
        const bool valid = i < sg.offset + sg.count;
        __syncthreads();   // the previous item's column reads are over
        // encoding: two threads per vertex (levels 0-7 + SH, levels 8-15 + misc lanes; the
        // reference network: levels 0-3 + direction blobs, levels 4-7 + roughness blob)
        if (REF) {
            if (valid) {
                float p[3];
                norm_pos(a.enc, a.v.pos, i, p);
                encode_levels8<4>(a, p, lead ? 0 : 4, act, m);
                float blob[16];
                ref_blob_lanes(a.v, i, blob);
#pragma unroll
                for (int k = 0; k < 8; ++k)
                    act[(16 + (lead ? 0 : 8) + k) * kLd + m] = lead ? blob[k] : blob[8 + k];
            } else {
                for (int k = lead ? 0 : 16; k < (lead ? 16 : 32); ++k) act[k * kLd + m] = 0.f;
            }
        } else if (valid) {
            float p[3];
            norm_pos(a.enc, a.v.pos, i, p);
            if (lead) {
                encode_levels8(a, p, 0, act, m);
                float sh[16];
                const size_t i3 = 3 * (size_t)i;
                sh16(a.v.wi[i3], a.v.wi[i3 + 1], a.v.wi[i3 + 2], sh);
#pragma unroll
                for (int k = 0; k < 16; ++k) act[(32 + k) * kLd + m] = sh[k];
            } else {
                encode_levels8(a, p, 8, act, m);
                float misc[16];
                misc_lanes(a.v, i, misc);
#pragma unroll
                for (int k = 0; k < 8; ++k) act[(48 + k) * kLd + m] = misc[k];
            }
        } else {
            for (int k = lead ? 0 : 28; k < (lead ? 28 : 56); ++k) act[k * kLd + m] = 0.f;
        }
        VertexAux aux{};
        if (lead && valid) aux = load_aux(a.v, i);
        // StatNet: 56 live input lanes (48..55 misc, 56..63 zero); the reference network's 32
        hidden_layer<WS>(s0, SIN, REF ? 32 : 56, act, wch, tid);
#pragma unroll 1
        for (int h = 1; h < HS; ++h)
            hidden_layer<WS>(s0 + (size_t)SIN * WS + (size_t)(h - 1) * WS * WS, WS, WS, act,
                             wch, tid);
        float y[SOUT];
#pragma unroll
        for (int k = 0; k < SOUT; ++k) y[k] = 0.f;
        if (lead) {
            output_layer<WS, SOUT>(s_out, act, m, y);
            // glue: the RRSNet input in this vertex's column (10 live lanes; the reference's 12)
            float x1[16];
            if (REF) glue16_ref_aux(y, aux, x1);
            else glue16_aux(a.fp, y, aux, x1);
#pragma unroll
            for (int k = 0; k < (REF ? kRefRrsLanes : 10); ++k) act[k * kLd + m] = x1[k];
        }
        hidden_layer<WR>(r0, kRrsIn, REF ? kRefRrsLanes : 10, act, wch, tid);
#pragma unroll 1
        for (int h = 1; h < HR; ++h)
            hidden_layer<WR>(r0 + (size_t)kRrsIn * WR + (size_t)(h - 1) * WR * WR, WR, WR, act,
                             wch, tid);
        long long term = 0;
        if (lead && valid) {
            float raw;
            output_layer<WR, 1>(r_out, act, m, &raw);
            const float rrs = rrs_factor_aux<REF>(a.fp, y, raw, aux);
            if (a.stats) {
#pragma unroll
                for (int k = 0; k < SOUT; ++k) a.stats[SOUT * (size_t)i + k] = y[k];
            }
            a.rrs[i] = rrs;
            if (a.scr || a.ext_acc)
                term = fixed_term(a.fp, rrs, a.scr ? &a.scr->status : &g_dummy_status);
        }
        if (a.scr || a.ext_acc) {
            term = warp_sum_ll(term);
            if ((tid & 31) == 0 && term != 0)
                atomicAdd(a.ext_acc ? a.ext_acc : &a.scr->sum_acc[si], (unsigned long long)term);
        }
    }
}

template <int WS, int HS, int WR, int HR>
cudaError_t launch_cfg(const InferArgs& a, int sm_count, int ctas_per_sm, cudaStream_t s) {
    using S = FpShape<WS>;
    auto kern = k_infer_fp32<WS, HS, WR, HR>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)S::kSmem);
    if (e != cudaSuccess) return e;
    int per_sm = resident_ctas((const void*)kern, kThr, S::kSmem, 32);
    if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
    const uint32_t items = 2u * a.segs.total_tiles;
    unsigned grid = (unsigned)(sm_count * per_sm);
    if (grid > items) grid = items;
    if (grid == 0) return cudaSuccess;
    g_last_grid = (int)grid;
    kern<<<grid, kThr, S::kSmem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_infer_fp32(const InferArgs& a, int ws, int hs, int wr, int hr, int sm_count,
                              int ctas_per_sm, cudaStream_t s) {
    if (ws == 64 && hs == 2 && wr == 64 && hr == 2)
        return launch_cfg<64, 2, 64, 2>(a, sm_count, ctas_per_sm, s);
    if (ws == 128 && hs == 3 && wr == 128 && hr == 3)
        return launch_cfg<128, 3, 128, 3>(a, sm_count, ctas_per_sm, s);
    if (ws == 64 && hs == 3 && wr == 64 && hr == 3)
        return launch_cfg<64, 3, 64, 3>(a, sm_count, ctas_per_sm, s);
    if (ws == 32 && hs == 3 && wr == 32 && hr == 3)   // the reference network
        return launch_cfg<32, 3, 32, 3>(a, sm_count, ctas_per_sm, s);
    return cudaErrorInvalidValue;
}

template <int WS, int HS, int WR, int HR>
int max_ctas_fp32() {
    using S = FpShape<WS>;
    auto kern = k_infer_fp32<WS, HS, WR, HR>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem) !=
        cudaSuccess)
        return 0;
    return resident_ctas((const void*)kern, kThr, S::kSmem, 32);
}

int infer_max_ctas_fp32(int ws, int hs) {
    if (ws == 64 && hs == 2) return max_ctas_fp32<64, 2, 64, 2>();
    if (ws == 64 && hs == 3) return max_ctas_fp32<64, 3, 64, 3>();
    if (ws == 128 && hs == 3) return max_ctas_fp32<128, 3, 128, 3>();
    if (ws == 32 && hs == 3) return max_ctas_fp32<32, 3, 32, 3>();
    return 0;
}

}  // namespace nrrs
