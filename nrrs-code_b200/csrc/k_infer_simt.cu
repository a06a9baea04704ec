// k_infer_simt.cu -- plain FP32 inference: hash grid + SH encoding, StatNet, glue, RRSNet,
// activation, clamp and the exact normalisation sum, one thread per vertex (SIMT FP32).
//
// This is the "plain FP32 per-depth path" the mixed-precision tcgen05 path is measured
// against. It fuses what the reference runs as nrrs_generate_inference_data (train.cu:269-287),
// tcnn inference_mixed_precision x2 (myNetworkLL2.cpp:206, network.cpp:346),
// nrrs_generate_inference_data_from_0to1 (train.cu:41-112) and the "Gen RRS Number" lambda
// (integrator.cpp:1184-1298), so the AoS round trips of the reference disappear.
//
// Layout: each thread keeps its activation column in shared memory (xs[lane][thread], conflict
// free); weights are stored transposed ([in][out], out padded to 4) and read as broadcast
// float4 loads from shared memory when they fit, else from global memory through L1.
#include "kernels.hpp"

namespace nrrs {

namespace {

template <int IN, int OUT, int OUTP, bool RELU>
__device__ __forceinline__ void dense_layer(const float* __restrict__ Wt, float* xs, int tid,
                                            float* out_reg) {
    float acc[OUT];
#pragma unroll
    for (int o = 0; o < OUT; ++o) acc[o] = 0.f;
#pragma unroll 2
    for (int k = 0; k < IN; ++k) {
        const float xk = xs[k * kTile + tid];
        const float4* w4 = reinterpret_cast<const float4*>(Wt + k * OUTP);
#pragma unroll
        for (int o4 = 0; o4 < OUTP / 4; ++o4) {
            const float4 w = w4[o4];
            if (4 * o4 + 0 < OUT) acc[4 * o4 + 0] = fmaf(w.x, xk, acc[4 * o4 + 0]);
            if (4 * o4 + 1 < OUT) acc[4 * o4 + 1] = fmaf(w.y, xk, acc[4 * o4 + 1]);
            if (4 * o4 + 2 < OUT) acc[4 * o4 + 2] = fmaf(w.z, xk, acc[4 * o4 + 2]);
            if (4 * o4 + 3 < OUT) acc[4 * o4 + 3] = fmaf(w.w, xk, acc[4 * o4 + 3]);
        }
    }
    if (out_reg) {
#pragma unroll
        for (int o = 0; o < OUT; ++o) out_reg[o] = RELU ? fmaxf(acc[o], 0.f) : acc[o];
    } else {
#pragma unroll
        for (int o = 0; o < OUT; ++o) xs[o * kTile + tid] = RELU ? fmaxf(acc[o], 0.f) : acc[o];
    }
}

constexpr int pad4(int x) { return (x + 3) / 4 * 4; }

template <int W, int H, int IN, int OUT>
struct MlpShape {
    static constexpr int kFloats = IN * W + (H - 1) * W * W + W * pad4(OUT);
};

// forward through a bias-free ReLU MLP whose input column is xs[0, IN_EFF)
template <int W, int H, int IN, int IN_EFF, int OUT>
__device__ __forceinline__ void mlp_simt(const float* __restrict__ Wt, float* xs, int tid,
                                         float* y) {
    dense_layer<IN_EFF, W, W, true>(Wt, xs, tid, nullptr);
    Wt += IN * W;
#pragma unroll 1
    for (int h = 1; h < H; ++h) {
        dense_layer<W, W, W, true>(Wt, xs, tid, nullptr);
        Wt += W * W;
    }
    dense_layer<W, OUT, pad4(OUT), false>(Wt, xs, tid, y);
}

// hash grid + SH + misc lanes of vertex i into this thread's column xs[0, 56)
__device__ __forceinline__ void encode_simt(const InferArgs& a, uint32_t i, float* xs, int tid) {
    float p[3];
    norm_pos(a.enc, a.v.pos, i, p);
    const float2* table = reinterpret_cast<const float2*>(a.table);
#pragma unroll 2
    for (int l = 0; l < kMaxLevels; ++l) {
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
        xs[(2 * l) * kTile + tid] = f0;
        xs[(2 * l + 1) * kTile + tid] = f1;
    }
    float sh[16];
    const size_t i3 = 3 * (size_t)i;
    sh16(a.v.wi[i3], a.v.wi[i3 + 1], a.v.wi[i3 + 2], sh);
#pragma unroll
    for (int k = 0; k < 16; ++k) xs[(32 + k) * kTile + tid] = sh[k];
    float m[16];
    misc_lanes(a.v, i, m);
#pragma unroll
    for (int k = 0; k < 8; ++k) xs[(48 + k) * kTile + tid] = m[k];
}

template <int WS, int HS, int WR, int HR, bool WSMEM>
__global__ void __launch_bounds__(kTile) k_infer_fp32(const __grid_constant__ InferArgs a) {
    extern __shared__ float4 smem4[];
    float* smem = reinterpret_cast<float*>(smem4);
    constexpr int NS = MlpShape<WS, HS, kStatIn, kStatOut>::kFloats;
    constexpr int NR = MlpShape<WR, HR, kRrsIn, 1>::kFloats;
    const int tid = threadIdx.x;
    const float* wst = a.wt_stat;
    const float* wrt = a.wt_rrs;
    float* xs = smem;
    if (WSMEM) {
        const float4* s4 = reinterpret_cast<const float4*>(a.wt_stat);
        const float4* r4 = reinterpret_cast<const float4*>(a.wt_rrs);
        for (int k = tid; k < NS / 4; k += kTile) smem4[k] = s4[k];
        for (int k = tid; k < NR / 4; k += kTile) smem4[NS / 4 + k] = r4[k];
        __syncthreads();
        wst = smem;
        wrt = smem + NS;
        xs = smem + NS + NR;
    }
    const SegmentTable& S = seg_table(a.segs);
    for (uint32_t t = blockIdx.x; t < S.total_tiles; t += gridDim.x) {
        const int si = find_segment(S, t);
        const Segment& sg = S.s[si];
        const uint32_t i = sg.offset + (t - sg.tile_start) * kTile + tid;
        const bool valid = i < sg.offset + sg.count;
        long long term = 0;
        if (valid) {
            encode_simt(a, i, xs, tid);
            float y[3];
            mlp_simt<WS, HS, kStatIn, 56, kStatOut>(wst, xs, tid, y);
            float x1[16];
            glue16(a.fp, y, a.v, i, x1);
#pragma unroll
            for (int k = 0; k < 10; ++k) xs[k * kTile + tid] = x1[k];
            float raw;
            mlp_simt<WR, HR, kRrsIn, 10, 1>(wrt, xs, tid, &raw);
            const float rrs = rrs_factor(a.fp, y, raw, a.v, i);
            if (a.stats) {
                a.stats[3 * (size_t)i] = y[0];
                a.stats[3 * (size_t)i + 1] = y[1];
                a.stats[3 * (size_t)i + 2] = y[2];
            }
            a.rrs[i] = rrs;
            if (a.scr || a.ext_acc) term = fixed_term(a.fp, rrs, a.scr ? &a.scr->status : &g_dummy_status);
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
    constexpr int NS = MlpShape<WS, HS, kStatIn, kStatOut>::kFloats;
    constexpr int NR = MlpShape<WR, HR, kRrsIn, 1>::kFloats;
    constexpr int XW = (WS > WR ? WS : WR) > kStatIn ? (WS > WR ? WS : WR) : kStatIn;
    constexpr size_t xs_bytes = (size_t)XW * kTile * sizeof(float);
    constexpr size_t w_bytes = (size_t)(NS + NR) * sizeof(float);
    constexpr bool fits = xs_bytes + w_bytes <= 200 * 1024;
    const size_t smem = fits ? xs_bytes + w_bytes : xs_bytes;
    auto kern = k_infer_fp32<WS, HS, WR, HR, fits>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = resident_ctas((const void*)kern, kTile, smem, 32);
    if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
    unsigned grid = (unsigned)(sm_count * per_sm);
    if (grid > a.segs.total_tiles) grid = a.segs.total_tiles;
    if (grid == 0) return cudaSuccess;
    g_last_grid = (int)grid;
    kern<<<grid, kTile, smem, s>>>(a);
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
    return cudaErrorInvalidValue;
}

template <int WS, int HS, int WR, int HR>
int max_ctas_fp32() {
    constexpr int NS = MlpShape<WS, HS, kStatIn, kStatOut>::kFloats;
    constexpr int NR = MlpShape<WR, HR, kRrsIn, 1>::kFloats;
    constexpr int XW = (WS > WR ? WS : WR) > kStatIn ? (WS > WR ? WS : WR) : kStatIn;
    constexpr size_t xs_bytes = (size_t)XW * kTile * sizeof(float);
    constexpr size_t w_bytes = (size_t)(NS + NR) * sizeof(float);
    constexpr bool fits = xs_bytes + w_bytes <= 200 * 1024;
    const size_t smem = fits ? xs_bytes + w_bytes : xs_bytes;
    auto kern = k_infer_fp32<WS, HS, WR, HR, fits>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    return resident_ctas((const void*)kern, kTile, smem, 32);
}

int infer_max_ctas_fp32(int ws, int hs) {
    if (ws == 64 && hs == 2) return max_ctas_fp32<64, 2, 64, 2>();
    if (ws == 64 && hs == 3) return max_ctas_fp32<64, 3, 64, 3>();
    if (ws == 128 && hs == 3) return max_ctas_fp32<128, 3, 128, 3>();
    return 0;
}

}  // namespace nrrs
