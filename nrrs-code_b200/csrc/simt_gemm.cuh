// simt_gemm.cuh -- the register-tiled FP32 SIMT GEMM of the plain FP32 path (inference and
// training kernels).
//
// A CTA of 128 threads holds the activations of 64 samples in one shared-memory tile, K-major
// ([k][64 samples + 4 pad]). A layer out[n][m] = epi(sum_k B[k][n] in[k][m]) is computed in place
// on that tile: each thread owns an 8 x (W/16) block of outputs (8 samples x 8, 4 or 2 neurons)
// and, per k, reads 8 activations and 8, 4 or 2 B values (float4 / float2) and issues 64, 32 or
// 16 FMAs.
// B ([k_rows][W] in global memory: a layer's transposed weights for a forward step, its row-major
// weights for a backward step) comes from L2 in 32-row chunks, double-buffered with cp.async.
// Every output is accumulated as fmaf(B[k][n], in[k][m], acc) over k ascending, the order of the
// one-thread-per-sample loops it replaces, so the results do not depend on the launch shape.
#pragma once
#include "kernels.hpp"

namespace nrrs {
namespace simt {

constexpr int kTM = 64;        // samples (vertices) per tile
// row stride of the activation tile: 4 floats of padding keep float4 alignment and spread the
// epilogue's stores (neuron rows 4 apart) over twice as many banks
constexpr int kLd = kTM + 4;
constexpr int kThr = 128;      // threads per CTA
constexpr int kKC = 32;        // B rows per chunk

constexpr int imax(int a, int b) { return a > b ? a : b; }

__device__ __forceinline__ void cp_async16(float* smem_dst, const float* gmem_src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// rows x W floats of B into a shared-memory chunk
template <int W>
__device__ __forceinline__ void load_chunk(float* dst, const float* __restrict__ src, int rows,
                                           int tid) {
    const int n4 = rows * (W / 4);
    for (int q = tid; q < n4; q += kThr) cp_async16(dst + 4 * q, src + 4 * q);
}

// out[n][m] = epi(n, m0, v[8]) with v[i] = sum_{k < k_eff} B[k][n] act[k][m0 + i], for the 8
// samples m0 .. m0+7 and the W/16 neurons each thread owns. Every read of the tile ends at the
// chunk loop's last barrier, so epi may overwrite it in place; a barrier follows epi. wch holds
// two chunks of kKC x W floats.
template <int W, class Epi>
__device__ __forceinline__ void tile_gemm(const float* __restrict__ B, int k_rows, int k_eff,
                                          const float* act, float* wch, int tid, Epi&& epi) {
    static_assert(W == 32 || W == 64 || W == 128, "tile widths");
    constexpr int C = W / 16;                 // neurons per thread: 8, 4 or 2 (W = 128, 64, 32)
    constexpr int CW = C < 4 ? C : 4;         // consecutive neurons of a thread's group
    const int lane = tid & 31, warp = tid >> 5;
    const int tx = lane & 15, ty = warp * 2 + (lane >> 4);   // ty 0..7: samples ty*8 .. +7
    float acc[8][C];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < C; ++j) acc[i][j] = 0.f;
    const int nch = (k_rows + kKC - 1) / kKC;
    load_chunk<W>(wch, B, k_rows < kKC ? k_rows : kKC, tid);
    cp_async_commit();
#pragma unroll 1
    for (int c = 0; c < nch; ++c) {
        if (c + 1 < nch) {
            const int r = k_rows - (c + 1) * kKC;
            load_chunk<W>(wch + ((c + 1) & 1) * kKC * W, B + (size_t)(c + 1) * kKC * W,
                          r < kKC ? r : kKC, tid);
        }
        cp_async_commit();
        cp_async_wait1();   // every group but the newest: chunk c has landed
        __syncthreads();
        const float* Bc = wch + (c & 1) * kKC * W + tx * CW;
        const float* A = act + (size_t)(c * kKC) * kLd + ty * 8;
        const int kn = k_eff - c * kKC < kKC ? k_eff - c * kKC : kKC;
#pragma unroll 4
        for (int kk = 0; kk < kn; ++kk) {
            const float4 a0 = *reinterpret_cast<const float4*>(A + kk * kLd);
            const float4 a1 = *reinterpret_cast<const float4*>(A + kk * kLd + 4);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            float bv[C];
            if constexpr (C == 2) {
                const float2 b0 = *reinterpret_cast<const float2*>(Bc + kk * W);
                bv[0] = b0.x; bv[1] = b0.y;
            } else {
                const float4 b0 = *reinterpret_cast<const float4*>(Bc + kk * W);
                bv[0] = b0.x; bv[1] = b0.y; bv[2] = b0.z; bv[3] = b0.w;
            }
            if constexpr (C == 8) {
                const float4 b1 = *reinterpret_cast<const float4*>(Bc + kk * W + 64);
                bv[4] = b1.x; bv[5] = b1.y; bv[6] = b1.z; bv[7] = b1.w;
            }
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < C; ++j) acc[i][j] = fmaf(bv[j], av[i], acc[i][j]);
        }
        __syncthreads();    // the buffer read here is refilled by the next iteration's prefetch
    }
#pragma unroll
    for (int j = 0; j < C; ++j) {
        const int n = (j < 4 ? 0 : 64) + tx * CW + (j & 3);
        const float v[8] = {acc[0][j], acc[1][j], acc[2][j], acc[3][j],
                            acc[4][j], acc[5][j], acc[6][j], acc[7][j]};
        epi(n, ty * 8, v);
    }
    __syncthreads();
}

// 8 consecutive values of tile row n from samples m0 .. m0+7
__device__ __forceinline__ void tile_store8(float* act, int n, int m0, const float* v) {
    float* o = act + (size_t)n * kLd + m0;
    *reinterpret_cast<float4*>(o) = make_float4(v[0], v[1], v[2], v[3]);
    *reinterpret_cast<float4*>(o + 4) = make_float4(v[4], v[5], v[6], v[7]);
}

}  // namespace simt
}  // namespace nrrs
