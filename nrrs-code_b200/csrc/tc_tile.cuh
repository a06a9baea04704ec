// tc_tile.cuh -- 128-row activation tiles for the tcgen05 kernels (inference and training).
//
// A tile holds 128 rows (vertices or samples) x K features in the canonical no-swizzle K-major
// core-matrix layout: 8 rows x 16 bytes per core matrix, K-adjacent core matrices 128 B apart
// (LBO), 8-row groups K*16 B apart (SBO). Row m of the tile is produced and consumed by thread m
// (TMEM lane m), one 16-byte chunk of 8 features at a time. The same bytes read as an MN-major
// operand (features contiguous, rows as the reduction dimension) with SBO = 128 B and
// LBO = K*16 B, which the weight-gradient GEMM uses.
#pragma once
#include "nrrs_common.cuh"
#include "tc_ptx.cuh"

namespace nrrs {
namespace tile {

constexpr uint32_t kSpin = 1u << 24;

template <bool BF>
__device__ __forceinline__ uint32_t pack2(float a, float b) {
    if constexpr (BF) {
        __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    } else {
        __half2 h = __floats2half2_rn(a, b);
        return *reinterpret_cast<uint32_t*>(&h);
    }
}

// ReLU and the conversion in one instruction (cvt with .relu: negative results become 0);
// x0 goes to the low half like pack2
template <bool BF>
__device__ __forceinline__ uint32_t pack2_relu(float x0, float x1) {
    uint32_t d;
    if constexpr (BF)
        asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(x1), "f"(x0));
    else
        asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(x1), "f"(x0));
    return d;
}

template <bool BF>
__device__ __forceinline__ float2 unpack2(uint32_t u) {
    if constexpr (BF) {
        __nv_bfloat162 h = *reinterpret_cast<__nv_bfloat162*>(&u);
        return __bfloat1622float2(h);
    } else {
        __half2 h = *reinterpret_cast<__half2*>(&u);
        return __half22float2(h);
    }
}

template <bool BF>
__device__ __forceinline__ uint4 pack8(const float* f) {
    return make_uint4(pack2<BF>(f[0], f[1]), pack2<BF>(f[2], f[3]), pack2<BF>(f[4], f[5]),
                      pack2<BF>(f[6], f[7]));
}

__device__ __forceinline__ uint32_t chunk_offset(int m, int kchunk, int K) {
    return (uint32_t)(m >> 3) * (uint32_t)(K * 16) + (uint32_t)kchunk * 128u + (uint32_t)(m & 7) * 16u;
}

// 8 consecutive K elements of row m
__device__ __forceinline__ void store_chunk(uint8_t* sA, int m, int kchunk, int K, uint4 v) {
    *reinterpret_cast<uint4*>(sA + chunk_offset(m, kchunk, K)) = v;
}
__device__ __forceinline__ uint4 load_chunk(const uint8_t* sA, int m, int kchunk, int K) {
    return *reinterpret_cast<const uint4*>(sA + chunk_offset(m, kchunk, K));
}

__device__ __forceinline__ void zero_row(uint8_t* sA, int m, int K) {
    for (int kc = 0; kc < K / 8; ++kc) store_chunk(sA, m, kc, K, make_uint4(0u, 0u, 0u, 0u));
}

// generic smem writes of all threads -> visible to the tensor cores; TMEM reads done
__device__ __forceinline__ void sync_for_mma() {
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
}

// D[TMEM, 128 x N] = A[128 x K] * B[N x K]^T, both K-major tiles; thread 0 issues, all wait
template <int K, int N, bool BF>
__device__ __forceinline__ bool mma_layer(const uint8_t* sA, const uint8_t* sB, uint32_t tmem,
                                          uint64_t* bar, uint32_t& phase, int tid) {
    if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
        constexpr uint32_t idesc = tc::idesc_f16(N, BF ? 1u : 0u);
#pragma unroll
        for (int kk = 0; kk < K / 16; ++kk) {
            const uint64_t ad = tc::smem_desc(a0 + kk * 256, 128, K * 16);
            const uint64_t bd = tc::smem_desc(b0 + kk * 256, 128, K * 16);
            tc::mma_f16(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
        tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait(bar, phase, kSpin);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok;
}

// D[TMEM, 128 x N] = A[128 x K] * W^T for a forward weight image W of K output rows and KIN
// inputs (K-major, the B operand of mma_layer). Read as an MN-major operand (inputs contiguous,
// output rows as the reduction dimension: SBO = 128 B, LBO = KIN*16 B) the same bytes are W^T;
// its first N inputs are produced. Input gradients need no transposed copy of the weights.
template <int K, int N, int KIN, bool BF>
__device__ __forceinline__ bool mma_layer_t(const uint8_t* sA, const uint8_t* sW, uint32_t tmem,
                                            uint64_t* bar, uint32_t& phase, int tid) {
    static_assert(N % 16 == 0 && N <= KIN && K % 16 == 0, "transposed operand shape");
    if (tid == 0) {
        tc::fence_after_sync();
        const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sW);
        constexpr uint32_t idesc = tc::idesc_f16_major(N, BF ? 1u : 0u, 0u, 1u);
#pragma unroll
        for (int kk = 0; kk < K / 16; ++kk) {
            const uint64_t ad = tc::smem_desc(a0 + kk * 256, 128, K * 16);
            const uint64_t bd = tc::smem_desc(b0 + kk * 2 * KIN * 16, KIN * 16, 128);
            tc::mma_f16(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
        tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait(bar, phase, kSpin);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok;
}

// hidden-layer epilogue that also records the ReLU mask of row m: bit j of bits[c / 32] is set
// when column c = 32 * (c / 32) + j is positive (the backward of the same row, by the same
// thread, applies it; no activation tile has to stay resident)
template <int N, bool BF>
__device__ __forceinline__ void epilogue_relu_bits(uint32_t trow, uint8_t* sOut, int m,
                                                   uint32_t (&bits)[N / 32]) {
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 32) {
        float v[32];
        tc::tmem_ld16(trow + c0, v);
        tc::tmem_ld16(trow + c0 + 16, v + 16);
        tc::tmem_wait_ld();
        uint32_t b = 0u;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            if (v[j] > 0.f) b |= 1u << j;
            else v[j] = 0.f;
        }
        bits[c0 / 32] = b;
#pragma unroll
        for (int j = 0; j < 4; ++j) store_chunk(sOut, m, c0 / 8 + j, N, pack8<BF>(v + 8 * j));
    }
}

// backward epilogue with a recorded mask: TMEM row -> zero where the forward ReLU was inactive
template <int N, bool BF>
__device__ __forceinline__ void epilogue_mask_bits(uint32_t trow, const uint32_t (&bits)[N / 32],
                                                   uint8_t* sOut, int m) {
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 32) {
        float v[32];
        tc::tmem_ld16(trow + c0, v);
        tc::tmem_ld16(trow + c0 + 16, v + 16);
        tc::tmem_wait_ld();
        const uint32_t b = bits[c0 / 32];
#pragma unroll
        for (int j = 0; j < 32; ++j)
            if (!((b >> j) & 1u)) v[j] = 0.f;
#pragma unroll
        for (int j = 0; j < 4; ++j) store_chunk(sOut, m, c0 / 8 + j, N, pack8<BF>(v + 8 * j));
    }
}

// hidden-layer epilogue: TMEM row -> ReLU -> tile (K = N). At N = 128 ReLU and conversion are
// one cvt per pair of columns (fewer instructions in the 4K kernels' epilogues); the 64-wide
// kernels keep max + convert, which the compiler schedules into fewer registers (their
// 3-CTA launch bounds leave 80)
template <int N, bool BF>
__device__ __forceinline__ void epilogue_relu(uint32_t trow, uint8_t* sOut, int m) {
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 32) {
        float v[32];
        tc::tmem_ld16(trow + c0, v);
        tc::tmem_ld16(trow + c0 + 16, v + 16);
        tc::tmem_wait_ld();
        if constexpr (N >= 128) {
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float* w = v + 8 * j;
                store_chunk(sOut, m, c0 / 8 + j, N,
                            make_uint4(pack2_relu<BF>(w[0], w[1]), pack2_relu<BF>(w[2], w[3]),
                                       pack2_relu<BF>(w[4], w[5]), pack2_relu<BF>(w[6], w[7])));
            }
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = fmaxf(v[j], 0.f);
#pragma unroll
            for (int j = 0; j < 4; ++j) store_chunk(sOut, m, c0 / 8 + j, N, pack8<BF>(v + 8 * j));
        }
    }
}

// epilogue with the network's activation: ReLU, or LeakyReLU with slope 0.01 (the reference
// network)
template <int N, bool BF, bool LEAKY>
__device__ __forceinline__ void epilogue_act(uint32_t trow, uint8_t* sOut, int m) {
    if constexpr (!LEAKY) {
        epilogue_relu<N, BF>(trow, sOut, m);
    } else {
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 32) {
            float v[32];
            tc::tmem_ld16(trow + c0, v);
            tc::tmem_ld16(trow + c0 + 16, v + 16);
            tc::tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 32; ++j) v[j] = v[j] > 0.f ? v[j] : 0.01f * v[j];
#pragma unroll
            for (int j = 0; j < 4; ++j) store_chunk(sOut, m, c0 / 8 + j, N, pack8<BF>(v + 8 * j));
        }
    }
}

// hidden-layer epilogue into TMEM: the TMEM row of D (N FP32 columns at trow) -> activation ->
// FP16/BF16 pairs -> the next layer's A operand (N / 2 columns at trow_a); the caller waits for
// the stores (tcgen05.wait::st) before the next MMA is issued
template <int N, bool BF, bool LEAKY>
__device__ __forceinline__ void epilogue_act_tmem(uint32_t trow, uint32_t trow_a) {
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 32) {
        float v[32];
        tc::tmem_ld16(trow + c0, v);
        tc::tmem_ld16(trow + c0 + 16, v + 16);
        tc::tmem_wait_ld();
        uint32_t pk[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            float x0 = v[2 * j], x1 = v[2 * j + 1];
            if constexpr (LEAKY) {
                x0 = x0 > 0.f ? x0 : 0.01f * x0;
                x1 = x1 > 0.f ? x1 : 0.01f * x1;
                pk[j] = pack2<BF>(x0, x1);
            } else {
                pk[j] = pack2_relu<BF>(x0, x1);
            }
        }
        tc::tmem_st16(trow_a + c0 / 2, pk);
    }
    tc::tmem_wait_st();
}

}  // namespace tile
}  // namespace nrrs
