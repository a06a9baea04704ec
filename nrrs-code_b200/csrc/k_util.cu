// k_util.cu -- derived weight images and the FP16 table copy.
//
// The FP32 master weights are row-major W[out][in] per layer. Two derived images are rebuilt
// after every optimizer step or parameter upload:
//   * FP32 transposed Wt[in][out4] (out padded to a multiple of 4) for the SIMT path;
//   * FP16/BF16 UMMA image: per layer an [Npad][K] K-major operand in the canonical
//     no-swizzle core-matrix layout of tcgen05 (8 rows x 16 bytes per core matrix, adjacent
//     K core matrices 128 B apart (LBO), adjacent 8-row groups K*16 B apart (SBO)).
//     The output layers are padded to N = 16 rows with zeros.
#include "kernels.hpp"

namespace nrrs {

namespace {

struct LayerDesc {
    int in, out;
};

__host__ __device__ inline int pad4(int x) { return (x + 3) / 4 * 4; }
__host__ __device__ inline int npad16(int x) { return (x + 15) / 16 * 16; }

// layer list of a network: in -> w (hidden) -> out
__host__ __device__ inline LayerDesc layer_of(int in, int w, int hidden, int out, int l) {
    LayerDesc d;
    d.in = l == 0 ? in : w;
    d.out = l == hidden ? out : w;
    return d;
}

// element offset of (n, k) in a K-major core-matrix image with K columns
__host__ __device__ inline size_t umma_offset(int n, int k, int K) {
    return (size_t)(n >> 3) * (size_t)(K * 8) + (size_t)(k >> 3) * 64 + (size_t)(n & 7) * 8 +
           (size_t)(k & 7);
}

struct PackArgs {
    const float* master;
    float* wt;
    float* wrow;     // 16-byte aligned row-major copy of the master (backward passes)
    void* wpack;
    int ws, hs, wr, hr, prec;
};

__global__ void k_pack(PackArgs a) {
    // one thread per (network, layer, n, k) of the padded images; grid-stride
    const int nets = 2;
    size_t mofs = 0, tofs = 0, pofs = 0;
    for (int net = 0; net < nets; ++net) {
        const int in = net == 0 ? stat_in_of(a.ws) : kRrsIn;
        const int w = net == 0 ? a.ws : a.wr;
        const int h = net == 0 ? a.hs : a.hr;
        const int out = net == 0 ? stat_out_of(a.ws) : 1;
        for (int l = 0; l <= h; ++l) {
            const LayerDesc d = layer_of(in, w, h, out, l);
            const int op4 = pad4(d.out);
            const int np = l == h ? npad16(d.out) : d.out;
            const size_t cells = (size_t)np * d.in;
            for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < cells;
                 e += (size_t)gridDim.x * blockDim.x) {
                const int n = (int)(e / d.in), k = (int)(e % d.in);
                const float v = n < d.out ? a.master[mofs + (size_t)n * d.in + k] : 0.f;
                if (n < op4) a.wt[tofs + (size_t)k * op4 + n] = v;
                if (n < d.out && a.wrow) a.wrow[mofs + (size_t)n * d.in + k] = v;
                if (a.wpack) {
                    const size_t o = pofs + umma_offset(n, k, d.in);
                    if (a.prec == NRRS_PREC_BF16)
                        reinterpret_cast<__nv_bfloat16*>(a.wpack)[o] = __float2bfloat16_rn(v);
                    else
                        reinterpret_cast<__half*>(a.wpack)[o] = __float2half_rn(v);
                }
            }
            mofs += (size_t)d.out * d.in;
            tofs += (size_t)d.in * op4;
            pofs += cells;
        }
    }
}

// Training image: per network the forward layers [N][K] in the UMMA K-major layout (as k_pack).
// The backward passes read the same bytes as MN-major operands, which is W^T, so no transposed
// copy is kept. StatNet is stored in FP16 (its deltas are bounded), RRSNet in BF16 (its loss
// gradient r^2/q^2 can exceed FP16's range).
struct PackTrainArgs {
    const float* master;
    uint16_t* out;
    int ws, hs, wr, hr;
};

__device__ __forceinline__ uint16_t to_bits(float v, bool bf) {
    if (bf) {
        const __nv_bfloat16 b = __float2bfloat16_rn(v);
        return *reinterpret_cast<const uint16_t*>(&b);
    }
    const __half h = __float2half_rn(v);
    return *reinterpret_cast<const uint16_t*>(&h);
}

__global__ void k_pack_train(PackTrainArgs a) {
    size_t mofs = 0, pofs = 0;
    for (int net = 0; net < 2; ++net) {
        const int in = net == 0 ? stat_in_of(a.ws) : kRrsIn;
        const int w = net == 0 ? a.ws : a.wr;
        const int h = net == 0 ? a.hs : a.hr;
        const int out = net == 0 ? stat_out_of(a.ws) : 1;
        // forward images
        for (int l = 0; l <= h; ++l) {
            const LayerDesc d = layer_of(in, w, h, out, l);
            const int np = l == h ? npad16(d.out) : d.out;
            const size_t cells = (size_t)np * d.in;
            for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < cells;
                 e += (size_t)gridDim.x * blockDim.x) {
                const int n = (int)(e / d.in), k = (int)(e % d.in);
                const float v = n < d.out ? a.master[mofs + (size_t)n * d.in + k] : 0.f;
                a.out[pofs + umma_offset(n, k, d.in)] = to_bits(v, net == 1);
            }
            mofs += (size_t)d.out * d.in;
            pofs += cells;
        }
    }
}

__global__ void k_table_half(const float* t, __half* h, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        h[i] = __float2half_rn(t[i]);
}

// The cell image of the FP16 table's dense levels: cell (x, y, z) of level L gets its 8 corner
// entries (raw FP16 pairs) in corner order k = x-bit + 2 y-bit + 4 z-bit, the order in which
// the gathers sum them, so features from the image equal features from the table bit for bit.
// Threads walk cells in x-fastest order: the corner reads of a warp are mostly contiguous rows.
__global__ void k_cell_image(const uint32_t* __restrict__ rows,
                             const __grid_constant__ EncodeParams e, uint4* __restrict__ cells,
                             uint32_t n_cells) {
    for (uint32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < n_cells;
         g += gridDim.x * blockDim.x) {
        // the dense levels are a prefix of the levels (N_l grows with l)
        int l = 0;
        while (l + 1 < (int)e.n_levels && e.lv[l + 1].dense && e.lv[l + 1].cell <= g) ++l;
        const LevelDev L = e.lv[l];
        const uint32_t N = L.res, r = g - L.cell;
        const uint32_t x = r % N, y = (r / N) % N, z = r / (N * N);
        uint32_t t[8];
#pragma unroll
        for (int k = 0; k < 8; ++k)
            t[k] = rows[grid_row(L, e.hash_mask, x + (k & 1), y + ((k >> 1) & 1),
                                 z + ((k >> 2) & 1))];
        cells[2 * (size_t)g] = make_uint4(t[0], t[1], t[2], t[3]);
        cells[2 * (size_t)g + 1] = make_uint4(t[4], t[5], t[6], t[7]);
    }
}

}  // namespace

cudaError_t launch_cell_image(const __half* table_h, const EncodeParams& e, uint4* cells,
                              uint32_t n_cells, int sm_count, cudaStream_t s) {
    if (!cells || n_cells == 0) return cudaSuccess;
    k_cell_image<<<sm_count * 8, 256, 0, s>>>(reinterpret_cast<const uint32_t*>(table_h), e,
                                              cells, n_cells);
    return cudaGetLastError();
}

thread_local int g_last_grid = 0;

int resident_ctas(const void* kern, int threads, size_t dyn_smem, int cap) {
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, kern) != cudaSuccess) return 1;
    int dev = 0, smem_sm = 0, regs_sm = 0, thr_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    const size_t per_cta_smem = dyn_smem + fa.sharedSizeBytes + 1024;
    int by_smem = (int)((size_t)smem_sm / per_cta_smem);
    const int regs = (fa.numRegs + 7) / 8 * 8;  // allocation granularity per thread
    int by_regs = regs > 0 ? regs_sm / (regs * threads) : 32;
    int by_thr = thr_sm / threads;
    int n = by_smem < by_regs ? by_smem : by_regs;
    n = n < by_thr ? n : by_thr;
    n = n < cap ? n : cap;
    return n < 1 ? 1 : n;
}

size_t transposed_weight_floats(int ws, int hs, int wr, int hr) {
    size_t t = 0;
    for (int l = 0; l <= hs; ++l) {
        LayerDesc d = layer_of(stat_in_of(ws), ws, hs, stat_out_of(ws), l);
        t += (size_t)d.in * pad4(d.out);
    }
    for (int l = 0; l <= hr; ++l) {
        LayerDesc d = layer_of(kRrsIn, wr, hr, 1, l);
        t += (size_t)d.in * pad4(d.out);
    }
    return t;
}

size_t packed_weight_bytes(int ws, int hs, int wr, int hr) {
    size_t t = 0;
    for (int l = 0; l <= hs; ++l) {
        LayerDesc d = layer_of(stat_in_of(ws), ws, hs, stat_out_of(ws), l);
        t += (size_t)(l == hs ? npad16(d.out) : d.out) * d.in;
    }
    for (int l = 0; l <= hr; ++l) {
        LayerDesc d = layer_of(kRrsIn, wr, hr, 1, l);
        t += (size_t)(l == hr ? npad16(d.out) : d.out) * d.in;
    }
    return t * 2;
}

cudaError_t launch_pack_weights(const float* master_mlp, float* wt, float* wrow, void* wpack,
                                int ws, int hs, int wr, int hr, int prec, cudaStream_t s) {
    PackArgs a{master_mlp, wt, wrow, wpack, ws, hs, wr, hr, prec};
    k_pack<<<64, 256, 0, s>>>(a);
    return cudaGetLastError();
}

size_t train_pack_bytes(int ws, int hs, int wr, int hr) {
    size_t t = 0;
    for (int net = 0; net < 2; ++net) {
        const int in = net == 0 ? stat_in_of(ws) : kRrsIn;
        const int w = net == 0 ? ws : wr;
        const int h = net == 0 ? hs : hr;
        const int out = net == 0 ? stat_out_of(ws) : 1;
        for (int l = 0; l <= h; ++l) {
            const LayerDesc d = layer_of(in, w, h, out, l);
            t += (size_t)(l == h ? npad16(d.out) : d.out) * d.in;
        }
    }
    return t * 2;
}

cudaError_t launch_pack_train(const float* master_mlp, void* out, int ws, int hs, int wr, int hr,
                              cudaStream_t s) {
    PackTrainArgs a{master_mlp, reinterpret_cast<uint16_t*>(out), ws, hs, wr, hr};
    k_pack_train<<<64, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_table_to_half(const float* t, __half* h, size_t n, cudaStream_t s) {
    k_table_half<<<148 * 4, 256, 0, s>>>(t, h, n);
    return cudaGetLastError();
}

}  // namespace nrrs
