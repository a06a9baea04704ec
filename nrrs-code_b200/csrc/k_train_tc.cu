// k_train_tc.cu -- mixed-precision training step on the 5th-generation tensor cores (sm_100a).
//
// Same maths as k_train_simt.cu (losses of NRRSNetwork::train, network.cpp:196-295), with every
// matrix product on tcgen05 (FP32 accumulation in TMEM, FP32 master weights and Adam state).
// StatNet runs in FP16 (its activations and deltas are bounded); RRSNet in BF16, because its
// loss gradient r^2/q^2 can exceed FP16's range.
// Deltas are kept per sample (the 1/n of the batch mean is applied when the weight gradients are
// reduced and in the hash-grid scatter), so they stay O(1) in BF16.
//
//   k_ttc_stat   per 128-sample tile: FP16-table encode -> StatNet forward (tcgen05) -> loss
//                gradient -> input gradients with the forward weight images read as MN-major
//                (transposed) operands (tcgen05) -> hash-grid scatter-add (vector FP32
//                reductions); glue -> RRSNet input tile. Every activation and delta tile is
//                written to HBM with a bulk TMA store, in its shared-memory layout.
//   k_ttc_rrs    <false>: RRSNet forward for the batch sums V and C; <true>: forward again,
//                loss gradient with the final V and C, backward; tiles stored as above.
//   k_wgrad_tc   dW = sum over samples of delta (x) activation: split-K over sample chunks,
//                operands brought in by bulk TMA loads (double-buffered, mbarrier-tracked) and
//                read as MN-major UMMA operands, accumulated in TMEM; FP32 chunk partials.
//   k_wreduce / k_adam from k_train_simt.cu finish the step.
#include "context.hpp"
#include "tc_tile.cuh"

namespace nrrs {

namespace {

using namespace tile;

constexpr int kMaxH = 3;
constexpr uint32_t kTcChunk = 4096;  // samples per weight-gradient partial

struct Arr {
    uint64_t off;  // byte offset of the tile-blocked array in the scratch
    uint32_t F;    // features per row (tile = 128 rows x F BF16)
    uint32_t pad;
};

struct TcTrainArgs {
    VertexPtrs v;
    const float* target;
    uint32_t n;
    EncodeParams enc;
    FactorParams fp;
    float loss_clamp, cost_offset, inv_n;
    int32_t train_rrs;
    const __half* table_h;
    float* table_grad;
    const uint8_t* tpack;   // training image (forward layers)
    uint32_t s_bytes;       // StatNet image bytes (at tpack + 0)
    uint32_t r_off, r_bytes;// RRSNet image
    uint8_t* act;           // tile-blocked BF16 scratch
    Arr x0, hs[kMaxH], dhs[kMaxH], dy, x1, hr[kMaxH], dhr[kMaxH], draw;
    int32_t pre;            // the hash columns of the x0 tiles are already written (k_encode_levels)
    float* dxs;             // when set: per-sample hash-lane gradients [n][32] out, no scatter here
    double* part;           // [part_rows][4]: loss_S, V, C, R per CTA
    uint32_t part_rows;
    uint32_t part_used;     // rows the StatNet and RRSNet-forward grids write
    double* loss_out;
    LossWeights lw;         // per-sample loss weights (inactive: plain means)
    unsigned* status;       // the context's NRRS_DEV_* word: wait timeouts are reported there
};

__device__ __forceinline__ uint8_t* tile_ptr(uint8_t* act, const Arr& r, uint32_t t) {
    return act + r.off + (size_t)t * 128u * r.F * 2u;
}

// bulk TMA store of one shared-memory tile to HBM, committed as its own bulk group
__device__ __forceinline__ void store_tile(void* dst, const void* src, uint32_t bytes) {
    tc::bulk_s2g(dst, src, bytes);
    tc::bulk_commit();
}

// bulk-copy a weight image into shared memory and wait for it (thread 0 issues)
__device__ __forceinline__ bool load_weights(uint8_t* sW, const uint8_t* src, uint32_t bytes,
                                             uint64_t* bar, int tid) {
    if (tid == 0) {
        tc::mbar_arrive_expect_tx(bar, bytes);
        for (uint32_t off = 0; off < bytes; off += 32768u) {
            const uint32_t b = bytes - off < 32768u ? bytes - off : 32768u;
            tc::bulk_g2s(sW + off, src + off, b, bar);
        }
    }
    return tc::mbar_wait(bar, 0, kSpin);
}

__device__ __forceinline__ double block_sum_d(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    return t;
}

// named barrier of one warpgroup (id 0 is __syncthreads)
__device__ __forceinline__ void wg_bar(int wg) {
    asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory");
}
// sync_for_mma for the 128 threads of one warpgroup
__device__ __forceinline__ void sync_for_mma_wg(int wg) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    wg_bar(wg);
}

// ---------------------------------------------------------------------------------------------
// Shared-memory plan of the StatNet kernel: the forward weight images (the backward reads them
// as MN-major operands, i.e. transposed), then per warpgroup two [128 x W] tiles that take turns
// as the input tile, activations and deltas, and the two 16-wide tiles. The ReLU masks live in
// registers: row m of every tile is produced and consumed by thread m of the warpgroup.
//
// WGS warpgroups share one copy of the weights, each running its own 128-sample tiles with its
// own tiles, TMEM columns, mbarriers and named barrier, so that one warpgroup's MMAs run while
// another waits on its epilogue or its stores. With two warpgroups of the 128-wide networks the
// 16-wide tiles live in the first 8 KB of tile buffer (H + 1) % 2 (which then holds h[H-2],
// already stored), so the plan fits one SM.
template <int W, int H, int WGS>
struct StatSmem {
    static constexpr bool kAlias = WGS > 1;
    static constexpr uint32_t kFwd = 2u * (W * kStatIn + (H - 1) * W * W + 16 * W);
    static constexpr uint32_t kW = (kFwd + 1023u) / 1024u * 1024u;
    static constexpr uint32_t kTileW = 128u * W * 2u;   // one [128 x W] tile
    static constexpr uint32_t kT16 = 128u * 16u * 2u;   // one [128 x 16] tile
    static constexpr uint32_t kPerWg = 2u * kTileW + (kAlias ? 0u : 2u * kT16);
    static constexpr uint32_t kBar = kW + WGS * kPerWg;
    static constexpr uint32_t kNumBars = 1 + 2 * WGS;  // weights, then (mma, x0 tile) per warpgroup
    static constexpr size_t kSmem = 1024 + kBar + 8 * kNumBars + 16;
    static_assert(kSmem <= 232448u, "StatNet training plan exceeds shared memory");
    __device__ static uint8_t* buf(uint8_t* base, int wg, int b) {
        return base + kW + (uint32_t)wg * kPerWg + (uint32_t)b * kTileW;
    }
    __device__ static uint8_t* dy(uint8_t* base, int wg) {
        return kAlias ? buf(base, wg, (H + 1) % 2) : buf(base, wg, 2);
    }
    __device__ static uint8_t* x1(uint8_t* base, int wg) { return dy(base, wg) + kT16; }
};

// Layer h's activations go to buffer (h + 1) % 2 (buffer 0 first holds the input tile), its
// deltas to buffer h % 2. Before an epilogue overwrites a buffer, thread 0 of the warpgroup
// waits until the bulk store that last read it has finished: the counts below are the bulk
// groups it committed since (bulk groups are per thread, so the warpgroups do not see each
// other's).
template <int W, int H, int WGS>
__global__ void __launch_bounds__(128 * WGS, 1) k_ttc_stat(const __grid_constant__ TcTrainArgs a) {
    static_assert((W == 64 || W == 128) && (H == 2 || H == 3), "tensor-core training shapes");
    static_assert(WGS == 1 || WGS == 2, "one or two warpgroups");
    using S = StatSmem<W, H, WGS>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023u) &
                                               ~uintptr_t(1023));
    const int wg = (int)(threadIdx.x >> 7);
    const int tid = (int)(threadIdx.x & 127), warp = tid >> 5;  // row and lane quarter in the warpgroup
    uint8_t* sW = base;
    uint8_t* sB[2] = {S::buf(base, wg, 0), S::buf(base, wg, 1)};
    uint8_t* sDY = S::dy(base, wg);
    uint8_t* sX1 = S::x1(base, wg);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S::kBar);
    uint64_t* bar_mma = &bars[1 + 2 * wg];
    uint64_t* bar_x0 = &bars[2 + 2 * wg];
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + S::kNumBars);
    __shared__ int s_abort[WGS];
    __shared__ double red[4 * WGS];

    if (threadIdx.x == 0) {
        for (int k = 0; k < (int)S::kNumBars; ++k) tc::mbar_init(&bars[k], 1);
        tc::fence_mbar_init();
        for (int k = 0; k < WGS; ++k) s_abort[k] = 0;
    }
    if (threadIdx.x < 32) {
        tc::tmem_alloc(tslot, W * WGS);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot + (uint32_t)(wg * W);
    if (!load_weights(sW, a.tpack, S::kFwd, &bars[0], threadIdx.x))
        for (int k = 0; k < WGS; ++k) s_abort[k] = 1;
    __syncthreads();
    unsigned flags = s_abort[wg] ? NRRS_DEV_TIMEOUT : 0u;
    uint32_t phase = 0, xphase = 0;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);

    // forward images: [W x 64], (H - 1) x [W x W], [16 x W]
    const uint8_t* wF[H + 1];
    wF[0] = sW;
    wF[1] = sW + W * kStatIn * 2;
#pragma unroll
    for (int h = 2; h <= H; ++h) wF[h] = wF[h - 1] + W * W * 2;

    double lossS = 0.0;
    const __half2* table = reinterpret_cast<const __half2*>(a.table_h);
    const uint32_t tiles = (a.n + 127) / 128;
    for (uint32_t t = blockIdx.x * WGS + wg; t < tiles && !flags; t += gridDim.x * WGS) {
        if (tid == 0) tc::bulk_wait_read();  // the previous tile's stores have left smem
        wg_bar(wg);
        const uint32_t i = t * 128 + tid;
        const bool valid = i < a.n;
        float p[3] = {0.f, 0.f, 0.f};
        bool ok = true;
        if (a.pre) {
            // hash columns from k_encode_levels: bring the tile in, add the SH and misc lanes
            if (tid == 0) {
                tc::mbar_arrive_expect_tx(bar_x0, 128u * 64u * 2u);
                tc::bulk_g2s(sB[0], tile_ptr(a.act, a.x0, t), 128u * 64u * 2u, bar_x0);
            }
            float sh[16], misc[16];
            if (valid) {
                const size_t i3 = 3 * (size_t)i;
                sh16(a.v.wi[i3], a.v.wi[i3 + 1], a.v.wi[i3 + 2], sh);
                misc_lanes(a.v, i, misc);
                if (!a.dxs) norm_pos(a.enc, a.v.pos, i, p);  // for the in-kernel scatter
            }
            ok = tc::mbar_wait(bar_x0, xphase, kSpin);
            xphase ^= 1u;
            if (valid) {
                store_chunk(sB[0], tid, 4, 64, pack8<false>(sh));
                store_chunk(sB[0], tid, 5, 64, pack8<false>(sh + 8));
                store_chunk(sB[0], tid, 6, 64, pack8<false>(misc));
            } else {
                store_chunk(sB[0], tid, 4, 64, make_uint4(0u, 0u, 0u, 0u));
                store_chunk(sB[0], tid, 5, 64, make_uint4(0u, 0u, 0u, 0u));
                store_chunk(sB[0], tid, 6, 64, make_uint4(0u, 0u, 0u, 0u));
            }
            store_chunk(sB[0], tid, 7, 64, make_uint4(0u, 0u, 0u, 0u));
        } else if (valid) {
            // ---- encode (FP16 table, FP16 tile) into buffer 0 ----
            norm_pos(a.enc, a.v.pos, i, p);
#pragma unroll 1
            for (int lq = 0; lq < 4; ++lq) {
                float f[8];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const LevelDev L = a.enc.lv[lq * 4 + j];
                    const CellCoord c = cell_of(p, L.res);
                    const float2 fv =
                        level_features_h<(W < 128)>(table, a.enc.cells, L, a.enc.hash_mask, c);
                    f[2 * j] = fv.x;
                    f[2 * j + 1] = fv.y;
                }
                store_chunk(sB[0], tid, lq, 64, pack8<false>(f));
            }
            float sh[16], misc[16];
            const size_t i3 = 3 * (size_t)i;
            sh16(a.v.wi[i3], a.v.wi[i3 + 1], a.v.wi[i3 + 2], sh);
            store_chunk(sB[0], tid, 4, 64, pack8<false>(sh));
            store_chunk(sB[0], tid, 5, 64, pack8<false>(sh + 8));
            misc_lanes(a.v, i, misc);
            store_chunk(sB[0], tid, 6, 64, pack8<false>(misc));
            store_chunk(sB[0], tid, 7, 64, make_uint4(0u, 0u, 0u, 0u));
        } else {
            zero_row(sB[0], tid, 64);
        }
        sync_for_mma_wg(wg);
        if (tid == 0) store_tile(tile_ptr(a.act, a.x0, t), sB[0], 128u * 64u * 2u);

        // ---- StatNet forward ----
        uint32_t mk[H][W / 32];
        ok &= mma_layer<kStatIn, W, false>(sB[0], wF[0], tmem, bar_mma, phase, tid);
        epilogue_relu_bits<W, false>(trow, sB[1], tid, mk[0]);
        sync_for_mma_wg(wg);
        if (tid == 0) store_tile(tile_ptr(a.act, a.hs[0], t), sB[1], S::kTileW);
#pragma unroll
        for (int h = 1; h < H; ++h) {
            ok &= mma_layer<W, W, false>(sB[h % 2], wF[h], tmem, bar_mma, phase, tid);
            if (tid == 0) tc::bulk_wait_read_n<1>();
            wg_bar(wg);
            epilogue_relu_bits<W, false>(trow, sB[(h + 1) % 2], tid, mk[h]);
            sync_for_mma_wg(wg);
            if (tid == 0) store_tile(tile_ptr(a.act, a.hs[h], t), sB[(h + 1) % 2], S::kTileW);
        }
        ok &= mma_layer<W, 16, false>(sB[H % 2], wF[H], tmem, bar_mma, phase, tid);
        float y[16];
        tc::tmem_ld16(trow, y);
        tc::tmem_wait_ld();

        // ---- loss gradient (per sample) and RRSNet input ----
        float dyv[16], x1[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) dyv[k] = 0.f, x1[k] = 0.f;
        if (valid) {
            const size_t i3 = 3 * (size_t)i;
            const float ws = a.lw.active ? sample_mul(a.lw, i, a.n).stat : 1.f;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const float d = y[c] - logf(a.target[i3 + c] + a.fp.stat_eps);
                if (a.lw.active) {
                    lossS += (double)ws * (double)d * (double)d;
                    dyv[c] = ws * (2.0f * d / 3.0f);
                } else {
                    lossS += (double)d * (double)d;
                    dyv[c] = 2.0f * d / 3.0f;
                }
            }
            glue16(a.fp, y, a.v, i, x1);
        }
        if constexpr (S::kAlias) {
            // the 16-wide tiles overwrite buffer (H + 1) % 2, whose h[H-2] store is the second
            // most recent bulk group
            if (tid == 0) tc::bulk_wait_read_n<1>();
            wg_bar(wg);
        }
        store_chunk(sDY, tid, 0, 16, pack8<false>(dyv));
        store_chunk(sDY, tid, 1, 16, pack8<false>(dyv + 8));
        store_chunk(sX1, tid, 0, 16, pack8<true>(x1));  // RRSNet input: BF16
        store_chunk(sX1, tid, 1, 16, pack8<true>(x1 + 8));
        sync_for_mma_wg(wg);
        if (tid == 0) {
            store_tile(tile_ptr(a.act, a.dy, t), sDY, 128u * 16u * 2u);
            store_tile(tile_ptr(a.act, a.x1, t), sX1, 128u * 16u * 2u);
        }

        // ---- backward: delta of layer h -> buffer h % 2 ----
        ok &= mma_layer_t<16, W, W, false>(sDY, wF[H], tmem, bar_mma, phase, tid);
        if (tid == 0) {
            // the first delta goes to buffer (H - 1) % 2: with the 16-wide tiles inside it, the
            // dy and x1 stores must have left it as well
            if constexpr (S::kAlias) tc::bulk_wait_read();
            else tc::bulk_wait_read_n<3>();  // since: h[H-1], dy, x1
        }
        wg_bar(wg);
        epilogue_mask_bits<W, false>(trow, mk[H - 1], sB[(H - 1) % 2], tid);
        sync_for_mma_wg(wg);
        if (tid == 0) store_tile(tile_ptr(a.act, a.dhs[H - 1], t), sB[(H - 1) % 2], S::kTileW);
#pragma unroll
        for (int h = H - 1; h >= 1; --h) {
            ok &= mma_layer_t<W, W, W, false>(sB[h % 2], wF[h], tmem, bar_mma, phase, tid);
            if (tid == 0) {
                if (h == H - 1) tc::bulk_wait_read_n<3>();  // since: dy, x1, d[H-1]
                else tc::bulk_wait_read_n<1>();             // since: d[h]
            }
            wg_bar(wg);
            epilogue_mask_bits<W, false>(trow, mk[h - 1], sB[(h - 1) % 2], tid);
            sync_for_mma_wg(wg);
            if (tid == 0) store_tile(tile_ptr(a.act, a.dhs[h - 1], t), sB[(h - 1) % 2], S::kTileW);
        }
        // input gradient of the 32 hash lanes (per sample; 1/n applied below)
        ok &= mma_layer_t<W, 32, kStatIn, false>(sB[0], wF[0], tmem, bar_mma, phase, tid);
        float dx[32];
        tc::tmem_ld16(trow, dx);
        tc::tmem_ld16(trow + 16, dx + 16);
        tc::tmem_wait_ld();
        tc::fence_before_sync();
        wg_bar(wg);  // TMEM free for the next tile
        if (valid && a.dxs) {
            // the level-major scatter kernel applies them; stored level-major ([16][n] pairs),
            // so that kernel reads each level's gradients coalesced
            float2* d = reinterpret_cast<float2*>(a.dxs);
#pragma unroll
            for (int l = 0; l < kMaxLevels; ++l) d[(size_t)l * a.n + i] = make_float2(dx[2 * l], dx[2 * l + 1]);
        } else if (valid) {
            const unsigned lanes = valid_lanes(i - (uint32_t)(tid & 31), a.n);
#pragma unroll 2
            for (int l = 0; l < kMaxLevels; ++l) {
                const LevelDev L = a.enc.lv[l];
                const CellCoord c = cell_of(p, L.res);
                warp_scatter_level(a.table_grad, L, a.enc.hash_mask, c, dx[2 * l] * a.inv_n,
                                   dx[2 * l + 1] * a.inv_n, lanes);
            }
        }
        if (!ok) s_abort[wg] = 1;
        wg_bar(wg);
        if (s_abort[wg]) flags |= NRRS_DEV_TIMEOUT;
    }
    const double s0 = block_sum_d(lossS, red);
    if (threadIdx.x == 0) a.part[4 * blockIdx.x + 0] = s0;
    if (tid == 0) tc::bulk_wait_all();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_dealloc(*tslot, W * WGS);
    }
    if (flags && tid == 0) atomicOr(a.status, flags);
}

// ---------------------------------------------------------------------------------------------
// Level-major scatter of the hash-grid gradient (split training): work item (level l, tile t) in
// l-major order, so the reductions in flight target the gradient slice of one level (at most
// 2^T x 8 bytes), which stays in L2, instead of the whole table. dxs: the per-sample hash-lane
// gradients that k_ttc_stat wrote, [16][n] float pairs; the 1/n of the batch mean is applied
// here. Levels [level_begin, level_end) of the launch.
// FP32 table-gradient bytes per scatter launch of the split step (a fraction of L2)
constexpr uint64_t kScatterGroupBytes = 40ull << 20;

struct ScatterLvArgs {
    EncodeParams enc;
    const float* pos;
    const float* dxs;
    float* table_grad;
    uint32_t n;
    float inv_n;
    uint32_t level_begin, level_end;
};

__global__ void __launch_bounds__(128) k_scatter_levels(const __grid_constant__ ScatterLvArgs a) {
    const uint32_t tiles = (a.n + 127) / 128;
    const uint32_t items = (a.level_end - a.level_begin) * tiles;
    const float2* d = reinterpret_cast<const float2*>(a.dxs);
    for (uint32_t w = blockIdx.x; w < items; w += gridDim.x) {
        const uint32_t lq = w / tiles, t = w - lq * tiles;
        const uint32_t l = a.level_begin + lq;
        const uint32_t i = t * 128 + threadIdx.x;
        if (i >= a.n) continue;
        float p[3];
        norm_pos(a.enc, a.pos, i, p);
        const float2 g = d[(size_t)l * a.n + i];
        const LevelDev L = a.enc.lv[l];
        const CellCoord c = cell_of(p, L.res);
        warp_scatter_level(a.table_grad, L, a.enc.hash_mask, c, g.x * a.inv_n, g.y * a.inv_n,
                           valid_lanes(i - (threadIdx.x & 31u), a.n));
    }
}

// ---------------------------------------------------------------------------------------------
// RRSNet: forward images, then per warpgroup the BF16 input tile, two [128 x W] tiles
// (activations of layer h in buffer h % 2, deltas of layer h in buffer (h + 1) % 2) and the
// output-delta tile. WGS warpgroups share the weights as in the StatNet kernel.
template <int W, int H, int WGS>
struct RrsSmem {
    static constexpr uint32_t kFwd = 2u * (W * kRrsIn + (H - 1) * W * W + 16 * W);
    static constexpr uint32_t kW = (kFwd + 1023u) / 1024u * 1024u;
    static constexpr uint32_t kTileW = 128u * W * 2u;
    static constexpr uint32_t kT16 = 128u * 16u * 2u;
    static constexpr uint32_t kPerWg = kT16 + 2u * kTileW + kT16;  // x1, b0, b1, draw
    static constexpr uint32_t kBar = kW + WGS * kPerWg;
    static constexpr uint32_t kNumBars = 1 + 2 * WGS;  // weights, then (mma, x1 tile) per warpgroup
    static constexpr size_t kSmem = 1024 + kBar + 8 * kNumBars + 16;
    static_assert(kSmem <= 232448u, "RRSNet training plan exceeds shared memory");
    __device__ static uint8_t* x1(uint8_t* base, int wg) { return base + kW + (uint32_t)wg * kPerWg; }
    __device__ static uint8_t* buf(uint8_t* base, int wg, int b) {
        return x1(base, wg) + kT16 + (uint32_t)b * kTileW;
    }
    __device__ static uint8_t* dr(uint8_t* base, int wg) { return buf(base, wg, 2); }
};

__device__ __forceinline__ float rel_contrib_tc(const TcTrainArgs& a, uint32_t i) {
    const size_t i3 = 3 * (size_t)i;
    float acc = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) acc += a.v.thp[i3 + c] * a.target[i3 + c];
    const float ref = (a.v.ref ? a.v.ref[i] : 0.5f) + a.fp.ref_eps;
    const float r = acc / 3.0f / ref;
    return r < a.loss_clamp ? r : a.loss_clamp;
}

template <int W, int H, int WGS, bool BACKWARD>
__global__ void __launch_bounds__(128 * WGS, 1) k_ttc_rrs(const __grid_constant__ TcTrainArgs a) {
    static_assert((W == 64 || W == 128) && (H == 2 || H == 3), "tensor-core training shapes");
    static_assert(WGS == 1 || WGS == 2, "one or two warpgroups");
    using S = RrsSmem<W, H, WGS>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023u) &
                                               ~uintptr_t(1023));
    const int wg = (int)(threadIdx.x >> 7);
    const int tid = (int)(threadIdx.x & 127), warp = tid >> 5;  // row and lane quarter in the warpgroup
    uint8_t* sW = base;
    uint8_t* sX1 = S::x1(base, wg);
    uint8_t* sB[2] = {S::buf(base, wg, 0), S::buf(base, wg, 1)};
    uint8_t* sDR = S::dr(base, wg);
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S::kBar);
    uint64_t* bar_mma = &bars[1 + 2 * wg];
    uint64_t* bar_x1 = &bars[2 + 2 * wg];
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + S::kNumBars);
    __shared__ int s_abort[WGS];
    __shared__ double red[4 * WGS];
    __shared__ double s_tot[4];

    if (threadIdx.x == 0) {
        for (int k = 0; k < (int)S::kNumBars; ++k) tc::mbar_init(&bars[k], 1);
        tc::fence_mbar_init();
        for (int k = 0; k < WGS; ++k) s_abort[k] = 0;
    }
    if (BACKWARD) {
        // batch sums of the loss partials (rows written by the StatNet and forward launches),
        // in a fixed order, so every CTA holds the same V and C
        double t0 = 0.0, t1 = 0.0, t2 = 0.0, t3 = 0.0;
        for (uint32_t b = threadIdx.x; b < a.part_used; b += blockDim.x) {
            t0 += a.part[4 * b + 0];
            t1 += a.part[4 * b + 1];
            t2 += a.part[4 * b + 2];
            t3 += a.part[4 * b + 3];
        }
        t0 = block_sum_d(t0, red);
        t1 = block_sum_d(t1, red);
        t2 = block_sum_d(t2, red);
        t3 = block_sum_d(t3, red);
        if (threadIdx.x == 0) s_tot[0] = t0, s_tot[1] = t1, s_tot[2] = t2, s_tot[3] = t3;
        __syncthreads();
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            const double Vm = s_tot[1] / (double)a.n, Cm = s_tot[2] / (double)a.n;
            a.loss_out[0] = s_tot[0] / (3.0 * (double)a.n);
            a.loss_out[1] = a.train_rrs ? (a.lw.active ? Vm * Cm + s_tot[3] / (double)a.n : Vm * Cm)
                                        : 0.0;
        }
        if (!a.train_rrs) return;  // StatNet-only steps: losses are all this launch writes
    }
    if (threadIdx.x < 32) {
        tc::tmem_alloc(tslot, W * WGS);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot + (uint32_t)(wg * W);
    float Vf = 0.f, Cf = 0.f;
    if (BACKWARD) {
        Vf = (float)(s_tot[1] / (double)a.n);
        Cf = (float)(s_tot[2] / (double)a.n);
    }
    if (!load_weights(sW, a.tpack + a.r_off, S::kFwd, &bars[0], threadIdx.x))
        for (int k = 0; k < WGS; ++k) s_abort[k] = 1;
    __syncthreads();
    unsigned flags = s_abort[wg] ? NRRS_DEV_TIMEOUT : 0u;
    uint32_t phase = 0, xphase = 0;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    // forward images: [W x 16], (H - 1) x [W x W], [16 x W]
    const uint8_t* wF[H + 1];
    wF[0] = sW;
    wF[1] = sW + W * kRrsIn * 2;
#pragma unroll
    for (int h = 2; h <= H; ++h) wF[h] = wF[h - 1] + W * W * 2;

    double sumV = 0.0, sumC = 0.0, sumR = 0.0;
    const uint32_t tiles = (a.n + 127) / 128;
    for (uint32_t t = blockIdx.x * WGS + wg; t < tiles && !flags; t += gridDim.x * WGS) {
        if (tid == 0) {
            tc::bulk_wait_read();
            tc::mbar_arrive_expect_tx(bar_x1, 128u * 16u * 2u);
            tc::bulk_g2s(sX1, tile_ptr(a.act, a.x1, t), 128u * 16u * 2u, bar_x1);
        }
        bool ok = tc::mbar_wait(bar_x1, xphase, kSpin);
        xphase ^= 1u;
        wg_bar(wg);
        const uint32_t i = t * 128 + tid;
        const bool valid = i < a.n;

        uint32_t mk[H][W / 32];
        ok &= mma_layer<kRrsIn, W, true>(sX1, wF[0], tmem, bar_mma, phase, tid);
        epilogue_relu_bits<W, true>(trow, sB[0], tid, mk[0]);
        sync_for_mma_wg(wg);
        if (BACKWARD && tid == 0) store_tile(tile_ptr(a.act, a.hr[0], t), sB[0], S::kTileW);
#pragma unroll
        for (int h = 1; h < H; ++h) {
            ok &= mma_layer<W, W, true>(sB[(h - 1) % 2], wF[h], tmem, bar_mma, phase, tid);
            if (BACKWARD) {
                if (tid == 0) tc::bulk_wait_read_n<1>();  // since: h[h-1]
                wg_bar(wg);
            }
            epilogue_relu_bits<W, true>(trow, sB[h % 2], tid, mk[h]);
            sync_for_mma_wg(wg);
            if (BACKWARD && tid == 0) store_tile(tile_ptr(a.act, a.hr[h], t), sB[h % 2], S::kTileW);
        }
        ok &= mma_layer<W, 16, true>(sB[(H - 1) % 2], wF[H], tmem, bar_mma, phase, tid);
        float r16[16];
        tc::tmem_ld16(trow, r16);
        tc::tmem_wait_ld();
        const float raw = r16[0];
        float q = 0.f, r = 0.f;
        SampleMul mu{1.f, 1.f, 1.f, 0.f};
        if (valid) {
            q = act_sigma(raw);
            r = rel_contrib_tc(a, i);
            if (a.lw.active) mu = sample_mul(a.lw, i, a.n);
        }
        if (!BACKWARD) {
            if (valid) {
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
            tc::fence_before_sync();
            wg_bar(wg);
        } else {
            float dr[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) dr[k] = 0.f;
            if (valid) {
                if (a.lw.active)
                    dr[0] = (mu.var * (-(r * r) / (q * q)) * Cf + mu.cost * Vf +
                             mu.reg * (2.0f * logf(q) / q)) * act_sigma_grad(raw);
                else
                    dr[0] = (-(r * r) / (q * q) * Cf + Vf) * act_sigma_grad(raw);
            }
            store_chunk(sDR, tid, 0, 16, pack8<true>(dr));
            store_chunk(sDR, tid, 1, 16, pack8<true>(dr + 8));
            sync_for_mma_wg(wg);
            if (tid == 0) store_tile(tile_ptr(a.act, a.draw, t), sDR, 128u * 16u * 2u);
            ok &= mma_layer_t<16, W, W, true>(sDR, wF[H], tmem, bar_mma, phase, tid);
            if (tid == 0) tc::bulk_wait_read_n<2>();  // since: h[H-1], draw
            wg_bar(wg);
            epilogue_mask_bits<W, true>(trow, mk[H - 1], sB[H % 2], tid);
            sync_for_mma_wg(wg);
            if (tid == 0) store_tile(tile_ptr(a.act, a.dhr[H - 1], t), sB[H % 2], S::kTileW);
#pragma unroll
            for (int h = H - 1; h >= 1; --h) {
                ok &= mma_layer_t<W, W, W, true>(sB[(h + 1) % 2], wF[h], tmem, bar_mma, phase, tid);
                if (tid == 0) {
                    if (h == H - 1) tc::bulk_wait_read_n<2>();  // since: draw, d[H-1]
                    else tc::bulk_wait_read_n<1>();             // since: d[h]
                }
                wg_bar(wg);
                epilogue_mask_bits<W, true>(trow, mk[h - 1], sB[h % 2], tid);
                sync_for_mma_wg(wg);
                if (tid == 0) store_tile(tile_ptr(a.act, a.dhr[h - 1], t), sB[h % 2], S::kTileW);
            }
            tc::fence_before_sync();
            wg_bar(wg);
        }
        if (!ok) s_abort[wg] = 1;
        wg_bar(wg);
        if (s_abort[wg]) flags |= NRRS_DEV_TIMEOUT;
    }
    if (!BACKWARD) {
        const double v = block_sum_d(sumV, red);
        const double c = block_sum_d(sumC, red);
        const double rr = block_sum_d(sumR, red);
        if (threadIdx.x == 0) {
            a.part[4 * blockIdx.x + 1] = v;
            a.part[4 * blockIdx.x + 2] = c;
            a.part[4 * blockIdx.x + 3] = rr;
        }
    }
    if (tid == 0) tc::bulk_wait_all();
    tc::fence_before_sync();
    __syncthreads();
    if (threadIdx.x < 32) {
        tc::fence_after_sync();
        tc::tmem_dealloc(*tslot, W * WGS);
    }
    if (flags && tid == 0) atomicOr(a.status, flags);
}

// ---------------------------------------------------------------------------------------------
struct TcJob {
    uint32_t bf16;    // operand type of this layer's tiles: 1 = BF16 (RRSNet), 0 = FP16 (StatNet)
    uint32_t pad;
    uint64_t d_off;   // deltas: tile-blocked array
    uint32_t Fd, Mv;  // its features, valid output rows
    uint32_t Fa, Nv;  // activations: features (= N of the MMA), valid input columns
    uint64_t a_off;
    uint32_t out, ldw;  // offset of the layer in the MLP gradient vector, its row stride
};

struct TcWGradArgs {
    const uint8_t* act;
    uint32_t n, chunks, total;
    uint32_t chunk;             // samples per chunk (a multiple of 64, at least kTcChunk)
    float* partial;
    int32_t njobs;
    TcJob job[8];
    unsigned* status;           // the context's NRRS_DEV_* word
};

constexpr uint32_t kWgBuf = 16384;  // bytes per operand stage (64 samples x up to 128 features)

template <int N>
__device__ __forceinline__ void wgrad_epilogue(uint32_t trow, const TcJob& j, float* out, int m) {
#pragma unroll
    for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        tc::tmem_ld16(trow + c0, v);
        tc::tmem_wait_ld();
        if ((uint32_t)m < j.Mv) {
#pragma unroll
            for (int k = 0; k < 16; ++k)
                if ((uint32_t)(c0 + k) < j.Nv) out[(size_t)m * j.ldw + c0 + k] = v[k];
        }
    }
}

__global__ void __launch_bounds__(128, 1) k_wgrad_tc(const __grid_constant__ TcWGradArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023u) &
                                               ~uintptr_t(1023));
    uint8_t* sA[2] = {base, base + 2 * kWgBuf};
    uint8_t* sB[2] = {base + kWgBuf, base + 3 * kWgBuf};
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + 4 * kWgBuf);  // load[2], mma[2], done
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 5);
    __shared__ int s_fail;
    const int tid = threadIdx.x, warp = tid >> 5;
    const TcJob& j = a.job[blockIdx.y];
    const uint32_t c = blockIdx.x;
    const uint32_t s0 = c * a.chunk;
    const uint32_t s1 = min(a.n, s0 + a.chunk);
    const uint32_t stages = (s1 - s0 + 63) / 64;

    if (tid == 0) {
        for (int k = 0; k < 5; ++k) tc::mbar_init(&bars[k], 1);
        tc::fence_mbar_init();
        s_fail = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(tslot, 128);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot;

    if (tid == 0) {
        const uint32_t bytesA = 64u * j.Fd * 2u, bytesB = 64u * j.Fa * 2u;
        const uint32_t lboA = j.Fd * 16u, lboB = j.Fa * 16u;
        const uint32_t idesc = tc::idesc_f16_major(j.Fa, j.bf16, 1u, 1u);
        auto issue = [&](uint32_t s) {
            const uint32_t b = s & 1u;
            const uint32_t smp = s0 + 64u * s;        // first sample of the stage
            const uint32_t tile = smp >> 7, half = (smp >> 6) & 1u;
            const uint8_t* ga = a.act + j.d_off + (size_t)tile * 128u * j.Fd * 2u + half * bytesA;
            const uint8_t* gb = a.act + j.a_off + (size_t)tile * 128u * j.Fa * 2u + half * bytesB;
            tc::mbar_arrive_expect_tx(&bars[b], bytesA + bytesB);
            tc::bulk_g2s(sA[b], ga, bytesA, &bars[b]);
            tc::bulk_g2s(sB[b], gb, bytesB, &bars[b]);
        };
        bool ok = true;
        issue(0);
        for (uint32_t s = 0; s < stages && ok; ++s) {
            if (s + 1 < stages) {
                const uint32_t nb = (s + 1) & 1u;
                if (s + 1 >= 2) ok &= tc::mbar_wait(&bars[2 + nb], ((s - 1) >> 1) & 1u, kSpin);
                issue(s + 1);
            }
            const uint32_t b = s & 1u;
            ok &= tc::mbar_wait(&bars[b], (s >> 1) & 1u, kSpin);
            tc::fence_after_sync();
            const uint32_t a0 = tc::smem_u32(sA[b]), b0 = tc::smem_u32(sB[b]);
#pragma unroll
            for (int kk = 0; kk < 4; ++kk) {
                const uint64_t ad = tc::smem_desc(a0 + kk * 2 * lboA, lboA, 128);
                const uint64_t bd = tc::smem_desc(b0 + kk * 2 * lboB, lboB, 128);
                tc::mma_f16(tmem, ad, bd, idesc, (s > 0 || kk > 0) ? 1u : 0u);
            }
            tc::mma_commit(&bars[2 + b]);
        }
        tc::mma_commit(&bars[4]);
        if (!ok) s_fail = 1;
    }
    __syncwarp();
    const bool done = tc::mbar_wait(&bars[4], 0, kSpin);
    tc::fence_after_sync();
    __syncthreads();
    if (!s_fail && done) {
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        float* out = a.partial + (size_t)c * a.total + j.out;
        const int m = tid;
        if (j.Fa == 64) wgrad_epilogue<64>(trow, j, out, m);
        else if (j.Fa == 16) wgrad_epilogue<16>(trow, j, out, m);
        else wgrad_epilogue<128>(trow, j, out, m);
    }
    if (tid == 0 && (s_fail || !done)) atomicOr(a.status, NRRS_DEV_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, 128);
    }
}

// scratch layout of the tensor-core path: tile-blocked BF16 arrays
struct TcLayout {
    Arr x0, hs[kMaxH], dhs[kMaxH], dy, x1, hr[kMaxH], dhr[kMaxH], draw;
    uint64_t act_bytes;
};

TcLayout tc_layout(const nrrs_config& c, uint32_t max_n) {
    const uint64_t tiles = (max_n + 127) / 128;
    TcLayout L{};
    uint64_t off = 0;
    auto take = [&](Arr& r, uint32_t F) {
        r.off = off;
        r.F = F;
        off += tiles * 128u * F * 2u;
        off = (off + 255) / 256 * 256;
    };
    take(L.x0, 64);
    for (int h = 0; h < c.statnet_hidden; ++h) take(L.hs[h], c.statnet_width);
    for (int h = 0; h < c.statnet_hidden; ++h) take(L.dhs[h], c.statnet_width);
    take(L.dy, 16);
    take(L.x1, 16);
    for (int h = 0; h < c.rrsnet_hidden; ++h) take(L.hr[h], c.rrsnet_width);
    for (int h = 0; h < c.rrsnet_hidden; ++h) take(L.dhr[h], c.rrsnet_width);
    take(L.draw, 16);
    L.act_bytes = off;
    return L;
}

// after_stat() is called once the StatNet kernel is launched (the split step forks the
// table-gradient scatter there)
template <int W, int H, class AfterStat>
cudaError_t launch_ttc(nrrs_ctx* ctx, TcTrainArgs& a, cudaStream_t s, bool train_rrs,
                       AfterStat after_stat) {
    // the 128-wide networks run two warpgroups per CTA over one weight copy (one CTA per SM);
    // the 64-wide ones fit three single-warpgroup CTAs per SM
    constexpr int WGS = W == 128 ? 2 : 1;
    constexpr int kThreads = 128 * WGS;
    using SS = StatSmem<W, H, WGS>;
    using RS = RrsSmem<W, H, WGS>;
    auto ks = k_ttc_stat<W, H, WGS>;
    auto kr0 = k_ttc_rrs<W, H, WGS, false>;
    auto kr1 = k_ttc_rrs<W, H, WGS, true>;
    cudaError_t e = cudaFuncSetAttribute(ks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SS::kSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kr0, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS::kSmem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kr1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RS::kSmem);
    if (e != cudaSuccess) return e;
    // CTAs needed to give every warpgroup at least one tile
    const uint32_t ctas = ((a.n + 127) / 128 + WGS - 1) / WGS;
    auto grid_of = [&](const void* k, size_t smem) {
        uint32_t g = (uint32_t)(ctx->sm_count * resident_ctas(k, kThreads, smem, 8));
        return g > ctas ? ctas : g;
    };
    const uint32_t gs = grid_of((const void*)ks, SS::kSmem);
    const uint32_t g = grid_of((const void*)kr0, RS::kSmem);
    a.part_used = gs > g ? gs : g;
    if (a.part_used > a.part_rows) return cudaErrorInvalidConfiguration;
    {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_STAT, s);
        ks<<<gs, kThreads, SS::kSmem, s>>>(a);
    }
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = after_stat()) != cudaSuccess) return e;
    if (train_rrs) {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_RRS, s);
        kr0<<<g, kThreads, RS::kSmem, s>>>(a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        kr1<<<g, kThreads, RS::kSmem, s>>>(a);
    } else {
        // losses without the RRSNet: only the StatNet sum is present
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_RRS, s);
        kr1<<<1, kThreads, RS::kSmem, s>>>(a);
    }
    return cudaGetLastError();
}

}  // namespace

bool train_tc_supported(const nrrs_config& c) {
    return c.precision != NRRS_PREC_FP32 && c.statnet_width == c.rrsnet_width &&
           (c.statnet_width == 64 || c.statnet_width == 128) && c.statnet_hidden == c.rrsnet_hidden &&
           (c.statnet_hidden == 2 || c.statnet_hidden == 3);
}

size_t train_tc_scratch_bytes(const nrrs_config& c, uint32_t n, int sm_count) {
    const TcLayout L = tc_layout(c, n);
    const uint64_t mlp = (uint64_t)64 * c.statnet_width + (uint64_t)(c.statnet_hidden - 1) *
                         c.statnet_width * c.statnet_width + 3ull * c.statnet_width +
                         16ull * c.rrsnet_width + (uint64_t)(c.rrsnet_hidden - 1) * c.rrsnet_width *
                         c.rrsnet_width + (uint64_t)c.rrsnet_width;
    const uint64_t chunks = (n + kTcChunk - 1) / kTcChunk;
    // + split mode: the per-sample hash-lane gradients [n][32] FP32
    return L.act_bytes + sizeof(double) * 4 * (uint64_t)sm_count * 16 + sizeof(float) * chunks * mlp +
           sizeof(float) * 32ull * n + 1024;
}

cudaError_t launch_wreduce(const float* partial, uint32_t chunks, uint32_t total, float* grad,
                           float scale, cudaStream_t s);
int train_step_tc(nrrs_ctx* ctx, const VertexPtrs& v, const float* target, uint32_t n,
                  double* loss_dev, cudaStream_t s, bool apply, const LossWeights* lw) {
    const nrrs_config& c = ctx->cfg;
    const TcLayout L = tc_layout(c, c.max_train);
    const bool train_rrs = c.step >= 3;
    // Weight-gradient chunks: as many as fill one wave of the weight-gradient grid (one CTA per
    // chunk and layer), each at least kTcChunk samples so that the partials fit the scratch
    // sized by kTcChunk. 262,144 samples and 8 layers on 444 CTA slots: 55 chunks of 4,800
    // (64 chunks of 4,096 were 1.15 waves).
    const size_t wsm = 1024 + 4 * kWgBuf + 64;
    const uint32_t njobs = (uint32_t)(c.statnet_hidden + 1) * (train_rrs ? 2u : 1u);
    const uint32_t slots =
        (uint32_t)ctx->sm_count * (uint32_t)resident_ctas((const void*)k_wgrad_tc, 128, wsm, 4);
    const uint32_t per_wave = slots / njobs > 0 ? slots / njobs : 1u;
    uint32_t chunk_len = ((n + per_wave - 1) / per_wave + 63u) / 64u * 64u;
    if (chunk_len < kTcChunk) chunk_len = kTcChunk;
    const uint64_t chunks = (n + chunk_len - 1) / chunk_len;
    const uint64_t mlp = ctx->n_stat + ctx->n_rrs;
    uint8_t* act = reinterpret_cast<uint8_t*>(ctx->train_scratch);
    double* part = reinterpret_cast<double*>(act + L.act_bytes);
    const uint32_t part_rows = (uint32_t)ctx->sm_count * 16;
    float* partial = reinterpret_cast<float*>(reinterpret_cast<uint8_t*>(part) +
                                              sizeof(double) * 4 * (size_t)part_rows);
    const uint64_t chunks_max = (c.max_train + kTcChunk - 1) / kTcChunk;
    float* dxs = reinterpret_cast<float*>(
        (reinterpret_cast<uintptr_t>(partial + chunks_max * mlp) + 15u) & ~uintptr_t(15));
    const bool split = ctx->train_split != 0;
    // the split step zeroes the table gradient level group by level group right before that
    // group's scatter (below); here only what the other kernels accumulate into
    const uint64_t zero_from = split ? ctx->n_table : 0;
    cudaError_t e = cudaMemsetAsync(ctx->grads + zero_from, 0,
                                    sizeof(float) * (ctx->n_params - zero_from), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(part, 0, sizeof(double) * 4 * part_rows, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(partial, 0, sizeof(float) * chunks * mlp, s);
    if (e != cudaSuccess) {
        ctx->last_error = std::string("train memset: ") + cudaGetErrorString(e);
        return NRRS_ERR_CUDA;
    }
    TcTrainArgs a{};
    a.v = v;
    a.target = target;
    a.n = n;
    a.enc = ctx->enc;
    a.fp.stat_eps = c.stat_eps;
    a.fp.ref_eps = c.ref_eps;
    a.loss_clamp = c.loss_clamp_max;
    a.cost_offset = c.cost_offset;
    a.inv_n = 1.0f / (float)n;
    a.train_rrs = train_rrs;
    a.table_h = ctx->table_h;
    a.table_grad = ctx->grads;
    a.tpack = reinterpret_cast<const uint8_t*>(ctx->tpack);
    const int W = c.statnet_width, H = c.statnet_hidden;
    a.s_bytes = 2u * (uint32_t)(W * kStatIn + (H - 1) * W * W + 16 * W);
    a.r_off = a.s_bytes;
    a.r_bytes = 2u * (uint32_t)(W * kRrsIn + (H - 1) * W * W + 16 * W);
    a.act = act;
    a.x0 = L.x0; a.dy = L.dy; a.x1 = L.x1; a.draw = L.draw;
    for (int h = 0; h < kMaxH; ++h) {
        a.hs[h] = L.hs[h]; a.dhs[h] = L.dhs[h]; a.hr[h] = L.hr[h]; a.dhr[h] = L.dhr[h];
    }
    a.part = part;
    a.part_rows = part_rows;
    a.loss_out = loss_dev ? loss_dev : ctx->loss_dev;
    a.status = &ctx->scr->status;
    if (lw) a.lw = *lw;
    if (split) {
        // hash columns of the x0 tiles, level-major (FP16, the StatNet training precision)
        EncodeLvArgs ea{};
        ea.enc = ctx->enc;
        ea.segs.n = 1;
        ea.segs.s[0].offset = 0;
        ea.segs.s[0].count = n;
        ea.segs.s[0].tile_start = 0;
        ea.segs.total_tiles = (n + 127) / 128;
        ea.pos = v.pos;
        ea.table_h = ctx->table_h;
        ea.out = act + L.x0.off;
        ea.tile_bytes = 128u * 64u * 2u;
        ea.kdim = 64;
        {
            ProfScope ps(ctx, NRRS_KERNEL_TRAIN_ENCODE, s);
            e = launch_encode_levels(ea, false, ctx->sm_count, s);
        }
        if (e != cudaSuccess) {
            ctx->last_error = std::string("training encoding launch: ") + cudaGetErrorString(e);
            return NRRS_ERR_CUDA;
        }
        a.pre = 1;
        a.dxs = dxs;
    }
    // Split step: the table-gradient scatter needs only the StatNet kernel's lane gradients,
    // and nothing before Adam reads the table gradient, so it runs on the context's side
    // stream, forked after the StatNet launch, while the RRSNet kernels and the weight
    // gradients run here; the step joins it before Adam (or before returning the gradients).
    // Level groups of at most kScatterGroupBytes of FP32 gradient, each zeroed right before its
    // scatter: the zeroing writes whole sectors into L2, so the reductions that follow hit
    // there. Zeroed at the start of the step, the slices were evicted by the kernels in between,
    // and every first reduction into a sector read its zeros back from HBM as a random 32-byte
    // access.
    auto scatter_table = [&](cudaStream_t ss) -> cudaError_t {
        ScatterLvArgs sa{};
        sa.enc = ctx->enc;
        sa.pos = v.pos;
        sa.dxs = dxs;
        sa.table_grad = ctx->grads;
        sa.n = n;
        sa.inv_n = a.inv_n;
        const uint32_t tiles = (n + 127) / 128;
        const uint32_t g_max =
            (uint32_t)(ctx->sm_count * resident_ctas((const void*)k_scatter_levels, 128, 0, 16));
        const int nl = c.n_levels;
        auto level_rows = [&](int l) -> uint64_t {
            const LevelDev& lv = ctx->enc.lv[l];
            const uint64_t r = (uint64_t)lv.res + 1;
            return lv.dense ? r * r * r : (uint64_t)ctx->enc.hash_mask + 1;
        };
        cudaError_t es = cudaSuccess;
        for (int l0 = 0; l0 < nl && es == cudaSuccess;) {
            const uint64_t row0 = ctx->enc.lv[l0].offset;
            uint64_t row1 = row0 + level_rows(l0);
            int l1 = l0 + 1;
            while (l1 < nl && (ctx->enc.lv[l1].offset + level_rows(l1) - row0) * 8u <=
                                  kScatterGroupBytes) {
                row1 = ctx->enc.lv[l1].offset + level_rows(l1);
                ++l1;
            }
            es = cudaMemsetAsync(ctx->grads + 2 * row0, 0, sizeof(float) * 2 * (row1 - row0), ss);
            if (es != cudaSuccess) break;
            sa.level_begin = (uint32_t)l0;
            sa.level_end = (uint32_t)l1;
            const uint32_t items = (uint32_t)(l1 - l0) * tiles;
            const uint32_t g = g_max < items ? g_max : items;
            ProfScope ps(ctx, NRRS_KERNEL_TRAIN_SCATTER, ss);
            if (g) k_scatter_levels<<<g, 128, 0, ss>>>(sa);
            es = cudaGetLastError();
            l0 = l1;
        }
        return es;
    };
    bool forked = false;
    auto after_stat = [&]() -> cudaError_t {
        if (!split) return cudaSuccess;
        cudaError_t ef = cudaEventRecord(ctx->ev_fork, s);
        if (ef == cudaSuccess) ef = cudaStreamWaitEvent(ctx->side, ctx->ev_fork, 0);
        if (ef != cudaSuccess) return ef;
        forked = true;
        ef = scatter_table(ctx->side);
        const cudaError_t ej = cudaEventRecord(ctx->ev_join, ctx->side);
        return ef != cudaSuccess ? ef : ej;
    };
    auto join = [&]() {
        if (forked) cudaStreamWaitEvent(s, ctx->ev_join, 0);
        forked = false;
    };
    if (W == 64)
        e = H == 2 ? launch_ttc<64, 2>(ctx, a, s, train_rrs, after_stat)
                   : launch_ttc<64, 3>(ctx, a, s, train_rrs, after_stat);
    else
        e = H == 2 ? launch_ttc<128, 2>(ctx, a, s, train_rrs, after_stat)
                   : launch_ttc<128, 3>(ctx, a, s, train_rrs, after_stat);
    if (e != cudaSuccess) {
        join();
        ctx->last_error = std::string("tensor-core train launch: ") + cudaGetErrorString(e);
        return NRRS_ERR_CUDA;
    }

    TcWGradArgs w{};
    w.act = act;
    w.n = n;
    w.chunks = (uint32_t)chunks;
    w.chunk = chunk_len;
    w.status = &ctx->scr->status;
    w.total = (uint32_t)mlp;
    w.partial = partial;
    int nj = 0;
    uint32_t off = 0;
    w.job[nj++] = TcJob{0, 0, L.dhs[0].off, (uint32_t)W, (uint32_t)W, 64, 64, L.x0.off, off, kStatIn};
    off += W * kStatIn;
    for (int h = 1; h < H; ++h) {
        w.job[nj++] = TcJob{0, 0, L.dhs[h].off, (uint32_t)W, (uint32_t)W, (uint32_t)W, (uint32_t)W,
                            L.hs[h - 1].off, off, (uint32_t)W};
        off += W * W;
    }
    w.job[nj++] = TcJob{0, 0, L.dy.off, 16, 3, (uint32_t)W, (uint32_t)W, L.hs[H - 1].off, off, (uint32_t)W};
    off += 3 * W;
    if (train_rrs) {
        w.job[nj++] = TcJob{1, 0, L.dhr[0].off, (uint32_t)W, (uint32_t)W, 16, 16, L.x1.off, off, kRrsIn};
        off += W * kRrsIn;
        for (int h = 1; h < H; ++h) {
            w.job[nj++] = TcJob{1, 0, L.dhr[h].off, (uint32_t)W, (uint32_t)W, (uint32_t)W, (uint32_t)W,
                                L.hr[h - 1].off, off, (uint32_t)W};
            off += W * W;
        }
        w.job[nj++] = TcJob{1, 0, L.draw.off, 16, 1, (uint32_t)W, (uint32_t)W, L.hr[H - 1].off, off, (uint32_t)W};
    }
    w.njobs = nj;
    e = cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm);
    if (e == cudaSuccess) {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_WGRAD, s);
        k_wgrad_tc<<<dim3((unsigned)chunks, (unsigned)nj), 128, wsm, s>>>(w);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        ProfScope ps(ctx, NRRS_KERNEL_TRAIN_REDUCE, s);
        e = launch_wreduce(partial, (uint32_t)chunks, (uint32_t)mlp, ctx->grads + ctx->n_table,
                           1.0f / (float)n, s);
    }
    join();  // the table gradient is complete on s from here
    if (e != cudaSuccess) {
        ctx->last_error = std::string("tensor-core wgrad launch: ") + cudaGetErrorString(e);
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
