// k_infer_tc.cu -- mixed-precision inference on the 5th-generation tensor cores (sm_100a).
//
// Each warpgroup (128 threads) owns a 128-vertex tile at a time and runs the whole per-vertex
// chain of the reference's inference (train.cu:269-287 data prep, tcnn HashGrid +
// FullyFusedMLP for StatNet and RRSNet, train.cu:41-112 glue, integrator.cpp:1184-1298 factor):
//
//   FP16 hash-table gathers + SH + misc lanes -> A tile [128 x 64] fp16/bf16 in shared memory
//   for every layer: tcgen05.mma (M=128, N=width, K=16 steps) into a TMEM accumulator,
//                    tcgen05.commit -> mbarrier, tcgen05.ld (one row per thread), ReLU,
//                    convert, write the next A tile in place
//   glue -> A tile [128 x 16]; RRSNet layers; activation, clamp, exact-sum term.
//
// Weights of both networks stay resident in shared memory for the CTA's lifetime; they are
// loaded once by bulk TMA copies (cp.async.bulk, unicast) from an image that k_util.cu packs in
// the canonical no-swizzle K-major core-matrix layout. A CTA holds WGS warpgroups that share
// that weight copy, each with its own A tile, mbarrier, TMEM columns and named barrier, so the
// gather phase of one tile overlaps the MMA chain of another; CTAs per SM and WGS are the
// autotuner's knobs. Every wait is bounded (NRRS_DEV_TIMEOUT).
//
// Split mode (PRE): k_encode_levels has already written each tile's 32 hash features as a
// [128 x 32] core-matrix block; one thread brings it in with an 8 KB bulk copy (prefetched for
// the next tile as soon as the first layer has read the current one), the warpgroup computes
// the SH and misc lanes into a second [128 x 32] block, and the first layer reads its K = 64
// operand from the two blocks (K steps 0-1 and 2-3). No table gathers remain in this kernel.
//
// Activations in TMEM (TA, split mode 3): an SS MMA reads both operands from shared memory, and
// at M = 128, N = 128 that alone uses the SM's whole shared-memory bandwidth, so with the
// epilogue's tile writes on top the tensor pipe idles. With TA each warpgroup also owns an A
// region in TMEM: the epilogue of a hidden layer writes its FP16/BF16 activations there with
// tcgen05.st, and the next layer's tcgen05.mma reads A from TMEM and only the weights from
// shared memory. The first layer of each network still reads its input tile from shared memory.
#include "kernels.hpp"
#include "tc_tile.cuh"

namespace nrrs {

namespace {

using namespace tile;

template <int W, int H, int IN>
struct PackedNet {
    static constexpr int kElems = W * IN + (H - 1) * W * W + 16 * W;
};

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int tmem_cols(int w) { return w <= 32 ? 32 : (w <= 64 ? 64 : (w <= 128 ? 128 : 256)); }

// PART: 0 = both networks in one kernel; 1 = StatNet only (writes the RRSNet input tiles);
// 2 = RRSNet only (reads them). Each kernel holds only the weights of the networks it runs.
template <int WS, int HS, int WR, int HR, int WGS, bool PRE, int PART = 0, bool TA = false>
struct TcShape {
    static constexpr int kStatElems = PackedNet<WS, HS, stat_in_of(WS)>::kElems;
    static constexpr int kRrsElems = PackedNet<WR, HR, kRrsIn>::kElems;
    static constexpr uint32_t kWBytes =
        (uint32_t)(PART == 0 ? kStatElems + kRrsElems : (PART == 1 ? kStatElems : kRrsElems)) * 2u;
    static constexpr uint32_t kWSrcOff = PART == 2 ? (uint32_t)kStatElems * 2u : 0u;
    static constexpr int kKMax =
        PART == 0 ? cmax(64, cmax(WS, WR)) : (PART == 1 ? cmax(64, WS) : cmax(16, WR));
    static constexpr uint32_t kABytes = 128u * kKMax * 2u;
    // TMEM per warpgroup: the accumulator D, and with TA the A region after it
    static constexpr uint32_t kColsD =
        (uint32_t)tmem_cols(PART == 0 ? cmax(WS, WR) : (PART == 1 ? WS : WR));
    static constexpr uint32_t kColsWg = TA ? 2 * kColsD : kColsD;
    static constexpr uint32_t kCols = kColsWg * WGS;
    static constexpr uint32_t kAOff = (kWBytes + 1023u) / 1024u * 1024u;
    // split mode: per warpgroup a hash-feature block and an SH/misc block, kept apart from the
    // activation tile so the next tile's features can be fetched during the MLP chain; where
    // that does not fit the blocks are the first 16 KB of the warpgroup's activation tile and
    // the copy is issued when the tile is free again
    static constexpr uint32_t kSepBytes = 2u * kEncTileBytes;
    static constexpr bool kShare =
        PRE && PART != 2 && 1024 + kAOff + WGS * (kABytes + kSepBytes) + 64 > 232448u;
    static constexpr uint32_t kHBytes = PRE && PART != 2 && !kShare ? kSepBytes : 0u;
    static constexpr uint32_t kHOff = kAOff + WGS * kABytes;
    // PART 2: per warpgroup the RRSNet input tile, apart from the activation tile so that the
    // next tile's can be fetched while this one's chain runs
    static constexpr uint32_t kXBytes = PART == 2 ? kX1TileBytes : 0u;
    static constexpr uint32_t kXOff = kHOff + WGS * kHBytes;
    static constexpr uint32_t kBarOff = kXOff + WGS * kXBytes;
    static constexpr size_t kSmem = 1024 + kBarOff + 96;
    static_assert(!kShare || kABytes >= kSepBytes, "feature blocks inside the activation tile");
};

// named barrier of one warpgroup (id 0 is __syncthreads)
__device__ __forceinline__ void wg_sync(int wg) {
    asm volatile("bar.sync %0, 128;" ::"r"(1 + wg) : "memory");
}
__device__ __forceinline__ void wg_sync_for_mma(int wg) {
    tc::fence_async_smem();
    tc::fence_before_sync();
    wg_sync(wg);
}

// StatNet input row of vertex i into A (K = 64): hash grid (FP16 table) + SH + misc + zeros
template <bool BF>
__device__ __forceinline__ void encode_row_tc(const InferArgs& a, uint32_t i, uint8_t* sA, int m) {
    float p[3];
    norm_pos(a.enc, a.v.pos, i, p);
    const __half2* table = reinterpret_cast<const __half2*>(a.table_h);
#pragma unroll 1
    for (int lq = 0; lq < 4; ++lq) {
        float f[8];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const LevelDev L = a.enc.lv[lq * 4 + j];
            const CellCoord c = cell_of(p, L.res);
            const float2 fv = level_features_h(table, a.enc.cells, L, a.enc.hash_mask, c);
            f[2 * j] = fv.x;
            f[2 * j + 1] = fv.y;
        }
        store_chunk(sA, m, lq, 64, pack8<BF>(f));
    }
    float sh[16];
    const size_t i3 = 3 * (size_t)i;
    sh16(a.v.wi[i3], a.v.wi[i3 + 1], a.v.wi[i3 + 2], sh);
    store_chunk(sA, m, 4, 64, pack8<BF>(sh));
    store_chunk(sA, m, 5, 64, pack8<BF>(sh + 8));
    float misc[16];
    misc_lanes(a.v, i, misc);
    store_chunk(sA, m, 6, 64, pack8<BF>(misc));
    store_chunk(sA, m, 7, 64, make_uint4(0u, 0u, 0u, 0u));
}

// the reference network's StatNet input row of vertex i (K = 32): 8 hash levels (FP16 table),
// then the one-blob lanes of the lat-long direction and of the warped roughness
template <bool BF>
__device__ __forceinline__ void encode_row_tc_ref(const InferArgs& a, uint32_t i, uint8_t* sA,
                                                  int m) {
    float p[3];
    norm_pos(a.enc, a.v.pos, i, p);
    const __half2* table = reinterpret_cast<const __half2*>(a.table_h);
#pragma unroll 1
    for (int lq = 0; lq < 2; ++lq) {
        float f[8];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const LevelDev L = a.enc.lv[lq * 4 + j];
            const CellCoord c = cell_of(p, L.res);
            const float2 fv = level_features_h(table, a.enc.cells, L, a.enc.hash_mask, c);
            f[2 * j] = fv.x;
            f[2 * j + 1] = fv.y;
        }
        store_chunk(sA, m, lq, kRefStatIn, pack8<BF>(f));
    }
    float blob[16];
    ref_blob_lanes(a.v, i, blob);
    store_chunk(sA, m, 2, kRefStatIn, pack8<BF>(blob));
    store_chunk(sA, m, 3, kRefStatIn, pack8<BF>(blob + 8));
}

// split mode: SH and misc lanes of vertex i as row m of a [128 x 32] block (the StatNet
// input columns 32-63: SH 16, normal/albedo/warped roughness/bias 8, zeros 8)
template <bool BF>
__device__ __forceinline__ void sh_misc_row_tc(const InferArgs& a, uint32_t i, uint8_t* sS, int m) {
    float sh[16];
    const size_t i3 = 3 * (size_t)i;
    sh16(a.v.wi[i3], a.v.wi[i3 + 1], a.v.wi[i3 + 2], sh);
    store_chunk(sS, m, 0, 32, pack8<BF>(sh));
    store_chunk(sS, m, 1, 32, pack8<BF>(sh + 8));
    float misc[16];
    misc_lanes(a.v, i, misc);
    store_chunk(sS, m, 2, 32, pack8<BF>(misc));
    store_chunk(sS, m, 3, 32, make_uint4(0u, 0u, 0u, 0u));
}

// The SH and misc inputs of one vertex (wi, normal, albedo, roughness), loaded during the
// previous tile's MLP chain so that their memory latency is not on the tile's critical path.
struct ShMiscIn {
    float wi[3], nrm[3], alb[3], rough;
};

__device__ __forceinline__ ShMiscIn load_sh_misc(const InferArgs& a, uint32_t i) {
    ShMiscIn s;
    const size_t i3 = 3 * (size_t)i;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        s.wi[c] = a.v.wi[i3 + c];
        s.nrm[c] = a.v.normal[i3 + c];
        s.alb[c] = a.v.albedo[i3 + c];
    }
    s.rough = a.v.rough[i];
    return s;
}

// the lanes of sh_misc_row_tc from inputs already in registers (the same arithmetic)
template <bool BF>
__device__ __forceinline__ void sh_misc_row_from(const ShMiscIn& in, uint8_t* sS, int m) {
    float sh[16];
    sh16(in.wi[0], in.wi[1], in.wi[2], sh);
    store_chunk(sS, m, 0, 32, pack8<BF>(sh));
    store_chunk(sS, m, 1, 32, pack8<BF>(sh + 8));
    float misc[16];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        misc[c] = in.nrm[c];
        misc[3 + c] = in.alb[c];
    }
    misc[6] = warp_rough(in.rough);
    misc[7] = 1.0f;
#pragma unroll
    for (int k = 8; k < 16; ++k) misc[k] = 0.f;
    store_chunk(sS, m, 2, 32, pack8<BF>(misc));
    store_chunk(sS, m, 3, 32, make_uint4(0u, 0u, 0u, 0u));
}

// split mode, first StatNet layer: K = 64 from two [128 x 32] blocks (hash features, then SH
// and misc), the same four K steps in the same order as the fused kernel's single A tile
template <int N, bool BF>
__device__ __forceinline__ bool tc_layer0_pre(const uint8_t* sH, const uint8_t* sS,
                                              const uint8_t* sWl, uint32_t tmem, uint64_t* bar,
                                              uint32_t& phase, int ltid) {
    if (ltid == 0) {
        tc::fence_after_sync();
        const uint32_t h0 = tc::smem_u32(sH), s0 = tc::smem_u32(sS), b0 = tc::smem_u32(sWl);
        constexpr uint32_t idesc = tc::idesc_f16(N, BF ? 1u : 0u);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
            const uint32_t a0 = kk < 2 ? h0 + kk * 256 : s0 + (kk - 2) * 256;
            const uint64_t ad = tc::smem_desc(a0, 128, 32 * 16);
            const uint64_t bd = tc::smem_desc(b0 + kk * 256, 128, kStatIn * 16);
            tc::mma_f16(tmem, ad, bd, idesc, kk > 0 ? 1u : 0u);
        }
        tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait(bar, phase, kSpin);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok;
}

// one layer issued by the warpgroup's first thread; the warpgroup waits for its completion
template <int K, int N, bool BF>
__device__ __forceinline__ bool tc_layer(const uint8_t* sA, const uint8_t* sWl, uint32_t tmem,
                                         uint64_t* bar, uint32_t& phase, int ltid) {
    if (ltid == 0) {
        tc::fence_after_sync();
        const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sWl);
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

// a hidden or output layer with A in TMEM (8 columns per K = 16 step) and B in shared memory
template <int K, int N, bool BF>
__device__ __forceinline__ bool tc_layer_ts(uint32_t tmem_a, const uint8_t* sWl, uint32_t tmem,
                                            uint64_t* bar, uint32_t& phase, int ltid) {
    if (ltid == 0) {
        tc::fence_after_sync();
        const uint32_t b0 = tc::smem_u32(sWl);
        constexpr uint32_t idesc = tc::idesc_f16(N, BF ? 1u : 0u);
#pragma unroll
        for (int kk = 0; kk < K / 16; ++kk) {
            const uint64_t bd = tc::smem_desc(b0 + kk * 256, 128, K * 16);
            tc::mma_f16_ts(tmem, tmem_a + 8u * kk, bd, idesc, kk > 0 ? 1u : 0u);
        }
        tc::mma_commit(bar);
    }
    const bool ok = tc::mbar_wait(bar, phase, kSpin);
    phase ^= 1u;
    tc::fence_after_sync();
    return ok;
}

// the TMEM stores of the warpgroup's epilogue are complete before its next MMA is issued
__device__ __forceinline__ void wg_sync_tmem(int wg) {
    tc::fence_before_sync();
    wg_sync(wg);
}

template <int WS, int HS, int WR, int HR, bool BF, int WGS, bool PRE, int PART, bool TA = false>
__global__ void __launch_bounds__(128 * WGS, (WGS == 2 && WS <= 64 && !TA) ? 3 : 1)
    k_infer_tc(const __grid_constant__ InferArgs a) {
    using S = TcShape<WS, HS, WR, HR, WGS, PRE, PART, TA>;
    static_assert(!TA || PART != 0, "activations in TMEM: split mode 3 kernels");
    constexpr bool kStat = PART != 2, kRrs = PART != 1;
    constexpr bool REF = WS == 32;   // the reference's shipped network (fused mode only)
    static_assert(!REF || (!PRE && PART == 0), "the reference network runs fused");
    extern __shared__ uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023u) & ~uintptr_t(1023));
    uint8_t* sW = base;
    // [0] weights, [1+wg] mma, [1+WGS+wg] copies into the tile (feature block or RRSNet input)
    uint64_t* bars = reinterpret_cast<uint64_t*>(base + S::kBarOff);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + 1 + 2 * WGS);
    __shared__ int s_abort[WGS];
    __shared__ int s_wabort;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int wg = tid >> 7, ltid = tid & 127;
    uint8_t* sA = base + S::kAOff + wg * S::kABytes;
    uint8_t* sH = S::kShare ? sA : base + S::kHOff + wg * S::kHBytes;  // split mode only
    uint8_t* sS = sH + kEncTileBytes;
    uint8_t* sX = base + S::kXOff + wg * S::kXBytes;   // PART 2 only

    if (tid == 0) {
        for (int k = 0; k < 1 + 2 * WGS; ++k) tc::mbar_init(&bars[k], 1);
        tc::fence_mbar_init();
        for (int k = 0; k < WGS; ++k) s_abort[k] = 0;
        s_wabort = 0;
    }
    if (warp == 0) {
        tc::tmem_alloc(tslot, S::kCols);
        tc::tmem_relinquish();
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tslot + (uint32_t)wg * S::kColsWg;
    if (tid == 0) {
        tc::mbar_arrive_expect_tx(&bars[0], S::kWBytes);
        const uint8_t* src = reinterpret_cast<const uint8_t*>(a.wpack) + S::kWSrcOff;
        for (uint32_t off = 0; off < S::kWBytes; off += 32768u) {
            const uint32_t bytes = S::kWBytes - off < 32768u ? S::kWBytes - off : 32768u;
            tc::bulk_g2s(sW + off, src + off, bytes, &bars[0]);
        }
    }
    unsigned flags = 0;
    if (!tc::mbar_wait(&bars[0], 0, kSpin)) s_wabort = 1;
    __syncthreads();
    if (s_wabort) flags |= NRRS_DEV_TIMEOUT;  // uniform across the CTA
    uint64_t* mbar = &bars[1 + wg];
    uint32_t phase = 0;
    // warp w of a warpgroup reads TMEM lanes 32*(w % 4) .. +31, i.e. rows of its own threads
    const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);
    // TA: the A region after D (the whole warpgroup's for the MMA, this warp's rows for stores)
    const uint32_t tmem_a = tmem + S::kColsD, trow_a = trow + S::kColsD;

    // weight images in this kernel's shared copy: StatNet then RRSNet (each only if run here)
    const uint8_t* wS0 = sW;
    const uint8_t* wSh = wS0 + WS * stat_in_of(WS) * 2;
    const uint8_t* wSo = wSh + (HS - 1) * WS * WS * 2;
    const uint8_t* wR0 = kStat ? wSo + 16 * WS * 2 : sW;
    const uint8_t* wRh = wR0 + WR * kRrsIn * 2;
    const uint8_t* wRo = wRh + (HR - 1) * WR * WR * 2;

    // copies into the tile: feature blocks (split modes) or RRSNet input tiles (PART 2); one in
    // flight at most per warpgroup
    uint64_t* hbar = &bars[1 + WGS + wg];
    uint32_t hphase = 0;
    bool h_pending = false;
    const uint32_t t0 = blockIdx.x * WGS + wg, tstride = gridDim.x * WGS;
    auto fetch_features = [&](uint32_t tt) {
        if (ltid == 0) {
            tc::mbar_arrive_expect_tx(hbar, kEncTileBytes);
            tc::bulk_g2s(sH, a.enc_tiles + (size_t)tt * kEncTileBytes, kEncTileBytes, hbar);
        }
        h_pending = true;
    };
    auto fetch_x1 = [&](uint32_t tt) {
        if (ltid == 0) {
            tc::mbar_arrive_expect_tx(hbar, kX1TileBytes);
            tc::bulk_g2s(sX, a.x1_tiles + (size_t)tt * kX1TileBytes, kX1TileBytes, hbar);
        }
        h_pending = true;
    };
    const SegmentTable& ST = seg_table(a.segs);
    const uint32_t total_tiles = ST.total_tiles;
    // PART 1 requests every tile's feature block and SH/misc inputs one tile ahead: the first
    // here, the next ones during the previous tile's chain; PART 2 its RRSNet input tiles
    ShMiscIn shin{};
    if (t0 < total_tiles && !flags) {
        if (PRE && kStat && (!S::kShare || PART == 1)) fetch_features(t0);
        if constexpr (PART == 1) {
            const Segment& g0 = ST.s[find_segment(ST, t0)];
            const uint32_t i0 = g0.offset + (t0 - g0.tile_start) * kTile + ltid;
            if (i0 < g0.offset + g0.count) shin = load_sh_misc(a, i0);
        }
        if constexpr (PART == 2) fetch_x1(t0);
    }

    for (uint32_t t = t0; t < total_tiles && !flags; t += tstride) {
        const int si = find_segment(ST, t);
        const Segment& sg = ST.s[si];
        const uint32_t i = sg.offset + (t - sg.tile_start) * kTile + ltid;
        const bool valid = i < sg.offset + sg.count;
        // the glue's and the factor's inputs, in flight during the StatNet chain
        VertexAux aux{};
        if (kStat && valid) aux = load_aux(a.v, i);

        bool ok = true;
        float y[16];
        if constexpr (!kStat) {
#pragma unroll
            for (int k = 0; k < 16; ++k) y[k] = 0.f;  // not used by the RRSNet factor
        }
        if constexpr (kStat) {
            // shared layout (PART 0): the previous tile's chain has finished with the activation
            // tile
            if (PRE && S::kShare && PART != 1) fetch_features(t);
            if constexpr (PRE) {
                if constexpr (PART == 1) {
                    if (valid) sh_misc_row_from<BF>(shin, sS, ltid);
                } else {
                    if (valid) sh_misc_row_tc<BF>(a, i, sS, ltid);
                }
                if (!valid) zero_row(sS, ltid, 32);
                ok = tc::mbar_wait(hbar, hphase, kSpin);
                hphase ^= 1u;
                h_pending = false;
            } else {
                if (valid) {
                    if constexpr (REF) encode_row_tc_ref<BF>(a, i, sA, ltid);
                    else encode_row_tc<BF>(a, i, sA, ltid);
                }
                else zero_row(sA, ltid, REF ? kRefStatIn : 64);
            }
            wg_sync_for_mma(wg);

            // ---- StatNet ----
            if constexpr (PRE) {
                ok &= tc_layer0_pre<WS, BF>(sH, sS, wS0, tmem, mbar, phase, ltid);
                // the first layer has read the block: bring in the next tile's features
                if (!S::kShare && ok && t + tstride < total_tiles) fetch_features(t + tstride);
            } else {
                ok &= tc_layer<stat_in_of(WS), WS, BF>(sA, wS0, tmem, mbar, phase, ltid);
            }
            if constexpr (TA) {
                epilogue_act_tmem<WS, BF, REF>(trow, trow_a);
                wg_sync_tmem(wg);
#pragma unroll 1
                for (int h = 1; h < HS; ++h) {
                    ok &= tc_layer_ts<WS, WS, BF>(tmem_a, wSh + (h - 1) * WS * WS * 2, tmem, mbar,
                                                  phase, ltid);
                    epilogue_act_tmem<WS, BF, REF>(trow, trow_a);
                    wg_sync_tmem(wg);
                }
                ok &= tc_layer_ts<WS, 16, BF>(tmem_a, wSo, tmem, mbar, phase, ltid);
            } else {
                epilogue_act<WS, BF, REF>(trow, sA, ltid);
                wg_sync_for_mma(wg);
#pragma unroll 1
                for (int h = 1; h < HS; ++h) {
                    ok &= tc_layer<WS, WS, BF>(sA, wSh + (h - 1) * WS * WS * 2, tmem, mbar, phase,
                                               ltid);
                    epilogue_act<WS, BF, REF>(trow, sA, ltid);
                    wg_sync_for_mma(wg);
                }
                ok &= tc_layer<WS, 16, BF>(sA, wSo, tmem, mbar, phase, ltid);
            }
            // PART 1: every read of the tile is done: request the next tile's feature block,
            // which lands while this tile's glue and stores run; its SH/misc inputs are loaded
            // after the glue (issued before it, the loads measured slower)
            uint32_t next_i = 0xffffffffu;
            if constexpr (PART == 1) {
                const uint32_t tn = t + tstride;
                if (tn < total_tiles && ok) {
                    if (S::kShare) fetch_features(tn);
                    const Segment& gn = ST.s[find_segment(ST, tn)];
                    const uint32_t in_ = gn.offset + (tn - gn.tile_start) * kTile + ltid;
                    if (in_ < gn.offset + gn.count) next_i = in_;
                }
            }
            tc::tmem_ld16(trow, y);
            tc::tmem_wait_ld();

            // ---- glue -> RRSNet input (K = 16) ----
            float x1[16];
            if (valid) {
                if constexpr (REF) glue16_ref_aux(y, aux, x1);
                else glue16_aux(a.fp, y, aux, x1);
            } else {
#pragma unroll
                for (int k = 0; k < 16; ++k) x1[k] = 0.f;
            }
            if constexpr (PART == 1) {
                if (next_i != 0xffffffffu) shin = load_sh_misc(a, next_i);
                // the RRSNet input straight from registers into the tile's K-major core-matrix
                // layout in HBM
                uint8_t* dst = a.x1_tiles + (size_t)t * kX1TileBytes;
                *reinterpret_cast<uint4*>(dst + chunk_offset(ltid, 0, 16)) = pack8<BF>(x1);
                *reinterpret_cast<uint4*>(dst + chunk_offset(ltid, 1, 16)) = pack8<BF>(x1 + 8);
            } else {
                store_chunk(sA, ltid, 0, 16, pack8<BF>(x1));
                store_chunk(sA, ltid, 1, 16, pack8<BF>(x1 + 8));
                wg_sync_for_mma(wg);
            }
        } else {
            // PART 2: this tile's RRSNet input from the StatNet kernel, requested one tile ahead
            ok = tc::mbar_wait(hbar, hphase, kSpin);
            hphase ^= 1u;
            h_pending = false;
            tc::fence_after_sync();
        }

        float r[16];
        if constexpr (kRrs) {
            // ---- RRSNet ----
            ok &= tc_layer<kRrsIn, WR, BF>(PART == 2 ? sX : sA, wR0, tmem, mbar, phase, ltid);
            // PART 2: the first layer has read the input tile, and after the barrier below every
            // thread of the warpgroup has seen this tile's copy land (a copy requested before
            // that could complete the barrier's next phase under a thread still waiting for
            // this one, which would then wait forever): bring in the next tile's
            const bool next_x1 = PART == 2 && ok && t + tstride < total_tiles;
            if constexpr (TA) {
                epilogue_act_tmem<WR, BF, REF>(trow, trow_a);
                wg_sync_tmem(wg);
                if (next_x1) fetch_x1(t + tstride);
#pragma unroll 1
                for (int h = 1; h < HR; ++h) {
                    ok &= tc_layer_ts<WR, WR, BF>(tmem_a, wRh + (h - 1) * WR * WR * 2, tmem, mbar,
                                                  phase, ltid);
                    epilogue_act_tmem<WR, BF, REF>(trow, trow_a);
                    wg_sync_tmem(wg);
                }
                ok &= tc_layer_ts<WR, 16, BF>(tmem_a, wRo, tmem, mbar, phase, ltid);
            } else {
                epilogue_act<WR, BF, REF>(trow, sA, ltid);
                wg_sync_for_mma(wg);
                if (next_x1) fetch_x1(t + tstride);
#pragma unroll 1
                for (int h = 1; h < HR; ++h) {
                    ok &= tc_layer<WR, WR, BF>(sA, wRh + (h - 1) * WR * WR * 2, tmem, mbar, phase,
                                               ltid);
                    epilogue_act<WR, BF, REF>(trow, sA, ltid);
                    wg_sync_for_mma(wg);
                }
                ok &= tc_layer<WR, 16, BF>(sA, wRo, tmem, mbar, phase, ltid);
            }
            tc::tmem_ld16(trow, r);
            tc::tmem_wait_ld();
        } else {
            r[0] = 0.f;
        }
        tc::fence_before_sync();
        wg_sync(wg);  // TMEM columns and A tile free for the next tile

        if (!ok) flags |= NRRS_DEV_TIMEOUT;
        // the factor: here when this kernel has what it needs (PART 1 only for ADRRS factors,
        // whose RRSNet kernel is not launched)
        const bool factor_here = PART != 1 || a.fp.source == NRRS_FACTOR_ADRRS;
        long long term = 0;
        if (valid) {
            if (kStat && a.stats) {
#pragma unroll
                for (int k = 0; k < stat_out_of(WS); ++k) a.stats[stat_out_of(WS) * (size_t)i + k] = y[k];
            }
            if (factor_here) {
                const float rrs = rrs_factor_aux<REF>(a.fp, y, r[0], aux);
                a.rrs[i] = rrs;
                if (a.scr || a.ext_acc)
                    term = fixed_term(a.fp, rrs, a.scr ? &a.scr->status : &g_dummy_status);
            }
        }
        if (factor_here && (a.scr || a.ext_acc)) {
            term = warp_sum_ll(term);
            if ((tid & 31) == 0 && term != 0)
                atomicAdd(a.ext_acc ? a.ext_acc : &a.scr->sum_acc[si], (unsigned long long)term);
        }
        // the warpgroup agrees on the abort decision
        if (flags) s_abort[wg] = 1;
        wg_sync(wg);
        if (s_abort[wg]) flags |= NRRS_DEV_TIMEOUT;
    }

    // a copy still in flight (the loop ended early) lands before the CTA leaves
    if (h_pending && ltid == 0 && !tc::mbar_wait(hbar, hphase, kSpin)) flags |= NRRS_DEV_TIMEOUT;
    if (flags && a.scr) atomicOr(&a.scr->status, flags);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(*tslot, S::kCols);
    }
}

template <int WS, int HS, int WR, int HR, bool BF, int WGS, bool PRE, int PART, bool TA = false>
cudaError_t launch_tc(const InferArgs& a, int sm_count, int ctas_per_sm, cudaStream_t s) {
    using S = TcShape<WS, HS, WR, HR, WGS, PRE, PART, TA>;
    if (S::kSmem > 232448 || S::kCols > 512) return cudaErrorInvalidConfiguration;
    auto kern = k_infer_tc<WS, HS, WR, HR, BF, WGS, PRE, PART, TA>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)S::kSmem);
    if (e != cudaSuccess) return e;
    // TMEM: the CTAs resident on one SM must fit in its 512 columns
    int per_sm = resident_ctas((const void*)kern, 128 * WGS, S::kSmem, 512 / (int)S::kCols);
    if (ctas_per_sm > 0 && ctas_per_sm < per_sm) per_sm = ctas_per_sm;
    const uint32_t ctas_needed = (a.segs.total_tiles + WGS - 1) / WGS;
    unsigned grid = (unsigned)(sm_count * per_sm);
    if (grid > ctas_needed) grid = ctas_needed;
    if (grid == 0) return cudaSuccess;
    g_last_grid = (int)grid;
    kern<<<grid, 128 * WGS, S::kSmem, s>>>(a);
    return cudaGetLastError();
}

// part: 0 both networks (fused or split-1), 1 StatNet only, 2 RRSNet only (split-2); tmem_act:
// parts 1 and 2 with the activations in TMEM (split-3; 1 or 2 warpgroups)
template <int WS, int HS, int WR, int HR, bool BF>
cudaError_t launch_wgs(const InferArgs& a, int sm_count, int ctas_per_sm, int wgs, int part,
                       bool tmem_act, cudaStream_t s) {
    if (tmem_act) {
        if (part == 1) {
            if (wgs == 2) return launch_tc<WS, HS, WR, HR, BF, 2, true, 1, true>(a, sm_count, ctas_per_sm, s);
            if (wgs == 1) return launch_tc<WS, HS, WR, HR, BF, 1, true, 1, true>(a, sm_count, ctas_per_sm, s);
        }
        if (part == 2) {
            if (wgs == 2) return launch_tc<WS, HS, WR, HR, BF, 2, true, 2, true>(a, sm_count, ctas_per_sm, s);
            if (wgs == 1) return launch_tc<WS, HS, WR, HR, BF, 1, true, 2, true>(a, sm_count, ctas_per_sm, s);
        }
        return cudaErrorInvalidConfiguration;
    }
    if (part == 1) {
        if (wgs == 4) return launch_tc<WS, HS, WR, HR, BF, 4, true, 1>(a, sm_count, ctas_per_sm, s);
        if (wgs == 2) return launch_tc<WS, HS, WR, HR, BF, 2, true, 1>(a, sm_count, ctas_per_sm, s);
        return launch_tc<WS, HS, WR, HR, BF, 1, true, 1>(a, sm_count, ctas_per_sm, s);
    }
    if (part == 2) {
        if (wgs == 4) return launch_tc<WS, HS, WR, HR, BF, 4, true, 2>(a, sm_count, ctas_per_sm, s);
        if (wgs == 2) return launch_tc<WS, HS, WR, HR, BF, 2, true, 2>(a, sm_count, ctas_per_sm, s);
        return launch_tc<WS, HS, WR, HR, BF, 1, true, 2>(a, sm_count, ctas_per_sm, s);
    }
    if (a.enc_tiles) {
        if (wgs == 2) return launch_tc<WS, HS, WR, HR, BF, 2, true, 0>(a, sm_count, ctas_per_sm, s);
        if (wgs == 1) return launch_tc<WS, HS, WR, HR, BF, 1, true, 0>(a, sm_count, ctas_per_sm, s);
        return cudaErrorInvalidConfiguration;
    }
    if (wgs == 2) return launch_tc<WS, HS, WR, HR, BF, 2, false, 0>(a, sm_count, ctas_per_sm, s);
    if (wgs == 1) return launch_tc<WS, HS, WR, HR, BF, 1, false, 0>(a, sm_count, ctas_per_sm, s);
    return cudaErrorInvalidConfiguration;
}

template <int WS, int HS, int WR, int HR, bool BF, int WGS, bool PRE, int PART, bool TA = false>
int max_ctas_tc() {
    using S = TcShape<WS, HS, WR, HR, WGS, PRE, PART, TA>;
    if (S::kSmem > 232448 || S::kCols > 512) return 0;
    auto kern = k_infer_tc<WS, HS, WR, HR, BF, WGS, PRE, PART, TA>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::kSmem) !=
        cudaSuccess)
        return 0;
    return resident_ctas((const void*)kern, 128 * WGS, S::kSmem, 512 / (int)S::kCols);
}

template <int WS, int HS, bool BF, int WGS, bool TA = false>
int max_ctas_split2() {
    const int m1 = max_ctas_tc<WS, HS, WS, HS, BF, WGS, true, 1, TA>();
    const int m2 = max_ctas_tc<WS, HS, WS, HS, BF, WGS, true, 2, TA>();
    return m1 < m2 ? m1 : m2;
}

// split: 0 fused, 1 encoding kernel + one MLP kernel, 2 encoding + StatNet + RRSNet kernels,
// 3 as 2 with the hidden activations in TMEM
template <int WS, int HS, bool BF>
int max_ctas_of(int wgs, int split) {
    if (split == 3) {
        if (wgs == 2) return max_ctas_split2<WS, HS, BF, 2, true>();
        if (wgs == 1) return max_ctas_split2<WS, HS, BF, 1, true>();
        return 0;
    }
    if (split == 2) {
        if (wgs == 4) return max_ctas_split2<WS, HS, BF, 4>();
        if (wgs == 2) return max_ctas_split2<WS, HS, BF, 2>();
        if (wgs == 1) return max_ctas_split2<WS, HS, BF, 1>();
        return 0;
    }
    if (wgs != 1 && wgs != 2) return 0;
    if (split == 1)
        return wgs == 2 ? max_ctas_tc<WS, HS, WS, HS, BF, 2, true, 0>() : max_ctas_tc<WS, HS, WS, HS, BF, 1, true, 0>();
    return wgs == 2 ? max_ctas_tc<WS, HS, WS, HS, BF, 2, false, 0>() : max_ctas_tc<WS, HS, WS, HS, BF, 1, false, 0>();
}

}  // namespace

int infer_max_ctas_fp32(int ws, int hs);

int infer_max_ctas(int ws, int hs, int wr, int hr, int prec, int wgs, int split) {
    if (prec == NRRS_PREC_FP32) return wgs == 1 && !split ? infer_max_ctas_fp32(ws, hs) : 0;
    if (wr != ws || hr != hs) return 0;
    const bool bf = prec == NRRS_PREC_BF16;
    if (ws == 64 && hs == 2) return bf ? max_ctas_of<64, 2, true>(wgs, split) : max_ctas_of<64, 2, false>(wgs, split);
    if (ws == 64 && hs == 3) return bf ? max_ctas_of<64, 3, true>(wgs, split) : max_ctas_of<64, 3, false>(wgs, split);
    if (ws == 128 && hs == 3) return bf ? max_ctas_of<128, 3, true>(wgs, split) : max_ctas_of<128, 3, false>(wgs, split);
    if (ws == 32 && hs == 3) {   // the reference network: fused mode, 1 or 2 warpgroups
        if (split != 0 || (wgs != 1 && wgs != 2)) return 0;
        if (wgs == 2) return bf ? max_ctas_tc<32, 3, 32, 3, true, 2, false, 0>() : max_ctas_tc<32, 3, 32, 3, false, 2, false, 0>();
        return bf ? max_ctas_tc<32, 3, 32, 3, true, 1, false, 0>() : max_ctas_tc<32, 3, 32, 3, false, 1, false, 0>();
    }
    return 0;
}

size_t infer_tc_smem_bytes(int ws, int hs, int wr, int hr) {
    if (ws == 64 && hs == 2) return TcShape<64, 2, 64, 2, 1, false, 0>::kSmem;
    if (ws == 64 && hs == 3) return TcShape<64, 3, 64, 3, 1, false, 0>::kSmem;
    if (ws == 128 && hs == 3) return TcShape<128, 3, 128, 3, 1, false, 0>::kSmem;
    if (ws == 32 && hs == 3) return TcShape<32, 3, 32, 3, 1, false, 0>::kSmem;
    return 0;
}

cudaError_t launch_infer_tc(const InferArgs& a, int ws, int hs, int wr, int hr, int prec,
                            int sm_count, int ctas_per_sm, int wgs, int part, bool tmem_act,
                            cudaStream_t s) {
    const bool bf = prec == NRRS_PREC_BF16;
    const bool ta = tmem_act;
    if (ws == 64 && hs == 2 && wr == 64 && hr == 2)
        return bf ? launch_wgs<64, 2, 64, 2, true>(a, sm_count, ctas_per_sm, wgs, part, ta, s)
                  : launch_wgs<64, 2, 64, 2, false>(a, sm_count, ctas_per_sm, wgs, part, ta, s);
    if (ws == 64 && hs == 3 && wr == 64 && hr == 3)
        return bf ? launch_wgs<64, 3, 64, 3, true>(a, sm_count, ctas_per_sm, wgs, part, ta, s)
                  : launch_wgs<64, 3, 64, 3, false>(a, sm_count, ctas_per_sm, wgs, part, ta, s);
    if (ws == 128 && hs == 3 && wr == 128 && hr == 3)  // 158 KB of weights in one kernel
        return bf ? launch_wgs<128, 3, 128, 3, true>(a, sm_count, ctas_per_sm, wgs, part, ta, s)
                  : launch_wgs<128, 3, 128, 3, false>(a, sm_count, ctas_per_sm, wgs, part, ta, s);
    if (ws == 32 && hs == 3 && wr == 32 && hr == 3) {  // the reference network: fused only
        if (part != 0 || a.enc_tiles || tmem_act) return cudaErrorInvalidValue;
        if (wgs == 2)
            return bf ? launch_tc<32, 3, 32, 3, true, 2, false, 0>(a, sm_count, ctas_per_sm, s)
                      : launch_tc<32, 3, 32, 3, false, 2, false, 0>(a, sm_count, ctas_per_sm, s);
        if (wgs == 1)
            return bf ? launch_tc<32, 3, 32, 3, true, 1, false, 0>(a, sm_count, ctas_per_sm, s)
                      : launch_tc<32, 3, 32, 3, false, 1, false, 0>(a, sm_count, ctas_per_sm, s);
        return cudaErrorInvalidConfiguration;
    }
    return cudaErrorInvalidValue;
}

}  // namespace nrrs
