// nrrs_common.cuh -- device-side definitions shared by every NRRS kernel (sm_100a).
//
// The maths restated here follows banbao990/NRRS-Code:
//   activationSigma          src/render/nrrs/net/networkcommon.h:61-68
//   box_cox_transform        src/render/nrrs/train.cu:19-39 (lambda = 0.5)
//   warp_roughness           src/render/nrrs/train.h:95
//   normalizeSpatialCoord    src/render/nrc/nrctrain.h:111-115
//   RRSWeightWindow          src/render/common/commoncudautils.h:14-28
//   factor + clamp + ceil    src/render/nrrs/integrator.cpp:1184-1298
//   glue (RRSNet input)      src/render/nrrs/train.cu:41-112
// The hash grid and the SH basis are the published Instant-NGP and real-SH definitions (the
// reference takes them from its absent tiny-cuda-nn submodule).
#pragma once
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/nrrs.h"

namespace nrrs {

constexpr int kMaxLevels = 16;
constexpr int kStatIn = 64;      // StatNet input lanes
constexpr int kRrsIn = 16;       // RRSNet input lanes
constexpr int kStatOut = 3;      // log-statistics
constexpr int kMaxSegments = 16; // depths per batched launch
constexpr int kTile = 128;       // vertices per inference tile

struct LevelDev {
    uint32_t offset;  // first table row of the level
    uint32_t res;     // N_l cells per axis (N_l + 1 grid points)
    uint32_t dense;   // 1 = dense indexing
    uint32_t cell;    // dense levels: first cell of the level in the cell image
};

struct EncodeParams {
    LevelDev lv[kMaxLevels];
    uint32_t n_levels;
    uint32_t hash_mask;
    int32_t normalize;
    float center[3];
    float diag[3];
    // The cell image of the FP16 table's dense levels (NULL when absent): for every cell
    // (x, y, z) of a dense level, its 8 corner entries in corner order, 32 bytes, at
    // cells[2 * (L.cell + x + N (y + N z))]. One 32-byte load then fetches what four row
    // gathers fetch from the table. It is rebuilt from the table after every table update.
    const uint4* cells;
};

struct VertexPtrs {
    const float* pos;
    const float* wi;
    const float* normal;
    const float* rough;
    const float* albedo;
    const float* thp;
    const uint32_t* depth;
    const float* ref;
    const uint32_t* sidx;
};

struct FactorParams {
    float clamp_min, clamp_max;
    float ww;            // weight window size
    int32_t use_ww;
    int32_t use_ceil;
    int32_t source;      // NRRS_FACTOR_*
    float stat_eps, ref_eps;
    double fixed_scale;  // 2^shift for the exact sum
    float vmax;          // largest admissible summed term
};

// One depth of a (possibly batched) launch.
struct Segment {
    uint32_t offset;       // first vertex
    uint32_t count;        // vertices
    uint32_t tile_start;   // first inference tile / decision chunk of this segment
    uint32_t budget;
    uint32_t n_specular;
    uint32_t queue_offset;
    uint32_t queue_capacity;
    uint32_t pad;
};

struct SegmentTable {
    Segment s[kMaxSegments];
    int32_t n;
    uint32_t total_tiles;
    // When the queue sizes live on the device, the host table holds the largest counts (which
    // size the grid) and `resolved` points at the table k_resolve_segments built on the device
    // from the actual counts; kernels read that one (seg_table).
    const struct SegmentTable* resolved;
};

// the table a kernel works on: the device-resolved one when there is one
__device__ __forceinline__ const SegmentTable& seg_table(const SegmentTable& t) {
    return t.resolved ? *t.resolved : t;
}

// Scratch words of the decision kernel; lives in context memory (or a static array for the
// allocation-free entry point). Self-resetting: the last CTA of every launch restores it.
struct DecideScratch {
    unsigned long long sum_acc[kMaxSegments];  // exact fixed-point normalisation sums
    unsigned int ticket;                       // dynamic chunk ticket
    unsigned int done;                         // finished CTAs
    unsigned int epoch;                        // launch epoch tagging the look-back states
    unsigned int status;                       // NRRS_DEV_* bits
    unsigned long long pad[4];
    // followed by the look-back state words (one unsigned long long per chunk)
};

__device__ __forceinline__ int find_segment(const SegmentTable& t, uint32_t tile) {
    int s = 0;
#pragma unroll 1
    for (int k = 1; k < t.n; ++k)
        if (tile >= t.s[k].tile_start) s = k;
    return s;
}

// ---- scalar maths (FP32) ----
__device__ __forceinline__ float act_sigma(float x) {
    const float ln2 = 0.6931471805599453f;
    return (x < 0.f) ? logf(1.0f + expf(x)) : (0.5f * x + ln2);
}
// adds (a, b, c, d) to the 16-byte aligned float quad at p with one vector reduction
__device__ __forceinline__ void red_add4(float* p, float a, float b, float c, float d) {
    asm volatile("red.relaxed.gpu.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(a),
                 "f"(b), "f"(c), "f"(d)
                 : "memory");
}

// adds (a, b) to the 8-byte aligned float pair at p with one vector reduction (sm_90 and later)
__device__ __forceinline__ void red_add2(float* p, float a, float b) {
    asm volatile("red.relaxed.gpu.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p), "f"(a), "f"(b)
                 : "memory");
}

__device__ __forceinline__ float act_sigma_grad(float x) {
    if (x < 0.f) { const float e = expf(x); return e / (1.0f + e); }
    return 0.5f;
}
__device__ __forceinline__ float box_cox(float x) { return 2.0f * (sqrtf(x) - 1.0f); }
__device__ __forceinline__ float warp_rough(float r) { return 1.0f - expf(-r); }

// real SH bands 0..3 of a unit direction (16 coefficients)
__device__ __forceinline__ void sh16(float x, float y, float z, float* o) {
    const float xx = x * x, yy = y * y, zz = z * z;
    o[0] = 0.28209479177387814f;
    o[1] = -0.4886025119029199f * y;
    o[2] = 0.4886025119029199f * z;
    o[3] = -0.4886025119029199f * x;
    o[4] = 1.0925484305920792f * x * y;
    o[5] = -1.0925484305920792f * y * z;
    o[6] = 0.31539156525252005f * (3.0f * zz - 1.0f);
    o[7] = -1.0925484305920792f * x * z;
    o[8] = 0.5462742152960396f * (xx - yy);
    o[9] = -0.5900435899266435f * y * (3.0f * xx - yy);
    o[10] = 2.890611442640554f * x * y * z;
    o[11] = -0.4570457994644658f * y * (5.0f * zz - 1.0f);
    o[12] = 0.3731763325901154f * z * (5.0f * zz - 3.0f);
    o[13] = -0.4570457994644658f * x * (5.0f * zz - 1.0f);
    o[14] = 1.445305721320277f * z * (xx - yy);
    o[15] = -0.5900435899266435f * x * (xx - 3.0f * yy);
}

__device__ __forceinline__ float clamp01(float x) { return x < 0.f ? 0.f : (x > 1.f ? 1.f : x); }

// normalised grid coordinate of vertex i
__device__ __forceinline__ void norm_pos(const EncodeParams& e, const float* pos, uint32_t i,
                                         float* p) {
    const float x = pos[3 * (size_t)i], y = pos[3 * (size_t)i + 1], z = pos[3 * (size_t)i + 2];
    if (e.normalize) {
        p[0] = clamp01(__fadd_rn(0.5f, __fdiv_rn(__fsub_rn(x, e.center[0]), e.diag[0])));
        p[1] = clamp01(__fadd_rn(0.5f, __fdiv_rn(__fsub_rn(y, e.center[1]), e.diag[1])));
        p[2] = clamp01(__fadd_rn(0.5f, __fdiv_rn(__fsub_rn(z, e.center[2]), e.diag[2])));
    } else {
        p[0] = clamp01(x); p[1] = clamp01(y); p[2] = clamp01(z);
    }
}

struct CellCoord {
    uint32_t ix, iy, iz;
    float fx, fy, fz;
};

// cell and fraction of a level: scaled coordinate rounded to FP32, floor clamped to [0, N-1]
__device__ __forceinline__ CellCoord cell_of(const float* p, uint32_t N) {
    CellCoord c;
    const float Nf = (float)N;
    float s, f;
    int i;
    s = __fmul_rn(p[0], Nf); i = (int)floorf(s); i = min(max(i, 0), (int)N - 1);
    f = __fsub_rn(s, (float)i); c.ix = (uint32_t)i; c.fx = f;
    s = __fmul_rn(p[1], Nf); i = (int)floorf(s); i = min(max(i, 0), (int)N - 1);
    f = __fsub_rn(s, (float)i); c.iy = (uint32_t)i; c.fy = f;
    s = __fmul_rn(p[2], Nf); i = (int)floorf(s); i = min(max(i, 0), (int)N - 1);
    f = __fsub_rn(s, (float)i); c.iz = (uint32_t)i; c.fz = f;
    return c;
}

__device__ __forceinline__ uint32_t grid_row(const LevelDev& L, uint32_t mask, uint32_t x,
                                             uint32_t y, uint32_t z) {
    uint32_t idx;
    if (L.dense) {
        const uint32_t R = L.res + 1;
        idx = x + R * y + R * R * z;
    } else {
        idx = (x ^ (y * 2654435761u) ^ (z * 805459861u)) & mask;
    }
    return L.offset + idx;
}

__device__ __forceinline__ float corner_weight(const CellCoord& c, int k) {
    const float wx = (k & 1) ? c.fx : 1.0f - c.fx;
    const float wy = (k & 2) ? c.fy : 1.0f - c.fy;
    const float wz = (k & 4) ? c.fz : 1.0f - c.fz;
    return wx * wy * wz;
}

// The 8 corner rows of cell c with per-corner feature gradients v[2k], v[2k+1] (corner order);
// the x-neighbours of one (y, z) that share an aligned pair of rows go as one 16-byte
// reduction, the others as two 8-byte ones.
__device__ __forceinline__ void scatter_corners(float* table_grad, const LevelDev& L,
                                                uint32_t mask, const CellCoord& c, const float* v) {
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        const uint32_t y = c.iy + (k2 & 1), z = c.iz + ((k2 >> 1) & 1);
        const uint32_t r0 = grid_row(L, mask, c.ix, y, z);
        const uint32_t r1 = grid_row(L, mask, c.ix + 1, y, z);
        const float* a = v + 4 * k2;   // corner x: a[0], a[1]; corner x + 1: a[2], a[3]
        if ((r0 >> 1) == (r1 >> 1)) {
            float* q = table_grad + 4 * (size_t)(r0 >> 1);
            if (r0 & 1u) red_add4(q, a[2], a[3], a[0], a[1]);
            else red_add4(q, a[0], a[1], a[2], a[3]);
        } else {
            red_add2(table_grad + 2 * (size_t)r0, a[0], a[1]);
            red_add2(table_grad + 2 * (size_t)r1, a[2], a[3]);
        }
    }
}

// Hash-grid gradient of one level: this lane's sample adds (g0, g1) x the trilinear weights to
// the 8 corner rows of cell c. Every lane in `lanes` (a prefix of the warp: lanes 0 .. k-1) calls
// it together. Samples that come in pixel order (a tracer's batch) put runs of neighbouring lanes
// in the same cell, whose reductions would serialise on the same rows: such runs are summed by a
// segmented shuffle scan and reduced once, by the run's last lane. A warp without runs (uniform
// samples) reduces per lane.
__device__ __forceinline__ void warp_scatter_level(float* table_grad, const LevelDev& L,
                                                   uint32_t mask, const CellCoord& c, float g0,
                                                   float g1, unsigned lanes) {
    const uint32_t lane = threadIdx.x & 31u;
    float v[16];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float wk = corner_weight(c, k);
        v[2 * k] = wk * g0;
        v[2 * k + 1] = wk * g1;
    }
    const uint32_t px = __shfl_up_sync(lanes, c.ix, 1);
    const uint32_t py = __shfl_up_sync(lanes, c.iy, 1);
    const uint32_t pz = __shfl_up_sync(lanes, c.iz, 1);
    const bool head = lane == 0 || px != c.ix || py != c.iy || pz != c.iz;
    const unsigned heads = __ballot_sync(lanes, head);
    if (heads == lanes) {
        scatter_corners(table_grad, L, mask, c, v);
        return;
    }
    const uint32_t start = 31u - __clz(heads & (0xffffffffu >> (31u - lane)));
#pragma unroll
    for (int dd = 1; dd < 32; dd <<= 1) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const float u = __shfl_up_sync(lanes, v[k], dd);
            if (lane >= start + (uint32_t)dd) v[k] += u;
        }
    }
    const bool tail = lane == 31u || !((lanes >> (lane + 1)) & 1u) || ((heads >> (lane + 1)) & 1u);
    if (tail) scatter_corners(table_grad, L, mask, c, v);
}

// the lanes of this warp whose sample index (base of the warp's first lane + lane) is below n
__device__ __forceinline__ unsigned valid_lanes(uint32_t warp_base, uint32_t n) {
    const uint32_t k = n > warp_base ? n - warp_base : 0u;
    return k >= 32u ? 0xffffffffu : ((1u << k) - 1u);
}

// entry e (0..3) of a 16-byte quad of table rows
__device__ __forceinline__ uint32_t quad_pick(const uint4& q, uint32_t e) {
    const uint32_t lo = (e & 1u) ? q.y : q.x, hi = (e & 1u) ? q.w : q.z;
    return (e & 2u) ? hi : lo;
}

// The 8 corner entries (FP16 pairs, as raw 32-bit words) of a cell, in corner order. For each
// (y, z) the aligned 16-byte quad holding corner x is loaded; corner x+1 comes from the same
// quad when it lies there (dense rows are consecutive, and the hash multiplies x by 1, so x and
// x+1 differ in the low bits: 3 times in 4) and from a predicated 4-byte load otherwise. That is
// about 5 L1 requests per level instead of 8 for the same values; the table carries 16 bytes of
// padding for the last quad.
// the 8 corner entries of cell c of dense level L from the cell image: one 32-byte load
__device__ __forceinline__ void cell_corners(const uint4* cells, const LevelDev& L,
                                             const CellCoord& c, uint32_t* t) {
    const uint4* q = cells + 2 * ((size_t)L.cell + c.ix + L.res * (c.iy + (size_t)L.res * c.iz));
    asm("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]),
          "=r"(t[7])
        : "l"(q));
}

__device__ __forceinline__ void level_corners_h(const __half2* table, const uint4* cells,
                                                const LevelDev& L, uint32_t mask,
                                                const CellCoord& c, uint32_t* t) {
    if (cells && L.dense) {
        cell_corners(cells, L, c, t);
        return;
    }
    const uint4* q4 = reinterpret_cast<const uint4*>(table);
    const uint32_t* t1 = reinterpret_cast<const uint32_t*>(table);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        const uint32_t y = c.iy + (k2 & 1), z = c.iz + ((k2 >> 1) & 1);
        const uint32_t r0 = grid_row(L, mask, c.ix, y, z);
        const uint32_t r1 = grid_row(L, mask, c.ix + 1, y, z);
        const uint4 q = __ldg(q4 + (r0 >> 2));
        const bool same = (r0 >> 2) == (r1 >> 2);
        uint32_t v1 = 0u;
        if (!same) v1 = __ldg(t1 + r1);
        t[2 * k2] = quad_pick(q, r0 & 3u);
        t[2 * k2 + 1] = same ? quad_pick(q, r1 & 3u) : v1;
    }
}

// trilinear sum over the 8 corners in corner order 0..7
__device__ __forceinline__ float2 corners_sum_h(const uint32_t* t, const CellCoord& c) {
    float f0 = 0.f, f1 = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float w = corner_weight(c, k);
        const float2 tv = __half22float2(*reinterpret_cast<const __half2*>(&t[k]));
        f0 += w * tv.x;
        f1 += w * tv.y;
    }
    return make_float2(f0, f1);
}

// The same 8 entries with one 4-byte load each: fewer registers in flight, which measured
// faster in the 128-wide training kernel (one CTA of four warps per SM, latency-bound)
__device__ __forceinline__ void level_corners_h_scalar(const __half2* table, const uint4* cells,
                                                       const LevelDev& L, uint32_t mask,
                                                       const CellCoord& c, uint32_t* t) {
    if (cells && L.dense) {
        cell_corners(cells, L, c, t);
        return;
    }
    const uint32_t* t1 = reinterpret_cast<const uint32_t*>(table);
#pragma unroll
    for (int k = 0; k < 8; ++k)
        t[k] = __ldg(t1 + grid_row(L, mask, c.ix + (k & 1), c.iy + ((k >> 1) & 1),
                                   c.iz + ((k >> 2) & 1)));
}

// Features of one level from an FP16 table [rows][2] (half2 per row): trilinear over the 8
// corners, summed in corner order 0..7.
template <bool QUAD = true>
__device__ __forceinline__ float2 level_features_h(const __half2* table, const uint4* cells,
                                                   const LevelDev& L, uint32_t mask,
                                                   const CellCoord& c) {
    uint32_t t[8];
    if constexpr (QUAD) level_corners_h(table, cells, L, mask, c, t);
    else level_corners_h_scalar(table, cells, L, mask, c, t);
    return corners_sum_h(t, c);
}

// Features of LB consecutive levels l0 .. l0+LB-1 (FP16 table): every corner load of the batch
// is issued before any is used (8 * LB gathers in flight per thread), then each level's
// trilinear sum in corner order 0..7 -- the same arithmetic as level_features_h.
template <int LB>
__device__ __forceinline__ void levels_features_h(const __half2* table, const EncodeParams& enc,
                                                  const float* p, int l0, float* f /*2*LB*/) {
    uint32_t t[8 * LB];
    CellCoord cc[LB];
#pragma unroll
    for (int j = 0; j < LB; ++j) {
        const LevelDev L = enc.lv[l0 + j];
        cc[j] = cell_of(p, L.res);
        level_corners_h(table, enc.cells, L, enc.hash_mask, cc[j], t + 8 * j);
    }
#pragma unroll
    for (int j = 0; j < LB; ++j) {
        const float2 fv = corners_sum_h(t + 8 * j, cc[j]);
        f[2 * j] = fv.x;
        f[2 * j + 1] = fv.y;
    }
}

// Misc StatNet lanes [48, 64): normal, albedo, warped roughness, bias 1, zeros
__device__ __forceinline__ void misc_lanes(const VertexPtrs& v, uint32_t i, float* o /*16*/) {
    const size_t i3 = 3 * (size_t)i;
    o[0] = v.normal[i3]; o[1] = v.normal[i3 + 1]; o[2] = v.normal[i3 + 2];
    o[3] = v.albedo[i3]; o[4] = v.albedo[i3 + 1]; o[5] = v.albedo[i3 + 2];
    o[6] = warp_rough(v.rough[i]);
    o[7] = 1.0f;
#pragma unroll
    for (int k = 8; k < 16; ++k) o[k] = 0.f;
}

__device__ __forceinline__ float lin_stat(float y, float eps) {
    const float L = expf(fminf(y, 20.0f)) - eps;
    return L > 0.f ? L : 0.f;
}

// glue: RRSNet input lanes from the StatNet log-statistics (train.cu:41-112, 3-stat form)
__device__ __forceinline__ void glue16(const FactorParams& fp, const float* y, const VertexPtrs& v,
                                       uint32_t i, float* x1) {
    const size_t i3 = 3 * (size_t)i;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        x1[c] = box_cox(lin_stat(y[c], fp.stat_eps));
        x1[3 + c] = box_cox(v.thp[i3 + c]);
    }
    x1[6] = warp_rough(v.rough[i]);
    x1[7] = box_cox(v.ref ? v.ref[i] : 0.5f);
    x1[8] = (float)(v.depth ? v.depth[i] : 0u) * 0.125f;
    x1[9] = 1.0f;
#pragma unroll
    for (int k = 10; k < 16; ++k) x1[k] = 0.f;
}

// The per-vertex inputs of the glue and the factor, loaded at the start of a tile so that their
// memory latency overlaps the StatNet chain instead of stalling it.
struct VertexAux {
    float thp[3];
    float rough, ref;
    uint32_t depth;
};

__device__ __forceinline__ VertexAux load_aux(const VertexPtrs& v, uint32_t i) {
    VertexAux x;
    const size_t i3 = 3 * (size_t)i;
    x.thp[0] = v.thp[i3];
    x.thp[1] = v.thp[i3 + 1];
    x.thp[2] = v.thp[i3 + 2];
    x.rough = v.rough[i];
    x.ref = v.ref ? v.ref[i] : 0.5f;
    x.depth = v.depth ? v.depth[i] : 0u;
    return x;
}

// glue16 and rrs_factor on preloaded inputs (the same arithmetic)
__device__ __forceinline__ void glue16_aux(const FactorParams& fp, const float* y,
                                           const VertexAux& x, float* x1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        x1[c] = box_cox(lin_stat(y[c], fp.stat_eps));
        x1[3 + c] = box_cox(x.thp[c]);
    }
    x1[6] = warp_rough(x.rough);
    x1[7] = box_cox(x.ref);
    x1[8] = (float)x.depth * 0.125f;
    x1[9] = 1.0f;
#pragma unroll
    for (int k = 10; k < 16; ++k) x1[k] = 0.f;
}

// the reference network's glue (train.cu:41-112): [bc(max(L,0)) x3, bc(max(L^2,0)) x3, bc(thp) x3,
// warped roughness, bc(ref_mean), 1, 0 x4] from its 6 outputs
__device__ __forceinline__ void glue16_ref_aux(const float* y, const VertexAux& x, float* x1) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        x1[c] = box_cox(fmaxf(y[c], 0.f));
        x1[3 + c] = box_cox(fmaxf(y[3 + c], 0.f));
        x1[6 + c] = box_cox(x.thp[c]);
    }
    x1[9] = warp_rough(x.rough);
    x1[10] = box_cox(x.ref);
    x1[11] = 1.0f;
#pragma unroll
    for (int k = 12; k < 16; ++k) x1[k] = 0.f;
}

// REF: the reference network's StatNet outputs L itself (no log statistic)
template <bool REF = false>
__device__ __forceinline__ float rrs_factor_aux(const FactorParams& fp, const float* y, float raw,
                                                const VertexAux& x) {
    float rrs;
    if (fp.source == NRRS_FACTOR_ADRRS) {
        const float ref = x.ref + fp.ref_eps;
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float L = REF ? y[c] : expf(fminf(y[c], 20.0f)) - fp.stat_eps;
            L = L < 1e-4f ? 1e-4f : (L > 1e4f ? 1e4f : L);
            acc += L * x.thp[c] / ref;
        }
        rrs = acc / 3.0f;
    } else {
        rrs = act_sigma(raw);
    }
    if (fp.use_ww) {
        const float dminus = 2.0f / (1.0f + fp.ww);
        const float dplus = dminus * fp.ww;
        rrs = rrs < dminus ? rrs / dminus : (rrs > dplus ? rrs / dplus : 1.0f);
    }
    rrs = rrs < fp.clamp_min ? fp.clamp_min : (rrs > fp.clamp_max ? fp.clamp_max : rrs);
    return rrs;
}

// factor + weight window + clamp (integrator.cpp:1184-1298)
__device__ __forceinline__ float rrs_factor(const FactorParams& fp, const float* y, float raw,
                                            const VertexPtrs& v, uint32_t i) {
    float rrs;
    if (fp.source == NRRS_FACTOR_ADRRS) {
        const float ref = (v.ref ? v.ref[i] : 0.5f) + fp.ref_eps;
        const size_t i3 = 3 * (size_t)i;
        float acc = 0.f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float L = expf(fminf(y[c], 20.0f)) - fp.stat_eps;
            L = L < 1e-4f ? 1e-4f : (L > 1e4f ? 1e4f : L);
            acc += L * v.thp[i3 + c] / ref;
        }
        rrs = acc / 3.0f;
    } else {
        rrs = act_sigma(raw);
    }
    if (fp.use_ww) {
        const float dminus = 2.0f / (1.0f + fp.ww);
        const float dplus = dminus * fp.ww;
        rrs = rrs < dminus ? rrs / dminus : (rrs > dplus ? rrs / dplus : 1.0f);
    }
    rrs = rrs < fp.clamp_min ? fp.clamp_min : (rrs > fp.clamp_max ? fp.clamp_max : rrs);
    return rrs;
}

// ---- the reference's shipped network (NRRS_NET_REFERENCE): 32-wide LeakyReLU MLPs, a 32-lane
//      StatNet input (8 hash levels, one-blob of the lat-long direction and of the warped
//      roughness) and 6 outputs (L, L^2). Only this network is 32 wide, so kernels templated on
//      the width select it by W == 32. ----
constexpr int kRefStatIn = 32;
constexpr int kRefStatOut = 6;
constexpr int kRefLevels = 8;
constexpr int kRefRrsLanes = 12;   // live RRSNet input lanes of the reference glue

__host__ __device__ constexpr int stat_in_of(int w) { return w == 32 ? kRefStatIn : kStatIn; }
__host__ __device__ constexpr int stat_out_of(int w) { return w == 32 ? kRefStatOut : kStatOut; }

__device__ __forceinline__ float leaky(float x) { return x > 0.f ? x : 0.01f * x; }

// CDF of the quartic (biweight) kernel of radius 1/bins at offset t: 15/16 (u - 2u^3/3 + u^5/5)
// + 1/2 at u = t bins, clamped to [-1, 1]
__device__ __forceinline__ float quartic_cdf(float t, int bins) {
    float u = t * (float)bins;
    u = u < -1.f ? -1.f : (u > 1.f ? 1.f : u);
    const float u2 = u * u;
    return 15.f / 16.f * u * (1.f - 2.f / 3.f * u2 + u2 * u2 / 5.f) + 0.5f;
}
// one-blob encoding of x in [0,1] into `bins` lanes: the kernel mass in each bin
template <int BINS>
__device__ __forceinline__ void one_blob(float x, float* out) {
#pragma unroll
    for (int k = 0; k < BINS; ++k)
        out[k] = quartic_cdf((float)(k + 1) / (float)BINS - x, BINS) -
                 quartic_cdf((float)k / (float)BINS - x, BINS);
}
// the 16 non-hash StatNet lanes of the reference network: one-blob (4 bins) of the lat-long u
// and v of wi, u = atan2(y, x) / 2pi + 1/2, v = acos(z) / pi, and one-blob (8 bins) of the warped
// roughness
__device__ __forceinline__ void ref_blob_lanes(const VertexPtrs& v, uint32_t i, float* o /*16*/) {
    const size_t i3 = 3 * (size_t)i;
    const float z = fminf(fmaxf(v.wi[i3 + 2], -1.f), 1.f);
    const float u = atan2f(v.wi[i3 + 1], v.wi[i3]) * 0.15915494309189535f + 0.5f;
    const float w = acosf(z) * 0.3183098861837907f;
    one_blob<4>(u, o);
    one_blob<4>(w, o + 4);
    one_blob<8>(1.0f - expf(-v.rough[i]), o + 8);
}

// ---- per-sample weights of the two losses (nrrs_train_step_batch) ----
// The reference hands its losses per-sample side arrays (network.cpp:408-435, 532-557) whose
// arithmetic lives in the absent tiny-cuda-nn fork. This build defines them (restated, unpinned):
//   s_i   = sample_weight[i] (1 when absent)             the pixel share of the sample
//   w_i   = s_i, or 0 where rrs_target[i] < 0            (the -1 mark, train.cu:520-523)
//   e_i   = error[i] / e_mean, a_i = error_for_avg[i] / e_mean (1 when absent), each clamped to
//           clamp_max when clamp_on; e_mean = error_sum / n_pixels
//   u_i   = gamma1 + gamma2 e_i + gamma3 a_i             error emphasis of the variance term
//   k_i   = max(number_samples[i], 1) (1 when absent)    samples averaged by the pixel
//   loss_S = sum_i s_i sum_c d_ic^2 / (3 sum s)
//   V = sum w u r^2 / (k q) / sum w,  C = sum w (cost_offset + q) / sum w,
//   R = sum w (ln q)^2 / sum w,  loss_R = V C + gamma4 R
// The kernels keep their per-sample form with 1/n applied later, so each sample carries the
// multipliers below, relative to the batch mean (n / sum s, n / sum w).
struct LossWeights {
    int32_t active;                  // 0: plain means (every multiplier 1, reg 0)
    const float* sample_weight;
    const float* rrs_target;
    const float* error;
    const float* error_for_avg;
    const float* number_samples;
    float g1, g2, g3, g4;
    int32_t clamp_on;
    float clamp_max;
    const double* sums;              // [sum s, sum w, e_mean] from k_loss_sums
};

struct SampleMul {
    float stat;   // StatNet term
    float var;    // variance term of the RRSNet loss
    float cost;   // cost term
    float reg;    // gamma4 x regulariser
};

__device__ __forceinline__ float loss_w_stat(const LossWeights& w, uint32_t i) {
    return w.sample_weight ? w.sample_weight[i] : 1.0f;
}
__device__ __forceinline__ float loss_w_rrs(const LossWeights& w, uint32_t i) {
    const float s = loss_w_stat(w, i);
    return (w.rrs_target && w.rrs_target[i] < 0.f) ? 0.f : s;
}

__device__ __forceinline__ SampleMul sample_mul(const LossWeights& w, uint32_t i, uint32_t n) {
    SampleMul m{1.f, 1.f, 1.f, 0.f};
    if (!w.active) return m;
    const double sum_s = w.sums[0], sum_w = w.sums[1];
    const float emean = (float)w.sums[2];
    const float rs = sum_s > 0.0 ? (float)((double)n / sum_s) : 0.f;
    const float rw = sum_w > 0.0 ? (float)((double)n / sum_w) : 0.f;
    const float s = loss_w_stat(w, i), ww = loss_w_rrs(w, i);
    float e = w.error ? w.error[i] / emean : 1.f;
    float ea = w.error_for_avg ? w.error_for_avg[i] / emean : 1.f;
    if (w.clamp_on) {
        e = fminf(e, w.clamp_max);
        ea = fminf(ea, w.clamp_max);
    }
    const float u = w.g1 + w.g2 * e + w.g3 * ea;
    const float k = w.number_samples ? fmaxf(w.number_samples[i], 1.f) : 1.f;
    m.stat = s * rs;
    m.var = ww * rw * u / k;
    m.cost = ww * rw;
    m.reg = w.g4 * ww * rw;
    return m;
}

// status sink for kernels launched without a context scratch
static __device__ unsigned int g_dummy_status;

// exact fixed-point term of the normalisation sum (truncation toward zero)
__device__ __forceinline__ long long fixed_term(const FactorParams& fp, float rrs,
                                                unsigned int* status) {
    float x = fp.use_ceil ? ceilf(rrs) : rrs;
    if (!isfinite(x)) { atomicOr(status, NRRS_DEV_NAN); return 0; }
    if (x > fp.vmax) { atomicOr(status, NRRS_DEV_SATURATED); x = fp.vmax; }
    return __double2ll_rz((double)x * fp.fixed_scale);
}

__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace nrrs
