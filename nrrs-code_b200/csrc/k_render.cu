// k_render.cu -- the wavefront steps either side of the NRRS step: camera rays, BVH traversal
// (closest hit, optionally in a sorted ray order, and shadow any-hit), the hit/miss shading that
// forms the next vertex queue, and the scatter step that consumes the emitted queue (thp / rrs,
// next-event estimation, BSDF sampling) or runs fixed Russian roulette. Kernels, the host BVH
// build and the C-ABI (include/nrrs.h).
//
// Replaces, in banbao990/NRRS-Code:
//   OptiX closest-hit / any-hit programs        src/render/nrrs/device.cu:48-161
//   handleEmissiveHit / handleMiss              src/render/nrrs/integrator.cpp:688-735
//   handleIntersections, generateScatteredRays  src/render/nrrs/integrator.cpp:737-887
//   generateCameraRays                          src/render/nrrs/integrator.cpp:889-935
//
// Everything a frame computes is reproducible:
// - random numbers are a counter-based hash of (seed, depth, slot, dimension);
// - every FP32 operation is written out and rounded on its own, except the triangle test's
//   products, which are explicit fused multiply-adds;
// - ties between equally close triangles go to the lower triangle index, whatever the BVH or
//   the order the rays are walked in;
// - the film and the contributions are exact fixed-point sums.
// A C restatement of the same steps (brute-force intersection instead of the BVH) checks the
// kernels bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <numeric>
#include <vector>

#include "fixed_point.cuh"
#include "nrrs.h"

struct nrrs_scene {
    float* tris = nullptr;        // [nt][12] v0, e1, e2, pad in BVH leaf order
    uint32_t* tri_id = nullptr;   // [nt] input index of each leaf-order triangle
    uint32_t* tri_mat = nullptr;  // [nt] material, input order
    float* tri_in = nullptr;      // [nt][9] v0, e1, e2 in input order
    float* nodes = nullptr;       // [nn][8] bmin, left_or_first (bits), bmax, count | axis << 16
    float* mats = nullptr;        // [nm][6]
    uint32_t* lights = nullptr;   // [nl] emissive triangles (input index)
    float* light_area = nullptr;  // [nl]
    float env[3] = {0.f, 0.f, 0.f};
    uint32_t nt = 0, nn = 0, nl = 0, nm = 0, max_depth = 0;
    uint32_t nee = 1;             // next-event estimation on (mEnableNEE)
    uint8_t* mat_spec = nullptr;  // [nm] 1 = perfect mirror, 2 = thin glass (null: neither)
};

namespace nrrs {
namespace {

constexpr float kInvPi = 0.318309886183790671f;
constexpr float kOffset = 1e-4f;        // ray origins leave the surface along the normal
constexpr int kStack = 64;
constexpr int kLeafMax = 1;   // one triangle per leaf: its tight box culls the costly test
constexpr uint32_t kMiss = 0xffffffffu;
constexpr uint32_t kRRDim = 31;     // hash dimension of the fixed-RR decision

// ---- counter-based random numbers (shared with the C restatement) ----
// lowbias32 (C. Wellons), a published 32-bit integer hash
__host__ __device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float rnd(uint32_t seed, uint32_t depth, uint32_t slot, uint32_t dim) {
    const uint32_t h = hash32(hash32(hash32(seed) ^ (depth * 0x9e3779b9u)) ^ (slot * 32u + dim));
    return (float)(h >> 8) * 0x1p-24f;
}

// ---- FP32 vector arithmetic, every operation rounded on its own ----
struct V3 { float x, y, z; };
__device__ __forceinline__ V3 v3(const float* p) { return {p[0], p[1], p[2]}; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return {__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y), __fadd_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return {__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y), __fsub_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 mul(V3 a, float s) { return {__fmul_rn(a.x, s), __fmul_rn(a.y, s), __fmul_rn(a.z, s)}; }
__device__ __forceinline__ V3 vmul(V3 a, V3 b) { return {__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y), __fmul_rn(a.z, b.z)}; }
__device__ __forceinline__ V3 divs(V3 a, float s) { return {__fdiv_rn(a.x, s), __fdiv_rn(a.y, s), __fdiv_rn(a.z, s)}; }
__device__ __forceinline__ float dot(V3 a, V3 b) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)), __fmul_rn(a.z, b.z));
}
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {__fsub_rn(__fmul_rn(a.y, b.z), __fmul_rn(a.z, b.y)),
            __fsub_rn(__fmul_rn(a.z, b.x), __fmul_rn(a.x, b.z)),
            __fsub_rn(__fmul_rn(a.x, b.y), __fmul_rn(a.y, b.x))};
}
__device__ __forceinline__ V3 normalize(V3 a) { return divs(a, __fsqrt_rn(dot(a, a))); }
__device__ __forceinline__ void put(float* p, V3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
__device__ __forceinline__ bool nonzero(V3 a) { return a.x != 0.f || a.y != 0.f || a.z != 0.f; }

// the intersection's dot and cross products with fused multiply-adds (each fmaf rounded once; the
// C restatement calls fmaf in the same order)
__device__ __forceinline__ float fdot(V3 a, V3 b) {
    return __fmaf_rn(a.x, b.x, __fmaf_rn(a.y, b.y, __fmul_rn(a.z, b.z)));
}
__device__ __forceinline__ V3 fcross(V3 a, V3 b) {
    return {__fmaf_rn(a.y, b.z, -__fmul_rn(a.z, b.y)), __fmaf_rn(a.z, b.x, -__fmul_rn(a.x, b.z)),
            __fmaf_rn(a.x, b.y, -__fmul_rn(a.y, b.x))};
}

// Moller-Trumbore, two-sided; t in (0, tmax) and t <= bound (the closest hit so far: a hit at
// the same t must still reach the tie rule)
__device__ __forceinline__ bool intersect_v(V3 v0, V3 e1, V3 e2, V3 o, V3 d, float tmax,
                                            float bound, float* t, float* u, float* v) {
    const V3 pv = fcross(d, e2);
    const float det = fdot(e1, pv);
    if (fabsf(det) < 1e-12f) return false;
    const float inv = __fdiv_rn(1.0f, det);
    const V3 tv = sub(o, v0);
    const float uu = __fmul_rn(fdot(tv, pv), inv);
    if (uu < 0.f || uu > 1.f) return false;
    const V3 qv = fcross(tv, e1);
    const float vv = __fmul_rn(fdot(d, qv), inv);
    if (vv < 0.f || __fadd_rn(uu, vv) > 1.f) return false;
    const float tt = __fmul_rn(fdot(e2, qv), inv);
    if (!(tt > 0.f && tt < tmax && tt <= bound)) return false;
    *t = tt; *u = uu; *v = vv;
    return true;
}

// a leaf-order triangle of 12 floats, read as three 16-byte loads
__device__ __forceinline__ bool intersect_leaf(const float* tri, V3 o, V3 d, float tmax,
                                               float bound, float* t, float* u, float* v) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(tri));
    const float4 b = __ldg(reinterpret_cast<const float4*>(tri) + 1);
    const float4 c = __ldg(reinterpret_cast<const float4*>(tri) + 2);
    return intersect_v({a.x, a.y, a.z}, {a.w, b.x, b.y}, {b.z, b.w, c.x}, o, d, tmax, bound, t, u, v);
}

// slab test: the interval of the box along the ray, clipped to [0, tmax]. A 0 x inf product (a
// ray parallel to a slab, starting on its plane) is NaN, which fminf/fmaxf drop; the box is grown
// at build time, so such a ray cannot reach a triangle inside it and the miss it gives is right.
__device__ __forceinline__ bool box_hit(float4 lo, float4 hi, V3 o, V3 inv, float tmax,
                                        float* tnear) {
    const float ax = (lo.x - o.x) * inv.x, bx = (hi.x - o.x) * inv.x;
    const float ay = (lo.y - o.y) * inv.y, by = (hi.y - o.y) * inv.y;
    const float az = (lo.z - o.z) * inv.z, bz = (hi.z - o.z) * inv.z;
    const float t0 = fmaxf(fmaxf(fminf(ax, bx), fminf(ay, by)), fmaxf(fminf(az, bz), 0.f));
    const float t1 = fminf(fminf(fmaxf(ax, bx), fmaxf(ay, by)), fminf(fmaxf(az, bz), tmax));
    *tnear = t0;
    return t0 <= t1;
}

struct Hit { uint32_t prim; float t, u, v; };

// closest hit; ties in t go to the lower input index. any = true stops at the first hit.
// Closest hit; ties in t go to the lower input index. Stack traversal, near child first by the
// sign of the ray on the node's split axis: the near child is held in a register as the next
// node and only the far one goes onto the stack. Each pass of the outer loop first walks nodes
// until this lane holds a leaf whose box the ray enters (or the stack is empty), then tests that
// leaf: lanes of a warp reconverge between the two loops, so the triangle tests run with the
// warp together.
__device__ Hit closest_hit(const nrrs_scene& s, V3 o, V3 d, float tmax) {
    Hit h{kMiss, tmax, 0.f, 0.f};   // h.t is the culling bound: tmax until the first hit
    const V3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    const float4* nodes = reinterpret_cast<const float4*>(s.nodes);
    int stack[kStack];
    int sp = 0;
    int node = 0;   // the next node to visit, held in a register (-1: pop one)
    for (;;) {
        uint32_t first = 0, cnt = 0;
        for (;;) {
            if (node < 0) {
                if (sp == 0) break;
                node = stack[--sp];
            }
            const float4* nd = nodes + 2 * (size_t)node;
            const float4 lo = __ldg(nd), hi = __ldg(nd + 1);
            float tn;
            if (!box_hit(lo, hi, o, inv, h.t, &tn)) { node = -1; continue; }
            const uint32_t lf = __float_as_uint(lo.w), ca = __float_as_uint(hi.w);
            if (ca & 0xffffu) { first = lf; cnt = ca & 0xffffu; node = -1; break; }
            const uint32_t axis = ca >> 16;
            const float da = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
            if (sp + 1 > kStack) { node = -1; continue; }   // depth is bounded at build time
            // near child next, the far one on the stack
            if (da < 0.f) { stack[sp++] = (int)lf; node = (int)lf + 1; }
            else { stack[sp++] = (int)lf + 1; node = (int)lf; }
        }
        if (cnt == 0) break;
        for (uint32_t i = first; i < first + cnt; ++i) {
            float t, u, v;
            if (!intersect_leaf(s.tris + 12 * (size_t)i, o, d, tmax, h.t, &t, &u, &v)) continue;
            const uint32_t id = s.tri_id[i];
            if (h.prim == kMiss || t < h.t || (t == h.t && id < h.prim)) h = {id, t, u, v};
        }
    }
    return h;
}

// Any hit in (0, tmax): one node per pass, far child first, ending at the first triangle hit.
__device__ bool any_hit(const nrrs_scene& s, V3 o, V3 d, float tmax) {
    const V3 inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    const float4* nodes = reinterpret_cast<const float4*>(s.nodes);
    int stack[kStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const float4* nd = nodes + 2 * (size_t)stack[--sp];
        const float4 lo = __ldg(nd), hi = __ldg(nd + 1);
        float tn;
        if (!box_hit(lo, hi, o, inv, tmax, &tn)) continue;
        const uint32_t lf = __float_as_uint(lo.w), ca = __float_as_uint(hi.w);
        const uint32_t cnt = ca & 0xffffu;
        if (cnt) {
            for (uint32_t i = lf; i < lf + cnt; ++i) {
                float t, u, v;
                if (intersect_leaf(s.tris + 12 * (size_t)i, o, d, tmax, tmax, &t, &u, &v)) return true;
            }
        } else {
            if (sp + 2 > kStack) continue;   // depth is bounded at build time; never taken
            // far child first: a shadow ray starts on a surface, among the boxes it is just
            // leaving, and an occluder is found sooner from the light's side (measured: 42 %
            // less shadow time than the left child first, 50 % less than near first)
            const uint32_t axis = ca >> 16;
            const float da = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
            if (da >= 0.f) { stack[sp++] = (int)lf; stack[sp++] = (int)lf + 1; }
            else { stack[sp++] = (int)lf + 1; stack[sp++] = (int)lf; }
        }
    }
    return false;
}

__device__ __forceinline__ void film_add(int64_t* film, uint32_t pixel, V3 c) {
    const float cc[3] = {c.x, c.y, c.z};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        if (cc[k] == 0.f || !fixed_ok(cc[k])) continue;
        long long l[3];
        fixed_limbs(cc[k], l);
#pragma unroll
        for (int q = 0; q < 3; ++q)
            if (l[q]) atomicAdd(reinterpret_cast<unsigned long long*>(film + 9 * (size_t)pixel + 3 * k + q),
                                (unsigned long long)l[q]);
    }
}

__device__ __forceinline__ float power_heuristic(float a, float b) {
    const float a2 = __fmul_rn(a, a);
    return __fdiv_rn(a2, __fadd_rn(a2, __fmul_rn(b, b)));
}

// ---- kernels ----
__global__ void __launch_bounds__(256) k_camera(nrrs_camera c, uint32_t sample, uint32_t seed,
                                                nrrs_ray_soa r) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= c.width * c.height) return;
    const V3 fw = normalize(v3(c.forward));
    const V3 right = normalize(cross(fw, v3(c.up)));
    const V3 up = cross(right, fw);
    const float jx = rnd(seed, 0xffffffffu - sample, p, 0), jy = rnd(seed, 0xffffffffu - sample, p, 1);
    const float w = (float)c.width, hgt = (float)c.height;
    const float px = __fsub_rn(__fmul_rn(__fdiv_rn(__fadd_rn((float)(p % c.width), jx), w), 2.0f), 1.0f);
    const float py = __fsub_rn(1.0f, __fmul_rn(__fdiv_rn(__fadd_rn((float)(p / c.width), jy), hgt), 2.0f));
    const float sx = __fmul_rn(__fmul_rn(px, c.tan_half_fov_y), __fdiv_rn(w, hgt));
    const float sy = __fmul_rn(py, c.tan_half_fov_y);
    const V3 d = normalize(add(add(fw, mul(right, sx)), mul(up, sy)));
    put(r.origin + 3 * (size_t)p, v3(c.pos));
    put(r.dir + 3 * (size_t)p, d);
    put(r.thp + 3 * (size_t)p, {1.f, 1.f, 1.f});
    r.pdf[p] = 0.f;
    r.pixel[p] = p;
    r.node[p] = -1;
}

// ---- ray order for the closest-hit trace: a counting sort by (direction octant, 12-bit Morton
// code of the origin in the scene's box), so that the lanes of a warp start close together and
// head the same way. Hits are written at the rays' own indices: the result does not depend on
// the order. Scratch: kSortBins + 1 counters (the last one counts finished CTAs), then the order.
constexpr uint32_t kSortBins = 1u << 15;
constexpr uint32_t kSortMinRays = 65536;   // below this the sort costs more than it saves
constexpr int kSortThreads = 256;

__device__ __forceinline__ uint32_t ray_key(const nrrs_scene& s, const nrrs_ray_soa& r, uint32_t i) {
    const V3 o = v3(r.origin + 3 * (size_t)i), d = v3(r.dir + 3 * (size_t)i);
    const float oo[3] = {o.x, o.y, o.z};
    uint32_t q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {   // the root box: s.nodes[0..2] and [4..6]
        const float f = (oo[k] - s.nodes[k]) / (s.nodes[4 + k] - s.nodes[k]) * 16.0f;
        q[k] = f > 0.f ? min((uint32_t)f, 15u) : 0u;   // NaN and negative go to 0
    }
    uint32_t key = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b)
        key |= (((q[0] >> b) & 1u) << (3 * b)) | (((q[1] >> b) & 1u) << (3 * b + 1)) |
               (((q[2] >> b) & 1u) << (3 * b + 2));
    const uint32_t oct = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    return (oct << 12) | key;
}

// counts per key (lanes of a warp with the same key take one atomic); the last CTA turns the
// counts into exclusive offsets in place
__global__ void __launch_bounds__(kSortThreads) k_sort_count(const __grid_constant__ nrrs_scene s,
                                                             nrrs_ray_soa r, const uint32_t* n_dev,
                                                             uint32_t max_n, uint32_t* hist) {
    const uint32_t n = min(*n_dev, max_n);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (kSortThreads / 32);
    const uint32_t w = blockIdx.x * (kSortThreads / 32) + (threadIdx.x >> 5);
    for (uint32_t base = w * 32; base < n; base += warps * 32) {
        const uint32_t i = base + lane;
        const bool ok = i < n;
        const uint32_t key = ok ? ray_key(s, r, i) : 0xffffffffu;
        const unsigned same = __match_any_sync(0xffffffffu, key);
        if (ok && lane == (uint32_t)(__ffs(same) - 1)) atomicAdd(&hist[key], (uint32_t)__popc(same));
    }
    __shared__ bool s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = atomicAdd(&hist[kSortBins], 1u) == gridDim.x - 1;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    constexpr uint32_t kStrip = kSortBins / kSortThreads;   // 128 bins per thread
    __shared__ uint32_t s_part[kSortThreads];
    uint32_t* h = hist + threadIdx.x * kStrip;
    uint32_t sum = 0;
    for (uint32_t c = 0; c < kStrip; c += 32) {
        uint32_t v[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) v[k] = __ldcg(h + c + k);
#pragma unroll
        for (int k = 0; k < 32; ++k) sum += v[k];
    }
    s_part[threadIdx.x] = sum;
    __syncthreads();
    for (uint32_t off = 1; off < kSortThreads; off <<= 1) {
        const uint32_t t = threadIdx.x >= off ? s_part[threadIdx.x - off] : 0u;
        __syncthreads();
        s_part[threadIdx.x] += t;
        __syncthreads();
    }
    uint32_t run = s_part[threadIdx.x] - sum;
    for (uint32_t c = 0; c < kStrip; c += 32) {
        uint32_t v[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) v[k] = __ldcg(h + c + k);
#pragma unroll
        for (int k = 0; k < 32; ++k) { h[c + k] = run; run += v[k]; }
    }
}

// each ray index at its key's next slot
__global__ void __launch_bounds__(kSortThreads) k_sort_scatter(const __grid_constant__ nrrs_scene s,
                                                               nrrs_ray_soa r, const uint32_t* n_dev,
                                                               uint32_t max_n, uint32_t* hist,
                                                               uint32_t* order) {
    const uint32_t n = min(*n_dev, max_n);
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warps = gridDim.x * (kSortThreads / 32);
    const uint32_t w = blockIdx.x * (kSortThreads / 32) + (threadIdx.x >> 5);
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    for (uint32_t base = w * 32; base < n; base += warps * 32) {
        const uint32_t i = base + lane;
        const bool ok = i < n;
        const uint32_t key = ok ? ray_key(s, r, i) : 0xffffffffu;
        const unsigned same = __match_any_sync(0xffffffffu, key);
        const uint32_t leader = (uint32_t)(__ffs(same) - 1);
        uint32_t slot = 0;
        if (ok && lane == leader) slot = atomicAdd(&hist[key], (uint32_t)__popc(same));
        slot = __shfl_sync(0xffffffffu, slot, (int)leader) + (uint32_t)__popc(same & lt);
        if (ok && slot < n) order[slot] = i;
    }
}

// closest hits of the first *n_dev rays, walked in `order` when given (null = queue order)
__global__ void __launch_bounds__(128) k_trace(const __grid_constant__ nrrs_scene s,
                                               nrrs_ray_soa r, const uint32_t* n_dev,
                                               uint32_t max_n, nrrs_hit_soa h,
                                               const uint32_t* order) {
    const uint32_t n = min(*n_dev, max_n);
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = order ? order[k] : k;
        if (i >= n) continue;
        Hit x{kMiss, 0.f, 0.f, 0.f};
        if (nonzero(v3(r.thp + 3 * (size_t)i)))
            x = closest_hit(s, v3(r.origin + 3 * (size_t)i), v3(r.dir + 3 * (size_t)i), INFINITY);
        h.prim[i] = x.prim;
        h.t[i] = x.t;
        h.u[i] = x.u;
        h.v[i] = x.v;
    }
}

constexpr int kShadeChunk = 1024;

__device__ __forceinline__ bool mirror_hit(const nrrs_scene& s, uint32_t prim) {
    return s.mat_spec && s.mat_spec[s.tri_mat[prim]];
}

// exclusive scan of counts[0 .. chunks) into offsets by one CTA of 256 threads (a strip per
// thread); returns the total to every thread
__device__ uint32_t block_scan_chunks(const uint32_t* counts, uint32_t* offsets, uint32_t chunks,
                                      unsigned long long* s_w) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const uint32_t per = (chunks + 255) / 256;
    const uint32_t lo = min(chunks, threadIdx.x * per), hi = min(chunks, lo + per);
    unsigned long long strip = 0;
    for (uint32_t q = lo; q < hi; ++q) strip += __ldcg(counts + q);
    unsigned long long incl = strip;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __syncthreads();
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    unsigned long long run = incl - strip, total = 0;
    for (int w = 0; w < 8; ++w) {
        if (w < wid) run += s_w[w];
        total += s_w[w];
    }
    for (uint32_t q = lo; q < hi; ++q) {
        offsets[q] = (uint32_t)run;
        run += __ldcg(counts + q);
    }
    return (uint32_t)total;
}

// surface hits per chunk of rays (inference queue and, with split, mirror queue); the last CTA
// turns the counts into offsets and the totals
__global__ void __launch_bounds__(256) k_shade_count(const __grid_constant__ nrrs_scene s,
                                                     nrrs_ray_soa r, nrrs_hit_soa h,
                                                     const uint32_t* n_dev, uint32_t max_n,
                                                     uint32_t* scratch, uint32_t* n_out,
                                                     uint32_t* n_spec_out) {
    __shared__ unsigned s_part[2][8], s_last;
    __shared__ unsigned long long s_w[8];
    const uint32_t n = min(*n_dev, max_n);
    const uint32_t chunks = (max_n + kShadeChunk - 1) / kShadeChunk;
    uint32_t* counts = scratch + 4;
    uint32_t* offsets = counts + chunks;
    uint32_t* counts_s = offsets + chunks;
    uint32_t* offsets_s = counts_s + chunks;
    const bool split = n_spec_out != nullptr;
    const uint32_t c = blockIdx.x;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned k = 0, ks = 0;
    for (uint32_t i = c * kShadeChunk + threadIdx.x; i < min(n, (c + 1) * kShadeChunk); i += 256) {
        const uint32_t prim = h.prim[i];
        if (prim == kMiss || !nonzero(v3(r.thp + 3 * (size_t)i))) continue;
        if (split && mirror_hit(s, prim)) ++ks;
        else ++k;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        k += __shfl_xor_sync(0xffffffffu, k, o);
        ks += __shfl_xor_sync(0xffffffffu, ks, o);
    }
    if (lane == 0) { s_part[0][wid] = k; s_part[1][wid] = ks; }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0, ts = 0;
        for (int w = 0; w < 8; ++w) { t += s_part[0][w]; ts += s_part[1][w]; }
        counts[c] = t;
        counts_s[c] = ts;
        __threadfence();
        s_last = atomicAdd(scratch, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    // the last CTA: exclusive scans of the chunk counts
    __threadfence();
    const uint32_t total = block_scan_chunks(counts, offsets, chunks, s_w);
    const uint32_t total_s = split ? block_scan_chunks(counts_s, offsets_s, chunks, s_w) : 0u;
    if (threadIdx.x == 255) {
        *n_out = total;
        if (split) *n_spec_out = total_s;
        scratch[0] = 0;
        __threadfence();
    }
}

__device__ __forceinline__ void put_vertex(const nrrs_path_vertices& out, size_t o, V3 pos, V3 d,
                                           V3 nrm, V3 alb, float rough, V3 thp, uint32_t depth,
                                           uint32_t pixel, int32_t node) {
    put(out.pos + 3 * o, pos);
    put(out.wi + 3 * o, mul(d, -1.0f));
    put(out.normal + 3 * o, nrm);
    put(out.albedo + 3 * o, alb);
    out.roughness[o] = rough;
    put(out.thp + 3 * o, thp);
    out.depth[o] = depth;
    out.pixel[o] = pixel;
    out.node[o] = node;
}

// emission and misses into the film; surface hits compacted in ray order into the inference
// queue `out` or, when `split` and the material is a mirror, the specular queue `outs`
__global__ void __launch_bounds__(256) k_shade(const __grid_constant__ nrrs_scene s,
                                               nrrs_ray_soa r, nrrs_hit_soa h,
                                               const uint32_t* n_dev, uint32_t max_n,
                                               uint32_t depth, int64_t* film, float* contrib,
                                               nrrs_path_vertices out, nrrs_path_vertices outs,
                                               int split, const uint32_t* scratch) {
    __shared__ unsigned s_warp[2][8];
    const uint32_t n = min(*n_dev, max_n);
    const uint32_t chunks = (max_n + kShadeChunk - 1) / kShadeChunk;
    const uint32_t c = blockIdx.x;
    const uint32_t base = scratch[4 + chunks + c];
    const uint32_t base_s = split ? scratch[4 + 3 * chunks + c] : 0u;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned lt;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
    unsigned run = 0, run_s = 0;   // vertices of the earlier passes of this chunk
    for (uint32_t j = 0; j < kShadeChunk / 256; ++j) {
        const uint32_t i = c * kShadeChunk + j * 256 + threadIdx.x;
        bool vert = false, mirror = false;
        float spec_rough = 0.0f;   // specular queue: 0 = mirror, -1 = thin glass
        V3 add_c = {0.f, 0.f, 0.f};
        V3 pos{}, nrm{}, alb{}, thp{}, d{};
        if (i < n) {
            thp = v3(r.thp + 3 * (size_t)i);
            d = v3(r.dir + 3 * (size_t)i);
            const uint32_t prim = h.prim[i];
            if (nonzero(thp)) {
                if (prim == kMiss) {
                    add_c = vmul(v3(s.env), thp);
                } else {
                    const float* tri = s.tri_in + 9 * (size_t)prim;
                    const float t = h.t[i];
                    pos = add(v3(r.origin + 3 * (size_t)i), mul(d, t));
                    const V3 g = cross(v3(tri + 3), v3(tri + 6));
                    nrm = normalize(g);
                    if (dot(nrm, d) > 0.f) nrm = mul(nrm, -1.0f);
                    const float* m = s.mats + 6 * (size_t)s.tri_mat[prim];
                    alb = v3(m);
                    const V3 le = v3(m + 3);
                    if (nonzero(le)) {
                        float w = 1.0f;
                        const float pdf = r.pdf[i];
                        if (pdf > 0.f && s.nl && s.nee) {
                            // the light pdf (solid angle) of sampling this point by NEE
                            const float area = __fmul_rn(0.5f, __fsqrt_rn(dot(g, g)));
                            const float cosl = fabsf(dot(nrm, d));
                            const float pl = __fdiv_rn(__fmul_rn(t, t),
                                                       __fmul_rn(__fmul_rn(cosl, area), (float)s.nl));
                            w = power_heuristic(pdf, pl);
                        }
                        add_c = mul(vmul(le, thp), w);
                    }
                    mirror = split && mirror_hit(s, prim);
                    vert = !mirror;
                    if (mirror && s.mat_spec[s.tri_mat[prim]] == 2) spec_rough = -1.0f;
                }
            }
            if (contrib) put(contrib + 3 * (size_t)i, add_c);
            if (nonzero(add_c)) film_add(film, r.pixel[i], add_c);
        }
        const unsigned m = __ballot_sync(0xffffffffu, vert);
        const unsigned ms = __ballot_sync(0xffffffffu, mirror);
        if (lane == 0) { s_warp[0][wid] = __popc(m); s_warp[1][wid] = __popc(ms); }
        __syncthreads();
        unsigned before = 0, total = 0, before_s = 0, total_s = 0;
        for (int w = 0; w < 8; ++w) {
            before += w < wid ? s_warp[0][w] : 0u;
            total += s_warp[0][w];
            before_s += w < wid ? s_warp[1][w] : 0u;
            total_s += s_warp[1][w];
        }
        if (vert)
            put_vertex(out, (size_t)base + run + before + __popc(m & lt), pos, d, nrm, alb, 1.0f,
                       thp, depth, r.pixel[i], r.node[i]);
        if (mirror)
            put_vertex(outs, (size_t)base_s + run_s + before_s + __popc(ms & lt), pos, d, nrm, alb,
                       spec_rough, thp, depth, r.pixel[i], r.node[i]);
        run += total;
        run_s += total_s;
        __syncthreads();
    }
}

// the specular bounce of the first *n_dev specular vertices into ray slots *off_dev + j, with
// pdf 0 (the next emitter hit counts in full), no light sampling and no RRS (the reference pushes
// these vertices to the emitted queue once, with rrs 1). A mirror (roughness 0) reflects. Thin
// glass (roughness -1, index 1.5 between air on both sides) reflects with the sheet's
// reflectance 2F/(1+F), F the unpolarised Fresnel reflectance of one face, and otherwise passes
// straight through; the choice is dimension 30 of the slot's random hash. thp x albedo either
// way. Slots at or past max_rays are dropped; *n_rays_out = min(*off_dev + *n_dev, max_rays).
constexpr uint32_t kGlassDim = 30;
__device__ __forceinline__ float sq(float x) { return __fmul_rn(x, x); }
__device__ __forceinline__ float thin_glass_reflectance(float cosi) {
    const float eta = 1.5f;
    const float sin2t = __fdiv_rn(__fsub_rn(1.0f, sq(cosi)), sq(eta));
    const float cost = __fsqrt_rn(fmaxf(__fsub_rn(1.0f, sin2t), 0.0f));
    const float rs = sq(__fdiv_rn(__fsub_rn(cosi, __fmul_rn(eta, cost)),
                                  __fadd_rn(cosi, __fmul_rn(eta, cost))));
    const float rp = sq(__fdiv_rn(__fsub_rn(__fmul_rn(eta, cosi), cost),
                                  __fadd_rn(__fmul_rn(eta, cosi), cost)));
    const float f = __fmul_rn(0.5f, __fadd_rn(rs, rp));
    return __fdiv_rn(__fmul_rn(2.0f, f), __fadd_rn(1.0f, f));
}

__global__ void __launch_bounds__(128) k_scatter_specular(nrrs_path_vertices v,
                                                          const uint32_t* n_dev, uint32_t max_n,
                                                          const uint32_t* off_dev,
                                                          uint32_t max_rays, uint32_t depth,
                                                          uint32_t seed, nrrs_ray_soa r,
                                                          uint32_t* n_rays_out) {
    const uint32_t n = min(*n_dev, max_n);
    const uint32_t off = *off_dev;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint64_t slot = (uint64_t)off + j;
        if (slot >= max_rays) continue;
        const V3 nn = v3(v.normal + 3 * (size_t)j), din = mul(v3(v.wi + 3 * (size_t)j), -1.0f);
        const V3 p = v3(v.pos + 3 * (size_t)j);
        const float dn = dot(din, nn);
        bool reflect = true;
        if (v.roughness[j] < 0.0f)   // thin glass
            reflect = rnd(seed, depth, j, kGlassDim) < thin_glass_reflectance(fabsf(dn));
        const V3 dir = reflect ? normalize(sub(din, mul(nn, __fmul_rn(2.0f, dn)))) : din;
        put(r.origin + 3 * slot, add(p, mul(nn, reflect ? kOffset : -kOffset)));
        put(r.dir + 3 * slot, dir);
        put(r.thp + 3 * slot, vmul(v3(v.thp + 3 * (size_t)j), v3(v.albedo + 3 * (size_t)j)));
        r.pdf[slot] = 0.f;
        r.pixel[slot] = v.pixel[j];
        r.node[slot] = v.node[j];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0)
        *n_rays_out = (uint32_t)min((uint64_t)off + n, (uint64_t)max_rays);
}

// generateScatteredRays for vertex x into slot j, with its throughput already divided by the RRS
// (or fixed RR) factor: one next-event-estimation shadow ray and one BSDF ray
__device__ __forceinline__ void scatter_one(const nrrs_scene& s, const nrrs_path_vertices& v,
                                            uint32_t x, uint32_t j, V3 thp, uint32_t depth,
                                            uint32_t seed, const nrrs_ray_soa& r,
                                            const nrrs_shadow_soa& sh) {
    const V3 p = v3(v.pos + 3 * (size_t)x), nn = v3(v.normal + 3 * (size_t)x);
    const V3 alb = v3(v.albedo + 3 * (size_t)x);
    const V3 f = mul(alb, kInvPi);
    const V3 org = add(p, mul(nn, kOffset));
    const uint32_t px = v.pixel[x];
    const int node = v.node[x];
    // next-event estimation: a light by index, a point by area. The shading terms use the
    // direction from the vertex; the visibility test runs from the offset origin to the light
    // point itself and stops short of it, so the light's own triangle never occludes the sample.
    V3 sc = {0.f, 0.f, 0.f}, sdir = {0.f, 0.f, 1.f};
    float smax = 0.f;
    if (s.nl && s.nee) {
        const uint32_t k = min((uint32_t)(rnd(seed, depth, j, 0) * (float)s.nl), s.nl - 1);
        const uint32_t lt = s.lights[k];
        const float* tri = s.tri_in + 9 * (size_t)lt;
        const float su = __fsqrt_rn(rnd(seed, depth, j, 1));
        const float b1 = __fsub_rn(1.0f, su), b2 = __fmul_rn(rnd(seed, depth, j, 2), su);
        const V3 q = add(add(v3(tri), mul(v3(tri + 3), b1)), mul(v3(tri + 6), b2));
        const V3 dv = sub(q, p);
        const float d2 = dot(dv, dv);
        const V3 wl = divs(dv, __fsqrt_rn(d2));
        const float cosv = dot(nn, wl);
        const float cosl = fabsf(dot(normalize(cross(v3(tri + 3), v3(tri + 6))), wl));
        const V3 le = v3(s.mats + 6 * (size_t)s.tri_mat[lt] + 3);
        const V3 ds = sub(q, org);
        const float sl = __fsqrt_rn(dot(ds, ds));
        if (cosv > 0.f && cosl > 0.f && nonzero(le) && d2 > 0.f && sl > 0.f) {
            const float pl = __fdiv_rn(d2, __fmul_rn(__fmul_rn(cosl, s.light_area[k]), (float)s.nl));
            const float w = power_heuristic(pl, __fmul_rn(cosv, kInvPi));
            sc = divs(mul(mul(vmul(vmul(thp, f), le), cosv), w), pl);
            sdir = divs(ds, sl);
            smax = __fmul_rn(sl, 0.9999f);
        }
    }
    put(sh.origin + 3 * (size_t)j, org);
    put(sh.dir + 3 * (size_t)j, sdir);
    sh.tmax[j] = smax;
    put(sh.contrib + 3 * (size_t)j, sc);
    sh.pixel[j] = px;
    sh.node[j] = node;
    // BSDF: cosine-weighted, as normalize(n + a point uniform on the unit sphere), the
    // sphere point by bounded rejection from the cube
    V3 sp = {0.f, 0.f, 1.f};
    for (uint32_t t = 0; t < 8; ++t) {
        const V3 c = {__fsub_rn(__fmul_rn(rnd(seed, depth, j, 3 + 3 * t), 2.0f), 1.0f),
                      __fsub_rn(__fmul_rn(rnd(seed, depth, j, 4 + 3 * t), 2.0f), 1.0f),
                      __fsub_rn(__fmul_rn(rnd(seed, depth, j, 5 + 3 * t), 2.0f), 1.0f)};
        const float c2 = dot(c, c);
        if (c2 <= 1.0f && c2 > 1e-6f) {
            sp = divs(c, __fsqrt_rn(c2));
            break;
        }
    }
    V3 d = add(nn, sp);
    const float l2 = dot(d, d);
    d = l2 > 1e-12f ? divs(d, __fsqrt_rn(l2)) : nn;
    const float pdf = __fmul_rn(dot(nn, d), kInvPi);
    const V3 tn = pdf > 0.f ? vmul(thp, alb) : V3{0.f, 0.f, 0.f};
    put(r.origin + 3 * (size_t)j, org);
    put(r.dir + 3 * (size_t)j, d);
    put(r.thp + 3 * (size_t)j, tn);
    r.pdf[j] = pdf > 0.f ? pdf : 0.f;
    r.pixel[j] = px;
    r.node[j] = node;
}

__global__ void __launch_bounds__(128) k_scatter(const __grid_constant__ nrrs_scene s,
                                                 nrrs_path_vertices v, const float* rrs_norm,
                                                 const uint32_t* queue, const uint32_t* q_dev,
                                                 uint32_t max_q, uint32_t depth, uint32_t seed,
                                                 nrrs_ray_soa r, nrrs_shadow_soa sh) {
    const uint32_t n = min(*q_dev, max_q);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        const uint32_t x = queue[j];
        const float rr = rrs_norm[x];
        // sitem.mThp /= sitem.mRRS
        scatter_one(s, v, x, j, divs(v3(v.thp + 3 * (size_t)x), rr), depth, seed, r, sh);
    }
}

// the fixed Russian-roulette branch: vertex j survives when its uniform number (dimension 31 of
// the slot's hash) is below rr, with thp / rr; a killed vertex leaves an empty slot
__global__ void __launch_bounds__(128) k_scatter_fixed_rr(const __grid_constant__ nrrs_scene s,
                                                          nrrs_path_vertices v, const uint32_t* n_dev,
                                                          uint32_t max_n, float rr, uint32_t depth,
                                                          uint32_t seed, nrrs_ray_soa r,
                                                          nrrs_shadow_soa sh) {
    const uint32_t n = min(*n_dev, max_n);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (rnd(seed, depth, j, kRRDim) < rr) {
            scatter_one(s, v, j, j, divs(v3(v.thp + 3 * (size_t)j), rr), depth, seed, r, sh);
            continue;
        }
        const V3 zero = {0.f, 0.f, 0.f}, up = {0.f, 0.f, 1.f};
        put(sh.origin + 3 * (size_t)j, zero);
        put(sh.dir + 3 * (size_t)j, up);
        sh.tmax[j] = 0.f;
        put(sh.contrib + 3 * (size_t)j, zero);
        sh.pixel[j] = v.pixel[j];
        sh.node[j] = v.node[j];
        put(r.origin + 3 * (size_t)j, zero);
        put(r.dir + 3 * (size_t)j, up);
        put(r.thp + 3 * (size_t)j, zero);
        r.pdf[j] = 0.f;
        r.pixel[j] = v.pixel[j];
        r.node[j] = v.node[j];
    }
}

__global__ void __launch_bounds__(128) k_shadow(const __grid_constant__ nrrs_scene s,
                                                nrrs_shadow_soa sh, const uint32_t* n_dev,
                                                uint32_t max_n, int64_t* film, float* cout) {
    const uint32_t n = min(*n_dev, max_n);
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        V3 c = v3(sh.contrib + 3 * (size_t)j);
        if (nonzero(c)) {
            if (any_hit(s, v3(sh.origin + 3 * (size_t)j), v3(sh.dir + 3 * (size_t)j), sh.tmax[j]))
                c = {0.f, 0.f, 0.f};
            else film_add(film, sh.pixel[j], c);
        }
        if (cout) put(cout + 3 * (size_t)j, c);
    }
}

__global__ void __launch_bounds__(256) k_resolve(const int64_t* film, uint32_t n, float scale,
                                                 float* img) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int64_t* l = film + 9 * (size_t)p + 3 * k;
        img[3 * (size_t)p + k] = __fmul_rn(fixed_to_float(l[0], l[1], l[2]), scale);
    }
}

// ---- host: BVH over triangle centroids, median split on the longest axis ----
struct Build {
    const std::vector<float>* tri;   // [nt][9] input order
    std::vector<uint32_t> order;
    std::vector<float> nodes;
    uint32_t max_depth = 0;
    float margin = 0.f;   // 1e-5 of the scene's largest extent (set before the build)

    void bounds(uint32_t lo, uint32_t hi, float* bmin, float* bmax) const {
        for (int k = 0; k < 3; ++k) { bmin[k] = INFINITY; bmax[k] = -INFINITY; }
        for (uint32_t i = lo; i < hi; ++i) {
            const float* t = tri->data() + 9 * (size_t)order[i];
            for (int k = 0; k < 3; ++k) {
                const float a = t[k], b = t[k] + t[3 + k], c = t[k] + t[6 + k];
                bmin[k] = std::min({bmin[k], a, b, c});
                bmax[k] = std::max({bmax[k], a, b, c});
            }
        }
        // Grow the box so that the slab test never misses a triangle the exact test hits. A slab
        // distance (lo - o) * inv carries a relative error of about 1.2e-7 of |lo - o|; the margin,
        // relative to the coordinates and to the scene's extent, stays far above that for ray
        // origins within some 80 scene extents.
        for (int k = 0; k < 3; ++k) {
            const float e = 1e-5f * (std::fabs(bmin[k]) + std::fabs(bmax[k])) + margin;
            bmin[k] -= e;
            bmax[k] += e;
        }
    }
    static float area_of(const float* lo, const float* hi) {
        const float x = hi[0] - lo[0], y = hi[1] - lo[1], z = hi[2] - lo[2];
        return x * y + y * z + z * x;
    }
    float centroid(uint32_t id, int k) const {
        const float* t = tri->data() + 9 * (size_t)id;
        return t[k] + (t[3 + k] + t[6 + k]) / 3.0f;
    }
    uint32_t alloc() {
        nodes.resize(nodes.size() + 8);
        return (uint32_t)(nodes.size() / 8 - 1);
    }
    void set_word(uint32_t me, int at, uint32_t w) { std::memcpy(&nodes[8 * (size_t)me + at], &w, 4); }
    // fills node `me` for triangles [lo, hi); children are allocated as adjacent pairs
    void build(uint32_t me, uint32_t lo, uint32_t hi, uint32_t depth) {
        max_depth = std::max(max_depth, depth);
        float bmin[3], bmax[3];
        bounds(lo, hi, bmin, bmax);
        for (int k = 0; k < 3; ++k) {
            nodes[8 * (size_t)me + k] = bmin[k];
            nodes[8 * (size_t)me + 4 + k] = bmax[k];
        }
        if (hi - lo <= (uint32_t)kLeafMax || depth + 1 >= (uint32_t)(kStack / 2)) {
            set_word(me, 3, lo);
            set_word(me, 7, hi - lo);
            return;
        }
        // binned surface-area heuristic over the centroids (32 bins per axis); a median split
        // on the longest axis when no binned cut costs less than the node's own area × count
        // (leaves hold at most kLeafMax triangles, except at the depth cap)
        float cmin[3], cmax[3];
        for (int k = 0; k < 3; ++k) { cmin[k] = INFINITY; cmax[k] = -INFINITY; }
        for (uint32_t i = lo; i < hi; ++i)
            for (int k = 0; k < 3; ++k) {
                const float c = centroid(order[i], k);
                cmin[k] = std::min(cmin[k], c);
                cmax[k] = std::max(cmax[k], c);
            }
        constexpr int kBins = 32;
        int axis = -1, cut = 0;
        float best = (float)(hi - lo) * area_of(bmin, bmax);   // the leaf's cost
        for (int k = 0; k < 3; ++k) {
            const float ext = cmax[k] - cmin[k];
            if (!(ext > 0.f)) continue;
            float lo3[kBins][3], hi3[kBins][3];
            uint32_t cnt[kBins] = {};
            for (int q = 0; q < kBins; ++q)
                for (int j = 0; j < 3; ++j) { lo3[q][j] = INFINITY; hi3[q][j] = -INFINITY; }
            for (uint32_t i = lo; i < hi; ++i) {
                const uint32_t id = order[i];
                int q = (int)((centroid(id, k) - cmin[k]) / ext * kBins);
                q = std::min(std::max(q, 0), kBins - 1);
                ++cnt[q];
                const float* t = tri->data() + 9 * (size_t)id;
                for (int j = 0; j < 3; ++j) {
                    const float a0 = t[j], a1 = t[j] + t[3 + j], a2 = t[j] + t[6 + j];
                    lo3[q][j] = std::min({lo3[q][j], a0, a1, a2});
                    hi3[q][j] = std::max({hi3[q][j], a0, a1, a2});
                }
            }
            // sweep: the cost of cutting after bin q
            float rl[kBins][3], rh[kBins][3];
            uint32_t rc[kBins];
            float al[3] = {INFINITY, INFINITY, INFINITY}, ah[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t ac = 0;
            for (int q = kBins - 1; q > 0; --q) {
                for (int j = 0; j < 3; ++j) { al[j] = std::min(al[j], lo3[q][j]); ah[j] = std::max(ah[j], hi3[q][j]); }
                ac += cnt[q];
                for (int j = 0; j < 3; ++j) { rl[q][j] = al[j]; rh[q][j] = ah[j]; }
                rc[q] = ac;
            }
            float ll[3] = {INFINITY, INFINITY, INFINITY}, lh[3] = {-INFINITY, -INFINITY, -INFINITY};
            uint32_t lc = 0;
            for (int q = 0; q < kBins - 1; ++q) {
                for (int j = 0; j < 3; ++j) { ll[j] = std::min(ll[j], lo3[q][j]); lh[j] = std::max(lh[j], hi3[q][j]); }
                lc += cnt[q];
                if (lc == 0 || rc[q + 1] == 0) continue;
                const float c = (float)lc * area_of(ll, lh) + (float)rc[q + 1] * area_of(rl[q + 1], rh[q + 1]);
                if (c < best) { best = c; axis = k; cut = q; }
            }
        }
        uint32_t mid;
        if (axis >= 0) {
            const float ext = cmax[axis] - cmin[axis];
            const auto it = std::partition(order.begin() + lo, order.begin() + hi, [&](uint32_t id) {
                int q = (int)((centroid(id, axis) - cmin[axis]) / ext * kBins);
                q = std::min(std::max(q, 0), kBins - 1);
                return q <= cut;
            });
            mid = (uint32_t)(it - order.begin());
            if (mid == lo || mid == hi) axis = -1;
        }
        if (axis < 0) {
            axis = 0;
            for (int k = 1; k < 3; ++k)
                if (bmax[k] - bmin[k] > bmax[axis] - bmin[axis]) axis = k;
            mid = lo + (hi - lo) / 2;
            std::nth_element(order.begin() + lo, order.begin() + mid, order.begin() + hi,
                             [&](uint32_t a, uint32_t b) {
                                 const float ca = centroid(a, axis), cb = centroid(b, axis);
                                 return ca < cb || (ca == cb && a < b);
                             });
        }
        const uint32_t left = alloc();
        alloc();
        set_word(me, 3, left);
        set_word(me, 7, (uint32_t)axis << 16);
        build(left, lo, mid, depth + 1);
        build(left + 1, mid, hi, depth + 1);
    }
};

template <typename T>
cudaError_t upload(T** dst, const T* src, size_t count) {
    if (count == 0) { *dst = nullptr; return cudaSuccess; }
    cudaError_t e = cudaMalloc(dst, sizeof(T) * count);
    if (e == cudaSuccess) e = cudaMemcpy(*dst, src, sizeof(T) * count, cudaMemcpyHostToDevice);
    return e;
}

// a grid-stride kernel's grid: per_sm CTAs per SM, or fewer when n needs fewer. The traversal
// kernels take 64: rays differ widely in cost, and many short CTAs let the SMs refill as they end.
int grid_of(uint32_t n, int threads, int per_sm = 16) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t need = ((uint64_t)n + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sms * per_sm;
    return (int)std::max<uint64_t>(1, std::min(need, cap));
}

int ok(cudaError_t e) { return e == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA; }

}  // namespace
}  // namespace nrrs

using namespace nrrs;

extern "C" int nrrs_scene_create(const float* vertices, uint32_t n_vertices,
                                 const uint32_t* triangles, uint32_t n_triangles,
                                 const uint32_t* tri_material, const float* materials,
                                 uint32_t n_materials, const float* environment,
                                 nrrs_scene** out) {
    if (!out || !vertices || !triangles || !tri_material || !materials || n_triangles == 0 ||
        n_materials == 0 || n_triangles > (1u << 30))
        return NRRS_ERR_INVALID_ARG;
    if (nrrs_device_available() != 1) return NRRS_ERR_NO_DEVICE;
    std::vector<float> tri(9 * (size_t)n_triangles);
    std::vector<uint32_t> lights;
    std::vector<float> areas;
    for (uint32_t i = 0; i < n_triangles; ++i) {
        uint32_t idx[3];
        for (int k = 0; k < 3; ++k) {
            idx[k] = triangles[3 * (size_t)i + k];
            if (idx[k] >= n_vertices) return NRRS_ERR_INVALID_ARG;
        }
        if (tri_material[i] >= n_materials) return NRRS_ERR_INVALID_ARG;
        const float* a = vertices + 3 * (size_t)idx[0];
        const float* b = vertices + 3 * (size_t)idx[1];
        const float* c = vertices + 3 * (size_t)idx[2];
        float* t = &tri[9 * (size_t)i];
        for (int k = 0; k < 3; ++k) { t[k] = a[k]; t[3 + k] = b[k] - a[k]; t[6 + k] = c[k] - a[k]; }
        const float* m = materials + 6 * (size_t)tri_material[i];
        if (m[3] != 0.f || m[4] != 0.f || m[5] != 0.f) {
            // area = 0.5 |e1 x e2|, each operation rounded on its own
            const float cx = t[4] * t[8] - t[5] * t[7], cy = t[5] * t[6] - t[3] * t[8],
                        cz = t[3] * t[7] - t[4] * t[6];
            const float area = 0.5f * std::sqrt((cx * cx + cy * cy) + cz * cz);
            if (area > 0.f) { lights.push_back(i); areas.push_back(area); }
        }
    }
    Build b;
    b.tri = &tri;
    b.order.resize(n_triangles);
    std::iota(b.order.begin(), b.order.end(), 0u);
    {
        float lo[3], hi[3];
        b.bounds(0, n_triangles, lo, hi);   // margin 0 here: the scene's own bounds
        float ext = 0.f;
        for (int k = 0; k < 3; ++k) ext = std::max(ext, hi[k] - lo[k]);
        b.margin = 1e-5f * ext;
    }
    b.build(b.alloc(), 0, n_triangles, 0);
    std::vector<float> tri_leaf(12 * (size_t)n_triangles, 0.f);
    for (uint32_t i = 0; i < n_triangles; ++i)
        std::memcpy(&tri_leaf[12 * (size_t)i], &tri[9 * (size_t)b.order[i]], 36);
    nrrs_scene* s = new (std::nothrow) nrrs_scene();
    if (!s) return NRRS_ERR_INVALID_ARG;
    s->nt = n_triangles;
    s->nn = (uint32_t)(b.nodes.size() / 8);
    s->nl = (uint32_t)lights.size();
    s->nm = n_materials;
    s->max_depth = b.max_depth;
    if (environment) for (int k = 0; k < 3; ++k) s->env[k] = environment[k];
    cudaError_t e = upload(&s->tris, tri_leaf.data(), tri_leaf.size());
    if (e == cudaSuccess) e = upload(&s->tri_id, b.order.data(), b.order.size());
    if (e == cudaSuccess) e = upload(&s->tri_mat, tri_material, n_triangles);
    if (e == cudaSuccess) e = upload(&s->tri_in, tri.data(), tri.size());
    if (e == cudaSuccess) e = upload(&s->nodes, b.nodes.data(), b.nodes.size());
    if (e == cudaSuccess) e = upload(&s->mats, materials, 6 * (size_t)n_materials);
    if (e == cudaSuccess) e = upload(&s->lights, lights.data(), lights.size());
    if (e == cudaSuccess) e = upload(&s->light_area, areas.data(), areas.size());
    if (e != cudaSuccess) {
        nrrs_scene_destroy(s);
        return NRRS_ERR_CUDA;
    }
    *out = s;
    return NRRS_OK;
}

extern "C" void nrrs_scene_destroy(nrrs_scene* s) {
    if (!s) return;
    cudaFree(s->tris); cudaFree(s->tri_id); cudaFree(s->tri_mat); cudaFree(s->tri_in);
    cudaFree(s->nodes); cudaFree(s->mats); cudaFree(s->lights); cudaFree(s->light_area);
    cudaFree(s->mat_spec);
    delete s;
}

extern "C" int nrrs_scene_set_nee(nrrs_scene* s, int32_t enable) {
    if (!s || (enable != 0 && enable != 1)) return NRRS_ERR_INVALID_ARG;
    s->nee = (uint32_t)enable;
    return NRRS_OK;
}

extern "C" int nrrs_scene_info(const nrrs_scene* s, uint32_t* n_nodes, uint32_t* n_lights,
                               uint32_t* max_depth) {
    if (!s) return NRRS_ERR_INVALID_ARG;
    if (n_nodes) *n_nodes = s->nn;
    if (n_lights) *n_lights = s->nl;
    if (max_depth) *max_depth = s->max_depth;
    return NRRS_OK;
}

extern "C" int nrrs_camera_rays(const nrrs_camera* c, uint32_t sample, uint32_t seed,
                                const nrrs_ray_soa* rays, void* stream) {
    if (!c || !rays || c->width == 0 || c->height == 0) return NRRS_ERR_INVALID_ARG;
    const uint32_t n = c->width * c->height;
    k_camera<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*c, sample, seed, *rays);
    return ok(cudaGetLastError());
}

extern "C" int nrrs_trace(const nrrs_scene* s, const nrrs_ray_soa* rays, const uint32_t* n_dev,
                          uint32_t max_n, const nrrs_hit_soa* hits, void* stream) {
    if (!s || !rays || !n_dev || !hits) return NRRS_ERR_INVALID_ARG;
    if (max_n == 0) return NRRS_OK;
    k_trace<<<grid_of(max_n, 128, 64), 128, 0, (cudaStream_t)stream>>>(*s, *rays, n_dev, max_n,
                                                                        *hits, nullptr);
    return ok(cudaGetLastError());
}

extern "C" uint64_t nrrs_trace_scratch_bytes(uint32_t max_n) {
    return 4ull * (kSortBins + 64) + 4ull * max_n;
}

extern "C" int nrrs_trace_sorted(const nrrs_scene* s, const nrrs_ray_soa* rays,
                                 const uint32_t* n_dev, uint32_t max_n, const nrrs_hit_soa* hits,
                                 void* scratch, void* stream) {
    if (!s || !rays || !n_dev || !hits || !scratch) return NRRS_ERR_INVALID_ARG;
    if (max_n == 0) return NRRS_OK;
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t* order = nullptr;
    if (max_n >= kSortMinRays) {
        uint32_t* hist = static_cast<uint32_t*>(scratch);
        uint32_t* ord = hist + kSortBins + 64;
        if (cudaMemsetAsync(hist, 0, 4ull * (kSortBins + 1), st) != cudaSuccess)
            return NRRS_ERR_CUDA;
        const int g = grid_of(max_n, kSortThreads, 8);
        k_sort_count<<<g, kSortThreads, 0, st>>>(*s, *rays, n_dev, max_n, hist);
        k_sort_scatter<<<g, kSortThreads, 0, st>>>(*s, *rays, n_dev, max_n, hist, ord);
        order = ord;
    }
    k_trace<<<grid_of(max_n, 128, 64), 128, 0, st>>>(*s, *rays, n_dev, max_n, *hits, order);
    return ok(cudaGetLastError());
}

extern "C" uint64_t nrrs_shade_scratch_bytes(uint32_t max_n) {
    const uint64_t chunks = ((uint64_t)max_n + kShadeChunk - 1) / kShadeChunk;
    return 4ull * (4 + 4 * chunks);
}

extern "C" int nrrs_shade_split(const nrrs_scene* s, const nrrs_ray_soa* rays,
                                const nrrs_hit_soa* hits, const uint32_t* n_dev, uint32_t max_n,
                                uint32_t depth, int64_t* film, float* contrib,
                                const nrrs_path_vertices* out, uint32_t* n_out_dev,
                                const nrrs_path_vertices* out_specular, uint32_t* n_specular_dev,
                                void* scratch, void* stream) {
    if (!s || !rays || !hits || !n_dev || !film || !out || !n_out_dev || !scratch ||
        (!out_specular) != (!n_specular_dev))
        return NRRS_ERR_INVALID_ARG;
    cudaStream_t st = (cudaStream_t)stream;
    if (max_n == 0) {
        if (n_specular_dev && cudaMemsetAsync(n_specular_dev, 0, 4, st) != cudaSuccess)
            return NRRS_ERR_CUDA;
        return ok(cudaMemsetAsync(n_out_dev, 0, 4, st));
    }
    const uint32_t chunks = (max_n + kShadeChunk - 1) / kShadeChunk;
    uint32_t* sc = static_cast<uint32_t*>(scratch);
    if (cudaMemsetAsync(sc, 0, 4, st) != cudaSuccess) return NRRS_ERR_CUDA;   // the done counter
    const int split = out_specular != nullptr;
    k_shade_count<<<chunks, 256, 0, st>>>(*s, *rays, *hits, n_dev, max_n, sc, n_out_dev,
                                          n_specular_dev);
    k_shade<<<chunks, 256, 0, st>>>(*s, *rays, *hits, n_dev, max_n, depth, film, contrib, *out,
                                    split ? *out_specular : *out, split, sc);
    return ok(cudaGetLastError());
}

extern "C" int nrrs_shade(const nrrs_scene* s, const nrrs_ray_soa* rays, const nrrs_hit_soa* hits,
                          const uint32_t* n_dev, uint32_t max_n, uint32_t depth, int64_t* film,
                          float* contrib, const nrrs_path_vertices* out, uint32_t* n_out_dev,
                          void* scratch, void* stream) {
    return nrrs_shade_split(s, rays, hits, n_dev, max_n, depth, film, contrib, out, n_out_dev,
                            nullptr, nullptr, scratch, stream);
}

extern "C" int nrrs_scatter_specular(const nrrs_scene* s, const nrrs_path_vertices* v,
                                     const uint32_t* n_dev, uint32_t max_n,
                                     const uint32_t* ray_offset_dev, uint32_t max_rays,
                                     uint32_t depth, uint32_t seed, const nrrs_ray_soa* rays,
                                     uint32_t* n_rays_out_dev, void* stream) {
    if (!s || !v || !n_dev || !ray_offset_dev || !rays || !n_rays_out_dev ||
        n_rays_out_dev == ray_offset_dev)
        return NRRS_ERR_INVALID_ARG;
    k_scatter_specular<<<grid_of(std::max(max_n, 1u), 128), 128, 0, (cudaStream_t)stream>>>(
        *v, n_dev, max_n, ray_offset_dev, max_rays, depth, seed, *rays, n_rays_out_dev);
    return ok(cudaGetLastError());
}

extern "C" int nrrs_scene_set_specular(nrrs_scene* s, const uint8_t* specular,
                                       uint32_t n_materials) {
    if (!s || !specular || n_materials != s->nm) return NRRS_ERR_INVALID_ARG;
    for (uint32_t m = 0; m < n_materials; ++m)
        if (specular[m] > 2) return NRRS_ERR_INVALID_ARG;
    if (!s->mat_spec && cudaMalloc(&s->mat_spec, n_materials) != cudaSuccess) {
        s->mat_spec = nullptr;
        return NRRS_ERR_CUDA;
    }
    return ok(cudaMemcpy(s->mat_spec, specular, n_materials, cudaMemcpyHostToDevice));
}

extern "C" int nrrs_scatter(const nrrs_scene* s, const nrrs_path_vertices* v, const float* rrs_norm,
                            const uint32_t* queue, const uint32_t* queue_size_dev,
                            uint32_t max_queue, uint32_t depth, uint32_t seed,
                            const nrrs_ray_soa* rays, const nrrs_shadow_soa* shadow,
                            void* stream) {
    if (!s || !v || !rrs_norm || !queue || !queue_size_dev || !rays || !shadow)
        return NRRS_ERR_INVALID_ARG;
    if (max_queue == 0) return NRRS_OK;
    k_scatter<<<grid_of(max_queue, 128), 128, 0, (cudaStream_t)stream>>>(
        *s, *v, rrs_norm, queue, queue_size_dev, max_queue, depth, seed, *rays, *shadow);
    return ok(cudaGetLastError());
}

extern "C" int nrrs_scatter_fixed_rr(const nrrs_scene* s, const nrrs_path_vertices* v,
                                     const uint32_t* n_dev, uint32_t max_n, float rr,
                                     uint32_t depth, uint32_t seed, const nrrs_ray_soa* rays,
                                     const nrrs_shadow_soa* shadow, void* stream) {
    if (!s || !v || !n_dev || !rays || !shadow || !(rr > 0.f && rr <= 1.f))
        return NRRS_ERR_INVALID_ARG;
    if (max_n == 0) return NRRS_OK;
    k_scatter_fixed_rr<<<grid_of(max_n, 128), 128, 0, (cudaStream_t)stream>>>(
        *s, *v, n_dev, max_n, rr, depth, seed, *rays, *shadow);
    return ok(cudaGetLastError());
}

extern "C" int nrrs_trace_shadow(const nrrs_scene* s, const nrrs_shadow_soa* shadow,
                                 const uint32_t* n_dev, uint32_t max_n, int64_t* film,
                                 float* contrib_out, void* stream) {
    if (!s || !shadow || !n_dev || !film) return NRRS_ERR_INVALID_ARG;
    if (max_n == 0) return NRRS_OK;
    k_shadow<<<grid_of(max_n, 128, 64), 128, 0, (cudaStream_t)stream>>>(
        *s, *shadow, n_dev, max_n, film, contrib_out);
    return ok(cudaGetLastError());
}

extern "C" int nrrs_film_resolve(const int64_t* film, uint32_t n_pixels, float scale, float* image,
                                 void* stream) {
    if (!film || !image) return NRRS_ERR_INVALID_ARG;
    if (n_pixels == 0) return NRRS_OK;
    k_resolve<<<(n_pixels + 255) / 256, 256, 0, (cudaStream_t)stream>>>(film, n_pixels, scale, image);
    return ok(cudaGetLastError());
}
