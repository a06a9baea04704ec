// k_pixel_error.cu -- per-pixel error of the RRSNet loss: patch sample counts, the blended
// radiance estimate per patch, its relative error against the rendered film and the exact sum
// of the errors. Kernels and their C-ABI (include/nrrs.h).
//
// Replaces, in banbao990/NRRS-Code:
//   patch sample counts            src/render/nrrs/integrator.cpp:1027-1050, 803-808
//   weighted L (first frame, STEP#1.1)   src/render/nrrs/integrator.cpp:2358-2395
//   nrrs_update_weighted_L         src/render/nrrs/train.cu:344-363
//   nrrs_calculate_error           src/render/nrrs/train.cu:365-430
//   the error sum                  src/render/nrrs/integrator.cpp:2466-2471
//   nrrs_UBS_calc_error and its sum  src/render/nrrs/train.cu:594-608, integrator.cpp:2875-2886
//
// A patch is a scale x scale block of frame pixels (offsetFrame2Scaled, myFilm.h:6-15). The
// reference adds a patch's pixels with FP32 atomics in scheduling order; here one thread per
// patch adds them in pixel order, so the results do not depend on scheduling. Every FP32
// operation is written out (no contraction). The error sum is exact: fixed-point limbs added as
// integers, rounded once at the end.
#include <cmath>

#include "fixed_point.cuh"
#include "nrrs.h"

namespace nrrs {
namespace {

struct PatchGeom {
    uint32_t w, h, s;   // frame width, height, patch size
    uint32_t pw, ph;    // patches per row, rows of patches
};

PatchGeom geom_of(const nrrs_pixel_error_params& p) {
    PatchGeom g{};
    g.w = p.frame_width;
    g.h = p.frame_height;
    g.s = p.scale ? p.scale : 1u;
    g.pw = g.w / g.s;
    g.ph = g.h / g.s;
    return g;
}

__device__ __forceinline__ uint32_t patch_of(const PatchGeom& g, uint32_t px) {
    return (px % g.w) / g.s + ((px / g.w) / g.s) * g.pw;
}

__global__ void __launch_bounds__(256) k_count_patch(PatchGeom g, const uint32_t* pixel,
                                                     uint32_t n, float* spp) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t px = pixel[i];
    if (px >= g.w * g.h) return;
    atomicAdd(spp + patch_of(g, px), 1.0f);  // integer-valued: exact below 2^24, any order
}

__global__ void __launch_bounds__(256) k_accumulate(PatchGeom g, const float* __restrict__ pl,
                                                    uint32_t spp, int first, float* wl,
                                                    float* cur, uint32_t* acc) {
    const uint32_t ps = blockIdx.x * blockDim.x + threadIdx.x;
    if (ps >= g.pw * g.ph) return;
    const uint32_t x0 = (ps % g.pw) * g.s, y0 = (ps / g.pw) * g.s;
    const float fspp = (float)spp;
    float c[3] = {0.f, 0.f, 0.f}, f[3] = {0.f, 0.f, 0.f};
    for (uint32_t dy = 0; dy < g.s; ++dy)
        for (uint32_t dx = 0; dx < g.s; ++dx) {
            const size_t px = (size_t)(y0 + dy) * g.w + x0 + dx;
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                const float l = pl[3 * px + k];
                c[k] = __fadd_rn(c[k], l);
                if (first) f[k] = __fadd_rn(f[k], __fdiv_rn(l, fspp));
            }
        }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        cur[3 * (size_t)ps + k] = c[k];
        if (first) wl[3 * (size_t)ps + k] = f[k];
    }
    acc[ps] = spp * g.s * g.s;
}

__global__ void __launch_bounds__(256) k_update(PatchGeom g, const float* __restrict__ cur,
                                                const uint32_t* __restrict__ acc, float blend,
                                                float* wl) {
    const uint32_t ps = blockIdx.x * blockDim.x + threadIdx.x;
    if (ps >= g.pw * g.ph) return;
    const float n = (float)acc[ps];   // 0 gives the reference's division by zero
    const float keep = __fsub_rn(1.0f, blend);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float lc = __fdiv_rn(cur[3 * (size_t)ps + k], n);
        const float lb = wl[3 * (size_t)ps + k];
        wl[3 * (size_t)ps + k] = __fadd_rn(__fmul_rn(lb, keep), __fmul_rn(lc, blend));
    }
}

constexpr uint32_t kSumNaN = 0x80000000u;  // `done` bit: some error was not summable

// Adds each thread's limbs l (or its bad mark) into sum, one atomic per limb and CTA; the last
// CTA rounds the total once and leaves the accumulators at zero. Every thread of the CTA calls.
__device__ void add_to_sum(const long long l[3], bool bad, nrrs_error_sum* sum) {
    __shared__ long long s_part[3][8];
    __shared__ unsigned s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    if (bad) s_bad = 1;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        long long v = l[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) s_part[k][wid] = v;
    }
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int k = 0; k < 3; ++k) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x / 32); ++w) t += (unsigned long long)s_part[k][w];
        if (t) atomicAdd(reinterpret_cast<unsigned long long*>(&sum->acc[k]), t);
    }
    if (s_bad) atomicOr(&sum->done, kSumNaN);
    __threadfence();
    const unsigned old = atomicAdd(&sum->done, 1u);
    if ((old & ~kSumNaN) != gridDim.x - 1) return;
    __threadfence();
    long long a[3];
    for (int k = 0; k < 3; ++k)
        a[k] = (long long)atomicAdd(reinterpret_cast<unsigned long long*>(&sum->acc[k]), 0ull);
    const bool nan = (old & kSumNaN) || s_bad;
    sum->value = nan ? __int_as_float(0x7fc00000) : fixed_to_float(a[0], a[1], a[2]);
    sum->acc[0] = sum->acc[1] = sum->acc[2] = 0;
    sum->done = 0;
    __threadfence();
}

// mean_c (l_c - r_c)^2 / (r_c^2 + 0.01), FP32 written out
__device__ __forceinline__ float rel_error(const float* l, const float* r) {
    float q[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float d = __fsub_rn(l[k], r[k]);
        q[k] = __fdiv_rn(__fmul_rn(d, d), __fadd_rn(__fmul_rn(r[k], r[k]), 0.01f));
    }
    return __fdiv_rn(__fadd_rn(__fadd_rn(q[0], q[1]), q[2]), 3.0f);
}

__global__ void __launch_bounds__(256) k_error(PatchGeom g, const float* __restrict__ ref,
                                               uint32_t ch, const float* __restrict__ wl,
                                               const float* __restrict__ spp, int clamp,
                                               int mult, float* err_out, nrrs_error_sum* sum) {
    const uint32_t ps = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t np = g.pw * g.ph, npix = g.w * g.h;
    long long l[3] = {0, 0, 0};
    bool bad = false;
    if (ps < np) {
        float e = rel_error(wl + 3 * (size_t)ps, ref + (size_t)ps * ch);
        if (clamp) e = fminf(e, 100.0f);   // fminf: a NaN error becomes 100, as min() does there
        err_out[ps] = e;
        if (mult) e = __fmul_rn(e, __fsqrt_rn(spp[ps]));
        err_out[npix + ps] = e;
        if (fixed_ok(e)) fixed_limbs(e, l);
        else bad = true;
    }
    if (sum) add_to_sum(l, bad, sum);
}

// nrrs_UBS_calc_error (train.cu:594-608): per frame pixel, the film read at its patch
__global__ void __launch_bounds__(256) k_ubs_error(PatchGeom g, const float* __restrict__ pl,
                                                   uint32_t spp, const float* __restrict__ ref,
                                                   uint32_t ch, float* err_out,
                                                   nrrs_error_sum* sum) {
    const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x;
    long long l[3] = {0, 0, 0};
    bool bad = false;
    if (px < g.w * g.h) {
        const float fspp = (float)spp;
        float L[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) L[k] = __fdiv_rn(pl[3 * (size_t)px + k], fspp);
        const float e = rel_error(L, ref + (size_t)patch_of(g, px) * ch);
        err_out[px] = e;
        if (fixed_ok(e)) fixed_limbs(e, l);
        else bad = true;
    }
    if (sum) add_to_sum(l, bad, sum);
}

int check_geom(const nrrs_pixel_error_params* p) {
    if (!p || p->frame_width == 0 || p->frame_height == 0) return NRRS_ERR_INVALID_ARG;
    const uint32_t s = p->scale ? p->scale : 1u;
    if (p->frame_width % s || p->frame_height % s) return NRRS_ERR_INVALID_ARG;
    if ((uint64_t)p->frame_width * p->frame_height > 0xffffffffull / 2) return NRRS_ERR_INVALID_ARG;
    return NRRS_OK;
}

int done(cudaError_t e) { return e == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA; }

}  // namespace
}  // namespace nrrs

using namespace nrrs;

extern "C" int nrrs_count_patch_samples(const nrrs_pixel_error_params* p, const uint32_t* pixel,
                                        uint32_t n, float* samples_per_patch, void* stream) {
    int rc = check_geom(p);
    if (rc != NRRS_OK) return rc;
    if (n == 0) return NRRS_OK;
    if (!pixel || !samples_per_patch) return NRRS_ERR_INVALID_ARG;
    k_count_patch<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(geom_of(*p), pixel, n,
                                                                      samples_per_patch);
    return done(cudaGetLastError());
}

extern "C" int nrrs_accumulate_weighted_l(const nrrs_pixel_error_params* p, const float* pixel_l,
                                          uint32_t spp_this_frame, int32_t first_frame,
                                          float* weighted_l, float* weighted_l_current,
                                          uint32_t* weighted_l_current_acc, void* stream) {
    int rc = check_geom(p);
    if (rc != NRRS_OK) return rc;
    if (!pixel_l || !weighted_l_current || !weighted_l_current_acc || (first_frame && !weighted_l))
        return NRRS_ERR_INVALID_ARG;
    const PatchGeom g = geom_of(*p);
    const uint32_t np = g.pw * g.ph;
    k_accumulate<<<(np + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        g, pixel_l, spp_this_frame, first_frame ? 1 : 0, weighted_l, weighted_l_current,
        weighted_l_current_acc);
    return done(cudaGetLastError());
}

extern "C" int nrrs_update_weighted_l(const nrrs_pixel_error_params* p,
                                      const float* weighted_l_current,
                                      const uint32_t* weighted_l_current_acc, float* weighted_l,
                                      void* stream) {
    int rc = check_geom(p);
    if (rc != NRRS_OK) return rc;
    if (!weighted_l_current || !weighted_l_current_acc || !weighted_l) return NRRS_ERR_INVALID_ARG;
    const PatchGeom g = geom_of(*p);
    const uint32_t np = g.pw * g.ph;
    k_update<<<(np + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        g, weighted_l_current, weighted_l_current_acc, p->blend_weight, weighted_l);
    return done(cudaGetLastError());
}

extern "C" int nrrs_calculate_error(const nrrs_pixel_error_params* p, const float* ref,
                                    int32_t ref_channels, const float* weighted_l,
                                    const float* samples_per_patch, float* error,
                                    nrrs_error_sum* sum, void* stream) {
    int rc = check_geom(p);
    if (rc != NRRS_OK) return rc;
    if (!ref || (ref_channels != 3 && ref_channels != 4) || !weighted_l || !error)
        return NRRS_ERR_INVALID_ARG;
    if (p->multiply_samples && !samples_per_patch) return NRRS_ERR_INVALID_ARG;
    const PatchGeom g = geom_of(*p);
    const uint32_t np = g.pw * g.ph;
    k_error<<<(np + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        g, ref, (uint32_t)ref_channels, weighted_l, samples_per_patch, p->clamp ? 1 : 0,
        p->multiply_samples ? 1 : 0, error, sum);
    return done(cudaGetLastError());
}

extern "C" int nrrs_ubs_error(const nrrs_pixel_error_params* p, const float* pixel_l, uint32_t spp,
                              const float* ref, int32_t ref_channels, float* error,
                              nrrs_error_sum* sum, void* stream) {
    int rc = check_geom(p);
    if (rc != NRRS_OK) return rc;
    if (!pixel_l || !ref || (ref_channels != 3 && ref_channels != 4) || !error)
        return NRRS_ERR_INVALID_ARG;
    const PatchGeom g = geom_of(*p);
    const uint32_t n = g.w * g.h;
    k_ubs_error<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        g, pixel_l, spp, ref, (uint32_t)ref_channels, error, sum);
    return done(cudaGetLastError());
}
