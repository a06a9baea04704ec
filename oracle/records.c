/*
 * records.c -- CPU oracle of the path-node records and the training batch. TEST INFRASTRUCTURE
 * ONLY: only tests/ and bench.py's cpu_baseline leg load it, never the product library.
 *
 * A sequential restatement of, in banbao990/NRRS-Code:
 *   NRRSPathNodesBuffer::recordNode      src/render/nrrs/workqueue.h:142-170
 *   NRRSPathNodesBuffer::recordRadiance  src/render/nrrs/workqueue.h:122-136
 *   nrrs_generate_training_data          src/render/nrrs/train.cu:432-570
 *   nrrs_calculate_sample_weight         src/render/nrrs/train.cu:572-592
 * with the order the library defines where the reference's depends on atomics: nodes and samples
 * in input order, the lowest-index child keeping its RRSNet target, and radiance summed as exact
 * fixed-point integers (three signed 64-bit limbs per channel, lowest bit 2^-64). The radiance is
 * walked up the parent chain at record time, as the reference does; the library defers the
 * ancestors to one pass over the nodes, and both must give the same integers.
 *
 * The node block is the library's own struct, nrrs_path_nodes, pointing at HOST arrays; the
 * header words are size, dropped, radiance-complete mark and status, as in the library.
 * The fixed-point conversion is checked against gcc's correctly rounded __int128 -> float.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "nrrs_oracle.h"

enum { HDR_SIZE = 0, HDR_DROPPED = 1, HDR_STATUS = 4 };

#define FIXED_MAX 4611686018427387904.0f /* 2^62 */

/* trunc(|x| 2^64) split into bits [0,32), [32,64) and [64,128), each signed like x */
void oracle_fixed_limbs(float x, int64_t* l) {
    uint32_t bits;
    memcpy(&bits, &x, 4);
    const uint32_t e = (bits >> 23) & 0xffu;
    const uint64_t m = (bits & 0x7fffffu) | (e ? 0x800000u : 0u);
    const int sh = (int)(e ? e : 1u) - 150 + 64;
    unsigned __int128 X;
    if (sh >= 0) X = (unsigned __int128)m << sh;
    else X = (-sh) >= 24 ? 0 : (unsigned __int128)(m >> (-sh));
    const uint64_t lo = (uint64_t)X;
    int64_t l0 = (int64_t)(lo & 0xffffffffu), l1 = (int64_t)(lo >> 32);
    int64_t l2 = (int64_t)(uint64_t)(X >> 64);
    if (bits >> 31) { l0 = -l0; l1 = -l1; l2 = -l2; }
    l[0] = l0; l[1] = l1; l[2] = l2;
}

/* (l0 + l1 2^32 + l2 2^64) 2^-64 to the nearest float, ties to even, by integer arithmetic */
float oracle_fixed_to_float(int64_t l0, int64_t l1, int64_t l2) {
    typedef unsigned __int128 u128;
    const u128 U = ((u128)(__int128)l2 << 64) + ((u128)(__int128)l1 << 32) + (u128)(__int128)l0;
    const uint32_t neg = (uint32_t)(U >> 127) & 1u;
    const u128 mag = neg ? (u128)0 - U : U;
    if (mag == 0) return 0.0f;
    const uint64_t hi = (uint64_t)(mag >> 64), lo = (uint64_t)mag;
    const int msb = hi ? 127 - __builtin_clzll(hi) : 63 - __builtin_clzll(lo);
    int ex = msb - 64;
    uint32_t mant;
    if (msb <= 23) {
        mant = (uint32_t)(lo << (23 - msb));
    } else {
        const int sh = msb - 23;
        const u128 q = mag >> sh, rem = mag - (q << sh), half = (u128)1 << (sh - 1);
        mant = (uint32_t)q;
        if (rem > half || (rem == half && (mant & 1u))) {
            ++mant;
            if (mant == (1u << 24)) { mant >>= 1; ++ex; }
        }
    }
    const uint32_t bits = (neg << 31) | ((uint32_t)(ex + 127) << 23) | (mant & 0x7fffffu);
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

/* The library's formulation of the same rounding: the top 64 bits of the magnitude with the
 * bits below folded into bit 0, one correctly rounded u64 -> float conversion, an exact
 * power-of-two scale. Must equal oracle_fixed_to_float everywhere. */
float oracle_fixed_to_float_fast(int64_t l0, int64_t l1, int64_t l2) {
    typedef unsigned __int128 u128;
    const u128 U = ((u128)(__int128)l2 << 64) + ((u128)(__int128)l1 << 32) + (u128)(__int128)l0;
    const uint32_t neg = (uint32_t)(U >> 127) & 1u;
    const u128 mag = neg ? (u128)0 - U : U;
    const uint64_t hi = (uint64_t)(mag >> 64), lo = (uint64_t)mag;
    float f;
    if (hi == 0) {
        f = (float)lo * 0x1p-64f;
    } else {
        const int sh = 64 - __builtin_clzll(hi);
        const uint64_t top = (hi << (64 - sh)) | (lo >> sh) | ((lo << (64 - sh)) != 0 ? 1u : 0u);
        f = ldexpf((float)top, sh - 64);
    }
    return neg ? -f : f;
}

/* the same value through gcc's own __int128 -> float conversion (round to nearest), for tests */
float oracle_fixed_to_float_gcc(int64_t l0, int64_t l1, int64_t l2) {
    typedef unsigned __int128 u128;
    const u128 U = ((u128)(__int128)l2 << 64) + ((u128)(__int128)l1 << 32) + (u128)(__int128)l0;
    return (float)(__int128)U * 0x1p-64f;
}

void oracle_nodes_reset(nrrs_path_nodes* nb) {
    nb->header[HDR_SIZE] = 0;
    nb->header[HDR_DROPPED] = 0;
    nb->header[2] = 0;
    nb->header[3] = 0;
}

/* recordNode (workqueue.h:142-170) for each recorded vertex, in vertex order; node_out[i] =
 * the node, or parent[i] when the vertex records nothing or the buffer is full
 * (integrator.cpp:828-830, 1436-1438) */
void oracle_record_nodes(nrrs_path_nodes* nb, const nrrs_vertex_soa* v, const int32_t* parent,
                         const uint32_t* pixel, const float* rrs, const uint8_t* record,
                         uint64_t n, int32_t* node_out) {
    const uint32_t call0 = nb->header[HDR_SIZE];  /* nodes of earlier calls: [0, call0) */
    for (uint64_t i = 0; i < n; ++i) {
        const int32_t p = parent[i];
        /* a parent must be a node of an earlier call: any other link is cut and flagged */
        const int bad_parent = p >= 0 && (uint32_t)p >= call0;
        const int32_t pn = bad_parent ? -1 : p;
        int32_t out = p;
        if (!record || record[i]) {
            const uint32_t idx = nb->header[HDR_SIZE];
            if (idx < nb->capacity) {
                nb->header[HDR_SIZE] = idx + 1;
                for (int k = 0; k < 3; ++k) {
                    const uint64_t di = 3 * (uint64_t)idx + k, si = 3 * i + k;
                    nb->pos[di] = v->pos[si];
                    nb->wi[di] = v->wi[si];
                    nb->normal[di] = v->normal ? v->normal[si] : 0.f;
                    nb->albedo[di] = v->albedo ? v->albedo[si] : 0.f;
                    nb->thp[di] = v->thp[si];
                }
                nb->roughness[idx] = v->roughness ? v->roughness[i] : 0.f;
                nb->parent[idx] = pn;
                nb->pixel[idx] = pixel[i];
                nb->rrs[idx] = rrs ? rrs[i] : 1.f;  /* the work item's default (device.cu:83) */
                nb->depth[idx] = v->depth ? v->depth[i] : 0u;
                memset(nb->radiance + 9 * (uint64_t)idx, 0, 9 * sizeof(int64_t));
                nb->first_child[idx] = 0xffffffffu;
                nb->children[idx] = 0;
                nb->node_flags[idx] = 0;
                if (pn >= 0) {
                    if (idx < nb->first_child[pn]) nb->first_child[pn] = idx;
                    nb->children[pn] += 1;
                }
                if (bad_parent) nb->header[HDR_STATUS] |= NRRS_DEV_BAD_INDEX;
                out = (int32_t)idx;
            } else {
                nb->header[HDR_DROPPED] += 1;  /* mInvalidNode */
                nb->header[HDR_STATUS] |= NRRS_DEV_OVERFLOW;
            }
        }
        node_out[i] = out;
    }
}

/* recordRadiance (workqueue.h:122-136): the contribution is added to the node and every
 * ancestor; a non-finite (or >= 2^62) one marks them instead, as a NaN would poison the
 * reference's FP32 sums */
void oracle_record_radiance(nrrs_path_nodes* nb, const int32_t* node, const float* contrib,
                            uint64_t n) {
    const uint32_t size = nb->header[HDR_SIZE];
    for (uint64_t i = 0; i < n; ++i) {
        const int32_t nd = node[i];
        if (nd < 0 || (uint32_t)nd >= size) continue;
        const float* x = contrib + 3 * i;
        const int ok = fabsf(x[0]) < FIXED_MAX && fabsf(x[1]) < FIXED_MAX && fabsf(x[2]) < FIXED_MAX;
        int64_t l[9];
        if (ok) {
            oracle_fixed_limbs(x[0], l);
            oracle_fixed_limbs(x[1], l + 3);
            oracle_fixed_limbs(x[2], l + 6);
        } else {
            nb->header[HDR_STATUS] |= NRRS_DEV_NAN;
        }
        int32_t cur = nd;
        for (;;) {
            if (ok) {
                int64_t* r = nb->radiance + 9 * (uint64_t)cur;
                for (int k = 0; k < 9; ++k) r[k] = (int64_t)((uint64_t)r[k] + (uint64_t)l[k]);
            } else {
                nb->node_flags[cur] |= 1u;
            }
            const int32_t p = nb->parent[cur];
            if (p < 0) break;
            if (p >= cur) { nb->header[HDR_STATUS] |= NRRS_DEV_BAD_INDEX; break; }
            cur = p;
        }
    }
}

/* nrrs_generate_training_data (train.cu:432-570), in node order. Returns the number of samples
 * (it may exceed capacity; those past it are dropped). */
uint64_t oracle_generate_training_data(nrrs_path_nodes* nb, const nrrs_train_data_params* p,
                                       const float* image, int channels, uint32_t n_pixels,
                                       uint32_t* pixel_samples, const nrrs_train_batch* o,
                                       uint64_t capacity) {
    const uint32_t size = nb->header[HDR_SIZE];
    uint64_t t = 0;
    for (uint32_t i = 0; i < size; ++i) {
        const int64_t* r = nb->radiance + 9 * (uint64_t)i;
        float L[3];
        for (int ch = 0; ch < 3; ++ch) {
            /* LRGB / thpRGB where thp > M_EPSILON (train.cu:481-487), then max(L, 0) */
            const float rad = oracle_fixed_to_float(r[3 * ch], r[3 * ch + 1], r[3 * ch + 2]);
            const float th = nb->thp[3 * (uint64_t)i + ch];
            float l = 0.f;
            if (th > p->thp_eps) l = rad / th;
            L[ch] = l < 0.f ? 0.f : l;
        }
        const float mean = ((L[0] + L[1]) + L[2]) / 3.0f;
        int nan = 0;
        for (int k = 0; k < 3; ++k)
            nan |= isnan(nb->pos[3 * (uint64_t)i + k]) || isnan(nb->wi[3 * (uint64_t)i + k]) ||
                   isnan(L[k]);
        int same = 0;
        if (p->dedupe_rrs_target) {   /* train.cu:462-466 */
            const int32_t par = nb->parent[i];
            if (par >= 0) {
                if ((uint32_t)par < i) same = nb->first_child[par] != i;
                else nb->header[HDR_STATUS] |= NRRS_DEV_BAD_INDEX;
            }
        }
        const int keep = nb->node_flags[i] == 0 && !nan && (!p->ignore_zero_l || mean > 0.f);
        if (!keep) continue;
        if (t < capacity) {
            const float rrs = nb->rrs[i];
            const uint32_t px = nb->pixel[i];
            for (int k = 0; k < 3; ++k) {
                if (o->pos) o->pos[3 * t + k] = nb->pos[3 * (uint64_t)i + k];
                if (o->wi) o->wi[3 * t + k] = nb->wi[3 * (uint64_t)i + k];
                if (o->normal) o->normal[3 * t + k] = nb->normal[3 * (uint64_t)i + k];
                if (o->albedo) o->albedo[3 * t + k] = nb->albedo[3 * (uint64_t)i + k];
                if (o->target) o->target[3 * t + k] = L[k];
                const float th = nb->thp[3 * (uint64_t)i + k];
                if (o->thp) o->thp[3 * t + k] = p->copy_rrs_node ? th * rrs : th;  /* :503-506 */
            }
            if (o->roughness) o->roughness[t] = nb->roughness[i];
            if (o->depth) o->depth[t] = nb->depth[i];
            if (o->rrs_target) o->rrs_target[t] = same ? -1.0f : rrs;       /* :520-535 */
            if (o->pixel) o->pixel[t] = px;
            const int px_ok = px < n_pixels;
            if (!px_ok && (image || pixel_samples || p->error_per_pixel || p->samples_per_patch))
                nb->header[HDR_STATUS] |= NRRS_DEV_BAD_INDEX;
            /* the sample's patch of the film and error images (offsetFrame2Scaled) */
            const uint32_t sc = p->error_image_scale, fw = p->frame_width;
            const uint32_t pq = !px_ok ? 0u
                                : sc > 1u ? (px % fw) / sc + ((px / fw) / sc) * (fw / sc) : px;
            if (o->ref_mean && image) {                                        /* :528-529 */
                float rm = 0.f;
                if (px_ok) {
                    const float* q = image + (uint64_t)pq * (uint64_t)channels;
                    rm = ((q[0] + q[1]) + q[2]) / 3.0f;
                }
                o->ref_mean[t] = rm;
            }
            if (p->error_per_pixel) {                                          /* :537-545 */
                if (o->error) o->error[t] = px_ok ? p->error_per_pixel[pq] : 0.f;
                if (o->error_for_avg)
                    o->error_for_avg[t] = px_ok ? p->error_per_pixel[(uint64_t)n_pixels + pq] : 0.f;
            }
            if (p->samples_per_patch && o->number_samples)
                o->number_samples[t] = px_ok ? p->samples_per_patch[pq] : 0.f;
            if (!same && px_ok && pixel_samples) pixel_samples[px] += 1;     /* :532-533 */
        }
        ++t;
    }
    if (t > capacity) nb->header[HDR_STATUS] |= NRRS_DEV_OVERFLOW;
    return t;
}

/* nrrs_calculate_sample_weight (train.cu:572-592) */
void oracle_sample_weights(const uint32_t* pixel, const uint32_t* pixel_samples,
                           uint32_t n_pixels, uint64_t n, float* weight) {
    for (uint64_t t = 0; t < n; ++t) {
        const uint32_t c = pixel[t] < n_pixels ? pixel_samples[pixel[t]] : 0u;
        weight[t] = c ? 1.0f / (float)c : 0.0f;
    }
}

/* ---- per-pixel error of the RRSNet loss (one patch = scale x scale frame pixels) ---------------- */

typedef struct {
    uint32_t w, h, s, pw, ph;
} geom_t;

static geom_t geom_of(const nrrs_pixel_error_params* p) {
    geom_t g;
    g.w = p->frame_width;
    g.h = p->frame_height;
    g.s = p->scale ? p->scale : 1u;
    g.pw = g.w / g.s;
    g.ph = g.h / g.s;
    return g;
}

/* offsetFrame2Scaled (myFilm.h:6-15) */
static uint32_t patch_of(const geom_t* g, uint32_t px) {
    return (px % g->w) / g->s + ((px / g->w) / g->s) * g->pw;
}

/* patch sample counts: +1 per camera ray (integrator.cpp:1050) and scattered ray (:803-808) */
void oracle_count_patch_samples(const nrrs_pixel_error_params* p, const uint32_t* pixel,
                                uint64_t n, float* spp) {
    const geom_t g = geom_of(p);
    for (uint64_t i = 0; i < n; ++i)
        if (pixel[i] < g.w * g.h) spp[patch_of(&g, pixel[i])] += 1.0f;
}

/* STEP#1.1 after the per-frame reset (integrator.cpp:1027-1028, 2379-2395) and the first-frame
 * initialisation (:2358-2375); a patch's pixels are added in pixel order */
void oracle_accumulate_weighted_l(const nrrs_pixel_error_params* p, const float* pl, uint32_t spp,
                                  int first, float* wl, float* cur, uint32_t* acc) {
    const geom_t g = geom_of(p);
    const float fspp = (float)spp;
    for (uint32_t ps = 0; ps < g.pw * g.ph; ++ps) {
        const uint32_t x0 = (ps % g.pw) * g.s, y0 = (ps / g.pw) * g.s;
        float c[3] = {0.f, 0.f, 0.f}, f[3] = {0.f, 0.f, 0.f};
        for (uint32_t dy = 0; dy < g.s; ++dy)
            for (uint32_t dx = 0; dx < g.s; ++dx) {
                const uint64_t px = (uint64_t)(y0 + dy) * g.w + x0 + dx;
                for (int k = 0; k < 3; ++k) {
                    c[k] = c[k] + pl[3 * px + k];
                    if (first) f[k] = f[k] + pl[3 * px + k] / fspp;
                }
            }
        for (int k = 0; k < 3; ++k) {
            cur[3 * (uint64_t)ps + k] = c[k];
            if (first) wl[3 * (uint64_t)ps + k] = f[k];
        }
        acc[ps] = spp * g.s * g.s;
    }
}

/* nrrs_update_weighted_L (train.cu:344-363) */
void oracle_update_weighted_l(const nrrs_pixel_error_params* p, const float* cur,
                              const uint32_t* acc, float* wl) {
    const geom_t g = geom_of(p);
    const float keep = 1.0f - p->blend_weight;
    for (uint32_t ps = 0; ps < g.pw * g.ph; ++ps) {
        const float n = (float)acc[ps];
        for (int k = 0; k < 3; ++k) {
            const float lc = cur[3 * (uint64_t)ps + k] / n;
            const float lb = wl[3 * (uint64_t)ps + k];
            wl[3 * (uint64_t)ps + k] = lb * keep + lc * p->blend_weight;
        }
    }
}

/* nrrs_calculate_error (train.cu:365-430); returns the exact sum of error[npix + patch]
 * (integrator.cpp:2466-2471) rounded to float, NaN if a term is not finite or >= 2^62 */
float oracle_calculate_error(const nrrs_pixel_error_params* p, const float* ref, int ch,
                             const float* wl, const float* spp, float* err_out) {
    const geom_t g = geom_of(p);
    const uint64_t npix = (uint64_t)g.w * g.h;
    int64_t acc[3] = {0, 0, 0};
    int bad = 0;
    for (uint32_t ps = 0; ps < g.pw * g.ph; ++ps) {
        float q[3];
        for (int k = 0; k < 3; ++k) {
            const float r = ref[(uint64_t)ps * ch + k];
            const float d = wl[3 * (uint64_t)ps + k] - r;
            q[k] = (d * d) / (r * r + 0.01f);
        }
        float e = ((q[0] + q[1]) + q[2]) / 3.0f;
        if (p->clamp) e = fminf(e, 100.0f);
        err_out[ps] = e;
        if (p->multiply_samples) e = e * sqrtf(spp[ps]);
        err_out[npix + ps] = e;
        if (fabsf(e) < FIXED_MAX) {
            int64_t l[3];
            oracle_fixed_limbs(e, l);
            for (int k = 0; k < 3; ++k) acc[k] = (int64_t)((uint64_t)acc[k] + (uint64_t)l[k]);
        } else {
            bad = 1;
        }
    }
    return bad ? NAN : oracle_fixed_to_float(acc[0], acc[1], acc[2]);
}

/* nrrs_UBS_calc_error (train.cu:594-608) and the exact sum (integrator.cpp:2875-2886): the film
 * read at the pixel's patch, L = pixel_l / spp */
float oracle_ubs_error(const nrrs_pixel_error_params* p, const float* pl, uint32_t spp,
                       const float* ref, int ch, float* err_out) {
    const geom_t g = geom_of(p);
    int64_t acc[3] = {0, 0, 0};
    int bad = 0;
    const float fspp = (float)spp;
    for (uint32_t px = 0; px < g.w * g.h; ++px) {
        const float* r = ref + (uint64_t)patch_of(&g, px) * ch;
        float q[3];
        for (int k = 0; k < 3; ++k) {
            const float l = pl[3 * (uint64_t)px + k] / fspp;
            const float d = l - r[k];
            q[k] = (d * d) / (r[k] * r[k] + 0.01f);
        }
        const float e = ((q[0] + q[1]) + q[2]) / 3.0f;
        err_out[px] = e;
        if (fabsf(e) < FIXED_MAX) {
            int64_t l[3];
            oracle_fixed_limbs(e, l);
            for (int k = 0; k < 3; ++k) acc[k] = (int64_t)((uint64_t)acc[k] + (uint64_t)l[k]);
        } else {
            bad = 1;
        }
    }
    return bad ? NAN : oracle_fixed_to_float(acc[0], acc[1], acc[2]);
}
