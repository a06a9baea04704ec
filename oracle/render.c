/*
 * render.c -- CPU oracle of the wavefront steps around the NRRS step: camera rays, closest hit
 * (brute force over every triangle: no BVH), shading into the next vertex queue, the scatter step
 * (thp / rrs, next-event estimation, BSDF sampling), shadow rays and the exact film. TEST
 * INFRASTRUCTURE ONLY: tests/ and bench.py's cpu_baseline leg use it, never the product library.
 *
 * In banbao990/NRRS-Code the same steps are the OptiX programs (src/render/nrrs/device.cu:48-161),
 * handleEmissiveHit / handleMiss (integrator.cpp:688-735), handleIntersections and
 * generateScatteredRays (:737-887) and generateCameraRays (:889-935), with KiRaRay's diffuse BSDF
 * and area lights. This restatement follows the library's definitions operation by operation (FP32,
 * no contraction; the intersection's explicit fmaf calls are the library's __fmaf_rn), so its
 * results equal the GPU's bit for bit; intersection ties go to the lower
 * triangle index in both, so the BVH does not matter.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "nrrs_oracle.h"

#define INV_PI 0.318309886183790671f
#define OFFSET 1e-4f
#define RR_DIM 31u   /* hash dimension of the fixed-RR decision */
#define MISS 0xffffffffu
#define FIXED_MAX_R 4611686018427387904.0f

static uint32_t hash32(uint32_t x) {   /* lowbias32 (C. Wellons) */
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
static float rnd(uint32_t seed, uint32_t depth, uint32_t slot, uint32_t dim) {
    const uint32_t h = hash32(hash32(hash32(seed) ^ (depth * 0x9e3779b9u)) ^ (slot * 32u + dim));
    return (float)(h >> 8) * 0x1p-24f;
}

typedef struct { float x, y, z; } v3;
static v3 ld(const float* p) { v3 a = {p[0], p[1], p[2]}; return a; }
static void st(float* p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }
static v3 add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static v3 sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
static v3 mul(v3 a, float s) { v3 r = {a.x * s, a.y * s, a.z * s}; return r; }
static v3 vmul(v3 a, v3 b) { v3 r = {a.x * b.x, a.y * b.y, a.z * b.z}; return r; }
static v3 divs(v3 a, float s) { v3 r = {a.x / s, a.y / s, a.z / s}; return r; }
static float dot(v3 a, v3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
static v3 cross(v3 a, v3 b) {
    v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
    return r;
}
static v3 normalize(v3 a) { return divs(a, sqrtf(dot(a, a))); }
static int nonzero(v3 a) { return a.x != 0.f || a.y != 0.f || a.z != 0.f; }

/* the scene as the library keeps it: triangles as v0, e1, e2 in input order */
typedef struct {
    const float* tri;        /* [nt][9] */
    const uint32_t* mat;     /* [nt] */
    const float* mats;       /* [nm][6] */
    uint32_t nt;
    const uint32_t* lights;  /* [nl] input index */
    const float* area;       /* [nl] */
    uint32_t nl;
    v3 env;
} scene_t;

/* triangles (v0, e1, e2) and the light list of a mesh, as nrrs_scene_create builds them */
uint32_t oracle_scene_tris(const float* vertices, const uint32_t* tris, uint32_t nt,
                           const uint32_t* tri_mat, const float* mats, float* tri_out,
                           uint32_t* lights, float* areas) {
    uint32_t nl = 0;
    for (uint32_t i = 0; i < nt; ++i) {
        const float* a = vertices + 3 * (uint64_t)tris[3 * (uint64_t)i];
        const float* b = vertices + 3 * (uint64_t)tris[3 * (uint64_t)i + 1];
        const float* c = vertices + 3 * (uint64_t)tris[3 * (uint64_t)i + 2];
        float* t = tri_out + 9 * (uint64_t)i;
        for (int k = 0; k < 3; ++k) { t[k] = a[k]; t[3 + k] = b[k] - a[k]; t[6 + k] = c[k] - a[k]; }
        const float* m = mats + 6 * (uint64_t)tri_mat[i];
        if (m[3] != 0.f || m[4] != 0.f || m[5] != 0.f) {
            const float cx = t[4] * t[8] - t[5] * t[7], cy = t[5] * t[6] - t[3] * t[8],
                        cz = t[3] * t[7] - t[4] * t[6];
            const float ar = 0.5f * sqrtf((cx * cx + cy * cy) + cz * cz);
            if (ar > 0.f) { lights[nl] = i; areas[nl] = ar; ++nl; }
        }
    }
    return nl;
}

/* the intersection's dot and cross products with fused multiply-adds, as the library's (fmaf is
 * correctly rounded: one rounding per call) */
static float fdot(v3 a, v3 b) { return fmaf(a.x, b.x, fmaf(a.y, b.y, a.z * b.z)); }
static v3 fcross(v3 a, v3 b) {
    v3 r = {fmaf(a.y, b.z, -(a.z * b.y)), fmaf(a.z, b.x, -(a.x * b.z)), fmaf(a.x, b.y, -(a.y * b.x))};
    return r;
}

static int intersect(const float* tri, v3 o, v3 d, float tmax, float* t, float* u, float* v) {
    const v3 v0 = ld(tri), e1 = ld(tri + 3), e2 = ld(tri + 6);
    const v3 pv = fcross(d, e2);
    const float det = fdot(e1, pv);
    if (fabsf(det) < 1e-12f) return 0;
    const float inv = 1.0f / det;
    const v3 tv = sub(o, v0);
    const float uu = fdot(tv, pv) * inv;
    if (uu < 0.f || uu > 1.f) return 0;
    const v3 qv = fcross(tv, e1);
    const float vv = fdot(d, qv) * inv;
    if (vv < 0.f || uu + vv > 1.f) return 0;
    const float tt = fdot(e2, qv) * inv;
    if (!(tt > 0.f && tt < tmax)) return 0;
    *t = tt; *u = uu; *v = vv;
    return 1;
}

static uint32_t closest(const scene_t* s, v3 o, v3 d, float tmax, float* t, float* u, float* v,
                        int any) {
    uint32_t best = MISS;
    float bt = tmax, bu = 0.f, bv = 0.f;
    for (uint32_t i = 0; i < s->nt; ++i) {
        float tt, uu, vv;
        if (!intersect(s->tri + 9 * (uint64_t)i, o, d, tmax, &tt, &uu, &vv)) continue;
        if (best == MISS || tt < bt) { best = i; bt = tt; bu = uu; bv = vv; }   /* ties: lower i */
        if (any) break;
    }
    *t = bt; *u = bu; *v = bv;
    return best;
}

static void film_add(int64_t* film, uint32_t pixel, v3 c) {
    const float cc[3] = {c.x, c.y, c.z};
    for (int k = 0; k < 3; ++k) {
        if (cc[k] == 0.f || !(fabsf(cc[k]) < FIXED_MAX_R)) continue;
        int64_t l[3];
        oracle_fixed_limbs(cc[k], l);
        int64_t* f = film + 9 * (uint64_t)pixel + 3 * k;
        for (int q = 0; q < 3; ++q) f[q] = (int64_t)((uint64_t)f[q] + (uint64_t)l[q]);
    }
}

static float power_heuristic(float a, float b) { return (a * a) / (a * a + b * b); }

static scene_t mk(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                  const uint32_t* lights, const float* area, uint32_t nl, const float* env) {
    scene_t s;
    s.tri = tri; s.mat = mat; s.mats = mats; s.nt = nt;
    s.lights = lights; s.area = area; s.nl = nl;
    s.env.x = env ? env[0] : 0.f; s.env.y = env ? env[1] : 0.f; s.env.z = env ? env[2] : 0.f;
    return s;
}

/* generateCameraRays */
void oracle_camera_rays(const nrrs_camera* c, uint32_t sample, uint32_t seed, float* origin,
                        float* dir) {
    const v3 fw = normalize(ld(c->forward));
    const v3 right = normalize(cross(fw, ld(c->up)));
    const v3 up = cross(right, fw);
    const float w = (float)c->width, h = (float)c->height;
    for (uint32_t p = 0; p < c->width * c->height; ++p) {
        const float jx = rnd(seed, 0xffffffffu - sample, p, 0), jy = rnd(seed, 0xffffffffu - sample, p, 1);
        const float px = (((float)(p % c->width) + jx) / w) * 2.0f - 1.0f;
        const float py = 1.0f - (((float)(p / c->width) + jy) / h) * 2.0f;
        const float sx = (px * c->tan_half_fov_y) * (w / h);
        const float sy = py * c->tan_half_fov_y;
        st(origin + 3 * (uint64_t)p, ld(c->pos));
        st(dir + 3 * (uint64_t)p, normalize(add(add(fw, mul(right, sx)), mul(up, sy))));
    }
}

/* closest hits: prim, t, u, v per ray (rays with zero thp: miss with t = u = v = 0) */
void oracle_trace(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                  const float* origin, const float* dir, const float* thp, uint32_t n,
                  uint32_t* prim, float* t, float* u, float* v) {
    scene_t s = mk(tri, mat, mats, nt, NULL, NULL, 0, NULL);
    for (uint32_t i = 0; i < n; ++i) {
        if (!nonzero(ld(thp + 3 * (uint64_t)i))) { prim[i] = MISS; t[i] = u[i] = v[i] = 0.f; continue; }
        prim[i] = closest(&s, ld(origin + 3 * (uint64_t)i), ld(dir + 3 * (uint64_t)i), INFINITY,
                          t + i, u + i, v + i, 0);
    }
}

/* handleEmissiveHit / handleMiss and the vertex queue; returns the number of vertices */
/* a path vertex into output slot m */
static void put_vertex(float* o_pos, float* o_wi, float* o_nrm, float* o_alb, float* o_rough,
                       float* o_thp, uint32_t* o_depth, uint32_t* o_pixel, int32_t* o_node,
                       uint32_t m, v3 p, v3 d, v3 nn, const float* alb, float rough, v3 th,
                       uint32_t depth, uint32_t pixel, int32_t node) {
    st(o_pos + 3 * (uint64_t)m, p);
    st(o_wi + 3 * (uint64_t)m, mul(d, -1.0f));
    st(o_nrm + 3 * (uint64_t)m, nn);
    st(o_alb + 3 * (uint64_t)m, ld(alb));
    o_rough[m] = rough;
    st(o_thp + 3 * (uint64_t)m, th);
    o_depth[m] = depth;
    o_pixel[m] = pixel;
    o_node[m] = node;
}

/* handleEmissiveHit / handleMiss and the vertex queues. mat_spec (may be NULL) marks mirror
 * materials: with s_* outputs given, their hits go to the specular queue (roughness 0) instead
 * of the inference queue, as the reference's closest-hit program pushes specular hits straight
 * to the scatter queue (device.cu:91-95). Returns the inference-queue size; *n_spec the other. */
uint32_t oracle_shade_split(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                            uint32_t nl, const float* env, const uint8_t* mat_spec,
                            const float* origin, const float* dir, const float* thp,
                            const float* pdf, const uint32_t* pixel, const int32_t* node,
                            const uint32_t* prim, const float* t, uint32_t n, uint32_t depth,
                            int64_t* film, float* contrib, float* o_pos, float* o_wi,
                            float* o_nrm, float* o_alb, float* o_rough, float* o_thp,
                            uint32_t* o_depth, uint32_t* o_pixel, int32_t* o_node,
                            float* s_pos, float* s_wi, float* s_nrm, float* s_alb,
                            float* s_rough, float* s_thp, uint32_t* s_depth, uint32_t* s_pixel,
                            int32_t* s_node, uint32_t* n_spec) {
    scene_t s = mk(tri, mat, mats, nt, NULL, NULL, nl, env);
    uint32_t m = 0, ms = 0;
    for (uint32_t i = 0; i < n; ++i) {
        const v3 th = ld(thp + 3 * (uint64_t)i), d = ld(dir + 3 * (uint64_t)i);
        v3 c = {0.f, 0.f, 0.f};
        if (nonzero(th)) {
            if (prim[i] == MISS) {
                c = vmul(s.env, th);
            } else {
                const float* tr = tri + 9 * (uint64_t)prim[i];
                const v3 p = add(ld(origin + 3 * (uint64_t)i), mul(d, t[i]));
                const v3 g = cross(ld(tr + 3), ld(tr + 6));
                v3 nn = normalize(g);
                if (dot(nn, d) > 0.f) nn = mul(nn, -1.0f);
                const float* mm = mats + 6 * (uint64_t)mat[prim[i]];
                const v3 le = ld(mm + 3);
                if (nonzero(le)) {
                    float w = 1.0f;
                    if (pdf[i] > 0.f && nl) {
                        const float area = 0.5f * sqrtf(dot(g, g));
                        const float cosl = fabsf(dot(nn, d));
                        const float pl = (t[i] * t[i]) / ((cosl * area) * (float)nl);
                        w = power_heuristic(pdf[i], pl);
                    }
                    c = mul(vmul(le, th), w);
                }
                if (s_pos && mat_spec && mat_spec[mat[prim[i]]]) {
                    const float rough = mat_spec[mat[prim[i]]] == 2 ? -1.0f : 0.0f;
                    put_vertex(s_pos, s_wi, s_nrm, s_alb, s_rough, s_thp, s_depth, s_pixel, s_node,
                               ms++, p, d, nn, mm, rough, th, depth, pixel[i], node[i]);
                } else {
                    put_vertex(o_pos, o_wi, o_nrm, o_alb, o_rough, o_thp, o_depth, o_pixel, o_node,
                               m++, p, d, nn, mm, 1.0f, th, depth, pixel[i], node[i]);
                }
            }
        }
        st(contrib + 3 * (uint64_t)i, c);
        if (nonzero(c)) film_add(film, pixel[i], c);
    }
    if (n_spec) *n_spec = ms;
    return m;
}

uint32_t oracle_shade(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                      uint32_t nl, const float* env, const float* origin, const float* dir,
                      const float* thp, const float* pdf, const uint32_t* pixel,
                      const int32_t* node, const uint32_t* prim, const float* t, uint32_t n,
                      uint32_t depth, int64_t* film, float* contrib, float* o_pos, float* o_wi,
                      float* o_nrm, float* o_alb, float* o_rough, float* o_thp,
                      uint32_t* o_depth, uint32_t* o_pixel, int32_t* o_node) {
    return oracle_shade_split(tri, mat, mats, nt, nl, env, NULL, origin, dir, thp, pdf, pixel,
                              node, prim, t, n, depth, film, contrib, o_pos, o_wi, o_nrm, o_alb,
                              o_rough, o_thp, o_depth, o_pixel, o_node, NULL, NULL, NULL, NULL,
                              NULL, NULL, NULL, NULL, NULL, NULL);
}

/* thin glass (index 1.5, air on both sides): the sheet's reflectance 2F/(1+F), F the
 * unpolarised Fresnel reflectance of one face at incidence cosine cosi */
static float thin_glass_reflectance(float cosi) {
    const float eta = 1.5f;
    const float sin2t = (1.0f - cosi * cosi) / (eta * eta);
    const float ct = 1.0f - sin2t;
    const float cost = sqrtf(ct > 0.0f ? ct : 0.0f);
    const float a = (cosi - eta * cost) / (cosi + eta * cost);
    const float b = (eta * cosi - cost) / (eta * cosi + cost);
    const float f = 0.5f * (a * a + b * b);
    return (2.0f * f) / (1.0f + f);
}

/* the specular bounce of the first n specular vertices into ray slots off .. off + n - 1 (slots
 * at or past max_rays are dropped): a mirror (roughness 0) reflects; thin glass (roughness -1)
 * reflects when dimension 30 of the slot's hash is below the sheet's reflectance and otherwise
 * passes straight through; thp x albedo; no light sampling and no RRS (the reference pushes these
 * vertices to the emitted queue once, with rrs 1); pdf 0, so the emitter the ray hits counts
 * without an MIS weight. */
void oracle_scatter_specular(const float* pos, const float* wi, const float* nrm, const float* alb,
                             const float* thp, const float* rough, const uint32_t* pixel,
                             const int32_t* node, uint32_t n, uint32_t off, uint32_t max_rays,
                             uint32_t depth, uint32_t seed, float* r_origin, float* r_dir,
                             float* r_thp, float* r_pdf, uint32_t* r_pixel, int32_t* r_node) {
    for (uint32_t j = 0; j < n; ++j) {
        const uint64_t slot = (uint64_t)off + j;
        if (slot >= max_rays) continue;
        const v3 nn = ld(nrm + 3 * (uint64_t)j), din = mul(ld(wi + 3 * (uint64_t)j), -1.0f);
        const v3 p = ld(pos + 3 * (uint64_t)j);
        const float dn = dot(din, nn);
        int reflect = 1;
        if (rough[j] < 0.0f)
            reflect = rnd(seed, depth, j, 30u) < thin_glass_reflectance(fabsf(dn));
        const v3 dir = reflect ? normalize(sub(din, mul(nn, 2.0f * dn))) : din;
        st(r_origin + 3 * slot, add(p, mul(nn, reflect ? OFFSET : -OFFSET)));
        st(r_dir + 3 * slot, dir);
        st(r_thp + 3 * slot, vmul(ld(thp + 3 * (uint64_t)j), ld(alb + 3 * (uint64_t)j)));
        r_pdf[slot] = 0.f;
        r_pixel[slot] = pixel[j];
        r_node[slot] = node[j];
    }
}

/* the scene arrays of the scatter steps */
typedef struct {
    const float* tri;
    const uint32_t* mat;
    const float* mats;
    const uint32_t* lights;
    const float* area;
    uint32_t nl;
} lights_t;

/* the output arrays of the scatter steps */
typedef struct {
    float *r_origin, *r_dir, *r_thp, *r_pdf;
    uint32_t* r_pixel;
    int32_t* r_node;
    float *s_origin, *s_dir, *s_tmax, *s_contrib;
    uint32_t* s_pixel;
    int32_t* s_node;
} scatter_out_t;

/* generateScatteredRays for vertex x into slot j with its throughput already divided */
static void scatter_one(const lights_t* L, const float* pos, const float* nrm, const float* alb,
                        const uint32_t* pixel, const int32_t* node, uint32_t x, uint32_t j, v3 th,
                        uint32_t depth, uint32_t seed, const scatter_out_t* o) {
    const float* tri = L->tri;
    const uint32_t* mat = L->mat;
    const float* mats = L->mats;
    const uint32_t* lights = L->lights;
    const float* area = L->area;
    const uint32_t nl = L->nl;
    float *r_origin = o->r_origin, *r_dir = o->r_dir, *r_thp = o->r_thp, *r_pdf = o->r_pdf;
    uint32_t* r_pixel = o->r_pixel;
    int32_t* r_node = o->r_node;
    float *s_origin = o->s_origin, *s_dir = o->s_dir, *s_tmax = o->s_tmax, *s_contrib = o->s_contrib;
    uint32_t* s_pixel = o->s_pixel;
    int32_t* s_node = o->s_node;
    const v3 p = ld(pos + 3 * (uint64_t)x), nn = ld(nrm + 3 * (uint64_t)x);
    const v3 al = ld(alb + 3 * (uint64_t)x);
    const v3 f = mul(al, INV_PI);
    const v3 org = add(p, mul(nn, OFFSET));
    /* the shading terms use the direction from the vertex; the visibility test runs from the
     * offset origin to the light point and stops short of it */
    v3 sc = {0.f, 0.f, 0.f}, sdir = {0.f, 0.f, 1.f};
    float smax = 0.f;
    if (nl) {
        uint32_t k = (uint32_t)(rnd(seed, depth, j, 0) * (float)nl);
        if (k > nl - 1) k = nl - 1;
        const uint32_t lt = lights[k];
        const float* tr = tri + 9 * (uint64_t)lt;
        const float su = sqrtf(rnd(seed, depth, j, 1));
        const float b1 = 1.0f - su, b2 = rnd(seed, depth, j, 2) * su;
        const v3 q = add(add(ld(tr), mul(ld(tr + 3), b1)), mul(ld(tr + 6), b2));
        const v3 dv = sub(q, p);
        const float d2 = dot(dv, dv);
        const v3 wl = divs(dv, sqrtf(d2));
        const float cosv = dot(nn, wl);
        const float cosl = fabsf(dot(normalize(cross(ld(tr + 3), ld(tr + 6))), wl));
        const v3 le = ld(mats + 6 * (uint64_t)mat[lt] + 3);
        const v3 ds = sub(q, org);
        const float sl = sqrtf(dot(ds, ds));
        if (cosv > 0.f && cosl > 0.f && nonzero(le) && d2 > 0.f && sl > 0.f) {
            const float pl = d2 / ((cosl * area[k]) * (float)nl);
            const float w = power_heuristic(pl, cosv * INV_PI);
            sc = divs(mul(mul(vmul(vmul(th, f), le), cosv), w), pl);
            sdir = divs(ds, sl);
            smax = sl * 0.9999f;
        }
    }
    st(s_origin + 3 * (uint64_t)j, org);
    st(s_dir + 3 * (uint64_t)j, sdir);
    s_tmax[j] = smax;
    st(s_contrib + 3 * (uint64_t)j, sc);
    s_pixel[j] = pixel[x];
    s_node[j] = node[x];
    v3 sp = {0.f, 0.f, 1.f};
    for (uint32_t t = 0; t < 8; ++t) {
        const v3 c = {rnd(seed, depth, j, 3 + 3 * t) * 2.0f - 1.0f,
                      rnd(seed, depth, j, 4 + 3 * t) * 2.0f - 1.0f,
                      rnd(seed, depth, j, 5 + 3 * t) * 2.0f - 1.0f};
        const float c2 = dot(c, c);
        if (c2 <= 1.0f && c2 > 1e-6f) { sp = divs(c, sqrtf(c2)); break; }
    }
    v3 d = add(nn, sp);
    const float l2 = dot(d, d);
    d = l2 > 1e-12f ? divs(d, sqrtf(l2)) : nn;
    const float pdf = dot(nn, d) * INV_PI;
    const v3 zero = {0.f, 0.f, 0.f};
    st(r_origin + 3 * (uint64_t)j, org);
    st(r_dir + 3 * (uint64_t)j, d);
    st(r_thp + 3 * (uint64_t)j, pdf > 0.f ? vmul(th, al) : zero);
    r_pdf[j] = pdf > 0.f ? pdf : 0.f;
    r_pixel[j] = pixel[x];
    r_node[j] = node[x];
}

/* handleIntersections (RRS branch) + generateScatteredRays for queue entries [0, nq) */
void oracle_scatter(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                    const uint32_t* lights, const float* area, uint32_t nl, const float* pos,
                    const float* nrm, const float* alb, const float* thp, const uint32_t* pixel,
                    const int32_t* node, const float* rrs_norm, const uint32_t* queue,
                    uint32_t nq, uint32_t depth, uint32_t seed, float* r_origin, float* r_dir,
                    float* r_thp, float* r_pdf, uint32_t* r_pixel, int32_t* r_node,
                    float* s_origin, float* s_dir, float* s_tmax, float* s_contrib,
                    uint32_t* s_pixel, int32_t* s_node) {
    (void)nt;
    const lights_t L = {tri, mat, mats, lights, area, nl};
    const scatter_out_t o = {r_origin, r_dir, r_thp, r_pdf, r_pixel, r_node,
                             s_origin, s_dir, s_tmax, s_contrib, s_pixel, s_node};
    for (uint32_t j = 0; j < nq; ++j) {
        const uint32_t x = queue[j];
        const v3 th = divs(ld(thp + 3 * (uint64_t)x), rrs_norm[x]);
        scatter_one(&L, pos, nrm, alb, pixel, node, x, j, th, depth, seed, &o);
    }
}

/* handleIntersections' fixed Russian-roulette branch (integrator.cpp:744-769): vertex j survives
 * when dimension 31 of its slot's hash is below rr, with thp / rr; a killed vertex leaves an
 * empty slot (zero origin and throughput, direction +z, pixel and node kept) */
void oracle_scatter_fixed_rr(const float* tri, const uint32_t* mat, const float* mats,
                             const uint32_t* lights, const float* area, uint32_t nl,
                             const float* pos, const float* nrm, const float* alb,
                             const float* thp, const uint32_t* pixel, const int32_t* node,
                             uint32_t n, float rr, uint32_t depth, uint32_t seed, float* r_origin,
                             float* r_dir, float* r_thp, float* r_pdf, uint32_t* r_pixel,
                             int32_t* r_node, float* s_origin, float* s_dir, float* s_tmax,
                             float* s_contrib, uint32_t* s_pixel, int32_t* s_node) {
    const lights_t L = {tri, mat, mats, lights, area, nl};
    const scatter_out_t o = {r_origin, r_dir, r_thp, r_pdf, r_pixel, r_node,
                             s_origin, s_dir, s_tmax, s_contrib, s_pixel, s_node};
    const v3 zero = {0.f, 0.f, 0.f}, up = {0.f, 0.f, 1.f};
    for (uint32_t j = 0; j < n; ++j) {
        if (rnd(seed, depth, j, RR_DIM) < rr) {
            scatter_one(&L, pos, nrm, alb, pixel, node, j, j, divs(ld(thp + 3 * (uint64_t)j), rr),
                        depth, seed, &o);
            continue;
        }
        st(s_origin + 3 * (uint64_t)j, zero);
        st(s_dir + 3 * (uint64_t)j, up);
        s_tmax[j] = 0.f;
        st(s_contrib + 3 * (uint64_t)j, zero);
        s_pixel[j] = pixel[j];
        s_node[j] = node[j];
        st(r_origin + 3 * (uint64_t)j, zero);
        st(r_dir + 3 * (uint64_t)j, up);
        st(r_thp + 3 * (uint64_t)j, zero);
        r_pdf[j] = 0.f;
        r_pixel[j] = pixel[j];
        r_node[j] = node[j];
    }
}

/* shadow rays: a visible light adds the slot's contribution to the film */
void oracle_shadow(const float* tri, uint32_t nt, const float* origin, const float* dir,
                   const float* tmax, const float* contrib, const uint32_t* pixel, uint32_t n,
                   int64_t* film, float* cout) {
    scene_t s = mk(tri, NULL, NULL, nt, NULL, NULL, 0, NULL);
    for (uint32_t j = 0; j < n; ++j) {
        v3 c = ld(contrib + 3 * (uint64_t)j);
        if (nonzero(c)) {
            float t, u, v;
            if (closest(&s, ld(origin + 3 * (uint64_t)j), ld(dir + 3 * (uint64_t)j), tmax[j], &t,
                        &u, &v, 1) != MISS) {
                c.x = c.y = c.z = 0.f;
            } else {
                film_add(film, pixel[j], c);
            }
        }
        st(cout + 3 * (uint64_t)j, c);
    }
}

void oracle_film_resolve(const int64_t* film, uint32_t n, float scale, float* img) {
    for (uint32_t p = 0; p < n; ++p)
        for (int k = 0; k < 3; ++k) {
            const int64_t* l = film + 9 * (uint64_t)p + 3 * k;
            img[3 * (uint64_t)p + k] = oracle_fixed_to_float(l[0], l[1], l[2]) * scale;
        }
}
