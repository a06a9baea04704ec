/*
 * nrrs_oracle.c -- CPU oracle for the NRRS per-vertex step. TEST INFRASTRUCTURE ONLY:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load it.
 *
 * PARITY UNPINNED for the encodings, MLPs, losses and Adam: they live in the reference's
 * tiny-cuda-nn submodule (branch `use-bb`, no pinned commit, absent from the checkout), so they
 * are restated from the published algorithms and written definitions. The decision/emission,
 * normalisation, glue, activation and weight window are restated from the reference sources
 * cited below and pinned by hand-derived known answers (tests/golden/) and, for
 * RRSWeightWindow, by the reference's own header compiled into oracle/_ref.
 *
 * Build: oracle/Makefile (gcc -O2 -fopenmp -ffp-contract=off). FP contraction is off so the
 * FP32 decision arithmetic is the exact IEEE sequence the contract defines.
 */
#include "nrrs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* real SH normalisation constants: 0.5 sqrt(1/pi), sqrt(3/(4 pi)), 0.5 sqrt(15/pi),
 * 0.25 sqrt(5/pi), 0.25 sqrt(15/pi), 0.25 sqrt(35/(2 pi)), 0.5 sqrt(105/pi),
 * 0.25 sqrt(21/(2 pi)), 0.25 sqrt(7/pi), 0.25 sqrt(105/pi) */
#define SH_C0 0.28209479177387814
#define SH_C1 0.4886025119029199
#define SH_C2A 1.0925484305920792
#define SH_C2B 0.31539156525252005
#define SH_C2C 0.5462742152960396
#define SH_C3A 0.5900435899266435
#define SH_C3B 2.890611442640554
#define SH_C3C 0.4570457994644658
#define SH_C3D 0.3731763325901154
#define SH_C3E 1.445305721320277

typedef struct {
    uint32_t offset, entries, res, dense, hash_mask;
} level_t;

/* Level l of an Instant-NGP grid: N_l = floor(N_min * b^l) cells per axis, N_l + 1 grid points.
 * Dense when (N_l+1)^3 <= T (row = x + R y + R^2 z), hashed otherwise with the spatial hash
 * (x * 1) ^ (y * 2654435761) ^ (z * 805459861) mod T (uint32 wrap-around). */
static uint64_t build_levels(const nrrs_config* cfg, level_t* lv) {
    const uint64_t T = 1ull << cfg->log2_hashmap_size;
    uint64_t off = 0;
    for (int l = 0; l < cfg->n_levels; ++l) {
        const uint32_t N = (uint32_t)floor((double)cfg->base_resolution *
                                           pow((double)cfg->per_level_scale, (double)l));
        const uint64_t R = (uint64_t)N + 1;
        const uint64_t dense_n = R * R * R;
        lv[l].res = N;
        lv[l].dense = dense_n <= T;
        lv[l].entries = (uint32_t)(lv[l].dense ? dense_n : T);
        lv[l].offset = (uint32_t)off;
        lv[l].hash_mask = (uint32_t)(T - 1);
        off += lv[l].entries;
    }
    return off;
}

static inline uint32_t grid_index(const level_t* lv, uint32_t x, uint32_t y, uint32_t z) {
    if (lv->dense) {
        const uint32_t R = lv->res + 1;
        return x + R * y + R * R * z;
    }
    return (x ^ (y * 2654435761u) ^ (z * 805459861u)) & lv->hash_mask;
}

/* the shape of the two network families (include/nrrs.h, nrrs_network_family) */
static int net_ref(const nrrs_config* c) { return c->network == NRRS_NET_REFERENCE; }
static int net_stat_in(const nrrs_config* c) { return net_ref(c) ? 32 : 64; }
static int net_stat_out(const nrrs_config* c) { return net_ref(c) ? 6 : 3; }

static uint64_t statnet_params(const nrrs_config* c) {
    const uint64_t w = (uint64_t)c->statnet_width;
    return (uint64_t)net_stat_in(c) * w + (uint64_t)(c->statnet_hidden - 1) * w * w +
           (uint64_t)net_stat_out(c) * w;
}
static uint64_t rrsnet_params(const nrrs_config* c) {
    const uint64_t w = (uint64_t)c->rrsnet_width;
    return 16 * w + (uint64_t)(c->rrsnet_hidden - 1) * w * w + w;
}

uint64_t oracle_level_table(const nrrs_config* cfg, uint32_t* out) {
    level_t lv[32];
    uint64_t tot = build_levels(cfg, lv);
    for (int l = 0; l < cfg->n_levels; ++l) {
        out[l * 4 + 0] = lv[l].offset;
        out[l * 4 + 1] = lv[l].entries;
        out[l * 4 + 2] = lv[l].res;
        out[l * 4 + 3] = lv[l].dense;
    }
    return tot;
}

uint64_t oracle_param_count(const nrrs_config* cfg, uint64_t* table, uint64_t* stat,
                            uint64_t* rrs) {
    level_t lv[32];
    const uint64_t t = build_levels(cfg, lv) * 2;
    if (table) *table = t;
    if (stat) *stat = statnet_params(cfg);
    if (rrs) *rrs = rrsnet_params(cfg);
    return t + statnet_params(cfg) + rrsnet_params(cfg);
}

/* normalizeSpatialCoord, src/render/nrc/nrctrain.h:111-115: inflate the AABB by 0.5 % of its
 * diagonal length, then 0.5 + (p - center) / diagonal; clamped to [0,1] for the grid. */
void oracle_normalize_pos_f32(const nrrs_config* cfg, const float* p, float* out) {
    if (!cfg->normalize_pos) {
        for (int d = 0; d < 3; ++d) {
            float x = p[d];
            out[d] = x < 0.f ? 0.f : (x > 1.f ? 1.f : x);
        }
        return;
    }
    float dg[3], lo[3], hi[3], c[3], diag[3];
    for (int d = 0; d < 3; ++d) dg[d] = cfg->aabb_max[d] - cfg->aabb_min[d];
    const float inflate = sqrtf(dg[0] * dg[0] + dg[1] * dg[1] + dg[2] * dg[2]) * 0.005f;
    for (int d = 0; d < 3; ++d) {
        lo[d] = cfg->aabb_min[d] - inflate;
        hi[d] = cfg->aabb_max[d] + inflate;
        c[d] = (lo[d] + hi[d]) * 0.5f;
        diag[d] = hi[d] - lo[d];
    }
    for (int d = 0; d < 3; ++d) {
        float x = 0.5f + (p[d] - c[d]) / diag[d];
        out[d] = x < 0.f ? 0.f : (x > 1.f ? 1.f : x);
    }
}

void oracle_sh16_f64(const double* dir, double* o) {
    const double x = dir[0], y = dir[1], z = dir[2];
    const double xx = x * x, yy = y * y, zz = z * z;
    o[0] = SH_C0;
    o[1] = -SH_C1 * y;
    o[2] = SH_C1 * z;
    o[3] = -SH_C1 * x;
    o[4] = SH_C2A * x * y;
    o[5] = -SH_C2A * y * z;
    o[6] = SH_C2B * (3 * zz - 1);
    o[7] = -SH_C2A * x * z;
    o[8] = SH_C2C * (xx - yy);
    o[9] = -SH_C3A * y * (3 * xx - yy);
    o[10] = SH_C3B * x * y * z;
    o[11] = -SH_C3C * y * (5 * zz - 1);
    o[12] = SH_C3D * z * (5 * zz - 3);
    o[13] = -SH_C3C * x * (5 * zz - 1);
    o[14] = SH_C3E * z * (xx - yy);
    o[15] = -SH_C3A * x * (xx - 3 * yy);
}

float oracle_activation_sigma_f32(float x) {
    const float ln2 = 0.6931471805599453f;
    return (x < 0) ? logf(1.0f + expf(x)) : (0.5f * x + ln2);
}
float oracle_box_cox_f32(float x) { return 2.0f * (sqrtf(x) - 1.0f); }
/* warp_roughness, train.h:95 */
float oracle_warp_roughness_f32(float r) { return 1.0f - expf(-r); }
/* the StatNet's radiance estimate L from a log-statistic y = log(L + eps), before the ADRRS
 * clamp (the factor's first step, the same expression as factor() below) */
float oracle_stat_to_l_f32(float y, float eps) { return expf(y < 20.0f ? y : 20.0f) - eps; }

/* RRSWeightWindow, src/render/common/commoncudautils.h:14-28 */
float oracle_weight_window_f32(float x, float ww) {
    const float dminus = 2 / (1 + ww);
    const float dplus = dminus * ww;
    if (x < dminus) return x / dminus;
    if (x > dplus) return x / dplus;
    return 1.0f;
}

/* ---- precision-generic part ---- */
#define REAL double
#define REAL_IS_DOUBLE 1
#define SFX _f64
#include "nrrs_oracle_impl.h"
#undef REAL
#undef REAL_IS_DOUBLE
#undef SFX
#define REAL float
#define REAL_IS_DOUBLE 0
#define SFX _f32
#include "nrrs_oracle_impl.h"
#undef REAL
#undef REAL_IS_DOUBLE
#undef SFX

static double* promote(const float* p, uint64_t n) {
    double* d = (double*)malloc(sizeof(double) * n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) d[i] = (double)p[i];
    return d;
}

void oracle_infer_f64(const nrrs_config* cfg, const float* params, uint64_t n,
                      const nrrs_vertex_soa* v, const nrrs_decide_params* p, double* x0,
                      double* stats, double* x1, double* raw, double* rrs) {
    double* pd = promote(params, oracle_param_count(cfg, NULL, NULL, NULL));
    infer_impl_f64(cfg, pd, n, v, p, x0, stats, x1, raw, rrs);
    free(pd);
}
void oracle_infer_f32(const nrrs_config* cfg, const float* params, uint64_t n,
                      const nrrs_vertex_soa* v, const nrrs_decide_params* p, float* x0,
                      float* stats, float* x1, float* raw, float* rrs) {
    infer_impl_f32(cfg, params, n, v, p, x0, stats, x1, raw, rrs);
}
void oracle_train_grads_f64(const nrrs_config* cfg, const float* params, uint64_t n,
                            const nrrs_vertex_soa* v, const float* target, double* grads,
                            double* loss) {
    double* pd = promote(params, oracle_param_count(cfg, NULL, NULL, NULL));
    train_impl_f64(cfg, pd, n, v, target, grads, loss, NULL);
    free(pd);
}
void oracle_train_grads_f32(const nrrs_config* cfg, const float* params, uint64_t n,
                            const nrrs_vertex_soa* v, const float* target, float* grads,
                            double* loss) {
    train_impl_f32(cfg, params, n, v, target, grads, loss, NULL);
}
/* the same with the per-sample loss weights of nrrs_train_step_batch */
void oracle_train_grads_w_f64(const nrrs_config* cfg, const float* params, uint64_t n,
                              const nrrs_vertex_soa* v, const float* target,
                              const oracle_loss_w* w, double* grads, double* loss) {
    double* pd = promote(params, oracle_param_count(cfg, NULL, NULL, NULL));
    train_impl_f64(cfg, pd, n, v, target, grads, loss, w);
    free(pd);
}
void oracle_train_grads_w_f32(const nrrs_config* cfg, const float* params, uint64_t n,
                              const nrrs_vertex_soa* v, const float* target,
                              const oracle_loss_w* w, float* grads, double* loss) {
    train_impl_f32(cfg, params, n, v, target, grads, loss, w);
}

/* losses only, FP64 parameters (finite differences perturb them in FP64) */
void oracle_train_loss_f64(const nrrs_config* cfg, const double* params, uint64_t n,
                           const nrrs_vertex_soa* v, const float* target, double* loss) {
    oracle_train_loss_w_f64(cfg, params, n, v, target, NULL, loss);
}

void oracle_train_loss_w_f64(const nrrs_config* cfg, const double* params, uint64_t n,
                             const nrrs_vertex_soa* v, const float* target,
                             const oracle_loss_w* w, double* loss) {
    level_t lv[32];
    const uint64_t tab = build_levels(cfg, lv);
    const double* table = params;
    const double* Ws = params + tab * 2;
    const double* Wr = Ws + statnet_params(cfg);
    const int ws = cfg->statnet_width, wr = cfg->rrsnet_width;
    const int hs = cfg->statnet_hidden, hr = cfg->rrsnet_hidden;
    double lossS = 0, sumV = 0, sumC = 0, sumR = 0, sum_s = 0, sum_w = 0;
#pragma omp parallel for schedule(static) reduction(+ : lossS, sumV, sumC, sumR, sum_s, sum_w)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint64_t i = (uint64_t)ii;
        double x0[64], acts[4 * 128], y[6], x1[16], g[4 * 128], raw;
        const double sw = lw_s_f64(w, i), ww = lw_w_f64(w, i);
        sum_s += sw;
        sum_w += ww;
        build_x0_f64(cfg, lv, table, v, i, x0, NULL, NULL);
        mlp_fwd_f64(Ws, net_stat_in(cfg), ws, hs, net_stat_out(cfg), x0, acts, y, net_ref(cfg));
        if (net_ref(cfg)) {
            for (int c = 0; c < 6; ++c) {
                const double L = (double)target[3 * i + (c % 3)];
                const double T = c < 3 ? L : L * L;
                const double d = y[c] - T;
                lossS += sw * d * d / (T * T + 0.01);
            }
        } else {
            for (int c = 0; c < 3; ++c) {
                const double d = y[c] - log((double)target[3 * i + c] + (double)cfg->stat_eps);
                lossS += sw * d * d;
            }
        }
        if (cfg->step >= 3) {
            glue_f64(cfg, y, v, i, x1);
            mlp_fwd_f64(Wr, 16, wr, hr, 1, x1, g, &raw, net_ref(cfg));
            const double q = act_sigma_f64(raw);
            const double r = rel_contrib_f64(cfg, v, target, i);
            sumV += ww * lw_u_f64(w, i) * r * r / (lw_k_f64(w, i) * q);
            sumC += ww * ((double)cfg->cost_offset + q);
            sumR += ww * log(q) * log(q);
        }
    }
    const double g4 = w ? (double)w->gamma4 : 0.0;
    loss[0] = lossS / ((net_ref(cfg) ? 6.0 : 3.0) * sum_s);
    loss[1] = cfg->step >= 3 ? (sumV / sum_w) * (sumC / sum_w) + g4 * sumR / sum_w : 0.0;
}

/* ---- exact normalisation sum (replaces calcSum2PassAsync<true>, commoncudautilshost.cpp:6-22,
 *      whose FP32 order depends on the occupancy-chosen grid). Each term is converted to a
 *      64-bit fixed-point integer with `shift` fractional bits (truncation toward zero);
 *      integer addition is associative, so any summation order gives the same bits. ---- */
int oracle_sum_shift(uint64_t n, float vmax) {
    double prod = (double)(n ? n : 1) * (double)(vmax > 1.f ? vmax : 1.f);
    int e = 0;
    frexp(prod, &e);
    int s = 62 - e;
    return s > 40 ? 40 : s;
}

int64_t oracle_sum_fixed(const float* rrs, uint64_t n, int use_ceil, int shift, double* sum) {
    int64_t acc = 0;
    for (uint64_t i = 0; i < n; ++i) {
        float x = use_ceil ? ceilf(rrs[i]) : rrs[i];
        if (!isfinite(x)) continue;
        acc += (int64_t)ldexp((double)x, shift);
    }
    if (sum) *sum = ldexp((double)acc, -shift);
    return acc;
}

/* ---- decision and emission: "Gen Tids" (src/render/nrrs/integrator.cpp:1368-1460) and
 *      TidQueue::push(tid, cnt) (src/render/common/commonworkqueue.h:19-25), with the
 *      capacity guard of pushCheck (:34-42). FP32 sequence, exactly:
 *        rcp = 1 / (float)sum                                   (commoncudautils.cu:174-176)
 *        nf  = ((float)(budget - n_specular) * rcp) * (use_ceil ? 1 : rate)     (:1376-1377)
 *        r   = rrs * (scale_up ? nf : min(nf, 1))                              (:1391-1397)
 *        s   = int(r); s += (rnd <= r - s)                          (:1415-1416, :1454)
 *      Order of the queue: vertex order, the s copies of one vertex contiguous (the
 *      reference's order is atomic-arrival; the multiset is the same). ---- */
static uint64_t decide_core(const float* rrs, const float* rnd, const uint32_t* scatter_index,
                            uint64_t n, uint32_t budget, uint32_t n_specular,
                            const nrrs_decide_params* p, double sum, float* rrs_norm,
                            uint8_t* split, uint32_t* queue, uint64_t capacity, uint32_t flags,
                            uint32_t* status_flags);

uint64_t oracle_decide_emit(const float* rrs, const float* rnd, const uint32_t* scatter_index,
                            uint64_t n, uint32_t budget, uint32_t n_specular,
                            const nrrs_decide_params* p, uint64_t shift_n, float* rrs_norm,
                            uint8_t* split, uint32_t* queue, uint64_t capacity,
                            uint32_t* status_flags) {
    uint32_t flags = 0;
    const float vmax = p->use_ceil ? ceilf(p->clamp_max) : p->clamp_max;
    const int shift = oracle_sum_shift(shift_n ? shift_n : n, vmax);
    double sum = 0;
    for (uint64_t i = 0; i < n; ++i) {
        float x = p->use_ceil ? ceilf(rrs[i]) : rrs[i];
        if (!isfinite(x)) flags |= NRRS_DEV_NAN;
    }
    oracle_sum_fixed(rrs, n, p->use_ceil, shift, &sum);
    return decide_core(rrs, rnd, scatter_index, n, budget, n_specular, p, sum, rrs_norm, split,
                       queue, capacity, flags, status_flags);
}

/* the same decision for one shard of a queue, with the exact sum accumulated over all shards */
uint64_t oracle_decide_emit_acc(const float* rrs, const float* rnd, const uint32_t* scatter_index,
                                uint64_t n, uint32_t budget, uint32_t n_specular,
                                const nrrs_decide_params* p, int64_t acc, int shift,
                                float* rrs_norm, uint8_t* split, uint32_t* queue,
                                uint64_t capacity, uint32_t* status_flags) {
    return decide_core(rrs, rnd, scatter_index, n, budget, n_specular, p, ldexp((double)acc, -shift),
                       rrs_norm, split, queue, capacity, 0u, status_flags);
}

static uint64_t decide_core(const float* rrs, const float* rnd, const uint32_t* scatter_index,
                            uint64_t n, uint32_t budget, uint32_t n_specular,
                            const nrrs_decide_params* p, double sum, float* rrs_norm,
                            uint8_t* split, uint32_t* queue, uint64_t capacity, uint32_t flags,
                            uint32_t* status_flags) {
    volatile float sumf = (float)sum;
    volatile float rcp = 1.0f / sumf;
    volatile float bud = (float)(uint32_t)(budget - n_specular);
    volatile float nf = bud * rcp;
    nf = nf * (p->use_ceil ? 1.0f : p->normalize_rate);
    const float scale = p->scale_up ? nf : (nf < 1.0f ? nf : 1.0f);
    uint64_t total = 0;
    for (uint64_t i = 0; i < n; ++i) {
        volatile float r = rrs[i] * scale;
        const uint32_t stid = scatter_index ? scatter_index[i] : (uint32_t)i;
        if (rrs_norm) rrs_norm[stid] = r;
        int s;
        if (!(r == r)) {
            s = 0;
            flags |= NRRS_DEV_NAN;
        } else if (!(r < 256.0f)) {
            s = 255;
            flags |= NRRS_DEV_SATURATED;
        } else {
            s = (int)r;
            volatile float frac = r - (float)s;
            s += (rnd[i] <= frac) ? 1 : 0;
            if (s > 255) { s = 255; flags |= NRRS_DEV_SATURATED; }
        }
        if (split) split[i] = (uint8_t)s;
        for (int k = 0; k < s; ++k) {
            if (total < capacity) queue[total] = stid;
            else flags |= NRRS_DEV_OVERFLOW;
            ++total;
        }
    }
    if (status_flags) *status_flags = flags;
    return total;
}

/* Adam (Kingma & Ba 2015) in FP32 with an optional L2 term added to the gradient */
/* The RRSNet parameters use lr_rrsnet when it is set (the reference's level1 optimizer). */
void oracle_adam_f32(const nrrs_config* cfg, float* params, const float* grads, float* m,
                     float* v, uint64_t first, uint64_t count, uint64_t t) {
    const float b1 = cfg->beta1, b2 = cfg->beta2;
    const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
    uint64_t n_table = 0, n_stat = 0;
    oracle_param_count(cfg, &n_table, &n_stat, NULL);
    const int64_t rrs_first = (int64_t)(n_table + n_stat);
    const float lr_rrs = cfg->lr_rrsnet > 0.f ? cfg->lr_rrsnet : cfg->lr;
#pragma omp parallel for schedule(static)
    for (int64_t k = (int64_t)first; k < (int64_t)(first + count); ++k) {
        const float g = grads[k] + cfg->l2_reg * params[k];
        m[k] = b1 * m[k] + (1.0f - b1) * g;
        v[k] = b2 * v[k] + (1.0f - b2) * g * g;
        const float mh = m[k] / c1, vh = v[k] / c2;
        params[k] -= (k < rrs_first ? cfg->lr : lr_rrs) * mh / (sqrtf(vh) + cfg->eps);
    }
}

void oracle_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
int oracle_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
