/*
 * nrrs_oracle_impl.h -- precision-generic body of the CPU oracle. TEST INFRASTRUCTURE ONLY.
 * Included twice by nrrs_oracle.c with REAL = double (suffix _f64) and REAL = float (_f32).
 * See nrrs_oracle.h for the parity status and the reference citations.
 */
#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SFX)

#if REAL_IS_DOUBLE
#define R_EXP exp
#define R_ATAN2 atan2
#define R_ACOS acos
#define R_LOG log
#define R_SQRT sqrt
#define R_CEIL ceil
#else
#define R_EXP expf
#define R_ATAN2 atan2f
#define R_ACOS acosf
#define R_LOG logf
#define R_SQRT sqrtf
#define R_CEIL ceilf
#endif

/* activationSigma, networkcommon.h:61-68: softplus for x<0, else 0.5x + ln 2 */
static inline REAL FN(act_sigma)(REAL x) {
    const REAL ln2 = (REAL)0.6931471805599453;
    return (x < 0) ? R_LOG((REAL)1 + R_EXP(x)) : (REAL)0.5 * x + ln2;
}
/* derivative of activationSigma: sigmoid(x) for x<0, 0.5 otherwise */
static inline REAL FN(act_sigma_grad)(REAL x) {
    if (x < 0) { REAL e = R_EXP(x); return e / ((REAL)1 + e); }
    return (REAL)0.5;
}
/* box_cox_transform with lambda = 0.5, train.cu:19-39: 2 (sqrt(x) - 1) */
static inline REAL FN(box_cox)(REAL x) { return (REAL)2 * (R_SQRT(x) - (REAL)1); }

/* real spherical harmonics, bands 0..3 (16 coefficients) of a unit direction */
static void FN(sh16)(const float* d, REAL* o) {
    const REAL x = d[0], y = d[1], z = d[2];
    const REAL xx = x * x, yy = y * y, zz = z * z;
    o[0] = (REAL)SH_C0;
    o[1] = -(REAL)SH_C1 * y;
    o[2] = (REAL)SH_C1 * z;
    o[3] = -(REAL)SH_C1 * x;
    o[4] = (REAL)SH_C2A * x * y;
    o[5] = -(REAL)SH_C2A * y * z;
    o[6] = (REAL)SH_C2B * ((REAL)3 * zz - (REAL)1);
    o[7] = -(REAL)SH_C2A * x * z;
    o[8] = (REAL)SH_C2C * (xx - yy);
    o[9] = -(REAL)SH_C3A * y * ((REAL)3 * xx - yy);
    o[10] = (REAL)SH_C3B * x * y * z;
    o[11] = -(REAL)SH_C3C * y * ((REAL)5 * zz - (REAL)1);
    o[12] = (REAL)SH_C3D * z * ((REAL)5 * zz - (REAL)3);
    o[13] = -(REAL)SH_C3C * x * ((REAL)5 * zz - (REAL)1);
    o[14] = (REAL)SH_C3E * z * (xx - yy);
    o[15] = -(REAL)SH_C3A * x * (xx - (REAL)3 * yy);
}

/* Hash-grid encoding of one normalised FP32 position (Instant-NGP, Mueller et al. 2022):
 * the scaled coordinate p*N_l is rounded to FP32, the cell is floor() clamped to [0, N_l-1],
 * trilinear weights over the 8 corners (bit0 = x, bit1 = y, bit2 = z) in corner order.
 * corner_idx/corner_w (optional, [L][8]) record the table rows and weights for backward. */
static void FN(hash_encode)(const level_t* lv, int L, const REAL* table, const float* p,
                            REAL* feat, uint32_t* corner_idx, REAL* corner_w) {
    for (int l = 0; l < L; ++l) {
        const int N = (int)lv[l].res;
        int ic[3];
        float fr[3];
        for (int d = 0; d < 3; ++d) {
            float s = p[d] * (float)N;
            int i = (int)floorf(s);
            if (i > N - 1) i = N - 1;
            if (i < 0) i = 0;
            ic[d] = i;
            fr[d] = s - (float)i;
        }
        REAL f0 = 0, f1 = 0;
        for (int c = 0; c < 8; ++c) {
            const uint32_t gx = (uint32_t)(ic[0] + (c & 1));
            const uint32_t gy = (uint32_t)(ic[1] + ((c >> 1) & 1));
            const uint32_t gz = (uint32_t)(ic[2] + ((c >> 2) & 1));
            const uint32_t idx = grid_index(&lv[l], gx, gy, gz);
            const REAL wx = (c & 1) ? (REAL)fr[0] : (REAL)1 - (REAL)fr[0];
            const REAL wy = (c & 2) ? (REAL)fr[1] : (REAL)1 - (REAL)fr[1];
            const REAL wz = (c & 4) ? (REAL)fr[2] : (REAL)1 - (REAL)fr[2];
            const REAL w = wx * wy * wz;
            const uint64_t row = (uint64_t)lv[l].offset + idx;
            f0 += w * (REAL)table[row * 2 + 0];
            f1 += w * (REAL)table[row * 2 + 1];
            if (corner_idx) { corner_idx[l * 8 + c] = (uint32_t)row; corner_w[l * 8 + c] = w; }
        }
        feat[2 * l + 0] = f0;
        feat[2 * l + 1] = f1;
    }
}

/* One-blob encoding of x in [0,1] into `bins` lanes (Mueller et al. 2019) with the compact
 * quartic (biweight) kernel of radius 1/bins that tiny-cuda-nn's OneBlob uses: lane k holds the
 * kernel mass centred at x that falls into bin [k/bins, (k+1)/bins), F(b - x) - F(a - x), where
 * F is the kernel's CDF, F(t) = 15/16 (u - 2u^3/3 + u^5/5) + 1/2 at u = t bins clamped to [-1,1]. */
static REAL FN(quartic_cdf)(REAL t, int bins) {
    REAL u = t * (REAL)bins;
    u = u < (REAL)-1 ? (REAL)-1 : (u > (REAL)1 ? (REAL)1 : u);
    const REAL u2 = u * u;
    return (REAL)15 / (REAL)16 * u * ((REAL)1 - (REAL)2 / (REAL)3 * u2 + u2 * u2 / (REAL)5) +
           (REAL)0.5;
}
static void FN(one_blob)(REAL x, int bins, REAL* out) {
    for (int k = 0; k < bins; ++k)
        out[k] = FN(quartic_cdf)((REAL)(k + 1) / (REAL)bins - x, bins) -
                 FN(quartic_cdf)((REAL)k / (REAL)bins - x, bins);
}
/* lat-long coordinates of a unit direction (the reference's work item stores wi as lat-long,
 * workqueue.h:159, through KiRaRay's worldToLatLong, absent from the checkout):
 * u = atan2(y, x) / 2pi + 1/2, v = acos(z) / pi */
static void FN(latlong)(const float* d, REAL* uv) {
    const REAL z = (REAL)d[2] < (REAL)-1 ? (REAL)-1 : ((REAL)d[2] > (REAL)1 ? (REAL)1 : (REAL)d[2]);
    uv[0] = R_ATAN2((REAL)d[1], (REAL)d[0]) * (REAL)0.15915494309189535 + (REAL)0.5;
    uv[1] = R_ACOS(z) * (REAL)0.3183098861837907;
}

/* StatNet input row x0[64]: [0,32) hash features, [32,48) SH(wi), [48,51) normal,
 * [51,54) albedo, [54] 1-exp(-roughness) (warp_roughness, train.h:95), [55] 1 (bias), rest 0 */
static void FN(build_x0)(const nrrs_config* cfg, const level_t* lv, const REAL* table,
                         const nrrs_vertex_soa* v, uint64_t i, REAL* x0, uint32_t* cidx,
                         REAL* cw) {
    float pn[3];
    oracle_normalize_pos_f32(cfg, v->pos + 3 * i, pn);
    FN(hash_encode)(lv, cfg->n_levels, table, pn, x0, cidx, cw);
    if (net_ref(cfg)) {
        /* the reference network: [0,16) hash features, [16,20) and [20,24) one-blob of the
         * lat-long u and v, [24,32) one-blob of the warped roughness */
        REAL uv[2];
        FN(latlong)(v->wi + 3 * i, uv);
        FN(one_blob)(uv[0], 4, x0 + 16);
        FN(one_blob)(uv[1], 4, x0 + 20);
        FN(one_blob)((REAL)1 - R_EXP(-(REAL)v->roughness[i]), 8, x0 + 24);
        return;
    }
    FN(sh16)(v->wi + 3 * i, x0 + 32);
    for (int d = 0; d < 3; ++d) x0[48 + d] = (REAL)v->normal[3 * i + d];
    for (int d = 0; d < 3; ++d) x0[51 + d] = (REAL)v->albedo[3 * i + d];
    x0[54] = (REAL)1 - R_EXP(-(REAL)v->roughness[i]);
    x0[55] = (REAL)1;
    for (int d = 56; d < 64; ++d) x0[d] = 0;
}

/* y = W x for row-major W [out][in]  */
static void FN(matvec)(const REAL* W, int out, int in, const REAL* x, REAL* y) {
    for (int o = 0; o < out; ++o) {
        REAL acc = 0;
        const REAL* w = W + (uint64_t)o * in;
        for (int k = 0; k < in; ++k) acc += (REAL)w[k] * x[k];
        y[o] = acc;
    }
}
static void FN(relu)(REAL* x, int n) { for (int k = 0; k < n; ++k) x[k] = x[k] > 0 ? x[k] : 0; }
/* LeakyReLU with tiny-cuda-nn's slope 0.01 (the reference network's activation) */
static void FN(leaky)(REAL* x, int n) {
    for (int k = 0; k < n; ++k) x[k] = x[k] > 0 ? x[k] : (REAL)0.01 * x[k];
}

/* forward through a bias-free ReLU MLP; acts[l] receives the post-activation of hidden l;
 * layer widths: in -> w (hidden times) -> out */
static void FN(mlp_fwd)(const REAL* W, int in, int w, int hidden, int out, const REAL* x,
                        REAL* acts /* [hidden][w] */, REAL* y, int leaky) {
    const REAL* cur = x;
    int cur_in = in;
    for (int h = 0; h < hidden; ++h) {
        FN(matvec)(W, w, cur_in, cur, acts + h * w);
        if (leaky) FN(leaky)(acts + h * w, w);
        else FN(relu)(acts + h * w, w);
        W += (uint64_t)w * cur_in;
        cur = acts + h * w;
        cur_in = w;
    }
    FN(matvec)(W, out, cur_in, cur, y);
}

/* backward through the same MLP: dy -> weight grads (accumulated into dW) and dx (optional) */
static void FN(mlp_bwd)(const REAL* W, int in, int w, int hidden, int out, const REAL* x,
                        const REAL* acts, const REAL* dy, REAL* dW, REAL* dx, int leaky) {
    /* offsets of each layer in W / dW */
    uint64_t off[8];
    int ins[8], outs[8];
    uint64_t o = 0;
    for (int h = 0; h <= hidden; ++h) {
        ins[h] = h == 0 ? in : w;
        outs[h] = h == hidden ? out : w;
        off[h] = o;
        o += (uint64_t)ins[h] * outs[h];
    }
    REAL dcur[128], dprev[128];
    for (int k = 0; k < out; ++k) dcur[k] = dy[k];
    for (int h = hidden; h >= 0; --h) {
        const REAL* a = h == 0 ? x : acts + (h - 1) * w;
        const REAL* Wl = W + off[h];
        REAL* dWl = dW + off[h];
        for (int r = 0; r < outs[h]; ++r)
            for (int k = 0; k < ins[h]; ++k) dWl[(uint64_t)r * ins[h] + k] += dcur[r] * a[k];
        if (h == 0 && !dx) break;
        for (int k = 0; k < ins[h]; ++k) {
            REAL acc = 0;
            for (int r = 0; r < outs[h]; ++r) acc += (REAL)Wl[(uint64_t)r * ins[h] + k] * dcur[r];
            dprev[k] = acc;
        }
        if (h > 0) {
            for (int k = 0; k < ins[h]; ++k)
                dcur[k] = a[k] > 0 ? dprev[k] : (leaky ? (REAL)0.01 * dprev[k] : (REAL)0);
        } else {
            for (int k = 0; k < ins[h]; ++k) dx[k] = dprev[k];
        }
    }
}

/* glue, train.cu:41-112 restated for 3 log-statistics: RRSNet input x1[16] =
 * [bc(Lhat) x3, bc(thp) x3, warped roughness, bc(ref_mean), depth/8, 1, 0 x6],
 * Lhat_c = max(exp(min(y_c, 20)) - stat_eps, 0) */
static void FN(glue)(const nrrs_config* cfg, const REAL* y, const nrrs_vertex_soa* v, uint64_t i,
                     REAL* x1) {
    if (net_ref(cfg)) {
        /* the reference's own glue (train.cu:41-112): [bc(max(L,0)) x3, bc(max(L^2,0)) x3,
         * bc(thp) x3, warped roughness, bc(ref_mean), 1, 0 x4] */
        for (int c = 0; c < 3; ++c) {
            x1[c] = FN(box_cox)(y[c] > 0 ? y[c] : (REAL)0);
            x1[3 + c] = FN(box_cox)(y[3 + c] > 0 ? y[3 + c] : (REAL)0);
            x1[6 + c] = FN(box_cox)((REAL)v->thp[3 * i + c]);
        }
        x1[9] = (REAL)1 - R_EXP(-(REAL)v->roughness[i]);
        x1[10] = FN(box_cox)(v->ref_mean ? (REAL)v->ref_mean[i] : (REAL)0.5);
        x1[11] = 1;
        for (int k = 12; k < 16; ++k) x1[k] = 0;
        return;
    }
    for (int c = 0; c < 3; ++c) {
        REAL yc = y[c] < (REAL)20 ? y[c] : (REAL)20;
        REAL L = R_EXP(yc) - (REAL)cfg->stat_eps;
        if (!(L > 0)) L = 0;
        x1[c] = FN(box_cox)(L);
        x1[3 + c] = FN(box_cox)((REAL)v->thp[3 * i + c]);
    }
    x1[6] = (REAL)1 - R_EXP(-(REAL)v->roughness[i]);
    const REAL ref = v->ref_mean ? (REAL)v->ref_mean[i] : (REAL)0.5;
    x1[7] = FN(box_cox)(ref);
    x1[8] = (REAL)(v->depth ? v->depth[i] : 0) * (REAL)0.125;
    x1[9] = 1;
    for (int k = 10; k < 16; ++k) x1[k] = 0;
}

/* factor, clamp (integrator.cpp:1184-1298) */
static REAL FN(factor)(const nrrs_config* cfg, const nrrs_decide_params* p, const REAL* y,
                       REAL raw, const nrrs_vertex_soa* v, uint64_t i) {
    REAL rrs;
    if (p->factor_source == NRRS_FACTOR_ADRRS) {
        const REAL ref = (v->ref_mean ? (REAL)v->ref_mean[i] : (REAL)0.5) + (REAL)cfg->ref_eps;
        REAL acc = 0;
        for (int c = 0; c < 3; ++c) {
            REAL L;
            if (net_ref(cfg)) {
                L = y[c];   /* the reference network outputs L itself */
            } else {
                REAL yc = y[c] < (REAL)20 ? y[c] : (REAL)20;
                L = R_EXP(yc) - (REAL)cfg->stat_eps;
            }
            L = L < (REAL)1e-4 ? (REAL)1e-4 : (L > (REAL)1e4 ? (REAL)1e4 : L);
            acc += L * (REAL)v->thp[3 * i + c] / ref;
        }
        rrs = acc / (REAL)3;
    } else {
        rrs = FN(act_sigma)(raw);
    }
    if (p->use_weight_window) {
        const REAL dminus = (REAL)2 / ((REAL)1 + (REAL)p->weight_window_size);
        const REAL dplus = dminus * (REAL)p->weight_window_size;
        rrs = rrs < dminus ? rrs / dminus : (rrs > dplus ? rrs / dplus : (REAL)1);
    }
    const REAL lo = (REAL)p->clamp_min, hi = (REAL)p->clamp_max;
    rrs = rrs < lo ? lo : (rrs > hi ? hi : rrs);
    return rrs;
}

static void FN(infer_impl)(const nrrs_config* cfg, const REAL* params, uint64_t n,
                      const nrrs_vertex_soa* v, const nrrs_decide_params* p, REAL* x0o,
                      REAL* stats, REAL* x1o, REAL* rawo, REAL* rrso) {
    level_t lv[32];
    uint64_t tab = build_levels(cfg, lv);
    const REAL* table = params;
    const REAL* Ws = params + tab * 2;
    const REAL* Wr = Ws + statnet_params(cfg);
    const int ws = cfg->statnet_width, wr = cfg->rrsnet_width;
    const int hs = cfg->statnet_hidden, hr = cfg->rrsnet_hidden;
    const int sin_ = net_stat_in(cfg), sout = net_stat_out(cfg), leaky = net_ref(cfg);
#pragma omp parallel for schedule(static)
    for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
        const uint64_t i = (uint64_t)ii;
        REAL x0[64], acts[4 * 128], y[6], x1[16], g[4 * 128], raw;
        for (int k = 0; k < 64; ++k) x0[k] = 0;
        FN(build_x0)(cfg, lv, table, v, i, x0, NULL, NULL);
        FN(mlp_fwd)(Ws, sin_, ws, hs, sout, x0, acts, y, leaky);
        FN(glue)(cfg, y, v, i, x1);
        FN(mlp_fwd)(Wr, 16, wr, hr, 1, x1, g, &raw, leaky);
        if (x0o) for (int k = 0; k < 64; ++k) x0o[i * 64 + k] = x0[k];
        if (stats) for (int k = 0; k < sout; ++k) stats[i * sout + k] = y[k];
        if (x1o) for (int k = 0; k < 16; ++k) x1o[i * 16 + k] = x1[k];
        if (rawo) rawo[i] = raw;
        if (rrso) rrso[i] = FN(factor)(cfg, p, y, raw, v, i);
    }
}

/* relative contribution used by the RRSNet loss: min(mean_c(thp_c L_c) / (ref + ref_eps), clamp) */
static REAL FN(rel_contrib)(const nrrs_config* cfg, const nrrs_vertex_soa* v, const float* target,
                            uint64_t i) {
    REAL acc = 0;
    for (int c = 0; c < 3; ++c) acc += (REAL)v->thp[3 * i + c] * (REAL)target[3 * i + c];
    const REAL ref = (v->ref_mean ? (REAL)v->ref_mean[i] : (REAL)0.5) + (REAL)cfg->ref_eps;
    REAL r = acc / (REAL)3 / ref;
    return r < (REAL)cfg->loss_clamp_max ? r : (REAL)cfg->loss_clamp_max;
}

/* per-sample loss weights of nrrs_train_step_batch (the definition in include/nrrs.h):
 * stat weight s, RRSNet weight w (0 for a -1 RRSNet target), error emphasis u, sample count k */
static REAL FN(lw_s)(const oracle_loss_w* w, uint64_t i) {
    return (w && w->sample_weight) ? (REAL)w->sample_weight[i] : (REAL)1;
}
static REAL FN(lw_w)(const oracle_loss_w* w, uint64_t i) {
    return (w && w->rrs_target && w->rrs_target[i] < 0.f) ? (REAL)0 : FN(lw_s)(w, i);
}
static REAL FN(lw_u)(const oracle_loss_w* w, uint64_t i) {
    if (!w) return 1;
    REAL e = w->error ? (REAL)w->error[i] / (REAL)w->error_mean : (REAL)1;
    REAL a = w->error_for_avg ? (REAL)w->error_for_avg[i] / (REAL)w->error_mean : (REAL)1;
    if (w->clamp_on) {
        e = e < (REAL)w->clamp_max ? e : (REAL)w->clamp_max;
        a = a < (REAL)w->clamp_max ? a : (REAL)w->clamp_max;
    }
    return (REAL)w->gamma1 + (REAL)w->gamma2 * e + (REAL)w->gamma3 * a;
}
static REAL FN(lw_k)(const oracle_loss_w* w, uint64_t i) {
    if (!w || !w->number_samples) return 1;
    return w->number_samples[i] > 1.f ? (REAL)w->number_samples[i] : (REAL)1;
}

/* Losses and gradients of one training step (no update).
 * StatNet: loss_S = 1/(3n) sum_i sum_c (y_ic - log(L_ic + stat_eps))^2   (relative log-L2)
 * RRSNet:  q_i = activationSigma(raw_i), a_i = rel_contrib_i^2,
 *          V = 1/n sum a_i / q_i,  C = 1/n sum (cost_offset + q_i),  loss_R = V * C
 *          RRSNet inputs come from the (detached) StatNet forward of the same step. */
static void FN(train_impl)(const nrrs_config* cfg, const REAL* params, uint64_t n,
                            const nrrs_vertex_soa* v, const float* target, REAL* grads,
                            double* loss, const oracle_loss_w* w) {
    level_t lv[32];
    uint64_t tab = build_levels(cfg, lv);
    const uint64_t np_table = tab * 2, np_stat = statnet_params(cfg), np_rrs = rrsnet_params(cfg);
    const uint64_t np = np_table + np_stat + np_rrs;
    const REAL* table = params;
    const REAL* Ws = params + np_table;
    const REAL* Wr = Ws + np_stat;
    const int ws = cfg->statnet_width, wr = cfg->rrsnet_width;
    const int hs = cfg->statnet_hidden, hr = cfg->rrsnet_hidden;
    const int train_rrs = cfg->step >= 3;
    const int sin_ = net_stat_in(cfg), sout = net_stat_out(cfg), leaky = net_ref(cfg);
    memset(grads, 0, sizeof(REAL) * np);
    double lossS = 0, sumV = 0, sumC = 0, sumR = 0;
    /* weighted losses: the batch sums of the weights, and the divisors of the means */
    double sum_s = (double)n, sum_w = (double)n;
    if (w) {
        sum_s = 0;
        sum_w = 0;
        for (uint64_t i = 0; i < n; ++i) {
            sum_s += (double)FN(lw_s)(w, i);
            sum_w += (double)FN(lw_w)(w, i);
        }
    }

    /* pass 1: RRSNet forward for the batch sums V and C */
    if (train_rrs) {
#pragma omp parallel for schedule(static) reduction(+ : sumV, sumC, sumR)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint64_t i = (uint64_t)ii;
            REAL x0[64], acts[4 * 128], y[6], x1[16], g[4 * 128], raw;
            FN(build_x0)(cfg, lv, table, v, i, x0, NULL, NULL);
            FN(mlp_fwd)(Ws, sin_, ws, hs, sout, x0, acts, y, leaky);
            FN(glue)(cfg, y, v, i, x1);
            FN(mlp_fwd)(Wr, 16, wr, hr, 1, x1, g, &raw, leaky);
            const REAL q = FN(act_sigma)(raw);
            const REAL r = FN(rel_contrib)(cfg, v, target, i);
            if (w) {
                const REAL ww = FN(lw_w)(w, i), lq = R_LOG(q);
                sumV += (double)(ww * FN(lw_u)(w, i) * r * r / (FN(lw_k)(w, i) * q));
                sumC += (double)(ww * ((REAL)cfg->cost_offset + q));
                sumR += (double)(ww * lq * lq);
            } else {
                sumV += (double)(r * r / q);
                sumC += (double)((REAL)cfg->cost_offset + q);
            }
        }
    }
    const double Vm = sumV / sum_w, Cm = sumC / sum_w, Rm = sumR / sum_w;
    const double g4 = w ? (double)w->gamma4 : 0.0;

    /* pass 2: per-sample backward */
    int nt = 1;
#ifdef _OPENMP
    nt = omp_get_max_threads();
#endif
    const uint64_t np_mlp = np_stat + np_rrs;
    REAL* priv = (REAL*)calloc((size_t)nt * np_mlp, sizeof(REAL));
#pragma omp parallel reduction(+ : lossS)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        REAL* dWs = priv + (uint64_t)tid * np_mlp;
        REAL* dWr = dWs + np_stat;
#pragma omp for schedule(static)
        for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
            const uint64_t i = (uint64_t)ii;
            REAL x0[64], acts[4 * 128], y[6], dy[6], dx0[64], cw[16 * 8];
            uint32_t cidx[16 * 8];
            FN(build_x0)(cfg, lv, table, v, i, x0, cidx, cw);
            FN(mlp_fwd)(Ws, sin_, ws, hs, sout, x0, acts, y, leaky);
            const REAL sw = FN(lw_s)(w, i);
            if (leaky) {
                /* the reference network: relative squared error of L and L^2 against the target
                 * L and its square, (y - T)^2 / (T^2 + 0.01), mean over the 6 outputs */
                for (int c = 0; c < 6; ++c) {
                    const REAL L = (REAL)target[3 * i + (c % 3)];
                    const REAL T = c < 3 ? L : L * L;
                    const REAL den = T * T + (REAL)0.01;
                    const REAL d = y[c] - T;
                    lossS += (double)(sw * d * d / den);
                    dy[c] = (REAL)2 * sw * d / (den * (REAL)6 * (REAL)sum_s);
                }
            } else {
                for (int c = 0; c < 3; ++c) {
                    const REAL t = R_LOG((REAL)target[3 * i + c] + (REAL)cfg->stat_eps);
                    const REAL d = y[c] - t;
                    if (w) {
                        lossS += (double)(sw * d * d);
                        dy[c] = (REAL)2 * sw * d / ((REAL)3 * (REAL)sum_s);
                    } else {
                        lossS += (double)(d * d);
                        dy[c] = (REAL)2 * d / ((REAL)3 * (REAL)n);
                    }
                }
            }
            FN(mlp_bwd)(Ws, sin_, ws, hs, sout, x0, acts, dy, dWs, dx0, leaky);
            for (int l = 0; l < cfg->n_levels; ++l)
                for (int c = 0; c < 8; ++c) {
                    const uint64_t row = cidx[l * 8 + c];
                    const REAL w = cw[l * 8 + c];
                    const REAL g0 = w * dx0[2 * l], g1 = w * dx0[2 * l + 1];
#pragma omp atomic
                    grads[row * 2 + 0] += g0;
#pragma omp atomic
                    grads[row * 2 + 1] += g1;
                }
            if (train_rrs) {
                REAL x1[16], g[4 * 128], raw, draw;
                FN(glue)(cfg, y, v, i, x1);
                FN(mlp_fwd)(Wr, 16, wr, hr, 1, x1, g, &raw, leaky);
                const REAL q = FN(act_sigma)(raw);
                const REAL r = FN(rel_contrib)(cfg, v, target, i);
                REAL dq;
                if (w) {
                    const REAL ww = FN(lw_w)(w, i);
                    dq = (ww * FN(lw_u)(w, i) * (-(r * r)) / (FN(lw_k)(w, i) * q * q) * (REAL)Cm +
                          ww * (REAL)Vm + (REAL)g4 * ww * (REAL)2 * R_LOG(q) / q) / (REAL)sum_w;
                } else {
                    dq = (-(r * r) / (q * q) * (REAL)Cm + (REAL)Vm) / (REAL)n;
                }
                draw = dq * FN(act_sigma_grad)(raw);
                FN(mlp_bwd)(Wr, 16, wr, hr, 1, x1, g, &draw, dWr, NULL, leaky);
            }
        }
    }
    for (int t = 0; t < nt; ++t)
        for (uint64_t k = 0; k < np_mlp; ++k) grads[np_table + k] += priv[(uint64_t)t * np_mlp + k];
    free(priv);
    loss[0] = lossS / ((double)(leaky ? 6 : 3) * sum_s);
    loss[1] = train_rrs ? Vm * Cm + g4 * Rm : 0.0;
}

#undef R_EXP
#undef R_ATAN2
#undef R_ACOS
#undef R_LOG
#undef R_SQRT
#undef R_CEIL
#undef FN
#undef CAT
#undef CAT2
