// nrrs_api.cu -- the C-ABI of libnrrs_b200 (declared in include/nrrs.h).
//
// Host orchestration of the NRRS hot path. Each entry point validates its arguments, builds a
// by-value kernel argument block and enqueues kernels on the caller's stream; nothing here
// synchronises except the calls documented as synchronous. There is no CPU fallback: on a
// machine without an sm_100 device nrrs_create returns NRRS_ERR_NO_DEVICE.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <vector>

#include "context.hpp"

using namespace nrrs;

namespace {

thread_local std::string g_create_error;

int fail(nrrs_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_error = msg;
    else g_create_error = msg;
    return code;
}

int cuda_fail(nrrs_ctx* ctx, cudaError_t e, const char* where) {
    return fail(ctx, NRRS_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Level table of the Instant-NGP grid: N_l = floor(N_min * b^l), dense when (N_l+1)^3 <= T.
uint64_t build_levels(const nrrs_config& c, EncodeParams& e) {
    const uint64_t T = 1ull << c.log2_hashmap_size;
    uint64_t off = 0, cells = 0;
    for (int l = 0; l < c.n_levels; ++l) {
        const uint32_t N =
            (uint32_t)std::floor((double)c.base_resolution * std::pow((double)c.per_level_scale, (double)l));
        const uint64_t R = (uint64_t)N + 1;
        const uint64_t dense_n = R * R * R;
        e.lv[l].res = N;
        e.lv[l].dense = dense_n <= T;
        e.lv[l].offset = (uint32_t)off;
        e.lv[l].cell = e.lv[l].dense ? (uint32_t)cells : 0u;
        if (e.lv[l].dense) cells += (uint64_t)N * N * N;
        off += e.lv[l].dense ? dense_n : T;
    }
    e.cells = nullptr;
    e.n_levels = (uint32_t)c.n_levels;
    e.hash_mask = (uint32_t)(T - 1);
    return off;
}

// normalizeSpatialCoord's AABB terms (nrctrain.h:111-115), FP32 on the host
void aabb_terms(const nrrs_config& c, EncodeParams& e) {
    e.normalize = c.normalize_pos;
    float dg[3];
    for (int d = 0; d < 3; ++d) dg[d] = c.aabb_max[d] - c.aabb_min[d];
    const float inflate = sqrtf(dg[0] * dg[0] + dg[1] * dg[1] + dg[2] * dg[2]) * 0.005f;
    for (int d = 0; d < 3; ++d) {
        const float lo = c.aabb_min[d] - inflate, hi = c.aabb_max[d] + inflate;
        e.center[d] = (lo + hi) * 0.5f;
        e.diag[d] = hi - lo;
    }
}

uint64_t mlp_params(int in, int w, int h, int out) {
    return (uint64_t)in * w + (uint64_t)(h - 1) * w * w + (uint64_t)w * out;
}

// The shift depends only on the context capacity and the clamp, so a depth gives the same
// decisions whether it runs alone, batched, or sharded.
// the terms an exact sum can hold: max_queue per context, times the contexts added together
uint64_t sum_capacity(const nrrs_ctx* ctx) {
    return (uint64_t)ctx->cfg.max_queue * (ctx->cfg.sum_shards > 1 ? ctx->cfg.sum_shards : 1u);
}

FactorParams factor_params(const nrrs_ctx* ctx, const nrrs_decide_params* p) {
    const uint64_t n = sum_capacity(ctx);
    FactorParams f{};
    f.clamp_min = p->clamp_min;
    f.clamp_max = p->clamp_max;
    f.ww = p->weight_window_size;
    f.use_ww = p->use_weight_window;
    f.use_ceil = p->use_ceil;
    f.source = p->factor_source;
    f.stat_eps = ctx->cfg.stat_eps;
    f.ref_eps = ctx->cfg.ref_eps;
    f.vmax = p->use_ceil ? ceilf(p->clamp_max) : p->clamp_max;
    f.fixed_scale = std::ldexp(1.0, sum_shift(n, f.vmax));
    return f;
}

int check_decide_params(nrrs_ctx* ctx, const nrrs_decide_params* p, uint64_t n_total) {
    if (!p) return fail(ctx, NRRS_ERR_INVALID_ARG, "decide params are NULL");
    if (!(p->clamp_min >= 0.f) || !(p->clamp_max >= p->clamp_min) || !std::isfinite(p->clamp_max))
        return fail(ctx, NRRS_ERR_INVALID_ARG, "need 0 <= clamp_min <= clamp_max < inf");
    if (p->factor_source != NRRS_FACTOR_ADRRS && p->factor_source != NRRS_FACTOR_RRSNET)
        return fail(ctx, NRRS_ERR_INVALID_ARG, "factor_source must be 2 (ADRRS) or 3 (RRSNet)");
    (void)n_total;
    if (sum_shift(sum_capacity(ctx), p->use_ceil ? ceilf(p->clamp_max) : p->clamp_max) < 16)
        return fail(ctx, NRRS_ERR_UNSUPPORTED, "n * clamp_max too large for the exact sum");
    return NRRS_OK;
}

int check_vertices(nrrs_ctx* ctx, const nrrs_vertex_soa* v) {
    if (!v || !v->pos || !v->wi || !v->normal || !v->roughness || !v->albedo || !v->thp)
        return fail(ctx, NRRS_ERR_INVALID_ARG, "vertex SoA: pos/wi/normal/roughness/albedo/thp required");
    return NRRS_OK;
}

VertexPtrs vptrs(const nrrs_vertex_soa* v) {
    VertexPtrs p{};
    p.pos = v->pos; p.wi = v->wi; p.normal = v->normal; p.rough = v->roughness;
    p.albedo = v->albedo; p.thp = v->thp; p.depth = v->depth; p.ref = v->ref_mean;
    p.sidx = v->scatter_index;
    return p;
}

// segment table in units of `unit` vertices per tile
SegmentTable make_segments(const nrrs_segment* segs, int n, uint32_t unit) {
    SegmentTable t{};
    t.n = n;
    uint32_t tiles = 0;
    for (int k = 0; k < n; ++k) {
        t.s[k].offset = segs[k].offset;
        t.s[k].count = segs[k].count;
        t.s[k].tile_start = tiles;
        t.s[k].budget = segs[k].budget;
        t.s[k].n_specular = segs[k].n_specular;
        t.s[k].queue_offset = segs[k].queue_offset;
        t.s[k].queue_capacity = segs[k].queue_capacity;
        tiles += (segs[k].count + unit - 1) / unit;
    }
    t.total_tiles = tiles;
    return t;
}

// Restart the moving average at an upload of the parameters: e = 0, t = 0, and the inference
// weights are the uploaded ones.
int ema_restart(nrrs_ctx* ctx, cudaStream_t s) {
    if (!ctx->ema) return NRRS_OK;
    ctx->ema_t = 0;
    const size_t b = sizeof(float) * ctx->n_params;
    cudaError_t e = cudaMemsetAsync(ctx->ema, 0, b, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(ctx->params_inf, ctx->params, b, cudaMemcpyDeviceToDevice, s);
    return e == cudaSuccess ? NRRS_OK : cuda_fail(ctx, e, "moving average restart");
}

// The images derived from the weights: from params the training images (transposed and row-major
// FP32 MLP weights, the tensor-core training image, the FP16 table and its cell image); from the
// inference weights (params_inf with a moving average, else params) the inference images (the
// UMMA weight image, and with a moving average its own transposed weights, FP16 table and cell
// image). table = false skips the tables (the Adam and moving-average passes wrote them).
int refresh_derived(nrrs_ctx* ctx, cudaStream_t s, bool table = true) {
    const nrrs_config& c = ctx->cfg;
    const bool ema = ctx->ema != nullptr;
    cudaError_t e;
    {
        ProfScope ps(ctx, NRRS_KERNEL_PACK, s);
        e = launch_pack_weights(ctx->params + ctx->n_table, ctx->wt, ctx->wrow,
                                ema ? nullptr : ctx->wpack, c.statnet_width, c.statnet_hidden,
                                c.rrsnet_width, c.rrsnet_hidden, c.precision, s);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pack weights");
    if (ema) {
        ProfScope ps(ctx, NRRS_KERNEL_PACK, s);
        e = launch_pack_weights(ctx->params_inf + ctx->n_table, ctx->wt_inf, nullptr, ctx->wpack,
                                c.statnet_width, c.statnet_hidden, c.rrsnet_width,
                                c.rrsnet_hidden, c.precision, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "pack inference weights");
    }
    if (ctx->tpack) {
        ProfScope ps(ctx, NRRS_KERNEL_PACK, s);
        e = launch_pack_train(ctx->params + ctx->n_table, ctx->tpack, c.statnet_width,
                              c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "pack training weights");
    }
    if (ctx->table_h && table) {
        ProfScope ps(ctx, NRRS_KERNEL_TABLE_HALF, s);
        e = launch_table_to_half(ctx->params, ctx->table_h, ctx->n_table, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "table to half");
    }
    if (ctx->cells && table) {
        ProfScope ps(ctx, NRRS_KERNEL_CELL_IMAGE, s);
        e = launch_cell_image(ctx->table_h, ctx->enc, ctx->cells, ctx->n_cells, ctx->sm_count, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "cell image");
    }
    if (ema && ctx->table_h_inf && table) {
        ProfScope ps(ctx, NRRS_KERNEL_TABLE_HALF, s);
        e = launch_table_to_half(ctx->params_inf, ctx->table_h_inf, ctx->n_table, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "inference table to half");
    }
    if (ema && ctx->cells_inf && table) {
        ProfScope ps(ctx, NRRS_KERNEL_CELL_IMAGE, s);
        e = launch_cell_image(ctx->table_h_inf, ctx->enc, ctx->cells_inf, ctx->n_cells,
                              ctx->sm_count, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "inference cell image");
    }
    return NRRS_OK;
}

int run_infer(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const SegmentTable& segs,
              const nrrs_decide_params* p, uint64_t n_total, float* stats, float* rrs,
              bool accumulate, cudaStream_t s, unsigned long long* ext_acc = nullptr,
              const SegmentTable* resolved = nullptr) {
    InferArgs a{};
    a.v = vptrs(v);
    a.enc = ctx->enc;
    a.fp = factor_params(ctx, p);
    a.segs = segs;
    a.segs.resolved = resolved;
    // the inference weights: the debiased moving average when there is one
    const bool ema = ctx->ema != nullptr;
    if (ema) a.enc.cells = ctx->enc.cells ? ctx->cells_inf : nullptr;
    a.table = ema ? ctx->params_inf : ctx->params;
    a.table_h = ema ? ctx->table_h_inf : ctx->table_h;
    a.wt_stat = ema ? ctx->wt_inf : ctx->wt;
    a.wt_rrs = a.wt_stat + ctx->wt_rrs_offset;
    a.wpack = ctx->wpack;
    a.stats = stats;
    a.rrs = rrs;
    a.scr = accumulate ? ctx->scr : nullptr;
    a.ext_acc = ext_acc;
    const nrrs_config& c = ctx->cfg;
    cudaError_t e;
    if (segs.total_tiles == 0) return NRRS_OK;
    const int split = c.precision != NRRS_PREC_FP32 ? ctx->tc_split : 0;
    if (split) {
        // level-major encoding into the feature tiles, then the MLP kernel reads them. Running
        // the two concurrently in chunks (encoding of chunk c+1 on a second stream) was measured
        // 1.6x slower than back to back: the encoding's L1 gather traffic and the MLP kernel's
        // shared-memory traffic share the SM's L1/shared-memory pipeline.
        if (!ctx->enc_tiles || segs.total_tiles > ctx->enc_tiles_cap)
            return fail(ctx, NRRS_ERR_INVALID_ARG, "split inference: feature tiles too small");
        EncodeLvArgs ea{};
        ea.enc = a.enc;
        ea.segs = segs;
        ea.segs.resolved = resolved;
        ea.pos = a.v.pos;
        ea.table_h = a.table_h;
        ea.out = ctx->enc_tiles;
        ea.tile_bytes = kEncTileBytes;
        ea.kdim = 32;
        {
            ProfScope ps(ctx, NRRS_KERNEL_ENCODE, s);
            e = launch_encode_levels(ea, c.precision == NRRS_PREC_BF16, ctx->sm_count, s);
        }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "encoding launch");
        a.enc_tiles = ctx->enc_tiles;
    }
    if (split >= 2) {
        // StatNet kernel (writes the RRSNet input tiles; computes ADRRS factors itself), then
        // the RRSNet kernel when the factor comes from RRSNet. Each holds only its own weights,
        // so more 128-vertex tiles are in flight per SM. Mode 3 keeps the hidden activations in
        // TMEM as the next layer's A operand.
        if (!ctx->x1_tiles) return fail(ctx, NRRS_ERR_INVALID_ARG, "split inference: no RRSNet input tiles");
        a.x1_tiles = ctx->x1_tiles;
        const bool ta = split == 3;
        {
            ProfScope ps(ctx, NRRS_KERNEL_INFER_TC, s);
            e = launch_infer_tc(a, c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden,
                                c.precision, ctx->sm_count, ctx->tc_ctas_per_sm, ctx->tc_wgs, 1, ta, s);
        }
        if (e == cudaSuccess && a.fp.source == NRRS_FACTOR_RRSNET) {
            ProfScope ps(ctx, NRRS_KERNEL_INFER_RRS, s);
            e = launch_infer_tc(a, c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden,
                                c.precision, ctx->sm_count, ctx->tc_ctas_per_sm, ctx->tc_wgs, 2, ta, s);
        }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "inference launch");
        ctx->last_infer_grid = g_last_grid;
        return NRRS_OK;
    }
    {
        ProfScope ps(ctx, c.precision == NRRS_PREC_FP32 ? NRRS_KERNEL_INFER_FP32 : NRRS_KERNEL_INFER_TC, s);
        if (c.precision == NRRS_PREC_FP32)
            e = launch_infer_fp32(a, c.statnet_width, c.statnet_hidden, c.rrsnet_width,
                                  c.rrsnet_hidden, ctx->sm_count, ctx->simt_ctas_per_sm, s);
        else
            e = launch_infer_tc(a, c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden,
                                c.precision, ctx->sm_count, ctx->tc_ctas_per_sm, ctx->tc_wgs, 0, false, s);
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "inference launch");
    ctx->last_infer_grid = g_last_grid;
    return NRRS_OK;
}

int run_decide(nrrs_ctx* ctx, const float* rrs, const float* rnd, const uint32_t* sidx,
               const nrrs_segment* segs, int n_segs, uint64_t n_total,
               const uint32_t* n_spec_dev, const nrrs_decide_params* p, float* rrs_norm,
               uint8_t* split, uint32_t* queue, uint32_t* next_size, bool need_sum,
               cudaStream_t s, const long long* ext_sum = nullptr, bool resolved = false) {
    const FactorParams fp = factor_params(ctx, p);
    if (need_sum) {
        SumArgs sa{};
        sa.rrs = rrs;
        sa.scr = ctx->scr;
        sa.segs = make_segments(segs, n_segs, kTile);
        sa.segs.resolved = resolved ? &ctx->segs_dev[0] : nullptr;
        sa.fp = fp;
        cudaError_t e;
        if (sa.segs.total_tiles == 0) {
            e = cudaSuccess;
        } else {
            ProfScope ps(ctx, NRRS_KERNEL_SUM, s);
            e = launch_sum(sa, s);
        }
        if (e != cudaSuccess) return cuda_fail(ctx, e, "sum launch");
    }
    DecideArgs d{};
    d.rrs = rrs;
    d.rnd = rnd;
    d.sidx = sidx;
    d.rrs_norm = rrs_norm;
    // the two-pass decision reads the split counts back: the caller's array, or scratch
    d.split = split ? split : ctx->split_tmp;
    d.split_chunked = split ? 0 : 1;
    d.queue = queue;
    d.next_size = next_size;
    d.n_spec_dev = n_spec_dev;
    d.ext_sum = ext_sum;
    d.scr = ctx->scr;
    d.states = ctx->states;
    d.segs = make_segments(segs, n_segs, kDecChunk);
    d.segs.resolved = resolved ? &ctx->segs_dev[1] : nullptr;
    d.normalize_rate = p->normalize_rate;
    d.use_ceil = p->use_ceil;
    d.scale_up = p->scale_up;
    d.inv_fixed_scale = 1.0 / fp.fixed_scale;
    d.spin_limit = 1u << 22;
    if (d.segs.total_tiles > ctx->max_chunks)
        return fail(ctx, NRRS_ERR_INVALID_ARG, "too many decision chunks for max_queue");
    if (d.segs.total_tiles == 0) {
        cudaError_t e = cudaMemsetAsync(next_size, 0, sizeof(uint32_t) * n_segs, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "memset next_size");
        return NRRS_OK;
    }
    cudaError_t e;
    {
        ProfScope ps(ctx, NRRS_KERNEL_DECIDE, s);
        e = launch_decide_two_pass(d, s);
        ++ctx->prof.total_launches;  // the scope counts one of its two kernels
    }
    if (e != cudaSuccess) {
        cudaMemsetAsync(ctx->scr, 0, offsetof(DecideScratch, epoch), s);
        return cuda_fail(ctx, e, "decide launch");
    }
    return NRRS_OK;
}

// Device-resident queue sizes: the host segments carry the largest counts (they size every
// grid); k_resolve_segments builds the tables of the actual counts in ctx->segs_dev, which the
// kernels of this call read.
int resolve_counts(nrrs_ctx* ctx, const nrrs_segment* segs_max, int n_segs,
                   const uint32_t* counts_dev, cudaStream_t s) {
    const SegmentTable host = make_segments(segs_max, n_segs, kTile);
    const cudaError_t e = launch_resolve_segments(host, counts_dev, &ctx->segs_dev[0],
                                                  &ctx->segs_dev[1], &ctx->scr->status, s);
    return e == cudaSuccess ? NRRS_OK : cuda_fail(ctx, e, "resolve queue sizes");
}

void xavier_fill(std::vector<float>& h, uint64_t ofs, int in, int w, int hidden, int out,
                 uint64_t seed, uint64_t salt) {
    for (int l = 0; l <= hidden; ++l) {
        const int li = l == 0 ? in : w;
        const int lo = l == hidden ? out : w;
        std::mt19937_64 eng(splitmix64(seed ^ splitmix64(salt + (uint64_t)l)));
        const double a = std::sqrt(6.0 / (double)(li + lo));
        for (uint64_t k = 0; k < (uint64_t)li * lo; ++k) {
            const double u = (double)(eng() >> 11) * (1.0 / 9007199254740992.0);
            h[ofs + k] = (float)((2.0 * u - 1.0) * a);
        }
        ofs += (uint64_t)li * lo;
    }
}

}  // namespace

extern "C" {

void nrrs_config_default(nrrs_config* c) {
    std::memset(c, 0, sizeof(*c));
    c->n_levels = 16;
    c->n_features_per_level = 2;
    c->log2_hashmap_size = 19;
    c->base_resolution = 16;
    c->per_level_scale = 1.5f;
    c->sh_degree = 4;
    c->statnet_width = 64;
    c->statnet_hidden = 2;
    c->rrsnet_width = 64;
    c->rrsnet_hidden = 2;
    c->precision = NRRS_PREC_FP32;
    c->seed = 0;
    c->table_init_scale = 1e-4f;
    c->lr = 1e-2f;
    c->beta1 = 0.9f;
    c->beta2 = 0.99f;
    c->eps = 1e-15f;
    c->l2_reg = 0.f;
    c->stat_eps = 0.01f;
    c->ref_eps = 0.01f;
    c->loss_clamp_max = 10.f;
    c->cost_offset = 1.f;
    c->normalize_pos = 0;
    for (int d = 0; d < 3; ++d) { c->aabb_min[d] = 0.f; c->aabb_max[d] = 1.f; }
    c->max_queue = 1u << 20;
    c->max_train = 1u << 18;
    c->step = 3;
}

void nrrs_config_reference_network(nrrs_config* c) {
    if (!c) return;
    // common/configs/nrrs/nrrs/2net-simple.json level0 / level1
    c->network = NRRS_NET_REFERENCE;
    c->n_levels = 8;
    c->n_features_per_level = 2;
    c->log2_hashmap_size = 19;
    c->base_resolution = 16;
    c->per_level_scale = 2.0f;
    c->statnet_width = 32;
    c->statnet_hidden = 3;
    c->rrsnet_width = 32;
    c->rrsnet_hidden = 3;
    c->lr = 5e-3f;
    c->beta1 = 0.9f;
    c->beta2 = 0.99f;
    c->eps = 1e-15f;
    c->l2_reg = 3e-6f;
    c->ema_decay = 0.95f;   // "otype": "Ema", "decay": 0.95
    c->lr_rrsnet = 5e-4f;   // level1 (RRSNet) Adam
}

void nrrs_decide_params_default(nrrs_decide_params* p) {
    // the reference's shipped decision settings (common/configs/nrrs/render/test.json:63-67:
    // clamp_min 0.05, normalize_rate 0.85, use_ceil true, donnot_normalize_when_less_than_one
    // true) with the split cap of the benchmark workload (8 instead of 20)
    p->clamp_min = 0.05f;
    p->clamp_max = 8.0f;
    p->normalize_rate = 0.85f;
    p->use_ceil = 1;
    p->scale_up = 0;
    p->use_weight_window = 0;
    p->weight_window_size = 5.0f;
    p->factor_source = NRRS_FACTOR_RRSNET;
}

const char* nrrs_status_string(int s) {
    switch (s) {
        case NRRS_OK: return "ok";
        case NRRS_ERR_INVALID_ARG: return "invalid argument";
        case NRRS_ERR_CAPACITY_OVERFLOW: return "capacity overflow";
        case NRRS_ERR_NAN: return "non-finite value";
        case NRRS_ERR_TIMEOUT: return "device wait timed out";
        case NRRS_ERR_CUDA: return "CUDA error";
        case NRRS_ERR_NO_DEVICE: return "no sm_100 device";
        case NRRS_ERR_UNSUPPORTED: return "unsupported configuration";
        case NRRS_ERR_IO: return "file I/O error";
        default: return "unknown status";
    }
}

const char* nrrs_last_error(const nrrs_ctx* ctx) {
    return ctx ? ctx->last_error.c_str() : g_create_error.c_str();
}

int nrrs_device_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) { cudaGetLastError(); return 0; }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    return major == 10 ? 1 : 0;
}

int nrrs_create(const nrrs_config* cfg, nrrs_ctx** out) {
    if (!cfg || !out) return fail(nullptr, NRRS_ERR_INVALID_ARG, "NULL argument");
    *out = nullptr;
    const nrrs_config& c = *cfg;
    const bool ref_net = c.network == NRRS_NET_REFERENCE;
    if (c.network != NRRS_NET_WORKLOAD && !ref_net)
        return fail(nullptr, NRRS_ERR_INVALID_ARG, "network must be NRRS_NET_WORKLOAD or NRRS_NET_REFERENCE");
    if (ref_net) {
        // the reference's shipped network: its StatNet input is 16 hash lanes + 16 one-blob lanes
        if (c.n_levels != kRefLevels || c.n_features_per_level != 2)
            return fail(nullptr, NRRS_ERR_UNSUPPORTED, "reference network: 8 levels x 2 features");
        if (c.statnet_width != 32 || c.rrsnet_width != 32 || c.statnet_hidden != 3 ||
            c.rrsnet_hidden != 3)
            return fail(nullptr, NRRS_ERR_UNSUPPORTED, "reference network: 32 wide x 3 hidden");
    } else {
        if (c.n_levels != 16 || c.n_features_per_level != 2)
            return fail(nullptr, NRRS_ERR_UNSUPPORTED, "hash grid needs 16 levels x 2 features (32 lanes)");
        if (c.sh_degree != 4) return fail(nullptr, NRRS_ERR_UNSUPPORTED, "sh_degree must be 4");
    }
    if (c.log2_hashmap_size < 10 || c.log2_hashmap_size > 24 || c.base_resolution < 2 ||
        !(c.per_level_scale >= 1.0f))
        return fail(nullptr, NRRS_ERR_INVALID_ARG, "bad hash-grid parameters");
    const bool w64 = c.statnet_width == 64 && c.rrsnet_width == 64 && c.statnet_hidden == c.rrsnet_hidden &&
                     (c.statnet_hidden == 2 || c.statnet_hidden == 3);
    const bool w128 = c.statnet_width == 128 && c.rrsnet_width == 128 && c.statnet_hidden == 3 &&
                      c.rrsnet_hidden == 3;
    if (!w64 && !w128 && !ref_net)
        return fail(nullptr, NRRS_ERR_UNSUPPORTED, "networks: 64 wide x 2|3 hidden or 128 wide x 3 hidden");
    if (c.precision < NRRS_PREC_FP32 || c.precision > NRRS_PREC_BF16)
        return fail(nullptr, NRRS_ERR_INVALID_ARG, "bad precision");
    if (c.max_queue == 0 || c.max_train == 0)
        return fail(nullptr, NRRS_ERR_INVALID_ARG, "max_queue and max_train must be > 0");
    if (!(c.ema_decay >= 0.f && c.ema_decay < 1.f))
        return fail(nullptr, NRRS_ERR_INVALID_ARG, "ema_decay must be in [0, 1)");
    if (!(c.lr_rrsnet >= 0.f) || !std::isfinite(c.lr_rrsnet))
        return fail(nullptr, NRRS_ERR_INVALID_ARG, "lr_rrsnet must be finite and >= 0");
    if (!nrrs_device_available())
        return fail(nullptr, NRRS_ERR_NO_DEVICE, "no sm_100 CUDA device (this library has no CPU path)");

    nrrs_ctx* ctx = new nrrs_ctx();
    ctx->cfg = c;
    cudaGetDevice(&ctx->device);
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    ctx->table_rows = build_levels(c, ctx->enc);
    aabb_terms(c, ctx->enc);
    ctx->n_table = ctx->table_rows * 2;
    ctx->n_stat = mlp_params(stat_in_of(c.statnet_width), c.statnet_width, c.statnet_hidden,
                             stat_out_of(c.statnet_width));
    ctx->n_rrs = mlp_params(kRrsIn, c.rrsnet_width, c.rrsnet_hidden, 1);
    ctx->n_params = ctx->n_table + ctx->n_stat + ctx->n_rrs;
    ctx->wt_floats = transposed_weight_floats(c.statnet_width, c.statnet_hidden, c.rrsnet_width,
                                              c.rrsnet_hidden);
    ctx->wt_rrs_offset = 0;
    for (int l = 0; l <= c.statnet_hidden; ++l) {
        const int li = l == 0 ? stat_in_of(c.statnet_width) : c.statnet_width;
        const int lo = l == c.statnet_hidden ? stat_out_of(c.statnet_width) : c.statnet_width;
        ctx->wt_rrs_offset += (size_t)li * ((lo + 3) / 4 * 4);
    }
    ctx->wpack_bytes = packed_weight_bytes(c.statnet_width, c.statnet_hidden, c.rrsnet_width,
                                           c.rrsnet_hidden);
    ctx->max_chunks = (c.max_queue + kDecChunk - 1) / kDecChunk + kMaxSegments;

    cudaError_t e;
    const size_t pb = sizeof(float) * ctx->n_params;
#define NRRS_ALLOC(ptr, bytes)                                                         \
    do {                                                                               \
        e = cudaMalloc((void**)&(ptr), (bytes));                                       \
        if (e != cudaSuccess) {                                                        \
            nrrs_destroy(ctx);                                                         \
            return fail(nullptr, NRRS_ERR_CUDA, std::string("cudaMalloc: ") + cudaGetErrorString(e)); \
        }                                                                              \
    } while (0)
    NRRS_ALLOC(ctx->params, pb);
    NRRS_ALLOC(ctx->grads, pb);
    NRRS_ALLOC(ctx->adam_m, pb);
    NRRS_ALLOC(ctx->adam_v, pb);
    NRRS_ALLOC(ctx->wt, sizeof(float) * ctx->wt_floats);
    NRRS_ALLOC(ctx->wrow, sizeof(float) * (ctx->n_stat + ctx->n_rrs));
    if (c.precision != NRRS_PREC_FP32) {
        // 4 spare rows: the paired gathers read whole 16-byte blocks of 4 rows
        NRRS_ALLOC(ctx->table_h, sizeof(__half) * (ctx->n_table + 8));
        NRRS_ALLOC(ctx->wpack, ctx->wpack_bytes);
        // the cell image of the dense levels: 32 bytes per cell
        uint64_t nc = 0;
        for (int l = 0; l < c.n_levels; ++l)
            if (ctx->enc.lv[l].dense)
                nc = (uint64_t)ctx->enc.lv[l].cell +
                     (uint64_t)ctx->enc.lv[l].res * ctx->enc.lv[l].res * ctx->enc.lv[l].res;
        if (nc > 0 && nc < (1ull << 31)) {
            NRRS_ALLOC(ctx->cells, 32 * (size_t)nc);
            ctx->n_cells = (uint32_t)nc;
            ctx->enc.cells = ctx->cells;
        }
    }
    if (c.ema_decay > 0.f) {
        NRRS_ALLOC(ctx->ema, pb);
        NRRS_ALLOC(ctx->params_inf, pb);
        NRRS_ALLOC(ctx->wt_inf, sizeof(float) * ctx->wt_floats);
        if (ctx->table_h) NRRS_ALLOC(ctx->table_h_inf, sizeof(__half) * (ctx->n_table + 8));
        if (ctx->cells) NRRS_ALLOC(ctx->cells_inf, 32 * (size_t)ctx->n_cells);
    }
    if (train_tc_supported(c))
        NRRS_ALLOC(ctx->tpack, train_pack_bytes(c.statnet_width, c.statnet_hidden,
                                                c.rrsnet_width, c.rrsnet_hidden));
    const size_t scr_bytes = sizeof(DecideScratch) + sizeof(unsigned long long) * ctx->max_chunks;
    NRRS_ALLOC(ctx->scr, scr_bytes);
    ctx->states = reinterpret_cast<unsigned long long*>(ctx->scr + 1);
    NRRS_ALLOC(ctx->split_tmp, (size_t)ctx->max_chunks * kDecChunk);
    NRRS_ALLOC(ctx->loss_dev, sizeof(double) * 2);
    NRRS_ALLOC(ctx->segs_dev, sizeof(SegmentTable) * 2);
    NRRS_ALLOC(ctx->loss_sums, sizeof(double) * 4);
    ctx->train_scratch_bytes = train_scratch_bytes(c, c.max_train, ctx->sm_count);
    NRRS_ALLOC(ctx->train_scratch, ctx->train_scratch_bytes);
#undef NRRS_ALLOC

    // parameters: table ~ U(-s, s), MLPs Xavier-uniform (seeded, host side)
    std::vector<float> h(ctx->n_params);
    {
        std::mt19937_64 eng(splitmix64(c.seed ^ 0x7461626c65ull));
        for (uint64_t k = 0; k < ctx->n_table; ++k) {
            const double u = (double)(eng() >> 11) * (1.0 / 9007199254740992.0);
            h[k] = (float)((2.0 * u - 1.0) * c.table_init_scale);
        }
    }
    xavier_fill(h, ctx->n_table, stat_in_of(c.statnet_width), c.statnet_width, c.statnet_hidden,
                stat_out_of(c.statnet_width), c.seed, 100);
    xavier_fill(h, ctx->n_table + ctx->n_stat, kRrsIn, c.rrsnet_width, c.rrsnet_hidden, 1, c.seed, 200);
    e = cudaMemcpy(ctx->params, h.data(), pb, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(ctx->grads, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(ctx->adam_m, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(ctx->adam_v, 0, pb);
    if (e == cudaSuccess) e = cudaMemset(ctx->scr, 0, scr_bytes);
    if (e == cudaSuccess) {
        const unsigned one = 1;
        e = cudaMemcpy(&ctx->scr->epoch, &one, sizeof(one), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemset(ctx->loss_dev, 0, sizeof(double) * 2);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        nrrs_destroy(ctx);
        return fail(nullptr, NRRS_ERR_CUDA, std::string("init: ") + cudaGetErrorString(e));
    }
    int rc = ema_restart(ctx, 0);
    if (rc == NRRS_OK) rc = refresh_derived(ctx, 0);
    if (rc == NRRS_OK) {
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "init sync");
    }
    if (rc != NRRS_OK) {
        g_create_error = ctx->last_error;
        nrrs_destroy(ctx);
        return rc;
    }
    *out = ctx;
    return NRRS_OK;
}

void nrrs_destroy(nrrs_ctx* ctx) {
    if (!ctx) return;
    for (cudaEvent_t ev : ctx->prof.pool) cudaEventDestroy(ev);
    if (ctx->side) {
        cudaStreamSynchronize(ctx->side);
        cudaStreamDestroy(ctx->side);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
    cudaFree(ctx->params);
    cudaFree(ctx->grads);
    cudaFree(ctx->adam_m);
    cudaFree(ctx->adam_v);
    cudaFree(ctx->table_h);
    cudaFree(ctx->cells);
    cudaFree(ctx->ema);
    cudaFree(ctx->params_inf);
    cudaFree(ctx->wt_inf);
    cudaFree(ctx->table_h_inf);
    cudaFree(ctx->cells_inf);
    cudaFree(ctx->wt);
    cudaFree(ctx->wrow);
    cudaFree(ctx->wpack);
    cudaFree(ctx->tpack);
    cudaFree(ctx->enc_tiles);
    cudaFree(ctx->x1_tiles);
    cudaFree(ctx->scr);
    cudaFree(ctx->split_tmp);
    cudaFree(ctx->loss_dev);
    cudaFree(ctx->segs_dev);
    cudaFree(ctx->loss_sums);
    cudaFree(ctx->train_scratch);
    delete ctx;
}

int nrrs_set_step(nrrs_ctx* ctx, int32_t step) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    if (step < 0 || step > 3) return fail(ctx, NRRS_ERR_INVALID_ARG, "step must be 0..3");
    ctx->cfg.step = step;
    return NRRS_OK;
}

int nrrs_infer(nrrs_ctx* ctx, const nrrs_vertex_soa* v, uint32_t n, const nrrs_decide_params* p,
               float* stats, float* rrs, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    if ((rc = check_decide_params(ctx, p, n))) return rc;
    if (!rrs) return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs output is NULL");
    if (n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "n > max_queue");
    if (n == 0) return NRRS_OK;
    nrrs_segment sg{0, n, 0, 0, 0, 0};
    return run_infer(ctx, v, make_segments(&sg, 1, kTile), p, n, stats, rrs, false,
                     (cudaStream_t)stream);
}

int nrrs_decide_emit(nrrs_ctx* ctx, const float* rrs, const float* rnd,
                     const uint32_t* scatter_index, uint32_t n, uint32_t budget,
                     uint32_t n_specular, const uint32_t* n_specular_dev,
                     const nrrs_decide_params* p, float* rrs_norm, uint8_t* split,
                     uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev,
                     void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_decide_params(ctx, p, n);
    if (rc) return rc;
    if (n && (!rrs || !rnd)) return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs/rnd are NULL");
    if (!next_size_dev || (capacity && !next_queue))
        return fail(ctx, NRRS_ERR_INVALID_ARG, "next_queue/next_size are NULL");
    if (n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "n > max_queue");
    nrrs_segment sg{0, n, budget, n_specular, 0, capacity};
    return run_decide(ctx, rrs, rnd, scatter_index, &sg, 1, n, n_specular_dev, p, rrs_norm, split,
                      next_queue, next_size_dev, true, (cudaStream_t)stream);
}

int nrrs_step(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd, uint32_t n,
              uint32_t budget, uint32_t n_specular, const nrrs_decide_params* p, float* stats,
              float* rrs, float* rrs_norm, uint8_t* split, uint32_t* next_queue,
              uint32_t capacity, uint32_t* next_size_dev, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    if ((rc = check_decide_params(ctx, p, n))) return rc;
    if (!rrs || (n && !rnd) || !next_size_dev || (capacity && !next_queue))
        return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs/rnd/next_queue/next_size NULL");
    if (n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "n > max_queue");
    cudaStream_t s = (cudaStream_t)stream;
    nrrs_segment sg{0, n, budget, n_specular, 0, capacity};
    if (n) {
        rc = run_infer(ctx, v, make_segments(&sg, 1, kTile), p, n, stats, rrs, true, s);
        if (rc) return rc;
    }
    return run_decide(ctx, rrs, rnd, v->scatter_index, &sg, 1, n, nullptr, p, rrs_norm, split,
                      next_queue, next_size_dev, false, s);
}

int nrrs_step_batched(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                      const nrrs_segment* segs, int32_t n_segs, const nrrs_decide_params* p,
                      float* stats, float* rrs, float* rrs_norm, uint8_t* split,
                      uint32_t* next_queue, uint32_t* next_size_dev, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    if (!segs || n_segs < 1 || n_segs > kMaxSegments)
        return fail(ctx, NRRS_ERR_INVALID_ARG, "1..16 segments required");
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    uint64_t n_total = 0, n_max = 0;
    for (int k = 0; k < n_segs; ++k) {
        n_total += segs[k].count;
        n_max = segs[k].count > n_max ? segs[k].count : n_max;
        if (segs[k].queue_capacity && !next_queue)
            return fail(ctx, NRRS_ERR_INVALID_ARG, "next_queue is NULL");
    }
    if ((rc = check_decide_params(ctx, p, n_max))) return rc;
    if (n_total > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "sum of counts > max_queue");
    if (!rrs || !rnd || !next_size_dev) return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs/rnd/next_size NULL");
    cudaStream_t s = (cudaStream_t)stream;
    // the exact-sum scale is shared by all segments: use the largest segment
    rc = run_infer(ctx, v, make_segments(segs, n_segs, kTile), p, n_max, stats, rrs, true, s);
    if (rc) return rc;
    return run_decide(ctx, rrs, rnd, v->scatter_index, segs, n_segs, n_max, nullptr, p, rrs_norm,
                      split, next_queue, next_size_dev, false, s);
}

int nrrs_infer_dev(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const uint32_t* n_dev,
                   uint32_t max_n, const nrrs_decide_params* p, float* stats, float* rrs,
                   void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    if ((rc = check_decide_params(ctx, p, max_n))) return rc;
    if (!rrs || !n_dev) return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs/n_dev are NULL");
    if (max_n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "max_n > max_queue");
    if (max_n == 0) return NRRS_OK;
    cudaStream_t s = (cudaStream_t)stream;
    nrrs_segment sg{0, max_n, 0, 0, 0, 0};
    if ((rc = resolve_counts(ctx, &sg, 1, n_dev, s))) return rc;
    return run_infer(ctx, v, make_segments(&sg, 1, kTile), p, max_n, stats, rrs, false, s,
                     nullptr, &ctx->segs_dev[0]);
}

int nrrs_decide_emit_dev(nrrs_ctx* ctx, const float* rrs, const float* rnd,
                         const uint32_t* scatter_index, const uint32_t* n_dev, uint32_t max_n,
                         uint32_t budget, uint32_t n_specular, const uint32_t* n_specular_dev,
                         const nrrs_decide_params* p, float* rrs_norm, uint8_t* split,
                         uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev,
                         void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_decide_params(ctx, p, max_n);
    if (rc) return rc;
    if (!n_dev || (max_n && (!rrs || !rnd))) return fail(ctx, NRRS_ERR_INVALID_ARG, "n_dev/rrs/rnd are NULL");
    if (!next_size_dev || (capacity && !next_queue))
        return fail(ctx, NRRS_ERR_INVALID_ARG, "next_queue/next_size are NULL");
    if (max_n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "max_n > max_queue");
    cudaStream_t s = (cudaStream_t)stream;
    nrrs_segment sg{0, max_n, budget, n_specular, 0, capacity};
    if (max_n && (rc = resolve_counts(ctx, &sg, 1, n_dev, s))) return rc;
    return run_decide(ctx, rrs, rnd, scatter_index, &sg, 1, max_n, n_specular_dev, p, rrs_norm,
                      split, next_queue, next_size_dev, true, s, nullptr, true);
}

int nrrs_step_dev(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                  const uint32_t* n_dev, uint32_t max_n, uint32_t budget, uint32_t n_specular,
                  const uint32_t* n_specular_dev, const nrrs_decide_params* p, float* stats,
                  float* rrs, float* rrs_norm, uint8_t* split, uint32_t* next_queue,
                  uint32_t capacity, uint32_t* next_size_dev, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    if ((rc = check_decide_params(ctx, p, max_n))) return rc;
    if (!n_dev || !rrs || (max_n && !rnd) || !next_size_dev || (capacity && !next_queue))
        return fail(ctx, NRRS_ERR_INVALID_ARG, "n_dev/rrs/rnd/next_queue/next_size NULL");
    if (max_n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "max_n > max_queue");
    cudaStream_t s = (cudaStream_t)stream;
    nrrs_segment sg{0, max_n, budget, n_specular, 0, capacity};
    if (max_n) {
        if ((rc = resolve_counts(ctx, &sg, 1, n_dev, s))) return rc;
        rc = run_infer(ctx, v, make_segments(&sg, 1, kTile), p, max_n, stats, rrs, true, s,
                       nullptr, &ctx->segs_dev[0]);
        if (rc) return rc;
    }
    return run_decide(ctx, rrs, rnd, v->scatter_index, &sg, 1, max_n, n_specular_dev, p,
                      rrs_norm, split, next_queue, next_size_dev, false, s, nullptr, max_n != 0);
}

int nrrs_step_batched_dev(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                          const nrrs_segment* segs, const uint32_t* counts_dev, int32_t n_segs,
                          const nrrs_decide_params* p, float* stats, float* rrs, float* rrs_norm,
                          uint8_t* split, uint32_t* next_queue, uint32_t* next_size_dev,
                          void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    if (!segs || !counts_dev || n_segs < 1 || n_segs > kMaxSegments)
        return fail(ctx, NRRS_ERR_INVALID_ARG, "1..16 segments and their device counts required");
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    uint64_t n_total = 0, n_max = 0;
    for (int k = 0; k < n_segs; ++k) {
        n_total += segs[k].count;
        n_max = segs[k].count > n_max ? segs[k].count : n_max;
        if (segs[k].queue_capacity && !next_queue)
            return fail(ctx, NRRS_ERR_INVALID_ARG, "next_queue is NULL");
    }
    if ((rc = check_decide_params(ctx, p, n_max))) return rc;
    if (n_total > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "sum of counts > max_queue");
    if (!rrs || !rnd || !next_size_dev) return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs/rnd/next_size NULL");
    cudaStream_t s = (cudaStream_t)stream;
    if ((rc = resolve_counts(ctx, segs, n_segs, counts_dev, s))) return rc;
    rc = run_infer(ctx, v, make_segments(segs, n_segs, kTile), p, n_max, stats, rrs, true, s,
                   nullptr, &ctx->segs_dev[0]);
    if (rc) return rc;
    return run_decide(ctx, rrs, rnd, v->scatter_index, segs, n_segs, n_max, nullptr, p, rrs_norm,
                      split, next_queue, next_size_dev, false, s, nullptr, true);
}

int nrrs_infer_accumulate(nrrs_ctx* ctx, const nrrs_vertex_soa* v, uint32_t n,
                          const nrrs_decide_params* p, float* stats, float* rrs,
                          int64_t* sum_acc_dev, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    if ((rc = check_decide_params(ctx, p, n))) return rc;
    if (!rrs || !sum_acc_dev) return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs/sum_acc are NULL");
    if (n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "n > max_queue");
    if (n == 0) return NRRS_OK;
    nrrs_segment sg{0, n, 0, 0, 0, 0};
    return run_infer(ctx, v, make_segments(&sg, 1, kTile), p, n, stats, rrs, false,
                     (cudaStream_t)stream, reinterpret_cast<unsigned long long*>(sum_acc_dev));
}

int nrrs_decide_emit_with_sum(nrrs_ctx* ctx, const float* rrs, const float* rnd,
                              const uint32_t* scatter_index, uint32_t n, uint32_t budget,
                              uint32_t n_specular, const int64_t* sum_acc_dev,
                              const nrrs_decide_params* p, float* rrs_norm, uint8_t* split,
                              uint32_t* next_queue, uint32_t capacity, uint32_t* next_size_dev,
                              void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_decide_params(ctx, p, n);
    if (rc) return rc;
    if (!sum_acc_dev) return fail(ctx, NRRS_ERR_INVALID_ARG, "sum_acc is NULL");
    if (n && (!rrs || !rnd)) return fail(ctx, NRRS_ERR_INVALID_ARG, "rrs/rnd are NULL");
    if (!next_size_dev || (capacity && !next_queue))
        return fail(ctx, NRRS_ERR_INVALID_ARG, "next_queue/next_size are NULL");
    if (n > ctx->cfg.max_queue) return fail(ctx, NRRS_ERR_INVALID_ARG, "n > max_queue");
    nrrs_segment sg{0, n, budget, n_specular, 0, capacity};
    return run_decide(ctx, rrs, rnd, scatter_index, &sg, 1, n, nullptr, p, rrs_norm, split,
                      next_queue, next_size_dev, false, (cudaStream_t)stream,
                      reinterpret_cast<const long long*>(sum_acc_dev));
}

double nrrs_sum_from_accumulator(const nrrs_ctx* ctx, const nrrs_decide_params* p, int64_t acc) {
    if (!ctx || !p) return 0.0;
    return (double)acc / factor_params(ctx, p).fixed_scale;
}

int nrrs_train_grads(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* target, uint32_t n,
                     double* loss_dev, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    if (!target) return fail(ctx, NRRS_ERR_INVALID_ARG, "target is NULL");
    if (n == 0 || n > ctx->cfg.max_train) return fail(ctx, NRRS_ERR_INVALID_ARG, "need 0 < n <= max_train");
    return train_step_impl(ctx, vptrs(v), target, n, loss_dev, (cudaStream_t)stream, false);
}

int nrrs_copy_grads(nrrs_ctx* ctx, float* grads_dev, void* stream) {
    if (!ctx || !grads_dev) return NRRS_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpyAsync(grads_dev, ctx->grads, sizeof(float) * ctx->n_params,
                                    cudaMemcpyDeviceToDevice, (cudaStream_t)stream);
    return e == cudaSuccess ? NRRS_OK : cuda_fail(ctx, e, "copy grads");
}

int nrrs_adam_apply(nrrs_ctx* ctx, const float* grads_dev, float scale, void* stream) {
    if (!ctx || !grads_dev || !std::isfinite(scale)) return NRRS_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (grads_dev != ctx->grads) {
        cudaError_t e = cudaMemcpyAsync(ctx->grads, grads_dev, sizeof(float) * ctx->n_params,
                                        cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "copy grads in");
    }
    cudaError_t e = launch_adam_step(ctx, ctx->cfg.step >= 3, s, scale);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "adam launch");
    return refresh_derived(ctx, s, false);
}

void nrrs_loss_params_default(nrrs_loss_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma1 = 1.0f;          // u = 1: the plain variance term
    p->clamp_on = 0;
    p->clamp_max = 10.0f;      // the reference's clamp_max (2net-simple.json)
    p->n_pixels = 0;
}

int nrrs_train_step_batch(nrrs_ctx* ctx, const nrrs_train_batch* b, uint32_t n,
                          const float* sample_weight, const float* error_sum_dev,
                          const nrrs_loss_params* lp, double* loss_dev, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    if (!b || !lp) return fail(ctx, NRRS_ERR_INVALID_ARG, "batch/loss params are NULL");
    if (!b->pos || !b->wi || !b->normal || !b->roughness || !b->albedo || !b->thp || !b->target)
        return fail(ctx, NRRS_ERR_INVALID_ARG,
                    "batch: pos/wi/normal/roughness/albedo/thp/target required");
    if (n == 0 || n > ctx->cfg.max_train) return fail(ctx, NRRS_ERR_INVALID_ARG, "need 0 < n <= max_train");
    if (!std::isfinite(lp->gamma1) || !std::isfinite(lp->gamma2) || !std::isfinite(lp->gamma3) ||
        !std::isfinite(lp->gamma4) || (lp->clamp_on && !(lp->clamp_max > 0.f)))
        return fail(ctx, NRRS_ERR_INVALID_ARG, "loss params: finite gammas, clamp_max > 0");
    if (error_sum_dev && lp->n_pixels == 0)
        return fail(ctx, NRRS_ERR_INVALID_ARG, "an error sum needs n_pixels");
    VertexPtrs v{};
    v.pos = b->pos; v.wi = b->wi; v.normal = b->normal; v.rough = b->roughness;
    v.albedo = b->albedo; v.thp = b->thp; v.depth = b->depth; v.ref = b->ref_mean;
    LossWeights lw{};
    lw.active = 1;
    lw.sample_weight = sample_weight;
    lw.rrs_target = b->rrs_target;
    lw.error = b->error;
    lw.error_for_avg = b->error_for_avg;
    lw.number_samples = b->number_samples;
    lw.g1 = lp->gamma1; lw.g2 = lp->gamma2; lw.g3 = lp->gamma3; lw.g4 = lp->gamma4;
    lw.clamp_on = lp->clamp_on;
    lw.clamp_max = lp->clamp_max;
    lw.sums = ctx->loss_sums;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = launch_loss_sums(lw, n, error_sum_dev, lp->n_pixels, ctx->loss_sums, s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "loss weight sums");
    const int rc = train_step_impl(ctx, v, b->target, n, loss_dev, s, true, &lw);
    if (rc) return rc;
    // the Adam pass refreshed the FP16 table and its cell image; the MLP images follow
    return refresh_derived(ctx, s, false);
}

int nrrs_train_step(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* target, uint32_t n,
                    double* loss_dev, void* stream) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    int rc = check_vertices(ctx, v);
    if (rc) return rc;
    if (!target) return fail(ctx, NRRS_ERR_INVALID_ARG, "target is NULL");
    if (n == 0 || n > ctx->cfg.max_train) return fail(ctx, NRRS_ERR_INVALID_ARG, "need 0 < n <= max_train");
    rc = train_step_impl(ctx, vptrs(v), target, n, loss_dev, (cudaStream_t)stream);
    if (rc) return rc;
    // the Adam pass already refreshed the FP16 table
    return refresh_derived(ctx, (cudaStream_t)stream, false);
}

uint64_t nrrs_param_count(const nrrs_ctx* ctx) { return ctx ? ctx->n_params : 0; }

int nrrs_param_layout(const nrrs_ctx* ctx, uint64_t* t, uint64_t* s, uint64_t* r) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    if (t) *t = ctx->n_table;
    if (s) *s = ctx->n_stat;
    if (r) *r = ctx->n_rrs;
    return NRRS_OK;
}

int nrrs_get_params(const nrrs_ctx* ctx, float* dst, uint64_t count) {
    if (!ctx || !dst || count != ctx->n_params) return NRRS_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpy(dst, ctx->params, sizeof(float) * count, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

int nrrs_get_inference_params(const nrrs_ctx* ctx, float* dst, uint64_t count) {
    if (!ctx || !dst || count != ctx->n_params) return NRRS_ERR_INVALID_ARG;
    const float* src = ctx->ema ? ctx->params_inf : ctx->params;
    cudaError_t e = cudaMemcpy(dst, src, sizeof(float) * count, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

int nrrs_set_params(nrrs_ctx* ctx, const float* src, uint64_t count) {
    if (!ctx || !src || count != ctx->n_params) return ctx ? fail(ctx, NRRS_ERR_INVALID_ARG, "count mismatch") : NRRS_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpy(ctx->params, src, sizeof(float) * count, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "set params");
    int rc = ema_restart(ctx, 0);
    if (rc) return rc;
    rc = refresh_derived(ctx, 0);
    if (rc) return rc;
    e = cudaDeviceSynchronize();
    return e == cudaSuccess ? NRRS_OK : cuda_fail(ctx, e, "set params sync");
}

int nrrs_get_grads(const nrrs_ctx* ctx, float* dst, uint64_t count) {
    if (!ctx || !dst || count != ctx->n_params) return NRRS_ERR_INVALID_ARG;
    cudaError_t e = cudaMemcpy(dst, ctx->grads, sizeof(float) * count, cudaMemcpyDeviceToHost);
    return e == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

int nrrs_get_adam_state(const nrrs_ctx* ctx, float* m, float* v, uint64_t count, uint64_t* t) {
    if (!ctx || count != ctx->n_params) return NRRS_ERR_INVALID_ARG;
    cudaError_t e = cudaSuccess;
    if (m) e = cudaMemcpy(m, ctx->adam_m, sizeof(float) * count, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && v) e = cudaMemcpy(v, ctx->adam_v, sizeof(float) * count, cudaMemcpyDeviceToHost);
    if (t) *t = ctx->adam_t;
    return e == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

int nrrs_level_table(const nrrs_ctx* ctx, uint32_t* dst, int32_t max_levels) {
    if (!ctx || !dst || max_levels < ctx->cfg.n_levels) return NRRS_ERR_INVALID_ARG;
    for (int l = 0; l < ctx->cfg.n_levels; ++l) {
        const LevelDev& L = ctx->enc.lv[l];
        const uint64_t R = (uint64_t)L.res + 1;
        dst[4 * l + 0] = L.offset;
        dst[4 * l + 1] = (uint32_t)(L.dense ? R * R * R : (uint64_t)ctx->enc.hash_mask + 1);
        dst[4 * l + 2] = L.res;
        dst[4 * l + 3] = L.dense;
    }
    return NRRS_OK;
}

// checkpoint file: magic, version, config, adam step, params, m, v (all FP32)
int nrrs_save(const nrrs_ctx* ctx, const char* path) {
    if (!ctx || !path) return NRRS_ERR_INVALID_ARG;
    std::vector<float> p(ctx->n_params), m(ctx->n_params), v(ctx->n_params);
    if (nrrs_get_params(ctx, p.data(), ctx->n_params) ||
        nrrs_get_adam_state(ctx, m.data(), v.data(), ctx->n_params, nullptr))
        return NRRS_ERR_CUDA;
    FILE* f = std::fopen(path, "wb");
    if (!f) return NRRS_ERR_IO;
    const uint32_t hdr[2] = {0x5352524eu /* "NRRS" */, NRRS_ABI_VERSION};
    bool ok = std::fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
              std::fwrite(&ctx->cfg, sizeof(nrrs_config), 1, f) == 1 &&
              std::fwrite(&ctx->adam_t, sizeof(uint64_t), 1, f) == 1 &&
              std::fwrite(p.data(), sizeof(float), p.size(), f) == p.size() &&
              std::fwrite(m.data(), sizeof(float), m.size(), f) == m.size() &&
              std::fwrite(v.data(), sizeof(float), v.size(), f) == v.size();
    ok = (std::fclose(f) == 0) && ok;
    return ok ? NRRS_OK : NRRS_ERR_IO;
}

int nrrs_load(nrrs_ctx* ctx, const char* path) {
    if (!ctx || !path) return NRRS_ERR_INVALID_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return fail(ctx, NRRS_ERR_IO, "cannot open checkpoint");
    uint32_t hdr[2];
    nrrs_config c;
    uint64_t t = 0;
    std::vector<float> p(ctx->n_params), m(ctx->n_params), v(ctx->n_params);
    bool ok = std::fread(hdr, sizeof(hdr), 1, f) == 1 && hdr[0] == 0x5352524eu &&
              hdr[1] == NRRS_ABI_VERSION && std::fread(&c, sizeof(c), 1, f) == 1 &&
              std::fread(&t, sizeof(t), 1, f) == 1;
    ok = ok && c.n_levels == ctx->cfg.n_levels && c.log2_hashmap_size == ctx->cfg.log2_hashmap_size &&
         c.base_resolution == ctx->cfg.base_resolution && c.per_level_scale == ctx->cfg.per_level_scale &&
         c.statnet_width == ctx->cfg.statnet_width && c.statnet_hidden == ctx->cfg.statnet_hidden &&
         c.rrsnet_width == ctx->cfg.rrsnet_width && c.rrsnet_hidden == ctx->cfg.rrsnet_hidden;
    ok = ok && std::fread(p.data(), sizeof(float), p.size(), f) == p.size() &&
         std::fread(m.data(), sizeof(float), m.size(), f) == m.size() &&
         std::fread(v.data(), sizeof(float), v.size(), f) == v.size();
    std::fclose(f);
    if (!ok) return fail(ctx, NRRS_ERR_IO, "checkpoint does not match this configuration");
    const size_t b = sizeof(float) * ctx->n_params;
    cudaError_t e = cudaMemcpy(ctx->adam_m, m.data(), b, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(ctx->adam_v, v.data(), b, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "load moments");
    ctx->adam_t = t;
    return nrrs_set_params(ctx, p.data(), ctx->n_params);
}

int nrrs_get_device_status(nrrs_ctx* ctx, uint32_t* flags, void* stream) {
    if (!ctx || !flags) return NRRS_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned h = 0;
    cudaError_t e = cudaMemcpyAsync(&h, &ctx->scr->status, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(&ctx->scr->status, 0, sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "device status");
    *flags = h;
    if (h & NRRS_DEV_TIMEOUT) return NRRS_ERR_TIMEOUT;
    if (h & NRRS_DEV_OVERFLOW) return NRRS_ERR_CAPACITY_OVERFLOW;
    if (h & NRRS_DEV_NAN) return NRRS_ERR_NAN;
    return NRRS_OK;
}

uint64_t nrrs_launch_count(const nrrs_ctx* ctx) { return ctx ? ctx->prof.total_launches : 0; }

int32_t nrrs_last_infer_grid(const nrrs_ctx* ctx) { return ctx ? ctx->last_infer_grid : 0; }

const char* nrrs_kernel_name(int32_t kind) {
    static const char* names[NRRS_KERNEL_KINDS] = {
        "infer_fp32", "infer_tc", "sum", "decide", "pack_weights", "table_half",
        "train_statnet", "train_rrsnet", "train_wgrad", "train_reduce", "adam", "encode",
        "train_scatter", "train_encode", "infer_rrs", "cell_image"};
    return (kind >= 0 && kind < NRRS_KERNEL_KINDS) ? names[kind] : "unknown";
}

int nrrs_profile_enable(nrrs_ctx* ctx, int32_t enable) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    Profiler& p = ctx->prof;
    if (enable && p.pool.empty()) {
        p.pool.resize(16384);
        for (auto& ev : p.pool) {
            cudaError_t e = cudaEventCreate(&ev);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "event create");
        }
    }
    p.enabled = enable != 0;
    return NRRS_OK;
}

int nrrs_profile_read(nrrs_ctx* ctx, int32_t kind, uint64_t* launches, double* total_ms) {
    if (!ctx || kind < 0 || kind >= NRRS_KERNEL_KINDS) return NRRS_ERR_INVALID_ARG;
    Profiler& p = ctx->prof;
    // fold every pending pair of every kind, then recycle the pool
    for (int k = 0; k < NRRS_KERNEL_KINDS; ++k) {
        for (auto& pr : p.pending[k]) {
            cudaError_t e = cudaEventSynchronize(p.pool[pr.second]);
            if (e != cudaSuccess) return cuda_fail(ctx, e, "event sync");
            float ms = 0.f;
            cudaEventElapsedTime(&ms, p.pool[pr.first], p.pool[pr.second]);
            p.timed_ms[k] += ms;
            ++p.timed_launches[k];
        }
        p.pending[k].clear();
    }
    p.next = 0;
    if (launches) *launches = p.timed_launches[kind];
    if (total_ms) *total_ms = p.timed_ms[kind];
    p.timed_launches[kind] = 0;
    p.timed_ms[kind] = 0.0;
    return NRRS_OK;
}

int nrrs_set_launch_shape(nrrs_ctx* ctx, int32_t ctas_per_sm, int32_t warpgroups) {
    if (!ctx || ctas_per_sm < 0 || ctas_per_sm > 32) return NRRS_ERR_INVALID_ARG;
    const nrrs_config& c = ctx->cfg;
    if (c.precision == NRRS_PREC_FP32) {
        if (warpgroups != 1) return fail(ctx, NRRS_ERR_INVALID_ARG, "the FP32 path has one warpgroup per CTA");
        ctx->simt_ctas_per_sm = ctas_per_sm;
        return NRRS_OK;
    }
    if (warpgroups != 1 && warpgroups != 2 && warpgroups != 4)
        return fail(ctx, NRRS_ERR_INVALID_ARG, "warpgroups must be 1, 2 or 4");
    if (infer_max_ctas(c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden,
                       c.precision, warpgroups, ctx->tc_split) <= 0)
        return fail(ctx, NRRS_ERR_UNSUPPORTED, "launch shape not available for this network");
    ctx->tc_ctas_per_sm = ctas_per_sm;
    ctx->tc_wgs = warpgroups;
    return NRRS_OK;
}

int nrrs_set_infer_split(nrrs_ctx* ctx, int32_t split) {
    if (!ctx || split < 0 || split > 3) return NRRS_ERR_INVALID_ARG;
    const nrrs_config& c = ctx->cfg;
    if (split && c.precision == NRRS_PREC_FP32)
        return fail(ctx, NRRS_ERR_UNSUPPORTED, "split inference is a tensor-core path mode");
    if (split && infer_max_ctas(c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden,
                                c.precision, 1, split) <= 0 &&
        infer_max_ctas(c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden,
                       c.precision, 2, split) <= 0)
        return fail(ctx, NRRS_ERR_UNSUPPORTED, "split inference not available for this network");
    if (split >= 2 && !ctx->x1_tiles) {
        const uint32_t cap = c.max_queue / kTile + kMaxSegments + 1;
        if (cudaMalloc(&ctx->x1_tiles, (size_t)cap * kX1TileBytes) != cudaSuccess) {
            ctx->x1_tiles = nullptr;
            return fail(ctx, NRRS_ERR_CUDA, "split inference: RRSNet input tile allocation");
        }
    }
    if (split && !ctx->enc_tiles) {
        const uint32_t cap = c.max_queue / kTile + kMaxSegments + 1;
        if (cudaMalloc(&ctx->enc_tiles, (size_t)cap * kEncTileBytes) != cudaSuccess) {
            ctx->enc_tiles = nullptr;
            return fail(ctx, NRRS_ERR_CUDA, "split inference: feature tile allocation");
        }
        ctx->enc_tiles_cap = cap;
    }
    ctx->tc_split = split;
    // the warpgroup count must exist in the new mode
    if (infer_max_ctas(c.statnet_width, c.statnet_hidden, c.rrsnet_width, c.rrsnet_hidden,
                       c.precision, ctx->tc_wgs, split) <= 0)
        ctx->tc_wgs = infer_max_ctas(c.statnet_width, c.statnet_hidden, c.rrsnet_width,
                                     c.rrsnet_hidden, c.precision, 1, split) > 0 ? 1 : 2;
    return NRRS_OK;
}

int nrrs_set_train_split(nrrs_ctx* ctx, int32_t split) {
    if (!ctx || (split != 0 && split != 1)) return NRRS_ERR_INVALID_ARG;
    ctx->train_split = split;
    return NRRS_OK;
}

int nrrs_get_train_split(const nrrs_ctx* ctx, int32_t* split) {
    if (!ctx || !split) return NRRS_ERR_INVALID_ARG;
    *split = ctx->train_split;
    return NRRS_OK;
}

int nrrs_get_infer_split(const nrrs_ctx* ctx, int32_t* split) {
    if (!ctx || !split) return NRRS_ERR_INVALID_ARG;
    *split = ctx->tc_split;
    return NRRS_OK;
}

int nrrs_set_cell_image(nrrs_ctx* ctx, int32_t enable) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    if (enable && !ctx->cells)
        return fail(ctx, NRRS_ERR_UNSUPPORTED, "no cell image (FP32 context or no dense level)");
    ctx->enc.cells = enable ? ctx->cells : nullptr;
    return NRRS_OK;
}

int nrrs_get_cell_image(const nrrs_ctx* ctx, int32_t* enable) {
    if (!ctx || !enable) return NRRS_ERR_INVALID_ARG;
    *enable = ctx->enc.cells != nullptr;
    return NRRS_OK;
}

int nrrs_get_launch_shape(const nrrs_ctx* ctx, int32_t* ctas_per_sm, int32_t* warpgroups) {
    if (!ctx) return NRRS_ERR_INVALID_ARG;
    const bool fp32 = ctx->cfg.precision == NRRS_PREC_FP32;
    if (ctas_per_sm) *ctas_per_sm = fp32 ? ctx->simt_ctas_per_sm : ctx->tc_ctas_per_sm;
    if (warpgroups) *warpgroups = fp32 ? 1 : ctx->tc_wgs;
    return NRRS_OK;
}

namespace {

std::string tune_key(const nrrs_ctx* ctx) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, ctx->device);
    const nrrs_config& c = ctx->cfg;
    std::ostringstream k;
    k << prop.name << "|sm" << ctx->sm_count << "|w" << c.statnet_width << "h" << c.statnet_hidden
      << "|p" << c.precision << "|T" << c.log2_hashmap_size;
    return k.str();
}

// the cache is a JSON object of lines  "key": [ctas_per_sm, warpgroups, split],  (a missing
// split reads as 0, the fused mode)
bool cache_lookup(const char* path, const std::string& key, int* ctas, int* wgs, int* split) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    const std::string needle = "\"" + key + "\"";
    while (std::getline(f, line)) {
        const size_t pos = line.find(needle);
        if (pos == std::string::npos) continue;
        const size_t lb = line.find('[', pos);
        if (lb == std::string::npos) continue;
        *split = 0;
        if (std::sscanf(line.c_str() + lb, "[%d, %d, %d]", ctas, wgs, split) >= 2) return true;
    }
    return false;
}

void cache_store(const char* path, const std::string& key, int ctas, int wgs, int split) {
    std::vector<std::string> keep;
    {
        std::ifstream f(path);
        std::string line;
        const std::string needle = "\"" + key + "\"";
        while (std::getline(f, line))
            if (line.find("\": [") != std::string::npos && line.find(needle) == std::string::npos) {
                while (!line.empty() && (line.back() == ',' || line.back() == ' ')) line.pop_back();
                keep.push_back(line);
            }
    }
    char buf[512];
    std::snprintf(buf, sizeof(buf), "  \"%s\": [%d, %d, %d]", key.c_str(), ctas, wgs, split);
    keep.push_back(buf);
    std::ofstream o(path, std::ios::trunc);
    o << "{\n";
    for (size_t i = 0; i < keep.size(); ++i) o << keep[i] << (i + 1 < keep.size() ? ",\n" : "\n");
    o << "}\n";
}

}  // namespace

int nrrs_autotune(nrrs_ctx* ctx, uint32_t n, const char* cache_path, char* report,
                  size_t report_len) {
    if (!ctx || n == 0 || n > ctx->cfg.max_queue) return NRRS_ERR_INVALID_ARG;
    const nrrs_config& c = ctx->cfg;
    const std::string key = tune_key(ctx);
    std::ostringstream rep;
    int ctas = 0, wgs = 1, split = 0;
    if (cache_path && cache_lookup(cache_path, key, &ctas, &wgs, &split) &&
        nrrs_set_infer_split(ctx, split) == NRRS_OK && nrrs_set_launch_shape(ctx, ctas, wgs) == NRRS_OK) {
        rep << "{\"key\": \"" << key << "\", \"cached\": [" << ctas << ", " << wgs << ", " << split
            << "]}";
        if (report && report_len) std::snprintf(report, report_len, "%s", rep.str().c_str());
        return NRRS_OK;
    }
    // synthetic inputs on the device (the tuner's own buffers)
    std::vector<float> pos(3 * (size_t)n), wi(3 * (size_t)n), nrm(3 * (size_t)n), rough(n),
        alb(3 * (size_t)n), thp(3 * (size_t)n), ref(n);
    std::vector<uint32_t> dep(n);
    nrrs_synth_vertices(12345, 0, n, pos.data(), wi.data(), nrm.data(), rough.data(), alb.data(),
                        thp.data(), dep.data(), nullptr, ref.data(), nullptr);
    float* d = nullptr;
    const size_t floats = 3 * (size_t)n * 5 + 2 * (size_t)n + (size_t)n * 2;
    if (cudaMalloc(&d, sizeof(float) * floats + sizeof(uint32_t) * n) != cudaSuccess)
        return fail(ctx, NRRS_ERR_CUDA, "autotune allocation");
    float* p = d;
    auto put = [&](const void* h, size_t bytes) {
        cudaMemcpy(p, h, bytes, cudaMemcpyHostToDevice);
        float* r = p;
        p += bytes / sizeof(float);
        return r;
    };
    nrrs_vertex_soa v{};
    v.pos = put(pos.data(), 12 * (size_t)n);
    v.wi = put(wi.data(), 12 * (size_t)n);
    v.normal = put(nrm.data(), 12 * (size_t)n);
    v.albedo = put(alb.data(), 12 * (size_t)n);
    v.thp = put(thp.data(), 12 * (size_t)n);
    v.roughness = put(rough.data(), 4 * (size_t)n);
    v.ref_mean = put(ref.data(), 4 * (size_t)n);
    float* rrs = p;
    p += n;
    float* stats = p;
    p += n;  // stats are not written (NULL below); scratch only
    v.depth = reinterpret_cast<const uint32_t*>(put(dep.data(), 4 * (size_t)n));
    (void)stats;
    nrrs_decide_params dp;
    nrrs_decide_params_default(&dp);
    nrrs_segment sg{0, n, 0, 0, 0, 0};
    const SegmentTable segs = make_segments(&sg, 1, kTile);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const bool fp32 = c.precision == NRRS_PREC_FP32;
    const int saved_ctas = fp32 ? ctx->simt_ctas_per_sm : ctx->tc_ctas_per_sm;
    const int saved_wgs = ctx->tc_wgs, saved_split = ctx->tc_split;
    float best = 1e30f;
    int best_ctas = saved_ctas, best_wgs = saved_wgs, best_split = saved_split;
    rep << "{\"key\": \"" << key << "\", \"n\": " << n << ", \"trials\": [";
    bool first = true;
    for (int sp = 0; sp <= (fp32 ? 0 : 3); ++sp)
    for (int w = 1; w <= (fp32 ? 1 : 4); w *= 2) {
        const int maxc = infer_max_ctas(c.statnet_width, c.statnet_hidden, c.rrsnet_width,
                                        c.rrsnet_hidden, c.precision, w, sp);
        if (maxc > 0 && nrrs_set_infer_split(ctx, sp) != NRRS_OK) continue;
        for (int k = 1; k <= maxc; ++k) {
            if (nrrs_set_launch_shape(ctx, k, w) != NRRS_OK) continue;
            int rc = NRRS_OK;
            for (int it = 0; it < 2 && rc == NRRS_OK; ++it)
                rc = run_infer(ctx, &v, segs, &dp, n, nullptr, rrs, false, 0);
            cudaEventRecord(e0, 0);
            for (int it = 0; it < 5 && rc == NRRS_OK; ++it)
                rc = run_infer(ctx, &v, segs, &dp, n, nullptr, rrs, false, 0);
            cudaEventRecord(e1, 0);
            if (rc != NRRS_OK || cudaEventSynchronize(e1) != cudaSuccess) continue;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            ms /= 5.f;
            rep << (first ? "" : ", ") << "{\"ctas_per_sm\": " << k << ", \"warpgroups\": " << w
                << ", \"split\": " << sp << ", \"ms\": " << ms << "}";
            first = false;
            if (ms < best) {
                best = ms;
                best_ctas = k;
                best_wgs = w;
                best_split = sp;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    nrrs_set_infer_split(ctx, best_split);
    nrrs_set_launch_shape(ctx, best_ctas, best_wgs);
    rep << "], \"best\": [" << best_ctas << ", " << best_wgs << ", " << best_split
        << "], \"best_ms\": " << best << "}";
    if (cache_path) cache_store(cache_path, key, best_ctas, best_wgs, best_split);
    if (report && report_len) std::snprintf(report, report_len, "%s", rep.str().c_str());
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NRRS_OK : cuda_fail(ctx, e, "autotune");
}

struct nrrs_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

int nrrs_graph_capture_batched(nrrs_ctx* ctx, const nrrs_vertex_soa* v, const float* rnd,
                               const nrrs_segment* segs, int32_t n_segs,
                               const nrrs_decide_params* p, float* stats, float* rrs,
                               float* rrs_norm, uint8_t* split, uint32_t* next_queue,
                               uint32_t* next_size_dev, nrrs_graph** out) {
    if (!ctx || !out) return NRRS_ERR_INVALID_ARG;
    *out = nullptr;
    cudaStream_t cs;
    cudaError_t e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "capture stream");
    const bool prof = ctx->prof.enabled;
    ctx->prof.enabled = false;  // no event nodes in the graph
    nrrs_graph* g = new nrrs_graph();
    e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    int rc = NRRS_OK;
    if (e == cudaSuccess) {
        rc = nrrs_step_batched(ctx, v, rnd, segs, n_segs, p, stats, rrs, rrs_norm, split,
                               next_queue, next_size_dev, cs);
        const cudaError_t e2 = cudaStreamEndCapture(cs, &g->graph);
        if (e2 != cudaSuccess && rc == NRRS_OK) rc = cuda_fail(ctx, e2, "end capture");
    } else {
        rc = cuda_fail(ctx, e, "begin capture");
    }
    ctx->prof.enabled = prof;
    if (rc == NRRS_OK) {
        e = cudaGraphInstantiate(&g->exec, g->graph, 0);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "graph instantiate");
    }
    cudaStreamDestroy(cs);
    if (rc != NRRS_OK) {
        nrrs_graph_destroy(g);
        return rc;
    }
    *out = g;
    return NRRS_OK;
}

int nrrs_graph_launch(nrrs_graph* g, void* stream) {
    if (!g || !g->exec) return NRRS_ERR_INVALID_ARG;
    return cudaGraphLaunch(g->exec, (cudaStream_t)stream) == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

void nrrs_graph_destroy(nrrs_graph* g) {
    if (!g) return;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
}

}  // extern "C"
