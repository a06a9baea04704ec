/*
 * nrrs_oracle.h -- CPU oracle for the NRRS per-vertex step. TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference path (banbao990/NRRS-Code, src/render/nrrs) used by
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker and the timed
 * CPU baseline. The product library never links or calls it.
 *
 * Parity status: the decision/normalisation maths and the glue are restated from the reference
 * sources cited per function and pinned by hand-derived known answers (tests/golden). The
 * reference's RRSWeightWindow is additionally compiled from its own header into oracle/_ref
 * and compared. The encodings, MLPs, losses and optimizer live in the reference's tiny-cuda-nn
 * submodule, which is absent and unpinned (branch `use-bb`, no commit): for those the oracle
 * restates the published algorithms (Instant-NGP hash grid, real SH, bias-free MLP, Adam) and
 * the written loss definitions, so PARITY WITH THE REFERENCE IS UNPINNED for them.
 *
 * Every entry point exists in an FP64 (_f64) and FP32 (_f32) flavour where arithmetic is
 * floating point; the decision path is FP32 only because it must be bit-exact.
 */
#ifndef NRRS_ORACLE_H
#define NRRS_ORACLE_H
#include <stdint.h>
#include "../include/nrrs.h"

#ifdef __cplusplus
extern "C" {
#endif

/* level table: out[l*4 + {0,1,2,3}] = {offset, entries, resolution, dense}; returns total entries */
uint64_t oracle_level_table(const nrrs_config* cfg, uint32_t* out);
uint64_t oracle_param_count(const nrrs_config* cfg, uint64_t* table, uint64_t* stat, uint64_t* rrs);
void oracle_sh16_f64(const double* dir, double* out);
/* activationSigma (networkcommon.h:61-68) and box_cox_transform (train.cu:19-39) in FP32 */
float oracle_activation_sigma_f32(float x);
float oracle_box_cox_f32(float x);
float oracle_warp_roughness_f32(float r);
float oracle_stat_to_l_f32(float y, float eps);
float oracle_weight_window_f32(float x, float ww);
/* normalizeSpatialCoord (nrctrain.h:111-115) for one point, FP32 */
void oracle_normalize_pos_f32(const nrrs_config* cfg, const float* p, float* out);

/* inference: params = FP32 master params (nrrs_get_params layout).
 * Outputs (any may be NULL): x0 [n][64], stats [n][3], x1 [n][16], raw [n], rrs [n] (clamped). */
void oracle_infer_f64(const nrrs_config* cfg, const float* params, uint64_t n,
                      const nrrs_vertex_soa* v, const nrrs_decide_params* p,
                      double* x0, double* stats, double* x1, double* raw, double* rrs);
void oracle_infer_f32(const nrrs_config* cfg, const float* params, uint64_t n,
                      const nrrs_vertex_soa* v, const nrrs_decide_params* p,
                      float* x0, float* stats, float* x1, float* raw, float* rrs);

/* exact fixed-point sum of rrs (or ceil(rrs)): returns the 64-bit accumulator, *sum = acc*2^-shift */
int oracle_sum_shift(uint64_t n, float vmax);
int64_t oracle_sum_fixed(const float* rrs, uint64_t n, int use_ceil, int shift, double* sum);

/* decision + emission (integrator.cpp:1368-1460, commonworkqueue.h:19-25), FP32, bit-exact
 * contract. Returns the total queue size (may exceed capacity; extra entries are dropped).
 * shift_n sizes the exact sum's fixed-point shift (the library uses its max_queue; 0 = n).
 * status_flags receives NRRS_DEV_* bits. */
uint64_t oracle_decide_emit(const float* rrs, const float* rnd, const uint32_t* scatter_index,
                            uint64_t n, uint32_t budget, uint32_t n_specular,
                            const nrrs_decide_params* p, uint64_t shift_n, float* rrs_norm,
                            uint8_t* split, uint32_t* queue, uint64_t capacity,
                            uint32_t* status_flags);

/* decision of one shard given the exact accumulator of all shards (acc * 2^-shift = sum) */
uint64_t oracle_decide_emit_acc(const float* rrs, const float* rnd, const uint32_t* scatter_index,
                                uint64_t n, uint32_t budget, uint32_t n_specular,
                                const nrrs_decide_params* p, int64_t acc, int shift,
                                float* rrs_norm, uint8_t* split, uint32_t* queue,
                                uint64_t capacity, uint32_t* status_flags);

/* per-sample loss weights of nrrs_train_step_batch (include/nrrs.h gives the definition); any
 * array may be NULL (absent) */
typedef struct {
    const float* sample_weight;
    const float* rrs_target;
    const float* error;
    const float* error_for_avg;
    const float* number_samples;
    double error_mean;             /* error_sum / n_pixels, or 1 */
    float gamma1, gamma2, gamma3, gamma4;
    int32_t clamp_on;
    float clamp_max;
} oracle_loss_w;

/* training: losses and gradients (no update). grads has nrrs_param_count entries.
 * loss[0] = StatNet relative log-L2, loss[1] = RRSNet variance x cost (0 when step < 3). */
void oracle_train_grads_f64(const nrrs_config* cfg, const float* params, uint64_t n,
                            const nrrs_vertex_soa* v, const float* target, double* grads,
                            double* loss);
void oracle_train_grads_f32(const nrrs_config* cfg, const float* params, uint64_t n,
                            const nrrs_vertex_soa* v, const float* target, float* grads,
                            double* loss);
void oracle_train_grads_w_f64(const nrrs_config* cfg, const float* params, uint64_t n,
                              const nrrs_vertex_soa* v, const float* target,
                              const oracle_loss_w* w, double* grads, double* loss);
void oracle_train_grads_w_f32(const nrrs_config* cfg, const float* params, uint64_t n,
                              const nrrs_vertex_soa* v, const float* target,
                              const oracle_loss_w* w, float* grads, double* loss);
void oracle_train_loss_w_f64(const nrrs_config* cfg, const double* params, uint64_t n,
                             const nrrs_vertex_soa* v, const float* target,
                             const oracle_loss_w* w, double* loss);
/* loss only (for finite differences), FP64 */
void oracle_train_loss_f64(const nrrs_config* cfg, const double* params, uint64_t n,
                           const nrrs_vertex_soa* v, const float* target, double* loss);
/* Adam update in FP32 over [first, first+count); t = step number after increment */
void oracle_adam_f32(const nrrs_config* cfg, float* params, const float* grads, float* m,
                     float* v, uint64_t first, uint64_t count, uint64_t t);

/* path-node records and the training batch (records.c); the node block points at HOST arrays */
void oracle_fixed_limbs(float x, int64_t* l);
float oracle_fixed_to_float(int64_t l0, int64_t l1, int64_t l2);
float oracle_fixed_to_float_gcc(int64_t l0, int64_t l1, int64_t l2);
float oracle_fixed_to_float_fast(int64_t l0, int64_t l1, int64_t l2);
void oracle_nodes_reset(nrrs_path_nodes* nb);
void oracle_record_nodes(nrrs_path_nodes* nb, const nrrs_vertex_soa* v, const int32_t* parent,
                         const uint32_t* pixel, const float* rrs, const uint8_t* record,
                         uint64_t n, int32_t* node_out);
void oracle_record_radiance(nrrs_path_nodes* nb, const int32_t* node, const float* contrib,
                            uint64_t n);
uint64_t oracle_generate_training_data(nrrs_path_nodes* nb, const nrrs_train_data_params* p,
                                       const float* image, int channels, uint32_t n_pixels,
                                       uint32_t* pixel_samples, const nrrs_train_batch* o,
                                       uint64_t capacity);
void oracle_sample_weights(const uint32_t* pixel, const uint32_t* pixel_samples,
                           uint32_t n_pixels, uint64_t n, float* weight);

/* per-pixel error of the RRSNet loss (records.c); HOST arrays */
void oracle_count_patch_samples(const nrrs_pixel_error_params* p, const uint32_t* pixel,
                                uint64_t n, float* spp);
void oracle_accumulate_weighted_l(const nrrs_pixel_error_params* p, const float* pl, uint32_t spp,
                                  int first, float* wl, float* cur, uint32_t* acc);
void oracle_update_weighted_l(const nrrs_pixel_error_params* p, const float* cur,
                              const uint32_t* acc, float* wl);
float oracle_calculate_error(const nrrs_pixel_error_params* p, const float* ref, int ch,
                             const float* wl, const float* spp, float* err_out);
float oracle_ubs_error(const nrrs_pixel_error_params* p, const float* pl, uint32_t spp,
                       const float* ref, int ch, float* err_out);

/* the wavefront steps around the path (render.c); HOST arrays, triangles as v0, e1, e2 */
uint32_t oracle_scene_tris(const float* vertices, const uint32_t* tris, uint32_t nt,
                           const uint32_t* tri_mat, const float* mats, float* tri_out,
                           uint32_t* lights, float* areas);
void oracle_camera_rays(const nrrs_camera* c, uint32_t sample, uint32_t seed, float* origin,
                        float* dir);
void oracle_trace(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                  const float* origin, const float* dir, const float* thp, uint32_t n,
                  uint32_t* prim, float* t, float* u, float* v);
uint32_t oracle_shade(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                      uint32_t nl, const float* env, const float* origin, const float* dir,
                      const float* thp, const float* pdf, const uint32_t* pixel,
                      const int32_t* node, const uint32_t* prim, const float* t, uint32_t n,
                      uint32_t depth, int64_t* film, float* contrib, float* o_pos, float* o_wi,
                      float* o_nrm, float* o_alb, float* o_rough, float* o_thp,
                      uint32_t* o_depth, uint32_t* o_pixel, int32_t* o_node);
void oracle_scatter(const float* tri, const uint32_t* mat, const float* mats, uint32_t nt,
                    const uint32_t* lights, const float* area, uint32_t nl, const float* pos,
                    const float* nrm, const float* alb, const float* thp, const uint32_t* pixel,
                    const int32_t* node, const float* rrs_norm, const uint32_t* queue,
                    uint32_t nq, uint32_t depth, uint32_t seed, float* r_origin, float* r_dir,
                    float* r_thp, float* r_pdf, uint32_t* r_pixel, int32_t* r_node,
                    float* s_origin, float* s_dir, float* s_tmax, float* s_contrib,
                    uint32_t* s_pixel, int32_t* s_node);
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
                            int32_t* s_node, uint32_t* n_spec);
void oracle_scatter_specular(const float* pos, const float* wi, const float* nrm, const float* alb,
                             const float* thp, const float* rough, const uint32_t* pixel,
                             const int32_t* node, uint32_t n, uint32_t off, uint32_t max_rays,
                             uint32_t depth, uint32_t seed, float* r_origin, float* r_dir,
                             float* r_thp, float* r_pdf, uint32_t* r_pixel, int32_t* r_node);
void oracle_scatter_fixed_rr(const float* tri, const uint32_t* mat, const float* mats,
                             const uint32_t* lights, const float* area, uint32_t nl,
                             const float* pos, const float* nrm, const float* alb,
                             const float* thp, const uint32_t* pixel, const int32_t* node,
                             uint32_t n, float rr, uint32_t depth, uint32_t seed, float* r_origin,
                             float* r_dir, float* r_thp, float* r_pdf, uint32_t* r_pixel,
                             int32_t* r_node, float* s_origin, float* s_dir, float* s_tmax,
                             float* s_contrib, uint32_t* s_pixel, int32_t* s_node);
void oracle_shadow(const float* tri, uint32_t nt, const float* origin, const float* dir,
                   const float* tmax, const float* contrib, const uint32_t* pixel, uint32_t n,
                   int64_t* film, float* cout);
void oracle_film_resolve(const int64_t* film, uint32_t n, float scale, float* img);

/* threads used by the OpenMP loops (0 = runtime default) */
void oracle_set_threads(int n);
int oracle_get_threads(void);

#ifdef __cplusplus
}
#endif
#endif
