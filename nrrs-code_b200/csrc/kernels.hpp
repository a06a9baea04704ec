// kernels.hpp -- host-side launch wrappers of the NRRS kernels (internal to libnrrs_b200).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

#include "nrrs_common.cuh"

namespace nrrs {

// Fixed-point shift of the exact normalisation sum for queues of up to n vertices whose summed
// terms are at most vmax: n * vmax < 2^(62 - shift), capped at 40 fractional bits. Every path
// that decides a queue (context, sharded, allocation-free) takes its shift from here, so the
// same capacity gives the same bits.
inline int sum_shift(uint64_t n, float vmax) {
    const double prod = (double)(n ? n : 1) * (double)(vmax > 1.f ? vmax : 1.f);
    int e = 0;
    std::frexp(prod, &e);
    const int s = 62 - e;
    return s > 40 ? 40 : s;
}

constexpr int kDecThreads = 256;
constexpr int kDecVPT = 8;
constexpr int kDecChunk = kDecThreads * kDecVPT;  // vertices per decision chunk

struct DecideArgs {
    const float* rrs;
    const float* rnd;
    const uint32_t* sidx;
    float* rrs_norm;
    uint8_t* split;
    uint32_t* queue;
    uint32_t* next_size;          // [n segments]
    const uint32_t* n_spec_dev;   // optional override of segment 0's n_specular
    const long long* ext_sum;     // caller-owned exact sum of segment 0 (sharded decision) or null
    DecideScratch* scr;
    unsigned long long* states;   // one look-back word per chunk
    SegmentTable segs;            // tile_start counts decision chunks
    float normalize_rate;
    int32_t use_ceil;
    int32_t scale_up;
    double inv_fixed_scale;
    uint32_t spin_limit;
    int32_t split_chunked;        // two-pass decision: split is scratch with one block per chunk
};

struct SumArgs {
    const float* rrs;
    DecideScratch* scr;
    SegmentTable segs;            // tile_start counts sum tiles (kTile vertices)
    FactorParams fp;
};

struct InferArgs {
    VertexPtrs v;
    EncodeParams enc;
    FactorParams fp;
    SegmentTable segs;            // tile_start counts kTile-vertex tiles
    const float* table;           // FP32 table [rows][2]   (FP32 path)
    const __half* table_h;        // FP16 table [rows][2]   (mixed path)
    const float* wt_stat;         // transposed FP32 StatNet weights (FP32 path)
    const float* wt_rrs;          // transposed FP32 RRSNet weights
    const void* wpack;            // packed UMMA weights (mixed path)
    float* stats;                 // [n][3] optional
    float* rrs;                   // [n]
    DecideScratch* scr;           // accumulate the exact sum when not null
    unsigned long long* ext_acc;  // accumulate into this caller-owned sum instead (sharded)
    const uint8_t* enc_tiles;     // split mode: hash features per tile from k_encode_levels
    uint8_t* x1_tiles;            // split mode 2: RRSNet input per tile ([128 x 16], 4 KB)
};

// split inference mode: per tile, the 32 hash-grid features of its 128 vertices as a
// [128 x 32] K-major core-matrix block (8 KB), written level-major by k_encode_levels
constexpr uint32_t kEncTileBytes = 128u * 32u * 2u;
constexpr uint32_t kX1TileBytes = 128u * 16u * 2u;
struct EncodeLvArgs {
    EncodeParams enc;
    SegmentTable segs;
    const float* pos;
    const __half* table_h;
    uint8_t* out;                 // total_tiles x tile_bytes
    uint32_t tile_bytes;          // kEncTileBytes (inference) or the [128 x 64] training input tile
    uint32_t kdim;                // K of the tile layout: 32 (inference) or 64 (training input)
};
cudaError_t launch_encode_levels(const EncodeLvArgs& a, bool bf, int sm_count, cudaStream_t s);

// resident CTAs per SM of a kernel from its own resources (shared memory incl. the 1 KB the
// runtime reserves per CTA, registers, warps), capped by `cap` (TMEM columns or a tuning choice)
int resident_ctas(const void* kern, int threads, size_t dyn_smem, int cap);
// grid of the last inference launch (diagnostics)
extern thread_local int g_last_grid;

// decision + emission (single pass, decoupled look-back)
cudaError_t launch_decide(const DecideArgs& a, cudaStream_t s);
// the same decision and queue in two passes without a look-back (count + prefix scan, emission);
// needs a.split (the caller's array or context scratch of one byte per vertex)
cudaError_t launch_decide_two_pass(const DecideArgs& a, cudaStream_t s);
// device-side segment tables of device-resident queue sizes (counts_dev[host_max.n]), in units
// of kTile (tiles_dev) and kDecChunk (chunks_dev); counts above the host maxima are clamped and
// flag NRRS_DEV_OVERFLOW in *status
cudaError_t launch_resolve_segments(const SegmentTable& host_max, const uint32_t* counts_dev,
                                    SegmentTable* tiles_dev, SegmentTable* chunks_dev,
                                    unsigned* status, cudaStream_t s);
// exact sum of rrs (or ceil) per segment into scr->sum_acc
cudaError_t launch_sum(const SumArgs& a, cudaStream_t s);
// FP32 SIMT inference
cudaError_t launch_infer_fp32(const InferArgs& a, int ws, int hs, int wr, int hr, int sm_count,
                              int ctas_per_sm, cudaStream_t s);
// largest resident CTAs per SM of the inference kernel for a shape (0 = unsupported)
// split: 0 fused, 1 encoding + MLP kernel, 2 encoding + StatNet kernel + RRSNet kernel,
// 3 as 2 with the hidden activations in TMEM
int infer_max_ctas(int ws, int hs, int wr, int hr, int prec, int wgs, int split = 0);
// tcgen05 mixed-precision inference; part: 0 both networks, 1 StatNet only, 2 RRSNet only;
// tmem_act: parts 1 and 2 with the hidden activations in TMEM
cudaError_t launch_infer_tc(const InferArgs& a, int ws, int hs, int wr, int hr, int prec,
                            int sm_count, int ctas_per_sm, int wgs, int part, bool tmem_act,
                            cudaStream_t s);
size_t infer_tc_smem_bytes(int ws, int hs, int wr, int hr);
// derived weight copies: FP32 transposed and the UMMA-packed FP16/BF16 images
cudaError_t launch_pack_weights(const float* master_mlp, float* wt, float* wrow, void* wpack,
                                int ws, int hs, int wr, int hr, int prec, cudaStream_t s);
size_t packed_weight_bytes(int ws, int hs, int wr, int hr);
size_t transposed_weight_floats(int ws, int hs, int wr, int hr);
// BF16 training image: forward layers + transposed layers for input gradients
cudaError_t launch_pack_train(const float* master_mlp, void* out, int ws, int hs, int wr, int hr,
                              cudaStream_t s);
size_t train_pack_bytes(int ws, int hs, int wr, int hr);
// FP32 table -> FP16 copy
cudaError_t launch_table_to_half(const float* t, __half* h, size_t n, cudaStream_t s);
// the cell image of the dense levels (EncodeParams::cells) from the FP16 table
cudaError_t launch_cell_image(const __half* table_h, const EncodeParams& e, uint4* cells,
                              uint32_t n_cells, int sm_count, cudaStream_t s);

}  // namespace nrrs
