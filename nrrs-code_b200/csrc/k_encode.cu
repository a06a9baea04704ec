// k_encode.cu -- level-major hash-grid encoding into feature tiles (sm_100a), the first kernel
// of the split inference mode.
//
// With a table larger than L2 (16 levels of 2^22 FP16 pairs: 178 MB), the fused inference
// kernel gathers each vertex's 128 corners from all 16 levels at once, so the lines in flight
// span the whole table and most gathers are random HBM reads (about 3.6 KB of DRAM traffic per
// vertex for 512 B of features). This kernel sweeps the queue four levels at a time: work item
// (quad q, tile t) in q-major order, so the CTAs in flight read the slices of one quad of levels
// (at most 4 x 16 MB), which stay in L2, and a table line is brought from HBM about once per
// sweep instead of once per use.
//
// A work item writes the 8 features (levels 4q .. 4q+3, 2 each) of its 128 vertices as one
// 16-byte chunk per vertex into chunk q of tile t, in the no-swizzle K-major core-matrix layout
// of a [128 x kdim] tile: the A-operand layout of the first tcgen05 layer. Inference uses 8 KB
// [128 x 32] blocks; training writes the hash columns of its [128 x 64] input tiles, whose
// other columns the training kernel fills. Rows past the end of a segment are zero.
// The per-level arithmetic is that of the fused kernel (levels_features_h), so the features and
// everything downstream are bit-identical between the two modes. The encoding is the
// reference's tcnn HashGrid (common/configs/nrrs/nrrs/2net-simple.json:46).
#include "kernels.hpp"
#include "tc_tile.cuh"

namespace nrrs {

namespace {

template <bool BF>
__global__ void __launch_bounds__(kTile) k_encode_levels(const __grid_constant__ EncodeLvArgs a) {
    // work items are (level group, tile) over the tiles the host sized the launch for; with
    // device-resident sizes the tiles past the actual total are skipped
    const uint32_t tiles = a.segs.total_tiles;
    const uint32_t items = 4u * tiles;
    const SegmentTable& S = seg_table(a.segs);
    const __half2* table = reinterpret_cast<const __half2*>(a.table_h);
    const int m = threadIdx.x;
    for (uint32_t w = blockIdx.x; w < items; w += gridDim.x) {
        const uint32_t q = w / tiles, t = w - q * tiles;
        if (t >= S.total_tiles) continue;
        const int si = find_segment(S, t);
        const Segment& sg = S.s[si];
        const uint32_t i = sg.offset + (t - sg.tile_start) * kTile + m;
        uint4 v = make_uint4(0u, 0u, 0u, 0u);
        if (i < sg.offset + sg.count) {
            float p[3];
            norm_pos(a.enc, a.pos, i, p);
            // two levels per batch of loads: half the registers of four, twice the CTAs per SM
            float f[8];
            levels_features_h<2>(table, a.enc, p, 4 * (int)q, f);
            levels_features_h<2>(table, a.enc, p, 4 * (int)q + 2, f + 4);
            v = tile::pack8<BF>(f);
        }
        *reinterpret_cast<uint4*>(a.out + (size_t)t * a.tile_bytes +
                                  tile::chunk_offset(m, (int)q, (int)a.kdim)) = v;
    }
}

}  // namespace

cudaError_t launch_encode_levels(const EncodeLvArgs& a, bool bf, int sm_count, cudaStream_t s) {
    const uint32_t items = 4u * a.segs.total_tiles;
    if (items == 0) return cudaSuccess;
    auto k = bf ? k_encode_levels<true> : k_encode_levels<false>;
    const int per_sm = resident_ctas((const void*)k, kTile, 0, 16);
    uint32_t grid = (uint32_t)(sm_count * per_sm);
    if (grid > items) grid = items;
    k<<<grid, kTile, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nrrs
