// records.hpp -- device layout and launchers of the path-node records and the training batch.
//
// The node block is one caller allocation carved into SoA arrays (nrrs_path_nodes in nrrs.h).
// Its first 64 bytes are the header words below; then the look-back states of the
// order-preserving scans; then the node arrays.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "nrrs.h"

namespace nrrs {

// header words (uint32)
enum : int {
    kHdrSize = 0,        // nodes recorded, <= capacity
    kHdrDropped = 1,     // records refused at capacity (mInvalidNode)
    kHdrPropagated = 2,  // 1 once node radiance includes the descendants' contributions
    kHdrLevels = 3,      // record calls since the reset (kMaxLevels + 1: too many to keep)
    kHdrStatus = 4,      // NRRS_DEV_* bits
    kHdrTicket = 5,      // scan chunk tickets of the running launch
    kHdrDone = 6,        // CTAs finished in the running launch
    kHdrEpoch = 7,       // launch counter tagging the look-back states
    kHdrBarCount = 8,    // grid barrier of the radiance pass: arrivals
    kHdrBarGen = 9,      //   and generation
    kHdrCallBase = 10,   // u64 (words 10-11): epoch << 32 | node count when the call started
    kHdrLevelTable = 32, // node count after each record call since the reset
    kHdrWords = 128
};
constexpr int kMaxLevels = 64;

constexpr int kRecThreads = 256;
constexpr int kRecPasses = 4;
constexpr int kRecChunk = kRecThreads * kRecPasses;  // vertices (or nodes) per scan chunk
constexpr int kLimbs = 9;                            // 3 channels x 3 limbs of the radiance

struct NodeView {
    float* pos;
    float* wi;
    float* normal;
    float* albedo;
    float* rough;
    float* thp;
    int32_t* parent;
    uint32_t* pixel;
    float* rrs;
    uint32_t* depth;
    long long* rad;  // [capacity][kLimbs]
    uint32_t* first_child;
    uint32_t* children;
    uint32_t* arrived;
    uint32_t* flags;
    uint32_t* hdr;
    unsigned long long* states;
    uint32_t capacity;
};

struct RecordArgs {
    NodeView nb;
    const float* pos;
    const float* wi;
    const float* normal;
    const float* albedo;
    const float* rough;
    const float* thp;
    const uint32_t* depth;
    const int32_t* parent;
    const uint32_t* pixel;
    const float* rrs;
    const uint8_t* record;
    int32_t* node_out;
    uint32_t* chunk_count;   // [chunks] records per chunk (scratch)
    uint32_t* chunk_offset;  // [chunks] first node index of each chunk (scratch)
    uint32_t n, chunks, spin_limit;
};

struct RadianceArgs {
    NodeView nb;
    const int32_t* node;
    const float* contrib;
    uint32_t n;
};

struct GenerateArgs {
    NodeView nb;
    nrrs_train_batch out;
    const float* image;
    uint32_t* pixel_samples;
    uint32_t* size_dev;
    uint32_t channels, n_pixels, capacity, spin_limit;
    int32_t ignore_zero_l, copy_rrs_node, dedupe;
    float thp_eps;
    const float* error_pp;      // [2][n_pixels] per-pixel error, or null
    const float* spp_patch;     // [patches] samples per patch, or null
    uint32_t frame_width, scale;  // scale > 1: image and error arrays are per patch
};

struct WeightArgs {
    const uint32_t* pixel;
    const uint32_t* pixel_samples;
    const uint32_t* size_dev;
    float* weight;
    uint32_t n_pixels, max_n;
};

// two launches: per-chunk counts, whose last CTA turns them into offsets, then the writes
cudaError_t launch_record_nodes(const RecordArgs& a, cudaStream_t s);
// device scratch of nrrs_record_nodes inside the node block's scan region
inline uint32_t state_words(uint32_t capacity) { return (capacity + kRecChunk - 1) / kRecChunk + 1; }
inline uint32_t record_chunks_max(uint32_t max_record) {
    return (max_record + kRecChunk - 1) / kRecChunk + 1;
}
cudaError_t launch_record_radiance(const RadianceArgs& a, cudaStream_t s);
// completes every node's radiance with its descendants' (once per reset): level by level in one
// cooperative launch when the record calls since the reset are at most kMaxLevels, else by
// walking the parent chains
cudaError_t launch_propagate(const NodeView& nb, cudaStream_t s);
cudaError_t launch_generate(const GenerateArgs& a, int grid, cudaStream_t s);
cudaError_t launch_sample_weights(const WeightArgs& a, cudaStream_t s);

}  // namespace nrrs
