// records_api.cu -- C-ABI of the path-node records and the training batch (include/nrrs.h).
//
// No context: every buffer, the node block included, belongs to the caller. The node block's
// layout is fixed by nrrs_path_nodes_bytes/nrrs_path_nodes_init; the kernels are in
// k_records.cu.
#include <cstring>
#include <mutex>

#include "records.hpp"

namespace nrrs {
namespace {

constexpr uint64_t kAlign = 256;
constexpr uint32_t kSpinLimit = 1u << 22;

uint64_t align_up(uint64_t x) { return (x + kAlign - 1) / kAlign * kAlign; }

// the scan region: look-back states of the batch (one per node chunk), then the record calls'
// per-chunk counts and offsets
uint64_t scan_bytes(uint32_t capacity, uint32_t max_record) {
    return sizeof(unsigned long long) * (uint64_t)state_words(capacity) +
           2ull * sizeof(uint32_t) * record_chunks_max(max_record);
}

// byte offsets of every array in the block; returns the total
struct Layout {
    uint64_t hdr, states, pos, wi, normal, albedo, rough, thp, parent, pixel, rrs, depth, rad,
        first_child, children, arrived, flags, total;
};

Layout layout(uint32_t capacity, uint32_t max_record) {
    Layout L{};
    const uint64_t C = capacity;
    uint64_t o = 0;
    auto take = [&](uint64_t bytes) { const uint64_t at = o; o = align_up(o + bytes); return at; };
    L.hdr = take(sizeof(uint32_t) * kHdrWords);
    L.states = take(scan_bytes(capacity, max_record));
    L.pos = take(12 * C);
    L.wi = take(12 * C);
    L.normal = take(12 * C);
    L.albedo = take(12 * C);
    L.rough = take(4 * C);
    L.thp = take(12 * C);
    L.parent = take(4 * C);
    L.pixel = take(4 * C);
    L.rrs = take(4 * C);
    L.depth = take(4 * C);
    L.rad = take(8ull * kLimbs * C);
    L.first_child = take(4 * C);
    L.children = take(4 * C);
    L.arrived = take(4 * C);
    L.flags = take(4 * C);
    L.total = o;
    return L;
}

NodeView view(const nrrs_path_nodes* n) {
    NodeView v{};
    v.pos = n->pos;
    v.wi = n->wi;
    v.normal = n->normal;
    v.albedo = n->albedo;
    v.rough = n->roughness;
    v.thp = n->thp;
    v.parent = n->parent;
    v.pixel = n->pixel;
    v.rrs = n->rrs;
    v.depth = n->depth;
    v.rad = reinterpret_cast<long long*>(n->radiance);
    v.first_child = n->first_child;
    v.children = n->children;
    v.arrived = n->arrived;
    v.flags = n->node_flags;
    v.hdr = n->header;
    v.states = reinterpret_cast<unsigned long long*>(n->scan_states);
    v.capacity = n->capacity;
    return v;
}

bool valid(const nrrs_path_nodes* n) {
    return n && n->capacity && n->header && n->scan_states && n->pos && n->wi && n->normal &&
           n->albedo && n->roughness && n->thp && n->parent && n->pixel && n->rrs && n->depth &&
           n->radiance && n->first_child && n->children && n->arrived && n->node_flags;
}

// persistent grids: SMs x resident CTAs, looked up once per device
constexpr int kMaxDevices = 64;
std::mutex g_mu;
int g_sms[kMaxDevices] = {};

int sm_count() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return 0;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_sms[dev]) {
        int s = 0;
        if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
        g_sms[dev] = s;
    }
    return g_sms[dev];
}

int persistent_grid(uint64_t units, uint64_t per_cta, int ctas_per_sm) {
    const int sms = sm_count();
    if (sms <= 0) return 0;
    uint64_t need = (units + per_cta - 1) / per_cta;
    if (need == 0) need = 1;
    const uint64_t cap = (uint64_t)sms * ctas_per_sm;
    return (int)(need < cap ? need : cap);
}

}  // namespace
}  // namespace nrrs

using namespace nrrs;

extern "C" uint64_t nrrs_path_nodes_bytes(uint32_t capacity, uint32_t max_record) {
    return layout(capacity, max_record).total;
}

extern "C" int nrrs_path_nodes_init(void* dev_mem, uint64_t bytes, uint32_t capacity,
                                    uint32_t max_record, nrrs_path_nodes* out, void* stream) {
    if (!dev_mem || !out || capacity == 0) return NRRS_ERR_INVALID_ARG;
    if (reinterpret_cast<uintptr_t>(dev_mem) % kAlign) return NRRS_ERR_INVALID_ARG;
    const Layout L = layout(capacity, max_record);
    if (bytes < L.total) return NRRS_ERR_INVALID_ARG;
    char* b = static_cast<char*>(dev_mem);
    nrrs_path_nodes n{};
    n.capacity = capacity;
    n.max_record = max_record;
    n.pos = reinterpret_cast<float*>(b + L.pos);
    n.wi = reinterpret_cast<float*>(b + L.wi);
    n.normal = reinterpret_cast<float*>(b + L.normal);
    n.albedo = reinterpret_cast<float*>(b + L.albedo);
    n.roughness = reinterpret_cast<float*>(b + L.rough);
    n.thp = reinterpret_cast<float*>(b + L.thp);
    n.parent = reinterpret_cast<int32_t*>(b + L.parent);
    n.pixel = reinterpret_cast<uint32_t*>(b + L.pixel);
    n.rrs = reinterpret_cast<float*>(b + L.rrs);
    n.depth = reinterpret_cast<uint32_t*>(b + L.depth);
    n.radiance = reinterpret_cast<int64_t*>(b + L.rad);
    n.first_child = reinterpret_cast<uint32_t*>(b + L.first_child);
    n.children = reinterpret_cast<uint32_t*>(b + L.children);
    n.arrived = reinterpret_cast<uint32_t*>(b + L.arrived);
    n.node_flags = reinterpret_cast<uint32_t*>(b + L.flags);
    n.header = reinterpret_cast<uint32_t*>(b + L.hdr);
    n.scan_states = reinterpret_cast<uint64_t*>(b + L.states);
    // header and look-back states start at zero (epoch 0, no state ready)
    if (cudaMemsetAsync(b, 0, L.pos, (cudaStream_t)stream) != cudaSuccess) return NRRS_ERR_CUDA;
    *out = n;
    return NRRS_OK;
}

extern "C" int nrrs_path_nodes_reset(const nrrs_path_nodes* nodes, void* stream) {
    if (!valid(nodes)) return NRRS_ERR_INVALID_ARG;
    // size, dropped, the radiance-complete mark and the record calls; the epoch and the barrier
    // keep counting so that no stale look-back state or arrival can match a later launch
    static_assert(kHdrSize == 0 && kHdrDropped == 1 && kHdrPropagated == 2 && kHdrLevels == 3,
                  "header layout");
    return cudaMemsetAsync(nodes->header, 0, 4 * sizeof(uint32_t), (cudaStream_t)stream) ==
                   cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

extern "C" int nrrs_path_nodes_status(const nrrs_path_nodes* nodes, uint32_t* size,
                                      uint32_t* dropped, uint32_t* flags, void* stream) {
    if (!valid(nodes)) return NRRS_ERR_INVALID_ARG;
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t h[kHdrWords];
    if (cudaMemcpyAsync(h, nodes->header, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return NRRS_ERR_CUDA;
    if (cudaMemsetAsync(nodes->header + kHdrStatus, 0, sizeof(uint32_t), s) != cudaSuccess)
        return NRRS_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return NRRS_ERR_CUDA;
    if (size) *size = h[kHdrSize];
    if (dropped) *dropped = h[kHdrDropped];
    if (flags) *flags = h[kHdrStatus];
    return NRRS_OK;
}

extern "C" int nrrs_record_nodes(const nrrs_path_nodes* nodes, const nrrs_vertex_soa* v,
                                 const int32_t* parent, const uint32_t* pixel, const float* rrs,
                                 const uint8_t* record, uint32_t n, int32_t* node_out,
                                 void* stream) {
    if (!valid(nodes) || !v) return NRRS_ERR_INVALID_ARG;
    if (n > nodes->max_record) return NRRS_ERR_INVALID_ARG;
    if (n == 0) return NRRS_OK;
    if (!v->pos || !v->wi || !v->thp || !parent || !pixel || !node_out) return NRRS_ERR_INVALID_ARG;
    RecordArgs a{};
    a.nb = view(nodes);
    a.pos = v->pos;
    a.wi = v->wi;
    a.normal = v->normal;
    a.albedo = v->albedo;
    a.rough = v->roughness;
    a.thp = v->thp;
    a.depth = v->depth;
    a.parent = parent;
    a.pixel = pixel;
    a.rrs = rrs;
    a.record = record;
    a.node_out = node_out;
    a.n = n;
    a.chunks = (n + kRecChunk - 1) / kRecChunk;
    a.spin_limit = kSpinLimit;
    uint32_t* scratch = reinterpret_cast<uint32_t*>(
        reinterpret_cast<unsigned long long*>(nodes->scan_states) + state_words(nodes->capacity));
    a.chunk_count = scratch;
    a.chunk_offset = scratch + record_chunks_max(nodes->max_record);
    if (sm_count() <= 0) return NRRS_ERR_NO_DEVICE;
    return launch_record_nodes(a, (cudaStream_t)stream) == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

extern "C" int nrrs_record_radiance(const nrrs_path_nodes* nodes, const int32_t* node,
                                    const float* contrib, uint32_t n, void* stream) {
    if (!valid(nodes)) return NRRS_ERR_INVALID_ARG;
    if (n == 0) return NRRS_OK;
    if (!node || !contrib) return NRRS_ERR_INVALID_ARG;
    RadianceArgs a{};
    a.nb = view(nodes);
    a.node = node;
    a.contrib = contrib;
    a.n = n;
    return launch_record_radiance(a, (cudaStream_t)stream) == cudaSuccess ? NRRS_OK
                                                                         : NRRS_ERR_CUDA;
}

extern "C" int nrrs_generate_training_data(const nrrs_path_nodes* nodes,
                                           const nrrs_train_data_params* p, const float* image,
                                           int32_t image_channels, uint32_t n_pixels,
                                           uint32_t* pixel_samples, const nrrs_train_batch* out,
                                           uint32_t capacity, uint32_t* size_dev, void* stream) {
    if (!valid(nodes) || !p || !out || !size_dev) return NRRS_ERR_INVALID_ARG;
    if (image && image_channels != 3 && image_channels != 4) return NRRS_ERR_INVALID_ARG;
    if (!(p->thp_eps >= 0.f)) return NRRS_ERR_INVALID_ARG;
    if (p->error_image_scale > 1u) {   // whole patches only
        const uint32_t w = p->frame_width, sc = p->error_image_scale;
        if (w == 0 || n_pixels % w || w % sc || (n_pixels / w) % sc) return NRRS_ERR_INVALID_ARG;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const NodeView nb = view(nodes);
    if (sm_count() <= 0) return NRRS_ERR_NO_DEVICE;
    if (launch_propagate(nb, s) != cudaSuccess) return NRRS_ERR_CUDA;
    GenerateArgs a{};
    a.nb = nb;
    a.out = *out;
    a.image = image;
    a.pixel_samples = pixel_samples;
    a.size_dev = size_dev;
    a.channels = image ? (uint32_t)image_channels : 0u;
    a.n_pixels = n_pixels;
    a.capacity = capacity;
    a.spin_limit = kSpinLimit;
    a.ignore_zero_l = p->ignore_zero_l;
    a.copy_rrs_node = p->copy_rrs_node;
    a.dedupe = p->dedupe_rrs_target;
    a.thp_eps = p->thp_eps;
    a.error_pp = p->error_per_pixel;
    a.spp_patch = p->samples_per_patch;
    a.frame_width = p->frame_width;
    a.scale = p->error_image_scale;
    const int gg = persistent_grid(nodes->capacity, kRecChunk, 8);
    return launch_generate(a, gg, s) == cudaSuccess ? NRRS_OK : NRRS_ERR_CUDA;
}

extern "C" int nrrs_sample_weights(const uint32_t* pixel, const uint32_t* pixel_samples,
                                   uint32_t n_pixels, const uint32_t* size_dev, uint32_t max_n,
                                   float* weight, void* stream) {
    if (max_n == 0) return NRRS_OK;
    if (!pixel || !pixel_samples || !size_dev || !weight) return NRRS_ERR_INVALID_ARG;
    WeightArgs a{};
    a.pixel = pixel;
    a.pixel_samples = pixel_samples;
    a.size_dev = size_dev;
    a.weight = weight;
    a.n_pixels = n_pixels;
    a.max_n = max_n;
    return launch_sample_weights(a, (cudaStream_t)stream) == cudaSuccess ? NRRS_OK
                                                                        : NRRS_ERR_CUDA;
}
