// noalloc.cu -- decision + emission that allocates no device memory.
//
// nrrs_decide_emit needs a context, and nrrs_create allocates device memory with cudaMalloc.
// Some callers cannot do that: a renderer plugin whose host framework owns every device
// allocation through its own arena (the way the reference's integrator gets its queues from
// KiRaRay's allocator) and forbids a plugin to allocate; a frame loop with a device-memory
// budget fixed at start-up; code where cudaMalloc's implicit device synchronisation would stall
// the pipeline. This entry point serves them: it runs the same exact-sum and decide/emit
// kernels as nrrs_decide_emit, with their scratch in a file-scope device array instead of
// context memory.
//
// The array holds NRRS_NOALLOC_MAX_N vertices' worth of look-back state (about 66 KB) and stays
// resident on every GPU that loads the library until the process exits. In host code its name
// is only a host-side stand-in, so its device address is looked up with cudaGetSymbolAddress,
// once per device, the first time the entry point runs with that device current.
#include <cmath>
#include <mutex>

#include "kernels.hpp"

namespace nrrs {
namespace {

constexpr uint32_t kNoAllocChunks = (NRRS_NOALLOC_MAX_N + kDecChunk - 1) / kDecChunk + 1;
constexpr size_t kNoAllocBytes = sizeof(DecideScratch) + sizeof(unsigned long long) * kNoAllocChunks;

// shared by every call on a device; keeps the last call's contents
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return NRRS_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) return NRRS_ERR_CUDA;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return NRRS_OK;
}

int sum_shift_noalloc(float vmax) {
    const double prod = (double)NRRS_NOALLOC_MAX_N * (double)(vmax > 1.f ? vmax : 1.f);
    int e = 0;
    std::frexp(prod, &e);
    const int s = 62 - e;
    return s > 40 ? 40 : s;
}

}  // namespace
}  // namespace nrrs

using namespace nrrs;

extern "C" int nrrs_decide_emit_noalloc(const float* rrs, const float* rnd,
                                        const uint32_t* scatter_index, uint32_t n,
                                        uint32_t budget, uint32_t n_specular,
                                        const nrrs_decide_params* p, float* rrs_norm,
                                        uint8_t* split, uint32_t* next_queue, uint32_t capacity,
                                        uint32_t* next_size_dev, void* stream) {
    if (!p) return NRRS_ERR_INVALID_ARG;
    if (n > NRRS_NOALLOC_MAX_N) return NRRS_ERR_INVALID_ARG;  // beyond the static scratch
    if (n && (!rrs || !rnd)) return NRRS_ERR_INVALID_ARG;
    if (!next_size_dev || (capacity && !next_queue)) return NRRS_ERR_INVALID_ARG;
    if (!(p->clamp_min >= 0.f) || !(p->clamp_max >= p->clamp_min) || !std::isfinite(p->clamp_max))
        return NRRS_ERR_INVALID_ARG;
    if (p->factor_source != NRRS_FACTOR_ADRRS && p->factor_source != NRRS_FACTOR_RRSNET)
        return NRRS_ERR_INVALID_ARG;
    const float vmax = p->use_ceil ? ceilf(p->clamp_max) : p->clamp_max;
    const int shift = sum_shift_noalloc(vmax);
    if (shift < 16) return NRRS_ERR_UNSUPPORTED;

    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc != NRRS_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        return cudaMemsetAsync(next_size_dev, 0, sizeof(uint32_t), s) == cudaSuccess
                   ? NRRS_OK : NRRS_ERR_CUDA;
    }

    Segment sg{};
    sg.offset = 0;
    sg.count = n;
    sg.tile_start = 0;
    sg.budget = budget;
    sg.n_specular = n_specular;
    sg.queue_offset = 0;
    sg.queue_capacity = capacity;
    const uint32_t chunks = (n + kDecChunk - 1) / kDecChunk;

    // The array keeps whatever the previous call (or an aborted one) left: clear the header
    // (sums, ticket, done counter, status) and the look-back states this call will use.
    DecideScratch* scr = reinterpret_cast<DecideScratch*>(base);
    if (cudaMemsetAsync(base, 0, sizeof(DecideScratch) + sizeof(unsigned long long) * chunks, s) !=
        cudaSuccess)
        return NRRS_ERR_CUDA;

    SumArgs sa{};
    sa.rrs = rrs;
    sa.scr = scr;
    sa.segs.n = 1;
    sa.segs.s[0] = sg;
    sa.segs.total_tiles = (n + kTile - 1) / kTile;
    sa.fp.use_ceil = p->use_ceil;
    sa.fp.vmax = vmax;
    sa.fp.fixed_scale = std::ldexp(1.0, shift);
    if (launch_sum(sa, s) != cudaSuccess) return NRRS_ERR_CUDA;

    DecideArgs d{};
    d.rrs = rrs;
    d.rnd = rnd;
    d.sidx = scatter_index;
    d.rrs_norm = rrs_norm;
    d.split = split;
    d.queue = next_queue;
    d.next_size = next_size_dev;
    d.n_spec_dev = nullptr;
    d.scr = scr;
    d.states = reinterpret_cast<unsigned long long*>(scr + 1);
    d.segs.n = 1;
    d.segs.s[0] = sg;
    d.segs.total_tiles = chunks;
    d.normalize_rate = p->normalize_rate;
    d.use_ceil = p->use_ceil;
    d.scale_up = p->scale_up;
    d.inv_fixed_scale = 1.0 / sa.fp.fixed_scale;
    d.spin_limit = 1u << 22;
    if (launch_decide(d, s) != cudaSuccess) return NRRS_ERR_CUDA;
    return NRRS_OK;
}
