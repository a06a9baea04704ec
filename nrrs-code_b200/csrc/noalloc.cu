// noalloc.cu -- decision + emission that allocates no device memory.
//
// nrrs_decide_emit needs a context, and nrrs_create allocates device memory with cudaMalloc.
// Some callers cannot do that: a renderer plugin whose host framework owns every device
// allocation through its own arena (the way the reference's integrator gets its queues from
// KiRaRay's allocator) and forbids a plugin to allocate; a frame loop with a device-memory
// budget fixed at start-up; code where cudaMalloc's implicit device synchronisation would stall
// the pipeline. This entry point serves them: it runs the same exact-sum kernel as
// nrrs_decide_emit and the single-pass decision kernel (whose look-back state is a few bytes per
// 2,048 vertices; the context path's two-pass decision keeps a byte per vertex), with their
// scratch in a file-scope device array instead of context memory. The results are the same bits.
//
// The array holds NRRS_NOALLOC_MAX_N vertices' worth of look-back state (about 66 KB) and stays
// resident on every GPU that loads the library until the process exits. In host code its name
// is only a host-side stand-in, so its device address is looked up with cudaGetSymbolAddress
// with the device current. The lookup is cached per CUDA context (keyed by the driver's context
// id, which is never reused within a process), so a context that is destroyed and created again
// (cudaDeviceReset) gets a fresh lookup instead of a stale address. The first call in each
// context does the lookup; make it before any stream capture.
//
// The kernels' device status bits (look-back timeout, non-finite factor, saturated or
// overflowing counts) accumulate in the array's status word across calls; each call clears
// everything else it uses. nrrs_noalloc_device_status reads and clears them.
#include <cuda.h>

#include <cmath>
#include <cstddef>
#include <mutex>

#include "kernels.hpp"

namespace nrrs {
namespace {

constexpr uint32_t kNoAllocChunks = (NRRS_NOALLOC_MAX_N + kDecChunk - 1) / kDecChunk + 1;
constexpr size_t kNoAllocBytes = sizeof(DecideScratch) + sizeof(unsigned long long) * kNoAllocChunks;

// shared by every call on a device; keeps the last call's contents
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long*);

struct AddrCache {
    std::mutex mu;
    bool resolved = false;
    CtxGetCurrentFn get_current = nullptr;
    CtxGetIdFn get_id = nullptr;
    static constexpr int kSlots = 64;
    unsigned long long ctx_id[kSlots] = {};
    void* addr[kSlots] = {};
    int used = 0, next = 0;
};
AddrCache g_cache;

// id of the context current on this thread (0 when none is current or the driver lacks the call)
unsigned long long current_ctx_id(AddrCache& c) {
    if (!c.resolved) {
        c.resolved = true;
        cudaDriverEntryPointQueryResult q{};
        void* f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            c.get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            c.get_id = reinterpret_cast<CtxGetIdFn>(f);
        cudaGetLastError();
    }
    if (!c.get_current || !c.get_id) return 0;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (c.get_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    if (c.get_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// device address of the scratch array in the current context
int scratch_address(void** out) {
    std::lock_guard<std::mutex> lock(g_cache.mu);
    unsigned long long id = current_ctx_id(g_cache);
    if (id) {
        for (int k = 0; k < g_cache.used; ++k)
            if (g_cache.ctx_id[k] == id) {
                *out = g_cache.addr[k];
                return NRRS_OK;
            }
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return NRRS_ERR_CUDA;
    }
    if (!id) id = current_ctx_id(g_cache);  // the lookup made the primary context current
    if (id) {
        const int k = g_cache.used < AddrCache::kSlots ? g_cache.used++ : g_cache.next;
        g_cache.next = (k + 1) % AddrCache::kSlots;
        g_cache.ctx_id[k] = id;
        g_cache.addr[k] = p;
    }
    *out = p;
    return NRRS_OK;
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
    // the shift a context with max_queue = NRRS_NOALLOC_MAX_N uses, so both give the same bits
    const int shift = sum_shift(NRRS_NOALLOC_MAX_N, vmax);
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

    // The array keeps whatever the previous call (or an aborted one) left: clear the sums,
    // ticket, done counter and epoch, and the look-back states this call will use. The status
    // word is left alone so that nrrs_noalloc_device_status sees every call's flags.
    DecideScratch* scr = reinterpret_cast<DecideScratch*>(base);
    unsigned long long* states = reinterpret_cast<unsigned long long*>(scr + 1);
    if (cudaMemsetAsync(base, 0, offsetof(DecideScratch, status), s) != cudaSuccess ||
        cudaMemsetAsync(states, 0, sizeof(unsigned long long) * chunks, s) != cudaSuccess)
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
    d.states = states;
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

extern "C" int nrrs_noalloc_device_status(uint32_t* flags, void* stream) {
    if (!flags) return NRRS_ERR_INVALID_ARG;
    void* base = nullptr;
    int rc = scratch_address(&base);
    if (rc != NRRS_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned int* status = &reinterpret_cast<DecideScratch*>(base)->status;
    uint32_t h = 0;
    if (cudaMemcpyAsync(&h, status, sizeof(h), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemsetAsync(status, 0, sizeof(unsigned int), s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return NRRS_ERR_CUDA;
    *flags = h;
    if (h & NRRS_DEV_TIMEOUT) return NRRS_ERR_TIMEOUT;
    if (h & NRRS_DEV_OVERFLOW) return NRRS_ERR_CAPACITY_OVERFLOW;
    if (h & NRRS_DEV_NAN) return NRRS_ERR_NAN;
    return NRRS_OK;
}
