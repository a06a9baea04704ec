// k_records.cu -- path-node records, exact radiance accumulation and the training batch.
//
// Replaces, in banbao990/NRRS-Code:
//   NRRSPathNodesBuffer::recordNode      src/render/nrrs/workqueue.h:142-170
//   NRRSPathNodesBuffer::recordRadiance  src/render/nrrs/workqueue.h:122-136
//   nrrs_generate_training_data          src/render/nrrs/train.cu:432-570
//   nrrs_calculate_sample_weight         src/render/nrrs/train.cu:572-592
//
// The reference numbers nodes and training samples with atomicAdd and sums radiance with FP32
// atomics, so both its order and its bits depend on scheduling. Here:
//   * nodes and samples are compacted in input order by a single-pass scan with decoupled
//     look-back over 2048-element chunks (one ballot per warp and pass);
//   * radiance is a fixed-point integer, three signed 64-bit limbs per channel with the lowest
//     bit worth 2^-64: a contribution x (|x| < 2^62) becomes trunc(|x| 2^64) split into a
//     32-bit low limb, a 32-bit middle limb and the integer part, each signed like x. Integer
//     additions commute, so every node total is the same integer in any order;
//   * a contribution is added to its own node only; one pass then adds each node's complete
//     total into its parent once, a child that finds itself the last of its siblings carrying on
//     upwards. That is one addition per node instead of one per ancestor per contribution.
#include <cmath>

#include "records.hpp"

namespace nrrs {

namespace {

constexpr unsigned long long kFlagAgg = 1ull;
constexpr unsigned long long kFlagIncl = 2ull;
constexpr float kFixedMax = 4611686018427387904.0f;  // 2^62: larger contributions are refused

__device__ __forceinline__ unsigned long long pack_state(unsigned epoch, unsigned long long flag,
                                                         unsigned value) {
    return ((unsigned long long)(epoch & 0x3fffffffu) << 34) | (flag << 32) | value;
}

__device__ __forceinline__ unsigned long long load_state(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void store_state(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned sat_add(unsigned a, unsigned b) {
    const unsigned s = a + b;
    return s < a ? 0xffffffffu : s;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// Called by all of warp 0. Publishes this chunk's total, reads the predecessors' states 32 at a
// time until an inclusive prefix, publishes its own inclusive prefix and returns the exclusive
// one. Chunk 0 starts from seed. Every wait is bounded; running out sets NRRS_DEV_TIMEOUT.
__device__ unsigned lookback(unsigned long long* states, unsigned c, unsigned epoch,
                             unsigned total, unsigned seed, unsigned spin_limit, unsigned* flags) {
    const int lane = threadIdx.x & 31;
    if (c == 0) {
        if (lane == 0) store_state(&states[0], pack_state(epoch, kFlagIncl, sat_add(seed, total)));
        return seed;
    }
    if (lane == 0) store_state(&states[c], pack_state(epoch, kFlagAgg, total));
    int top = (int)c - 1;
    unsigned spins = 0;
    bool timed_out = false;
    unsigned long long acc = 0;
    for (;;) {
        const int idx = top - lane;
        bool ready = true, incl = true;
        unsigned val = 0;
        if (idx >= 0) {
            const unsigned long long w = load_state(&states[idx]);
            const unsigned long long wf = (w >> 32) & 3ull;
            ready = (unsigned)(w >> 34) == (epoch & 0x3fffffffu) && wf != 0;
            incl = wf == kFlagIncl;
            val = (unsigned)w;
        }
        if (!__all_sync(0xffffffffu, ready)) {
            if (++spins > spin_limit) {
                timed_out = true;
                break;
            }
            __nanosleep(32);
            continue;
        }
        const unsigned im = __ballot_sync(0xffffffffu, incl);
        const int stop = im ? __ffs(im) - 1 : 31;
        unsigned long long part = lane <= stop ? (unsigned long long)val : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        acc += part;
        if (im) break;
        top -= 32;
    }
    const unsigned prefix = acc > 0xffffffffull ? 0xffffffffu : (unsigned)acc;
    if (lane == 0) {
        if (timed_out) *flags |= NRRS_DEV_TIMEOUT;
        store_state(&states[c], pack_state(epoch, kFlagIncl, sat_add(prefix, total)));
    }
    return prefix;
}

// Exclusive scan of the 64 per-(pass, warp) counts in s_cnt (pass-major), by warp 0; returns
// the chunk total to every lane.
__device__ __forceinline__ unsigned scan64(unsigned* s_cnt) {
    const int lane = threadIdx.x & 31;
    const unsigned e0 = s_cnt[2 * lane], e1 = s_cnt[2 * lane + 1];
    const unsigned t = e0 + e1;
    unsigned incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    const unsigned excl = incl - t;
    s_cnt[2 * lane] = excl;
    s_cnt[2 * lane + 1] = excl + e0;
    return __shfl_sync(0xffffffffu, incl, 31);
}

// trunc(|x| 2^64) as three limbs signed like x; x finite with |x| < 2^62
__device__ __forceinline__ void fixed_limbs(float x, long long l[3]) {
    const unsigned bits = __float_as_uint(x);
    const unsigned e = (bits >> 23) & 0xffu;
    const unsigned long long m = (bits & 0x7fffffu) | (e ? 0x800000u : 0u);
    const int sh = (int)(e ? e : 1u) - 150 + 64;  // |x| 2^64 = m 2^sh
    unsigned __int128 X;
    if (sh >= 0) X = (unsigned __int128)m << sh;
    else X = (-sh) >= 24 ? (unsigned __int128)0 : (unsigned __int128)(m >> (-sh));
    const unsigned long long lo = (unsigned long long)X;
    long long l0 = (long long)(lo & 0xffffffffull);
    long long l1 = (long long)(lo >> 32);
    long long l2 = (long long)(unsigned long long)(X >> 64);
    if (bits >> 31) { l0 = -l0; l1 = -l1; l2 = -l2; }
    l[0] = l0; l[1] = l1; l[2] = l2;
}

// (l0 + l1 2^32 + l2 2^64) 2^-64 rounded to the nearest float, ties to even
__device__ __forceinline__ float fixed_to_float(long long l0, long long l1, long long l2) {
    using u128 = unsigned __int128;
    const u128 U = ((u128)(__int128)l2 << 64) + ((u128)(__int128)l1 << 32) + (u128)(__int128)l0;
    const unsigned neg = (unsigned)(U >> 127) & 1u;
    const u128 mag = neg ? (u128)0 - U : U;
    if (mag == 0) return 0.0f;
    const unsigned long long hi = (unsigned long long)(mag >> 64), lo = (unsigned long long)mag;
    const int msb = hi ? 127 - __clzll((long long)hi) : 63 - __clzll((long long)lo);
    int ex = msb - 64;
    unsigned mant;
    if (msb <= 23) {
        mant = (unsigned)(lo << (23 - msb));
    } else {
        const int sh = msb - 23;
        const u128 q = mag >> sh;
        const u128 rem = mag - (q << sh);
        const u128 half = (u128)1 << (sh - 1);
        mant = (unsigned)q;
        if (rem > half || (rem == half && (mant & 1u))) {
            ++mant;
            if (mant == (1u << 24)) { mant >>= 1; ++ex; }
        }
    }
    return __uint_as_float((neg << 31) | ((unsigned)(ex + 127) << 23) | (mant & 0x7fffffu));
}

__device__ __forceinline__ bool fixed_ok(float x) { return fabsf(x) < kFixedMax; }

__device__ __forceinline__ void add_limbs(long long* dst, const long long* l) {
#pragma unroll
    for (int k = 0; k < kLimbs; ++k)
        if (l[k]) atomicAdd(reinterpret_cast<unsigned long long*>(dst + k), (unsigned long long)l[k]);
}

// the end-of-launch protocol of the scan kernels: the last CTA restores ticket and done and
// advances the epoch; returns true in that CTA's thread 0
__device__ __forceinline__ bool finish_launch(uint32_t* hdr) {
    __syncthreads();
    if (threadIdx.x != 0) return false;
    __threadfence();
    const unsigned old = atomicAdd(&hdr[kHdrDone], 1u);
    if (old != gridDim.x - 1) return false;
    hdr[kHdrTicket] = 0;
    hdr[kHdrDone] = 0;
    hdr[kHdrEpoch] = hdr[kHdrEpoch] + 1;
    __threadfence();
    return true;
}

// ---- recordNode for a wavefront -------------------------------------------------------------
__global__ void __launch_bounds__(kRecThreads) k_record_nodes(const __grid_constant__ RecordArgs a) {
    __shared__ unsigned s_chunk, s_epoch, s_prefix;
    __shared__ unsigned s_cnt[kRecPasses * (kRecThreads / 32)];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const NodeView& nb = a.nb;
    if (tid == 0) s_epoch = *(volatile unsigned*)&nb.hdr[kHdrEpoch];
    unsigned flags = 0, dropped = 0;
    for (;;) {
        if (tid == 0) s_chunk = atomicAdd(&nb.hdr[kHdrTicket], 1u);
        __syncthreads();
        const unsigned c = s_chunk;
        if (c >= a.chunks) break;
        const unsigned v0 = c * kRecChunk;
        unsigned m[kRecPasses];
#pragma unroll
        for (int j = 0; j < kRecPasses; ++j) {
            const unsigned v = v0 + j * kRecThreads + tid;
            const bool r = v < a.n && (!a.record || a.record[v] != 0);
            m[j] = __ballot_sync(0xffffffffu, r);
            if (lane == 0) s_cnt[j * (kRecThreads / 32) + wid] = __popc(m[j]);
        }
        __syncthreads();
        if (wid == 0) {
            const unsigned total = scan64(s_cnt);
            unsigned seed = 0;
            if (c == 0) seed = __shfl_sync(0xffffffffu, lane == 0 ? *(volatile unsigned*)&nb.hdr[kHdrSize] : 0u, 0);
            const unsigned prefix = lookback(nb.states, c, s_epoch, total, seed, a.spin_limit, &flags);
            if (lane == 0) {
                s_prefix = prefix;
                if (c == a.chunks - 1) {
                    const unsigned end = sat_add(prefix, total);
                    nb.hdr[kHdrSize] = end < nb.capacity ? end : nb.capacity;
                }
            }
        }
        __syncthreads();
        const unsigned lt = lanemask_lt();
#pragma unroll
        for (int j = 0; j < kRecPasses; ++j) {
            const unsigned v = v0 + j * kRecThreads + tid;
            if (v >= a.n) continue;
            const int p = a.parent[v];
            int out = p;
            if ((m[j] >> lane) & 1u) {
                const unsigned long long idx64 = (unsigned long long)s_prefix +
                    s_cnt[j * (kRecThreads / 32) + wid] + __popc(m[j] & lt);
                if (idx64 < nb.capacity) {
                    const unsigned idx = (unsigned)idx64;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const size_t si = 3 * (size_t)v + k, di = 3 * (size_t)idx + k;
                        nb.pos[di] = a.pos[si];
                        nb.wi[di] = a.wi[si];
                        nb.normal[di] = a.normal ? a.normal[si] : 0.f;
                        nb.albedo[di] = a.albedo ? a.albedo[si] : 0.f;
                        nb.thp[di] = a.thp[si];
                    }
                    nb.rough[idx] = a.rough ? a.rough[v] : 0.f;
                    nb.parent[idx] = p;
                    nb.pixel[idx] = a.pixel[v];
                    nb.rrs[idx] = a.rrs ? a.rrs[v] : 1.f;
                    nb.depth[idx] = a.depth ? a.depth[v] : 0u;
                    long long* r = nb.rad + (size_t)idx * kLimbs;
#pragma unroll
                    for (int k = 0; k < kLimbs; ++k) r[k] = 0;
                    nb.first_child[idx] = 0xffffffffu;
                    nb.children[idx] = 0;
                    nb.flags[idx] = 0;
                    if (p >= 0) {
                        if ((unsigned)p < idx) {
                            atomicMin(&nb.first_child[p], idx);
                            atomicAdd(&nb.children[p], 1u);
                        } else {
                            flags |= NRRS_DEV_BAD_INDEX;
                        }
                    }
                    out = (int)idx;
                } else {
                    ++dropped;
                }
            }
            a.node_out[v] = out;
        }
        __syncthreads();
    }
    if (dropped) {
        atomicAdd(&nb.hdr[kHdrDropped], dropped);
        flags |= NRRS_DEV_OVERFLOW;
    }
    if (flags) atomicOr(&nb.hdr[kHdrStatus], flags);
    finish_launch(nb.hdr);
}

// ---- recordRadiance for a queue of contributions -------------------------------------------
__global__ void __launch_bounds__(256) k_record_radiance(const __grid_constant__ RadianceArgs a) {
    const unsigned i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const NodeView& nb = a.nb;
    const int node = a.node[i];
    const unsigned size = nb.hdr[kHdrSize];
    if (node < 0 || (unsigned)node >= size) return;
    const bool walk = nb.hdr[kHdrPropagated] != 0;
    const float x0 = a.contrib[3 * (size_t)i], x1 = a.contrib[3 * (size_t)i + 1],
                x2 = a.contrib[3 * (size_t)i + 2];
    unsigned flags = 0;
    if (!(fixed_ok(x0) && fixed_ok(x1) && fixed_ok(x2))) {
        flags |= NRRS_DEV_NAN;
        int cur = node;
        for (;;) {
            atomicOr(&nb.flags[cur], 1u);
            if (!walk) break;
            const int p = nb.parent[cur];
            if (p < 0) break;
            if (p >= cur) { flags |= NRRS_DEV_BAD_INDEX; break; }
            cur = p;
        }
    } else {
        long long l[kLimbs];
        fixed_limbs(x0, l);
        fixed_limbs(x1, l + 3);
        fixed_limbs(x2, l + 6);
        int cur = node;
        for (;;) {
            add_limbs(nb.rad + (size_t)cur * kLimbs, l);
            if (!walk) break;
            const int p = nb.parent[cur];
            if (p < 0) break;
            if (p >= cur) { flags |= NRRS_DEV_BAD_INDEX; break; }
            cur = p;
        }
    }
    if (flags) atomicOr(&nb.hdr[kHdrStatus], flags);
}

// ---- radiance of the descendants: each node's total into its parent, once --------------------
// A leaf (no children) starts a walk up its chain. After adding a complete node into its parent
// a thread decrements the parent's pending-children count; the child that brings it to zero
// continues with the parent, whose total is then complete. Indices strictly decrease along a
// chain, so every walk ends. Runs once per reset: a later launch returns at once.
__global__ void __launch_bounds__(256) k_propagate(const __grid_constant__ NodeView nb) {
    __shared__ unsigned s_skip;
    if (threadIdx.x == 0) s_skip = *(volatile unsigned*)&nb.hdr[kHdrPropagated];
    __syncthreads();
    unsigned flags = 0;
    if (!s_skip) {
        const unsigned size = nb.hdr[kHdrSize];
        for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < size;
             i += gridDim.x * blockDim.x) {
            if (nb.first_child[i] != 0xffffffffu) continue;  // not a leaf
            unsigned cur = i;
            for (;;) {
                const int p = nb.parent[cur];
                if (p < 0) break;
                if ((unsigned)p >= cur) { flags |= NRRS_DEV_BAD_INDEX; break; }
                long long l[kLimbs];
                const long long* src = nb.rad + (size_t)cur * kLimbs;
#pragma unroll
                for (int k = 0; k < kLimbs; ++k) l[k] = __ldcg(src + k);
                add_limbs(nb.rad + (size_t)p * kLimbs, l);
                const unsigned f = __ldcg(nb.flags + cur);
                if (f) atomicOr(&nb.flags[p], f);
                __threadfence();
                if (atomicSub(&nb.children[p], 1u) != 1u) break;
                __threadfence();
                cur = (unsigned)p;
            }
        }
    }
    if (flags) atomicOr(&nb.hdr[kHdrStatus], flags);
    // the last CTA marks the radiance complete
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned old = atomicAdd(&nb.hdr[kHdrDone], 1u);
        if (old == gridDim.x - 1) {
            nb.hdr[kHdrDone] = 0;
            nb.hdr[kHdrPropagated] = 1;
            __threadfence();
        }
    }
}

// ---- the training batch, in node order ------------------------------------------------------
__global__ void __launch_bounds__(kRecThreads) k_generate(const __grid_constant__ GenerateArgs a) {
    __shared__ unsigned s_chunk, s_epoch, s_prefix;
    __shared__ unsigned s_cnt[kRecPasses * (kRecThreads / 32)];
    __shared__ float s_L[kRecPasses][3][kRecThreads];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const NodeView& nb = a.nb;
    if (tid == 0) s_epoch = *(volatile unsigned*)&nb.hdr[kHdrEpoch];
    const unsigned size = *(volatile unsigned*)&nb.hdr[kHdrSize];
    const unsigned chunks = (size + kRecChunk - 1) / kRecChunk;
    unsigned flags = 0;
    for (;;) {
        if (tid == 0) s_chunk = atomicAdd(&nb.hdr[kHdrTicket], 1u);
        __syncthreads();
        const unsigned c = s_chunk;
        if (c >= chunks) break;
        const unsigned i0 = c * kRecChunk;
        unsigned m[kRecPasses], same_m[kRecPasses];
#pragma unroll
        for (int j = 0; j < kRecPasses; ++j) {
            const unsigned i = i0 + j * kRecThreads + tid;
            bool keep = false, same = false;
            if (i < size) {
                const long long* r = nb.rad + (size_t)i * kLimbs;
                float L[3];
                bool finite = nb.flags[i] == 0;
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    const float rad = fixed_to_float(r[3 * ch], r[3 * ch + 1], r[3 * ch + 2]);
                    const float t = nb.thp[3 * (size_t)i + ch];
                    float l = 0.f;
                    if (t > a.thp_eps) l = __fdiv_rn(rad, t);
                    L[ch] = l < 0.f ? 0.f : l;  // max(L, 0): a NaN stays NaN
                    s_L[j][ch][tid] = L[ch];
                }
                const float mean = __fdiv_rn(__fadd_rn(__fadd_rn(L[0], L[1]), L[2]), 3.0f);
                bool nan = false;
#pragma unroll
                for (int k = 0; k < 3; ++k)
                    nan |= isnan(nb.pos[3 * (size_t)i + k]) || isnan(L[k]);
                nan |= isnan(nb.wi[3 * (size_t)i]) || isnan(nb.wi[3 * (size_t)i + 1]) ||
                       isnan(nb.wi[3 * (size_t)i + 2]);
                keep = finite && !nan && (!a.ignore_zero_l || mean > 0.f);
                if (a.dedupe) {
                    const int p = nb.parent[i];
                    if (p >= 0) {
                        if ((unsigned)p < i) same = nb.first_child[p] != i;
                        else flags |= NRRS_DEV_BAD_INDEX;
                    }
                }
            }
            m[j] = __ballot_sync(0xffffffffu, keep);
            same_m[j] = __ballot_sync(0xffffffffu, same);
            if (lane == 0) s_cnt[j * (kRecThreads / 32) + wid] = __popc(m[j]);
        }
        __syncthreads();
        if (wid == 0) {
            const unsigned total = scan64(s_cnt);
            const unsigned prefix = lookback(nb.states, c, s_epoch, total, 0u, a.spin_limit, &flags);
            if (lane == 0) {
                s_prefix = prefix;
                if (c == chunks - 1) {
                    const unsigned end = sat_add(prefix, total);
                    *a.size_dev = end < a.capacity ? end : a.capacity;
                    if (end > a.capacity) flags |= NRRS_DEV_OVERFLOW;
                }
            }
        }
        __syncthreads();
        const unsigned lt = lanemask_lt();
        const nrrs_train_batch& o = a.out;
#pragma unroll
        for (int j = 0; j < kRecPasses; ++j) {
            if (!((m[j] >> lane) & 1u)) continue;
            const unsigned i = i0 + j * kRecThreads + tid;
            const unsigned long long t64 = (unsigned long long)s_prefix +
                s_cnt[j * (kRecThreads / 32) + wid] + __popc(m[j] & lt);
            if (t64 >= a.capacity) continue;
            const size_t t = (size_t)t64;
            const bool same = (same_m[j] >> lane) & 1u;
            const float rrs = nb.rrs[i];
            const unsigned px = nb.pixel[i];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                if (o.pos) o.pos[3 * t + k] = nb.pos[3 * (size_t)i + k];
                if (o.wi) o.wi[3 * t + k] = nb.wi[3 * (size_t)i + k];
                if (o.normal) o.normal[3 * t + k] = nb.normal[3 * (size_t)i + k];
                if (o.albedo) o.albedo[3 * t + k] = nb.albedo[3 * (size_t)i + k];
                if (o.target) o.target[3 * t + k] = s_L[j][k][tid];
                const float th = nb.thp[3 * (size_t)i + k];
                if (o.thp) o.thp[3 * t + k] = a.copy_rrs_node ? __fmul_rn(th, rrs) : th;
            }
            if (o.roughness) o.roughness[t] = nb.rough[i];
            if (o.depth) o.depth[t] = nb.depth[i];
            if (o.rrs_target) o.rrs_target[t] = same ? -1.0f : rrs;
            if (o.pixel) o.pixel[t] = px;
            const bool px_ok = px < a.n_pixels;
            if (!px_ok && (a.image || a.pixel_samples)) flags |= NRRS_DEV_BAD_INDEX;
            if (o.ref_mean && a.image) {
                float rm = 0.f;
                if (px_ok) {
                    const float* q = a.image + (size_t)px * a.channels;
                    rm = __fdiv_rn(__fadd_rn(__fadd_rn(q[0], q[1]), q[2]), 3.0f);
                }
                o.ref_mean[t] = rm;
            }
            if (!same && px_ok && a.pixel_samples) atomicAdd(&a.pixel_samples[px], 1u);
        }
        __syncthreads();
    }
    if (flags) atomicOr(&nb.hdr[kHdrStatus], flags);
    if (finish_launch(nb.hdr) && chunks == 0) *a.size_dev = 0;
}

// ---- 1 / samples of the sample's pixel -------------------------------------------------------
__global__ void __launch_bounds__(256) k_sample_weights(const __grid_constant__ WeightArgs a) {
    const unsigned t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.max_n || t >= *a.size_dev) return;
    const unsigned px = a.pixel[t];
    const unsigned cnt = px < a.n_pixels ? a.pixel_samples[px] : 0u;
    a.weight[t] = cnt ? __fdiv_rn(1.0f, (float)cnt) : 0.0f;
}

}  // namespace

cudaError_t launch_record_nodes(const RecordArgs& a, int grid, cudaStream_t s) {
    if (a.chunks == 0) return cudaSuccess;
    k_record_nodes<<<grid, kRecThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_record_radiance(const RadianceArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    k_record_radiance<<<(a.n + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_propagate(const NodeView& nb, int grid, cudaStream_t s) {
    k_propagate<<<grid, 256, 0, s>>>(nb);
    return cudaGetLastError();
}

cudaError_t launch_generate(const GenerateArgs& a, int grid, cudaStream_t s) {
    k_generate<<<grid, kRecThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sample_weights(const WeightArgs& a, cudaStream_t s) {
    if (a.max_n == 0) return cudaSuccess;
    k_sample_weights<<<(a.max_n + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nrrs
