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
//     look-back over 1024-element chunks (one ballot per warp and pass); the whole CTA reads
//     256 predecessor states per look-back step;
//   * radiance is a fixed-point integer, three signed 64-bit limbs per channel with the lowest
//     bit worth 2^-64: a contribution x (|x| < 2^62) becomes trunc(|x| 2^64) split into a
//     32-bit low limb, a 32-bit middle limb and the integer part, each signed like x. Integer
//     additions commute, so every node total is the same integer in any order;
//   * a contribution is added to its own node only; one pass then adds each node's complete
//     total into its parent once, walking up from the leaves: an only child hands its total up in
//     registers (plain loads and stores), siblings add theirs with atomics and the last to arrive
//     carries on. That is one addition per node instead of one per ancestor per contribution;
//   * a warp's compacted outputs form one contiguous run, so three-float fields go out through a
//     small per-warp shared-memory stage as contiguous words, and every field of an element is
//     loaded before any is stored.
#include <cmath>

#include "records.hpp"
#include "fixed_point.cuh"
#include "tc_ptx.cuh"

namespace nrrs {

namespace {

constexpr unsigned long long kFlagAgg = 1ull;
constexpr unsigned long long kFlagIncl = 2ull;

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

// Called by every thread of the CTA. Publishes this chunk's total, reads the 256 predecessor
// states below a window top until an inclusive prefix, publishes its own inclusive prefix and
// returns the exclusive one (to every thread). Chunk 0 starts from seed. Every wait is bounded;
// running out sets NRRS_DEV_TIMEOUT.
struct LookbackSmem {
    unsigned first[kRecThreads / 32];
    unsigned long long part[kRecThreads / 32];
};

__device__ unsigned lookback_block(unsigned long long* states, unsigned c, unsigned epoch,
                                   unsigned total, unsigned seed, unsigned spin_limit,
                                   unsigned* flags, LookbackSmem& sm) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (c == 0) {
        if (tid == 0) store_state(&states[0], pack_state(epoch, kFlagIncl, sat_add(seed, total)));
        return seed;
    }
    if (tid == 0) store_state(&states[c], pack_state(epoch, kFlagAgg, total));
    int top = (int)c - 1;
    unsigned spins = 0;
    bool timed_out = false;
    unsigned long long acc = 0;
    for (;;) {
        const int idx = top - tid;
        bool ready = true, incl = true;
        unsigned val = 0;
        if (idx >= 0) {
            const unsigned long long w = load_state(&states[idx]);
            const unsigned long long wf = (w >> 32) & 3ull;
            ready = (unsigned)(w >> 34) == (epoch & 0x3fffffffu) && wf != 0;
            incl = wf == kFlagIncl;
            val = (unsigned)w;
        }
        if (!__syncthreads_and(ready)) {
            if (++spins > spin_limit) {
                timed_out = true;
                break;
            }
            __nanosleep(64);
            continue;
        }
        const unsigned im = __ballot_sync(0xffffffffu, incl);
        if (lane == 0) sm.first[wid] = im ? (unsigned)(wid * 32 + __ffs(im) - 1) : 0xffffffffu;
        __syncthreads();
        unsigned stop = 0xffffffffu;
#pragma unroll
        for (int k = 0; k < kRecThreads / 32; ++k) stop = min(stop, sm.first[k]);
        unsigned long long part = (unsigned)tid <= stop ? (unsigned long long)val : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if (lane == 0) sm.part[wid] = part;
        __syncthreads();
#pragma unroll
        for (int k = 0; k < kRecThreads / 32; ++k) acc += sm.part[k];
        __syncthreads();
        if (stop != 0xffffffffu) break;
        top -= kRecThreads;
    }
    const unsigned prefix = acc > 0xffffffffull ? 0xffffffffu : (unsigned)acc;
    if (tid == 0) {
        if (timed_out) *flags |= NRRS_DEV_TIMEOUT;
        store_state(&states[c], pack_state(epoch, kFlagIncl, sat_add(prefix, total)));
    }
    return prefix;
}

// Exclusive scan, by warp 0, of the N (<= 32) per-(pass, warp) counts in s_cnt (pass-major,
// one per lane); returns the total to every lane of warp 0.
template <int N = kRecPasses * (kRecThreads / 32)>
__device__ __forceinline__ unsigned scan_counts(unsigned* s_cnt) {
    static_assert(N <= 32, "one count per lane");
    const int lane = threadIdx.x & 31;
    const unsigned t = lane < N ? s_cnt[lane] : 0u;
    unsigned incl = t;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane < N) s_cnt[lane] = incl - t;
    return __shfl_sync(0xffffffffu, incl, 31);
}

// A warp's compacted three-float records: lane `rank` holds one (when `active`), the warp's
// records go to dst[0 .. 3*cnt) as contiguous words through the per-warp stage of 96 floats.
__device__ __forceinline__ void store3_compact(float* dst, bool active, unsigned rank,
                                               unsigned cnt, float x, float y, float z,
                                               float* stage) {
    const int lane = threadIdx.x & 31;
    if (active) {
        stage[3 * rank] = x;
        stage[3 * rank + 1] = y;
        stage[3 * rank + 2] = z;
    }
    __syncwarp();
    for (unsigned j = lane; j < 3 * cnt; j += 32) dst[j] = stage[j];
    __syncwarp();
}

__device__ __forceinline__ unsigned atom_add_acq_rel(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

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
// One chunk of the wavefront's inputs at a time in shared memory: with BULK every array of a full
// chunk arrives by one unicast bulk copy each on one mbarrier (all bytes in flight at once); the
// last, partial chunk and inputs not 16-byte aligned are copied by the threads in coalesced
// loops. Two CTAs per SM.
constexpr int kWrThreads = 512;                      // write kernel: 16 warps, 2 passes
constexpr int kWrPasses = kRecChunk / kWrThreads;

struct RecordStage {
    float pos[3 * kRecChunk], wi[3 * kRecChunk], nrm[3 * kRecChunk], alb[3 * kRecChunk],
        thp[3 * kRecChunk];
    float rough[kRecChunk], rrs[kRecChunk];
    unsigned depth[kRecChunk], pixel[kRecChunk];
    int parent[kRecChunk];
    uint8_t record[kRecChunk];
    uint64_t bar;
};

template <typename T>
__device__ __forceinline__ void copy_in(T* dst, const T* __restrict__ src, unsigned count) {
    for (unsigned j = threadIdx.x; j < count; j += blockDim.x) dst[j] = src[j];
}

// Counts of the chunks' records; the last CTA to finish turns them into node offsets (from the
// node count at the start of the call), sets the new node count and appends the call to the
// level table. No CTA waits for another.
__global__ void __launch_bounds__(kRecThreads) k_record_count(const __grid_constant__ RecordArgs a) {
    __shared__ unsigned s_part[kRecThreads / 32];
    __shared__ unsigned s_last;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const NodeView& nb = a.nb;
    const unsigned c = blockIdx.x, v0 = c * kRecChunk;
    const unsigned cnt_c = min((unsigned)kRecChunk, a.n - v0);
    unsigned k = 0;
    if (a.record) {
#pragma unroll
        for (int j = 0; j < kRecPasses; ++j) {
            const unsigned lv = j * kRecThreads + tid;
            k += (lv < cnt_c && a.record[v0 + lv] != 0) ? 1u : 0u;
        }
    } else if (tid == 0) {
        k = cnt_c;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
    if (lane == 0) s_part[wid] = k;
    __syncthreads();
    if (tid == 0) {
        unsigned t = 0;
#pragma unroll
        for (int w = 0; w < kRecThreads / 32; ++w) t += s_part[w];
        a.chunk_count[c] = t;
        __threadfence();
        s_last = atomicAdd(&nb.hdr[kHdrDone], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    // ---- the last CTA: exclusive scan of every chunk's count ----
    __threadfence();
    const unsigned chunks = a.chunks;
    const unsigned per = (chunks + kRecThreads - 1) / kRecThreads;  // a strip per thread
    const unsigned lo = min(chunks, tid * per), hi = min(chunks, lo + per);
    unsigned long long strip = 0;
    for (unsigned q = lo; q < hi; ++q) strip += __ldcg(a.chunk_count + q);
    // block exclusive scan of the strip sums
    unsigned long long incl = strip;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    __shared__ unsigned long long s_w[kRecThreads / 32];
    if (lane == 31) s_w[wid] = incl;
    __syncthreads();
    unsigned long long before = 0;
    for (int w = 0; w < wid; ++w) before += s_w[w];
    const unsigned base = *(volatile unsigned*)&nb.hdr[kHdrSize];
    unsigned long long run = base + before + incl - strip;
    for (unsigned q = lo; q < hi; ++q) {
        a.chunk_offset[q] = run > 0xffffffffull ? 0xffffffffu : (unsigned)run;
        run += __ldcg(a.chunk_count + q);
    }
    __syncthreads();
    if (tid == kRecThreads - 1) {
        const unsigned long long end = run;   // the last thread's strip ends the scan
        const unsigned sz = end < nb.capacity ? (unsigned)end : nb.capacity;
        nb.hdr[kHdrCallBase] = base;
        nb.hdr[kHdrSize] = sz;
        const unsigned L = nb.hdr[kHdrLevels];
        if (L < (unsigned)kMaxLevels) nb.hdr[kHdrLevelTable + L] = sz;
        if (L <= (unsigned)kMaxLevels) nb.hdr[kHdrLevels] = L + 1;
        nb.hdr[kHdrDone] = 0;
        __threadfence();
    }
}

// The writes: every chunk knows its first node index, so chunks run independently. With BULK
// the inputs of a full chunk arrive by unicast bulk copies on one mbarrier.
template <bool BULK>
__global__ void __launch_bounds__(kWrThreads, 2)
k_record_nodes(const __grid_constant__ RecordArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    RecordStage& S = *reinterpret_cast<RecordStage*>(smem_raw);
    __shared__ unsigned s_cnt[kWrPasses * (kWrThreads / 32)];
    __shared__ float s_stage[kWrThreads / 32][96];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const NodeView& nb = a.nb;
    const unsigned c = blockIdx.x, v0 = c * kRecChunk;
    const unsigned cnt_c = min((unsigned)kRecChunk, a.n - v0);
    unsigned flags = 0, dropped = 0;
    if (BULK && cnt_c == (unsigned)kRecChunk) {
        if (tid == 0) {
            tc::mbar_init(&S.bar, 1);
            tc::fence_mbar_init();
            const unsigned v3 = 3 * kRecChunk * 4, v1 = kRecChunk * 4;
            const unsigned bytes = v3 * (3 + (a.normal ? 1 : 0) + (a.albedo ? 1 : 0)) +
                                   v1 * (2 + (a.rough ? 1 : 0) + (a.rrs ? 1 : 0) +
                                         (a.depth ? 1 : 0)) +
                                   (a.record ? kRecChunk : 0);
            tc::mbar_arrive_expect_tx(&S.bar, bytes);
            tc::bulk_g2s(S.pos, a.pos + 3 * (size_t)v0, v3, &S.bar);
            tc::bulk_g2s(S.wi, a.wi + 3 * (size_t)v0, v3, &S.bar);
            tc::bulk_g2s(S.thp, a.thp + 3 * (size_t)v0, v3, &S.bar);
            if (a.normal) tc::bulk_g2s(S.nrm, a.normal + 3 * (size_t)v0, v3, &S.bar);
            if (a.albedo) tc::bulk_g2s(S.alb, a.albedo + 3 * (size_t)v0, v3, &S.bar);
            tc::bulk_g2s(S.pixel, a.pixel + v0, v1, &S.bar);
            tc::bulk_g2s(S.parent, a.parent + v0, v1, &S.bar);
            if (a.rough) tc::bulk_g2s(S.rough, a.rough + v0, v1, &S.bar);
            if (a.rrs) tc::bulk_g2s(S.rrs, a.rrs + v0, v1, &S.bar);
            if (a.depth) tc::bulk_g2s(S.depth, a.depth + v0, v1, &S.bar);
            if (a.record) tc::bulk_g2s(S.record, a.record + v0, kRecChunk, &S.bar);
        }
        __syncthreads();  // the barrier is initialised before anyone waits on it
        if (!tc::mbar_wait(&S.bar, 0, a.spin_limit)) {
            // the copies must land before this CTA's shared memory can be given up
            tc::mbar_wait(&S.bar, 0, a.spin_limit);
            if (tid == 0) atomicOr(&nb.hdr[kHdrStatus], NRRS_DEV_TIMEOUT);
            return;
        }
    } else {
        copy_in(S.pos, a.pos + 3 * (size_t)v0, 3 * cnt_c);
        copy_in(S.wi, a.wi + 3 * (size_t)v0, 3 * cnt_c);
        copy_in(S.thp, a.thp + 3 * (size_t)v0, 3 * cnt_c);
        if (a.normal) copy_in(S.nrm, a.normal + 3 * (size_t)v0, 3 * cnt_c);
        if (a.albedo) copy_in(S.alb, a.albedo + 3 * (size_t)v0, 3 * cnt_c);
        copy_in(S.pixel, a.pixel + v0, cnt_c);
        copy_in(S.parent, a.parent + v0, cnt_c);
        if (a.rough) copy_in(S.rough, a.rough + v0, cnt_c);
        if (a.rrs) copy_in(S.rrs, a.rrs + v0, cnt_c);
        if (a.depth) copy_in(S.depth, a.depth + v0, cnt_c);
        if (a.record) copy_in(S.record, a.record + v0, cnt_c);
        __syncthreads();
    }
    const unsigned call0 = *(volatile unsigned*)&nb.hdr[kHdrCallBase];
    const unsigned prefix = a.chunk_offset[c];
    unsigned m[kWrPasses];
#pragma unroll
    for (int j = 0; j < kWrPasses; ++j) {
        const unsigned lv = j * kWrThreads + tid;
        const bool r = lv < cnt_c && (!a.record || S.record[lv] != 0);
        m[j] = __ballot_sync(0xffffffffu, r);
        if (lane == 0) s_cnt[j * (kWrThreads / 32) + wid] = __popc(m[j]);
    }
    __syncthreads();
    if (wid == 0) scan_counts<kWrPasses * (kWrThreads / 32)>(s_cnt);
    __syncthreads();
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int j = 0; j < kWrPasses; ++j) {
        const unsigned lv = j * kWrThreads + tid;
        const unsigned v = v0 + lv;
        const bool valid = lv < cnt_c;
        const bool active = (m[j] >> lane) & 1u;
        const unsigned rank = __popc(m[j] & lt);
        const unsigned long long base = (unsigned long long)prefix + s_cnt[j * (kWrThreads / 32) + wid];
        const unsigned cnt = __popc(m[j]);
        const unsigned room = base >= nb.capacity ? 0u
                              : (unsigned)min((unsigned long long)cnt, nb.capacity - base);
        const bool keep = active && rank < room;
        const int p = valid ? S.parent[lv] : 0;
        // a parent must be a node of an earlier call: any other link is cut and flagged
        const bool bad_parent = p >= 0 && (unsigned)p >= call0;
        const int pn = bad_parent ? -1 : p;
        const unsigned idx = (unsigned)(base + rank);
        if (room) {  // warp-uniform
            const unsigned l3 = 3 * lv;
            store3_compact(nb.pos + 3 * base, keep, rank, room, S.pos[l3], S.pos[l3 + 1],
                           S.pos[l3 + 2], s_stage[wid]);
            store3_compact(nb.wi + 3 * base, keep, rank, room, S.wi[l3], S.wi[l3 + 1],
                           S.wi[l3 + 2], s_stage[wid]);
            store3_compact(nb.normal + 3 * base, keep, rank, room,
                           a.normal ? S.nrm[l3] : 0.f, a.normal ? S.nrm[l3 + 1] : 0.f,
                           a.normal ? S.nrm[l3 + 2] : 0.f, s_stage[wid]);
            store3_compact(nb.albedo + 3 * base, keep, rank, room,
                           a.albedo ? S.alb[l3] : 0.f, a.albedo ? S.alb[l3 + 1] : 0.f,
                           a.albedo ? S.alb[l3 + 2] : 0.f, s_stage[wid]);
            store3_compact(nb.thp + 3 * base, keep, rank, room, S.thp[l3], S.thp[l3 + 1],
                           S.thp[l3 + 2], s_stage[wid]);
            long long* r = nb.rad + (size_t)base * kLimbs;
            for (unsigned k = lane; k < kLimbs * room; k += 32) r[k] = 0;
        }
        if (keep) {
            nb.rough[idx] = a.rough ? S.rough[lv] : 0.f;
            nb.parent[idx] = pn;
            nb.pixel[idx] = S.pixel[lv];
            nb.rrs[idx] = a.rrs ? S.rrs[lv] : 1.f;
            nb.depth[idx] = a.depth ? S.depth[lv] : 0u;
            nb.first_child[idx] = 0xffffffffu;
            nb.children[idx] = 0;
            nb.arrived[idx] = 0;
            nb.flags[idx] = 0;
            if (pn >= 0) {
                atomicMin(&nb.first_child[pn], idx);
                atomicAdd(&nb.children[pn], 1u);
            }
            if (bad_parent) flags |= NRRS_DEV_BAD_INDEX;
        } else if (active) {
            ++dropped;
        }
        if (valid) a.node_out[v] = keep ? (int)idx : p;
    }
    if (dropped) {
        atomicAdd(&nb.hdr[kHdrDropped], dropped);
        flags |= NRRS_DEV_OVERFLOW;
    }
    if (flags) atomicOr(&nb.hdr[kHdrStatus], flags);
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

// ---- radiance of the descendants ------------------------------------------------------------
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Barrier of a cooperative (co-resident) grid on two header words; the wait is bounded and
// running out sets NRRS_DEV_TIMEOUT.
__device__ void grid_barrier(uint32_t* hdr, unsigned spin_limit, unsigned* flags) {
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned* count = hdr + kHdrBarCount;
        unsigned* gen = hdr + kHdrBarGen;
        const unsigned g = ld_acquire(gen);
        __threadfence();
        if (atomicAdd(count, 1u) == gridDim.x - 1) {
            *(volatile unsigned*)count = 0;
            st_release(gen, g + 1u);
        } else {
            unsigned spins = 0;
            while (ld_acquire(gen) == g) {
                if (++spins > spin_limit) {
                    *flags |= NRRS_DEV_TIMEOUT;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
    }
    __syncthreads();
}

// Level by level: the nodes of one record call all have their parents in earlier calls, so going
// from the last call to the first, every node's total is complete when its level comes and is
// added into its parent once, with atomics and no waiting; a grid barrier separates levels.
__device__ void propagate_levels(const NodeView& nb, unsigned levels, unsigned spin_limit,
                                 unsigned* flags) {
    const unsigned* lt = nb.hdr + kHdrLevelTable;
    const int lane = threadIdx.x & 31;
    const unsigned warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const unsigned warps = (gridDim.x * blockDim.x) >> 5;
    constexpr int G = 2;  // 32-node groups per warp and step, loaded before any addition
    for (int k = (int)levels - 1; k >= 1; --k) {
        const unsigned lo = lt[k - 1], hi = lt[k];
        for (unsigned g0 = lo + 32u * warp * G; g0 < hi; g0 += 32u * warps * G) {
            // lane l holds limb word l + 32 q of each group's 32 x 9 words, and the group's
            // parent and flags of node l
            long long w[G][kLimbs];
            int par[G];
            unsigned fl[G];
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const unsigned gb = g0 + 32u * g;
                const unsigned nn = gb < hi ? min(32u, hi - gb) : 0u;
                par[g] = lane < (int)nn ? __ldcg(nb.parent + gb + lane) : -1;
                fl[g] = lane < (int)nn ? __ldcg(nb.flags + gb + lane) : 0u;
                const long long* src = nb.rad + (size_t)gb * kLimbs;
#pragma unroll
                for (int q = 0; q < kLimbs; ++q) {
                    const unsigned word = lane + 32u * q;
                    w[g][q] = word < kLimbs * nn ? __ldcg(src + word) : 0ll;
                }
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
#pragma unroll
                for (int q = 0; q < kLimbs; ++q) {
                    const unsigned word = lane + 32u * q;
                    const int node = word / kLimbs;   // 0..31 within the group
                    const int pp = __shfl_sync(0xffffffffu, par[g], node);
                    if (pp >= 0 && w[g][q] != 0)
                        atomicAdd(reinterpret_cast<unsigned long long*>(nb.rad + (size_t)pp * kLimbs +
                                                                        (word - node * kLimbs)),
                                  (unsigned long long)w[g][q]);
                }
                if (par[g] >= 0 && (fl[g] & 1u)) atomicOr(&nb.flags[par[g]], 1u);
            }
        }
        grid_barrier(nb.hdr, spin_limit, flags);
    }
}

// Walking the parent chains, for more record calls than the level table keeps. A leaf starts a
// walk carrying the complete total of the node it stands on. Into an only child's parent the
// total goes by plain loads and stores: nobody else touches that parent. Into a parent with
// siblings it goes by atomic additions, and an acquire-release count of arrivals tells the last
// sibling, which reads the parent's now complete total and carries on. Indices strictly
// decrease along a chain, so every walk ends.
__device__ void propagate_chains(const NodeView& nb, unsigned* flags) {
    const unsigned size = nb.hdr[kHdrSize];
    for (unsigned i = blockIdx.x * blockDim.x + threadIdx.x; i < size;
         i += gridDim.x * blockDim.x) {
        if (nb.first_child[i] != 0xffffffffu) continue;  // not a leaf
        unsigned cur = i;
        long long t[kLimbs];
        const long long* src = nb.rad + (size_t)i * kLimbs;
#pragma unroll
        for (int k = 0; k < kLimbs; ++k) t[k] = src[k];
        unsigned bad = nb.flags[i] & 1u;
        for (;;) {
            const int p = nb.parent[cur];
            if (p < 0) break;
            if ((unsigned)p >= cur) { *flags |= NRRS_DEV_BAD_INDEX; break; }
            long long* dst = nb.rad + (size_t)p * kLimbs;
            const unsigned nc = nb.children[p];
            if (nc == 1u) {
                long long own[kLimbs];
#pragma unroll
                for (int k = 0; k < kLimbs; ++k) own[k] = dst[k];
                const unsigned pf = nb.flags[p];
#pragma unroll
                for (int k = 0; k < kLimbs; ++k) {
                    t[k] = (long long)((unsigned long long)t[k] + (unsigned long long)own[k]);
                    dst[k] = t[k];
                }
                bad |= pf & 1u;
                if (bad && !(pf & 1u)) nb.flags[p] = pf | 1u;
            } else {
                add_limbs(dst, t);
                if (bad) atomicOr(&nb.flags[p], 1u);
                if (atom_add_acq_rel(&nb.arrived[p], 1u) + 1u != nc) break;
#pragma unroll
                for (int k = 0; k < kLimbs; ++k) t[k] = __ldcg(dst + k);
                bad = __ldcg(nb.flags + p) & 1u;
            }
            cur = (unsigned)p;
        }
    }
}

// One cooperative launch; runs once per reset (a later launch returns at once).
__global__ void __launch_bounds__(256) k_propagate(const __grid_constant__ NodeView nb,
                                                   unsigned spin_limit) {
    __shared__ unsigned s_skip, s_levels;
    if (threadIdx.x == 0) {
        s_skip = *(volatile unsigned*)&nb.hdr[kHdrPropagated];
        s_levels = *(volatile unsigned*)&nb.hdr[kHdrLevels];
    }
    __syncthreads();
    if (s_skip) return;  // the same in every CTA: the mark is only set after the last barrier
    unsigned flags = 0;
    if (s_levels <= (unsigned)kMaxLevels) propagate_levels(nb, s_levels, spin_limit, &flags);
    else propagate_chains(nb, &flags);
    if (flags) atomicOr(&nb.hdr[kHdrStatus], flags);
    grid_barrier(nb.hdr, spin_limit, &flags);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        nb.hdr[kHdrPropagated] = 1;
        if (flags & NRRS_DEV_TIMEOUT) atomicOr(&nb.hdr[kHdrStatus], NRRS_DEV_TIMEOUT);
    }
}

// ---- the training batch, in node order ------------------------------------------------------
__global__ void __launch_bounds__(kRecThreads, 5) k_generate(const __grid_constant__ GenerateArgs a) {
    __shared__ unsigned s_chunk, s_epoch;
    __shared__ unsigned s_cnt[kRecPasses * (kRecThreads / 32)];
    __shared__ unsigned s_keep[kRecPasses][kRecThreads / 32], s_same[kRecPasses][kRecThreads / 32];
    __shared__ LookbackSmem s_lb;
    __shared__ float s_L[kRecPasses][3][kRecThreads];
    __shared__ float s_stage[kRecThreads / 32][96];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const NodeView& nb = a.nb;
    if (tid == 0) s_epoch = *(volatile unsigned*)&nb.hdr[kHdrEpoch];
    const unsigned size = *(volatile unsigned*)&nb.hdr[kHdrSize];
    const unsigned chunks = (size + kRecChunk - 1) / kRecChunk;
    const unsigned lt = lanemask_lt();
    unsigned flags = 0;
    for (;;) {
        if (tid == 0) s_chunk = atomicAdd(&nb.hdr[kHdrTicket], 1u);
        __syncthreads();
        const unsigned c = s_chunk;
        if (c >= chunks) break;
        const unsigned i0 = c * kRecChunk;
#pragma unroll
        for (int j = 0; j < kRecPasses; ++j) {
            const unsigned i = i0 + j * kRecThreads + tid;
            bool keep = false, same = false;
            if (i < size) {
                long long r[kLimbs];
                const long long* rp = nb.rad + (size_t)i * kLimbs;
#pragma unroll
                for (int k = 0; k < kLimbs; ++k) r[k] = rp[k];
                float th[3], ps[3], w[3];
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    th[k] = nb.thp[3 * (size_t)i + k];
                    ps[k] = nb.pos[3 * (size_t)i + k];
                    w[k] = nb.wi[3 * (size_t)i + k];
                }
                const unsigned nf = nb.flags[i];
                const int p = a.dedupe ? nb.parent[i] : -1;
                unsigned fc = 0;
                if (p >= 0) {
                    if ((unsigned)p < i) fc = nb.first_child[p];
                    else flags |= NRRS_DEV_BAD_INDEX;
                }
                float L[3];
#pragma unroll
                for (int ch = 0; ch < 3; ++ch) {
                    const float rad = fixed_to_float(r[3 * ch], r[3 * ch + 1], r[3 * ch + 2]);
                    float l = 0.f;
                    if (th[ch] > a.thp_eps) l = __fdiv_rn(rad, th[ch]);
                    L[ch] = l < 0.f ? 0.f : l;  // max(L, 0): a NaN stays NaN
                    s_L[j][ch][tid] = L[ch];
                }
                const float mean = __fdiv_rn(__fadd_rn(__fadd_rn(L[0], L[1]), L[2]), 3.0f);
                bool nan = false;
#pragma unroll
                for (int k = 0; k < 3; ++k) nan |= isnan(ps[k]) || isnan(w[k]) || isnan(L[k]);
                keep = (nf & 1u) == 0 && !nan && (!a.ignore_zero_l || mean > 0.f);
                same = p >= 0 && (unsigned)p < i && fc != i;
            }
            const unsigned mk = __ballot_sync(0xffffffffu, keep);
            const unsigned ms = __ballot_sync(0xffffffffu, same);
            if (lane == 0) {
                s_cnt[j * (kRecThreads / 32) + wid] = __popc(mk);
                s_keep[j][wid] = mk;
                s_same[j][wid] = ms;
            }
        }
        __syncthreads();
        unsigned total = 0;
        if (wid == 0) total = scan_counts(s_cnt);
        if (tid == 0) s_lb.part[0] = total;
        __syncthreads();
        total = (unsigned)s_lb.part[0];
        __syncthreads();
        const unsigned prefix = lookback_block(nb.states, c, s_epoch, total, 0u, a.spin_limit,
                                               &flags, s_lb);
        if (tid == 0 && c == chunks - 1) {
            const unsigned end = sat_add(prefix, total);
            *a.size_dev = end < a.capacity ? end : a.capacity;
            if (end > a.capacity) flags |= NRRS_DEV_OVERFLOW;
        }
        const nrrs_train_batch& o = a.out;
#pragma unroll
        for (int j = 0; j < kRecPasses; ++j) {
            const unsigned i = i0 + j * kRecThreads + tid;
            const unsigned mk = s_keep[j][wid];
            const bool active = (mk >> lane) & 1u;
            const unsigned rank = __popc(mk & lt);
            const unsigned long long base = (unsigned long long)prefix + s_cnt[j * (kRecThreads / 32) + wid];
            const unsigned cnt = __popc(mk);
            const unsigned room = base >= a.capacity ? 0u
                                  : (unsigned)min((unsigned long long)cnt, a.capacity - base);
            if (room == 0) continue;  // warp-uniform
            const bool keep = active && rank < room;
            const bool same = (s_same[j][wid] >> lane) & 1u;
            // every field first, then the stores
            float q[15], rough = 0.f, rrs = 0.f, rm = 0.f, er = 0.f, era = 0.f, ns = 0.f;
            unsigned px = 0, dep = 0;
#pragma unroll
            for (int k = 0; k < 15; ++k) q[k] = 0.f;
            bool px_ok = false;
            if (keep) {
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const size_t si = 3 * (size_t)i + k;
                    q[k] = nb.pos[si];
                    q[3 + k] = nb.wi[si];
                    q[6 + k] = nb.normal[si];
                    q[9 + k] = nb.albedo[si];
                    q[12 + k] = nb.thp[si];
                }
                rough = nb.rough[i];
                rrs = nb.rrs[i];
                dep = nb.depth[i];
                px = nb.pixel[i];
                px_ok = px < a.n_pixels;
                if (px_ok) {
                    // the sample's patch of the film and error images (offsetFrame2Scaled)
                    const unsigned pq = a.scale > 1u
                        ? (px % a.frame_width) / a.scale +
                              ((px / a.frame_width) / a.scale) * (a.frame_width / a.scale)
                        : px;
                    if (a.image) {
                        const float* im = a.image + (size_t)pq * a.channels;
                        rm = __fdiv_rn(__fadd_rn(__fadd_rn(im[0], im[1]), im[2]), 3.0f);
                    }
                    if (a.error_pp) {
                        er = a.error_pp[pq];
                        era = a.error_pp[(size_t)a.n_pixels + pq];
                    }
                    if (a.spp_patch) ns = a.spp_patch[pq];
                }
                if (a.copy_rrs_node) {
#pragma unroll
                    for (int k = 12; k < 15; ++k) q[k] = __fmul_rn(q[k], rrs);
                }
            }
            const size_t t = (size_t)(base + rank);
            if (o.pos) store3_compact(o.pos + 3 * base, keep, rank, room, q[0], q[1], q[2], s_stage[wid]);
            if (o.wi) store3_compact(o.wi + 3 * base, keep, rank, room, q[3], q[4], q[5], s_stage[wid]);
            if (o.normal) store3_compact(o.normal + 3 * base, keep, rank, room, q[6], q[7], q[8], s_stage[wid]);
            if (o.albedo) store3_compact(o.albedo + 3 * base, keep, rank, room, q[9], q[10], q[11], s_stage[wid]);
            if (o.thp) store3_compact(o.thp + 3 * base, keep, rank, room, q[12], q[13], q[14], s_stage[wid]);
            if (o.target) store3_compact(o.target + 3 * base, keep, rank, room, s_L[j][0][tid],
                                         s_L[j][1][tid], s_L[j][2][tid], s_stage[wid]);
            if (keep) {
                if (o.roughness) o.roughness[t] = rough;
                if (o.depth) o.depth[t] = dep;
                if (o.rrs_target) o.rrs_target[t] = same ? -1.0f : rrs;
                if (o.pixel) o.pixel[t] = px;
                if (!px_ok && (a.image || a.pixel_samples || a.error_pp || a.spp_patch))
                    flags |= NRRS_DEV_BAD_INDEX;
                if (o.ref_mean && a.image) o.ref_mean[t] = rm;
                if (o.error && a.error_pp) o.error[t] = er;
                if (o.error_for_avg && a.error_pp) o.error_for_avg[t] = era;
                if (o.number_samples && a.spp_patch) o.number_samples[t] = ns;
                if (!same && px_ok && a.pixel_samples) atomicAdd(&a.pixel_samples[px], 1u);
            }
        }
        __syncthreads();
    }
    if (flags) atomicOr(&nb.hdr[kHdrStatus], flags);
    if (finish_launch(nb.hdr) && chunks == 0) *a.size_dev = 0;
}

// ---- 1 / samples of the sample's pixel -------------------------------------------------------
__global__ void __launch_bounds__(256) k_sample_weights(const __grid_constant__ WeightArgs a) {
    const unsigned n = min(a.max_n, *a.size_dev);
    for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const unsigned px = a.pixel[t];
        const unsigned cnt = px < a.n_pixels ? a.pixel_samples[px] : 0u;
        a.weight[t] = cnt ? __fdiv_rn(1.0f, (float)cnt) : 0.0f;
    }
}

}  // namespace

cudaError_t launch_record_nodes(const RecordArgs& a, cudaStream_t s) {
    if (a.chunks == 0) return cudaSuccess;
    auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    const bool bulk = al(a.pos) && al(a.wi) && al(a.thp) && al(a.normal) && al(a.albedo) &&
                      al(a.pixel) && al(a.parent) && al(a.rough) && al(a.rrs) && al(a.depth) &&
                      al(a.record);
    const int smem = (int)sizeof(RecordStage);
    static bool attr_set = false;  // the attribute is per function, not per device
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(k_record_nodes<true>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_record_nodes<false>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        attr_set = true;
    }
    k_record_count<<<a.chunks, kRecThreads, 0, s>>>(a);
    if (bulk) k_record_nodes<true><<<a.chunks, kWrThreads, smem, s>>>(a);
    else k_record_nodes<false><<<a.chunks, kWrThreads, smem, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_record_radiance(const RadianceArgs& a, cudaStream_t s) {
    if (a.n == 0) return cudaSuccess;
    k_record_radiance<<<(a.n + 255) / 256, 256, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_propagate(const NodeView& nb, cudaStream_t s) {
    // co-resident grid: SMs x resident CTAs of k_propagate
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_propagate, 256, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = sms * per_sm;
    NodeView v = nb;
    unsigned spin = 1u << 22;
    void* args[] = {&v, &spin};
    return cudaLaunchCooperativeKernel((const void*)k_propagate, dim3(grid), dim3(256), args, 0, s);
}

cudaError_t launch_generate(const GenerateArgs& a, int grid, cudaStream_t s) {
    k_generate<<<grid, kRecThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sample_weights(const WeightArgs& a, cudaStream_t s) {
    if (a.max_n == 0) return cudaSuccess;
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    const unsigned need = (a.max_n + 255) / 256, cap = (unsigned)sms * 8u;
    k_sample_weights<<<need < cap ? need : cap, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nrrs
