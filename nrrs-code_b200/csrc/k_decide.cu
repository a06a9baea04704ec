// k_decide.cu -- RRS normalisation, kill/split decision and next-bounce queue emission.
//
// Replaces, in banbao990/NRRS-Code:
//   calcSum2PassAsync<true>   src/render/common/commoncudautilshost.cpp:6-22
//   SumTwoPassInterleaved...  src/render/common/commoncudautils.cu:144-181
//   "Gen Tids" lambda         src/render/nrrs/integrator.cpp:1368-1460
//   TidQueue::push(tid, cnt)  src/render/common/commonworkqueue.h:19-25 (+ pushCheck :34-42)
//
// The sum is exact: every term is a 64-bit fixed-point integer, so the order in which CTAs add
// them does not change a bit (the reference's FP32 sum depends on the occupancy-chosen grid).
// Two emissions give the same queue, in vertex order with the s copies of a vertex contiguous,
// over 2048-vertex chunks:
//  * the context path runs two passes (k_decide_count, k_decide_emit): decide and count every
//    chunk, scan the chunk totals in the count pass's last CTA, then emit each chunk at its
//    prefix from its split counts. No CTA waits on another (4K bounce: 0.063 ms against
//    0.098 ms for the single pass, whose CTAs spent most of their time at block barriers);
//  * the allocation-free entry point keeps the single-pass prefix sum with decoupled look-back
//    (k_decide), which needs no per-vertex scratch: chunks are taken in ticket order, so every
//    predecessor of a waiting chunk has already started and the wait ends; each wait is bounded
//    and reports NRRS_DEV_TIMEOUT. One warp reads 32 predecessor states at a time.
#include "kernels.hpp"

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

// s = int(r) + (rnd <= r - int(r)), with NaN -> 0 and a cap of 255 (flagged)
__device__ __forceinline__ unsigned split_count(float r, float rnd, unsigned* flags) {
    if (!(r == r)) { *flags |= NRRS_DEV_NAN; return 0; }
    if (!(r < 256.0f)) { *flags |= NRRS_DEV_SATURATED; return 255; }
    int s = (int)r;
    const float frac = __fsub_rn(r, (float)s);
    s += (rnd <= frac) ? 1 : 0;
    if (s > 255) { *flags |= NRRS_DEV_SATURATED; s = 255; }
    return (unsigned)s;
}

// queue entries of one chunk staged in shared memory (E[s] is about 1: 2,048 per chunk)
constexpr unsigned kDecStage = 4096;

// normalisation scale of segment si (FP32 sequence of integrator.cpp:1376-1397)
__device__ __forceinline__ float decide_scale(const DecideArgs& a, const Segment& sg, int si) {
    const long long acc = a.ext_sum ? *(const volatile long long*)a.ext_sum
                                    : (long long)*(volatile unsigned long long*)&a.scr->sum_acc[si];
    const float sumf = (float)((double)acc * a.inv_fixed_scale);
    const float rcp = __fdiv_rn(1.0f, sumf);
    const unsigned nspec = (a.n_spec_dev && si == 0) ? *a.n_spec_dev : sg.n_specular;
    const float bud = (float)(unsigned)(sg.budget - nspec);
    float nf = __fmul_rn(bud, rcp);
    nf = __fmul_rn(nf, a.use_ceil ? 1.0f : a.normalize_rate);
    return a.scale_up ? nf : (nf < 1.0f ? nf : 1.0f);
}

__global__ void __launch_bounds__(kDecThreads) k_decide(const __grid_constant__ DecideArgs a) {
    __shared__ unsigned s_chunk, s_epoch, s_prefix;
    __shared__ uint32_t s_stage[kDecStage];
    __shared__ unsigned s_warp[kDecThreads / 32];
    const int tid = threadIdx.x;
    if (tid == 0) {
        s_chunk = atomicAdd(&a.scr->ticket, 1u);
        s_epoch = *(volatile unsigned*)&a.scr->epoch;
    }
    __syncthreads();
    const unsigned c = s_chunk;
    const unsigned epoch = s_epoch;
    unsigned flags = 0;
    const SegmentTable& S = seg_table(a.segs);

    if (c < S.total_tiles) {
        const int si = find_segment(S, c);
        const Segment& sg = S.s[si];
        const unsigned lc = c - sg.tile_start;
        const unsigned base = sg.offset + lc * kDecChunk;
        const unsigned end = sg.offset + min(sg.count, (lc + 1) * kDecChunk);

        const float scale = decide_scale(a, sg, si);

        unsigned sv[kDecVPT];
        unsigned st[kDecVPT];
        unsigned local = 0;
        const unsigned v0 = base + tid * kDecVPT;
        // a thread's 8 consecutive vertices: 16-byte loads and stores when the whole run is in
        // the segment and aligned (the common case), element-wise otherwise
        const bool vec = v0 + kDecVPT <= end &&
                         ((reinterpret_cast<uintptr_t>(a.rrs + v0) |
                           reinterpret_cast<uintptr_t>(a.rnd + v0)) & 15u) == 0;
        constexpr int kQ = kDecVPT / 4;  // 16-byte groups per thread
        float rv[kDecVPT], nv[kDecVPT];
        if (vec) {
#pragma unroll
            for (int g = 0; g < kQ; ++g) {
                const float4 r4 = *reinterpret_cast<const float4*>(a.rrs + v0 + 4 * g);
                const float4 n4 = *reinterpret_cast<const float4*>(a.rnd + v0 + 4 * g);
                rv[4 * g] = r4.x; rv[4 * g + 1] = r4.y; rv[4 * g + 2] = r4.z; rv[4 * g + 3] = r4.w;
                nv[4 * g] = n4.x; nv[4 * g + 1] = n4.y; nv[4 * g + 2] = n4.z; nv[4 * g + 3] = n4.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kDecVPT; ++j) {
                rv[j] = v0 + j < end ? a.rrs[v0 + j] : 0.f;
                nv[j] = v0 + j < end ? a.rnd[v0 + j] : 0.f;
            }
        }
        float rn[kDecVPT];
        uint32_t sp[kQ];
#pragma unroll
        for (int g = 0; g < kQ; ++g) sp[g] = 0u;
#pragma unroll
        for (int j = 0; j < kDecVPT; ++j) {
            const unsigned v = v0 + j;
            sv[j] = 0;
            st[j] = 0;
            rn[j] = 0.f;
            if (v < end) {
                const float r = __fmul_rn(rv[j], scale);
                const unsigned stid = a.sidx ? a.sidx[v] : v;
                rn[j] = r;
                if (a.rrs_norm && (a.sidx || !vec)) a.rrs_norm[stid] = r;
                const unsigned s = split_count(r, nv[j], &flags);
                if (a.split && !vec) a.split[v] = (uint8_t)s;
                sp[j >> 2] |= s << (8 * (j & 3));
                sv[j] = s;
                st[j] = stid;
                local += s;
            }
        }
        if (vec) {
            if (a.rrs_norm && !a.sidx &&
                (reinterpret_cast<uintptr_t>(a.rrs_norm + v0) & 15u) == 0) {
#pragma unroll
                for (int g = 0; g < kQ; ++g)
                    *reinterpret_cast<float4*>(a.rrs_norm + v0 + 4 * g) =
                        make_float4(rn[4 * g], rn[4 * g + 1], rn[4 * g + 2], rn[4 * g + 3]);
            } else if (a.rrs_norm && !a.sidx) {
#pragma unroll
                for (int j = 0; j < kDecVPT; ++j) a.rrs_norm[v0 + j] = rn[j];
            }
            if (a.split) {
                if ((reinterpret_cast<uintptr_t>(a.split + v0) & 3u) == 0) {
#pragma unroll
                    for (int g = 0; g < kQ; ++g) reinterpret_cast<uint32_t*>(a.split + v0)[g] = sp[g];
                } else {
#pragma unroll
                    for (int j = 0; j < kDecVPT; ++j) a.split[v0 + j] = (uint8_t)sv[j];
                }
            }
        }

        // block exclusive scan of the per-thread counts
        const int lane = tid & 31, wid = tid >> 5;
        unsigned incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) s_warp[wid] = incl;
        __syncthreads();
        if (wid == 0) {
            unsigned w = lane < kDecThreads / 32 ? s_warp[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < kDecThreads / 32) s_warp[lane] = w;  // inclusive warp prefix
        }
        __syncthreads();
        const unsigned warp_excl = wid ? s_warp[wid - 1] : 0;
        const unsigned thread_excl = warp_excl + incl - local;
        const unsigned chunk_total = s_warp[kDecThreads / 32 - 1];

        // decoupled look-back by warp 0: each read covers the 32 chunks before a window top;
        // the closest inclusive prefix ends it, otherwise the window moves down by 32
        if (wid == 0) {
            unsigned long long* states = a.states;
            unsigned prefix = 0;
            if (lc == 0) {
                if (lane == 0) store_state(&states[c], pack_state(epoch, kFlagIncl, chunk_total));
            } else {
                if (lane == 0) store_state(&states[c], pack_state(epoch, kFlagAgg, chunk_total));
                const int first = (int)sg.tile_start;  // the segment's first chunk: inclusive
                int top = (int)c - 1;
                unsigned spins = 0;
                bool timed_out = false;
                unsigned long long acc = 0;
                for (;;) {
                    const int idx = top - lane;
                    bool ready = true, incl = true;
                    unsigned val = 0;
                    if (idx >= first) {
                        const unsigned long long w = load_state(&states[idx]);
                        const unsigned long long wf = (w >> 32) & 3ull;
                        ready = (unsigned)(w >> 34) == (epoch & 0x3fffffffu) && wf != 0;
                        incl = wf == kFlagIncl;
                        val = (unsigned)w;
                    }
                    if (!__all_sync(0xffffffffu, ready)) {
                        if (++spins > a.spin_limit) {
                            timed_out = true;
                            break;
                        }
                        __nanosleep(32);
                        continue;
                    }
                    const unsigned im = __ballot_sync(0xffffffffu, incl);
                    const int stop = im ? __ffs(im) - 1 : 31;  // lanes 0..stop contribute
                    unsigned long long part = lane <= stop ? (unsigned long long)val : 0ull;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
                    acc += part;
                    if (im) break;
                    top -= 32;
                }
                prefix = acc > 0xffffffffull ? 0xffffffffu : (unsigned)acc;
                if (lane == 0) {
                    if (timed_out) flags |= NRRS_DEV_TIMEOUT;
                    store_state(&states[c], pack_state(epoch, kFlagIncl, sat_add(prefix, chunk_total)));
                }
            }
            if (lane == 0) {
                s_prefix = prefix;
                if (c == sg.tile_start + (sg.count + kDecChunk - 1) / kDecChunk - 1)
                    a.next_size[si] = sat_add(prefix, chunk_total);
            }
        }
        __syncthreads();

        // emission: s copies of stid, vertex order, capacity-guarded. The chunk's entries are
        // one contiguous range of the queue; staged in shared memory, they go out in coalesced
        // stores (written straight from each thread's runs, a warp's stores touched a sector per
        // entry). A chunk with more entries than the stage holds writes them directly.
        // room: queue slots left from the chunk's first entry (0 when the prefix is past the
        // capacity, including a saturated prefix)
        uint32_t* q = a.queue + sg.queue_offset + s_prefix;
        const unsigned room = s_prefix < sg.queue_capacity ? sg.queue_capacity - s_prefix : 0u;
        if (chunk_total <= kDecStage) {
            unsigned pos = thread_excl;
#pragma unroll
            for (int j = 0; j < kDecVPT; ++j)
                for (unsigned k = 0; k < sv[j]; ++k, ++pos) s_stage[pos] = st[j];
            __syncthreads();
            for (unsigned e = tid; e < chunk_total; e += kDecThreads) {
                if (e < room) q[e] = s_stage[e];
                else flags |= NRRS_DEV_OVERFLOW;
            }
        } else {
            unsigned pos = thread_excl;
#pragma unroll
            for (int j = 0; j < kDecVPT; ++j) {
                for (unsigned k = 0; k < sv[j]; ++k, ++pos) {
                    if (pos < room) q[pos] = st[j];
                    else flags |= NRRS_DEV_OVERFLOW;
                }
            }
        }
    }

    if (flags) atomicOr(&a.scr->status, flags);

    // the last CTA restores the scratch for the next launch
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        const unsigned old = atomicAdd(&a.scr->done, 1u);
        if (old == gridDim.x - 1) {
            for (int k = 0; k < S.n; ++k) {
                if (S.s[k].count == 0) a.next_size[k] = 0;
                a.scr->sum_acc[k] = 0ull;
            }
            a.scr->ticket = 0;
            a.scr->done = 0;
            a.scr->epoch = a.scr->epoch + 1;
            __threadfence();
        }
    }
}

// ---- two-pass decision (context path): no look-back ------------------------------------------
// Pass 1 (k_decide_count) normalises, decides and writes rrs_norm and the split counts of every
// chunk, streaming, and stores the chunk's total; its last CTA turns the totals into exclusive
// per-segment prefixes (and the next-queue sizes). Pass 2 (k_decide_emit) reads a chunk's split
// counts back (1 byte per vertex) and writes its queue entries at its prefix. Same decisions and
// the same queue as the single-pass kernel, bit for bit; each CTA runs without waiting on any
// other, which the single-pass kernel's per-chunk look-back and block barriers did.

__device__ __forceinline__ unsigned block_sum_u(unsigned v, unsigned* s_red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = v;
    __syncthreads();
    unsigned t = 0;
#pragma unroll
    for (int k = 0; k < kDecThreads / 32; ++k) t += s_red[k];
    return t;
}

// the split counts of chunk c, whose first vertex is `first`: the caller's array (indexed by
// vertex), or the context's scratch, one kDecChunk-byte block per chunk (segment offsets are the
// caller's and need not fit the scratch)
__device__ __forceinline__ uint8_t* split_of_chunk(const DecideArgs& a, unsigned c, unsigned first) {
    return a.split_chunked ? a.split + (size_t)c * kDecChunk : a.split + first;
}

__global__ void __launch_bounds__(kDecThreads) k_decide_count(const __grid_constant__ DecideArgs a) {
    __shared__ unsigned s_red[kDecThreads / 32];
    __shared__ int s_last;
    __shared__ unsigned long long s_scan[kDecThreads];
    const int tid = threadIdx.x;
    const unsigned c = blockIdx.x;
    unsigned flags = 0;
    const SegmentTable& S = seg_table(a.segs);
    unsigned local = 0;
    if (c < S.total_tiles) {
        const int si = find_segment(S, c);
        const Segment& sg = S.s[si];
        const unsigned lc = c - sg.tile_start;
        const unsigned end = sg.offset + min(sg.count, (lc + 1) * kDecChunk);
        const float scale = decide_scale(a, sg, si);
        const unsigned v0 = sg.offset + lc * kDecChunk + tid * kDecVPT;
        uint8_t* cs = split_of_chunk(a, c, sg.offset + lc * kDecChunk) + tid * kDecVPT;
        const bool vec = v0 + kDecVPT <= end &&
                         ((reinterpret_cast<uintptr_t>(a.rrs + v0) |
                           reinterpret_cast<uintptr_t>(a.rnd + v0)) & 15u) == 0;
        constexpr int kQ = kDecVPT / 4;
        float rv[kDecVPT], nv[kDecVPT];
        if (vec) {
#pragma unroll
            for (int g = 0; g < kQ; ++g) {
                const float4 r4 = *reinterpret_cast<const float4*>(a.rrs + v0 + 4 * g);
                const float4 n4 = *reinterpret_cast<const float4*>(a.rnd + v0 + 4 * g);
                rv[4 * g] = r4.x; rv[4 * g + 1] = r4.y; rv[4 * g + 2] = r4.z; rv[4 * g + 3] = r4.w;
                nv[4 * g] = n4.x; nv[4 * g + 1] = n4.y; nv[4 * g + 2] = n4.z; nv[4 * g + 3] = n4.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < kDecVPT; ++j) {
                rv[j] = v0 + j < end ? a.rrs[v0 + j] : 0.f;
                nv[j] = v0 + j < end ? a.rnd[v0 + j] : 0.f;
            }
        }
        float rn[kDecVPT];
        uint32_t sp[kQ];
#pragma unroll
        for (int g = 0; g < kQ; ++g) sp[g] = 0u;
#pragma unroll
        for (int j = 0; j < kDecVPT; ++j) {
            const unsigned v = v0 + j;
            rn[j] = 0.f;
            if (v < end) {
                const float r = __fmul_rn(rv[j], scale);
                rn[j] = r;
                if (a.rrs_norm && (a.sidx || !vec)) a.rrs_norm[a.sidx ? a.sidx[v] : v] = r;
                const unsigned s = split_count(r, nv[j], &flags);
                if (!vec) cs[j] = (uint8_t)s;
                sp[j >> 2] |= s << (8 * (j & 3));
                local += s;
            }
        }
        if (vec) {
            if (a.rrs_norm && !a.sidx && (reinterpret_cast<uintptr_t>(a.rrs_norm + v0) & 15u) == 0) {
#pragma unroll
                for (int g = 0; g < kQ; ++g)
                    *reinterpret_cast<float4*>(a.rrs_norm + v0 + 4 * g) =
                        make_float4(rn[4 * g], rn[4 * g + 1], rn[4 * g + 2], rn[4 * g + 3]);
            } else if (a.rrs_norm && !a.sidx) {
#pragma unroll
                for (int j = 0; j < kDecVPT; ++j) a.rrs_norm[v0 + j] = rn[j];
            }
            if ((reinterpret_cast<uintptr_t>(cs) & 3u) == 0) {
#pragma unroll
                for (int g = 0; g < kQ; ++g) reinterpret_cast<uint32_t*>(cs)[g] = sp[g];
            } else {
#pragma unroll
                for (int j = 0; j < kDecVPT; ++j) cs[j] = (uint8_t)(sp[j >> 2] >> (8 * (j & 3)));
            }
        }
    }
    // chunk total (split counts are at most 255, 2,048 per chunk: no overflow)
    const unsigned total = block_sum_u(local, s_red);
    if (flags) atomicOr(&a.scr->status, flags);
    if (tid == 0) {
        if (c < S.total_tiles) a.states[c] = total;
        __threadfence();
        s_last = atomicAdd(&a.scr->done, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // the last CTA: exclusive prefix of the chunk totals per segment, saturating like the
    // single-pass kernel; thread t scans a contiguous run of each segment's chunks
    for (int k = 0; k < S.n; ++k) {
        const Segment& sg = S.s[k];
        const unsigned nch = (sg.count + kDecChunk - 1) / kDecChunk;
        const unsigned per = (nch + kDecThreads - 1) / kDecThreads;
        const unsigned lo = sg.tile_start + min(nch, tid * per);
        const unsigned hi = sg.tile_start + min(nch, (tid + 1) * per);
        // the totals come in batches of independent L2 loads (the other CTAs' stores are visible
        // after their fences and the done counter)
        unsigned long long mine = 0;
        for (unsigned q0 = lo; q0 < hi; q0 += 8) {
            unsigned t8[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) t8[j] = q0 + j < hi ? (unsigned)__ldcg(&a.states[q0 + j]) : 0u;
#pragma unroll
            for (int j = 0; j < 8; ++j) mine += t8[j];
        }
        s_scan[tid] = mine;
        __syncthreads();
#pragma unroll 1
        for (int o = 1; o < kDecThreads; o <<= 1) {
            const unsigned long long y = tid >= o ? s_scan[tid - o] : 0ull;
            __syncthreads();
            s_scan[tid] += y;
            __syncthreads();
        }
        unsigned long long run = tid ? s_scan[tid - 1] : 0ull;
        for (unsigned q0 = lo; q0 < hi; q0 += 8) {
            unsigned t8[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) t8[j] = q0 + j < hi ? (unsigned)__ldcg(&a.states[q0 + j]) : 0u;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (q0 + j < hi) __stcg(&a.states[q0 + j], run > 0xffffffffull ? 0xffffffffull : run);
                run += t8[j];
            }
        }
        if (tid == kDecThreads - 1) {
            const unsigned long long tot = s_scan[tid];
            a.next_size[k] = tot > 0xffffffffull ? 0xffffffffu : (unsigned)tot;
        }
        __syncthreads();
    }
    // restore the scratch for the next launch
    if (tid == 0) {
        for (int k = 0; k < S.n; ++k) a.scr->sum_acc[k] = 0ull;
        a.scr->ticket = 0;
        a.scr->done = 0;
        a.scr->epoch = a.scr->epoch + 1;
        __threadfence();
    }
}

// Pass 2: the queue entries of chunk c at its prefix (capacity-guarded, vertex order, the s
// copies of a vertex contiguous), staged in shared memory for coalesced stores.
__global__ void __launch_bounds__(kDecThreads) k_decide_emit(const __grid_constant__ DecideArgs a) {
    __shared__ uint32_t s_stage[kDecStage];
    __shared__ unsigned s_warp[kDecThreads / 32];
    const int tid = threadIdx.x;
    const unsigned c = blockIdx.x;
    const SegmentTable& S = seg_table(a.segs);
    if (c >= S.total_tiles) return;
    unsigned flags = 0;
    const int si = find_segment(S, c);
    const Segment& sg = S.s[si];
    const unsigned lc = c - sg.tile_start;
    const unsigned end = sg.offset + min(sg.count, (lc + 1) * kDecChunk);
    const unsigned v0 = sg.offset + lc * kDecChunk + tid * kDecVPT;
    const unsigned prefix = (unsigned)a.states[c];
    const uint8_t* cs = split_of_chunk(a, c, sg.offset + lc * kDecChunk) + tid * kDecVPT;
    unsigned sv[kDecVPT];
    unsigned local = 0;
    if (v0 + kDecVPT <= end && (reinterpret_cast<uintptr_t>(cs) & 7u) == 0) {
        const unsigned long long w = *reinterpret_cast<const unsigned long long*>(cs);
#pragma unroll
        for (int j = 0; j < kDecVPT; ++j) sv[j] = (unsigned)(w >> (8 * j)) & 0xffu;
    } else {
#pragma unroll
        for (int j = 0; j < kDecVPT; ++j) sv[j] = v0 + j < end ? cs[j] : 0u;
    }
#pragma unroll
    for (int j = 0; j < kDecVPT; ++j) local += sv[j];

    // block exclusive scan of the per-thread counts
    const int lane = tid & 31, wid = tid >> 5;
    unsigned incl = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) s_warp[wid] = incl;
    __syncthreads();
    if (wid == 0) {
        unsigned w = lane < kDecThreads / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < kDecThreads / 32) s_warp[lane] = w;
    }
    __syncthreads();
    const unsigned thread_excl = (wid ? s_warp[wid - 1] : 0) + incl - local;
    const unsigned chunk_total = s_warp[kDecThreads / 32 - 1];

    uint32_t* q = a.queue + sg.queue_offset + prefix;
    const unsigned room = prefix < sg.queue_capacity ? sg.queue_capacity - prefix : 0u;
    if (chunk_total <= kDecStage) {
        unsigned pos = thread_excl;
#pragma unroll
        for (int j = 0; j < kDecVPT; ++j) {
            if (sv[j] == 0u) continue;  // vertices past the chunk's end have no copies
            const unsigned stid = a.sidx ? a.sidx[v0 + j] : v0 + j;
            for (unsigned k = 0; k < sv[j]; ++k, ++pos) s_stage[pos] = stid;
        }
        __syncthreads();
        for (unsigned e = tid; e < chunk_total; e += kDecThreads) {
            if (e < room) q[e] = s_stage[e];
            else flags |= NRRS_DEV_OVERFLOW;
        }
    } else {
        unsigned pos = thread_excl;
#pragma unroll
        for (int j = 0; j < kDecVPT; ++j) {
            for (unsigned k = 0; k < sv[j]; ++k, ++pos) {
                if (pos < room) q[pos] = a.sidx ? a.sidx[v0 + j] : v0 + j;
                else flags |= NRRS_DEV_OVERFLOW;
            }
        }
    }
    if (flags) atomicOr(&a.scr->status, flags);
}

__global__ void __launch_bounds__(kTile) k_sum(const __grid_constant__ SumArgs a) {
    __shared__ long long s_part[kTile / 32];
    unsigned flags = 0;
    const SegmentTable& S = seg_table(a.segs);
    for (unsigned t = blockIdx.x; t < S.total_tiles; t += gridDim.x) {
        const int si = find_segment(S, t);
        const Segment& sg = S.s[si];
        const unsigned v = sg.offset + (t - sg.tile_start) * kTile + threadIdx.x;
        long long term = 0;
        if (v < sg.offset + sg.count) term = fixed_term(a.fp, a.rrs[v], &a.scr->status);
        term = warp_sum_ll(term);
        if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = term;
        __syncthreads();
        if (threadIdx.x == 0) {
            long long tot = 0;
#pragma unroll
            for (int k = 0; k < kTile / 32; ++k) tot += s_part[k];
            atomicAdd(&a.scr->sum_acc[si], (unsigned long long)tot);
        }
        __syncthreads();
    }
    (void)flags;
}

// Builds, on the device, the segment tables of the actual queue sizes: count k is
// min(counts[k], the largest count the host sized the launch for; more flags NRRS_DEV_OVERFLOW),
// and the tile starts are the prefix sums in units of kTile (inference, sum, encoding) and of
// kDecChunk (decision). One thread: at most 16 segments.
__global__ void k_resolve_segments(const __grid_constant__ SegmentTable host, const uint32_t* counts,
                                   SegmentTable* tiles, SegmentTable* chunks, unsigned* status) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    uint32_t t_tiles = 0, t_chunks = 0;
    unsigned flags = 0;
    for (int k = 0; k < host.n; ++k) {
        Segment sg = host.s[k];
        uint32_t c = counts[k];
        if (c > sg.count) { c = sg.count; flags |= NRRS_DEV_OVERFLOW; }
        sg.count = c;
        sg.tile_start = t_tiles;
        tiles->s[k] = sg;
        sg.tile_start = t_chunks;
        chunks->s[k] = sg;
        t_tiles += (c + kTile - 1) / kTile;
        t_chunks += (c + kDecChunk - 1) / kDecChunk;
    }
    tiles->n = chunks->n = host.n;
    tiles->total_tiles = t_tiles;
    chunks->total_tiles = t_chunks;
    tiles->resolved = chunks->resolved = nullptr;
    if (flags) atomicOr(status, flags);
}

}  // namespace

cudaError_t launch_resolve_segments(const SegmentTable& host_max, const uint32_t* counts_dev,
                                    SegmentTable* tiles_dev, SegmentTable* chunks_dev,
                                    unsigned* status, cudaStream_t s) {
    k_resolve_segments<<<1, 32, 0, s>>>(host_max, counts_dev, tiles_dev, chunks_dev, status);
    return cudaGetLastError();
}

cudaError_t launch_decide(const DecideArgs& a, cudaStream_t s) {
    if (a.segs.total_tiles == 0) return cudaSuccess;
    k_decide<<<a.segs.total_tiles, kDecThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_decide_two_pass(const DecideArgs& a, cudaStream_t s) {
    if (a.segs.total_tiles == 0) return cudaSuccess;
    k_decide_count<<<a.segs.total_tiles, kDecThreads, 0, s>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_decide_emit<<<a.segs.total_tiles, kDecThreads, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sum(const SumArgs& a, cudaStream_t s) {
    if (a.segs.total_tiles == 0) return cudaSuccess;
    const unsigned grid = a.segs.total_tiles < 148u * 8u ? a.segs.total_tiles : 148u * 8u;
    k_sum<<<grid, kTile, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace nrrs
