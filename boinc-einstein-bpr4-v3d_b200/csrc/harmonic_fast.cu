// Harmonic summing + candidate compaction, register-blocked form.
//
// Semantics: shaders/harmonic.comp:5-35 with the summation order of
// shaders/hs_sum.glsl:2-9.  For trial bin i the dyadic sums are
//     s2  = P[i] + P[(8i+8)>>4]
//     s4  = s2 + (P[(12i+8)>>4] + P[(4i+8)>>4])
//     s8  = s4 + (((P[(14i+8)>>4] + P[(10i+8)>>4]) + P[(6i+8)>>4]) + P[(2i+8)>>4])
//     s16 = s8 + (((((((P15 + P13) + P11) + P9) + P7) + P5) + P3) + P1)
// (Pk = P[(k i + 8) >> 4]), each addition rounded in FP32 in that order.  For
// level h (w = 2^h) and fundamental bin j the trial bins are
// [max(window, jw - w/2), min(harmonic, jw + w/2)); the value is the largest sum
// when it exceeds threshold[h], else the sum at the first trial bin, else 0 for
// an empty range.  Level 0 is P[j].
//
// Layout: thread m of a CTA owns 16 consecutive trial bins i0 + r (i0 = 16 m').
// Then (i k + 8) >> 4 = m' k + ((r k + 8) >> 4): for factor k a thread needs the
// k or k+1 consecutive power values starting at m' k, so each value is loaded
// once per thread and reused by up to 16/k trial bins.  The CTA stages, for
// every k, the contiguous power range its threads need in shared memory (one
// region per k, padded per k so that the stride-k reads of a warp hit distinct
// banks).  Level h's fundamental bins j = i0/w + u own trial bins
// [uw - w/2, uw + w/2) of the thread; for u = 0 the first w/2 of them are the
// previous thread's last bins, whose maximum and first value arrive by warp
// shuffle (and through shared memory across warps).  Thread 0 of each CTA only
// computes that halo for thread 1.
#include <cooperative_groups.h>
#include "async_device.cuh"
#include "brp_internal.h"

namespace brp {
namespace {

constexpr int kHThreads = 128;
constexpr int kHBlocks = kHThreads - 1;  // owned 16-bin blocks per CTA

// Odd factors are staged in shared memory: region k holds the power values
// P[first*k - d_k + e] for e < region_floats(k) (d_k = (first*k) & 3, so the
// copy starts 16-byte aligned); thread m reads region[m*k + o + d_k], a
// stride-k pattern that is conflict-free for odd k.  Even factors are read
// straight from global memory: thread m's values P[m'k .. m'k + k] are
// contiguous and 8-byte (k = 2 mod 4) or 16-byte (k = 0 mod 4) aligned.
__host__ __device__ constexpr int region_floats(int k) { return ((kHThreads * k + 1 + 3 + 3) / 4) * 4; }
__host__ __device__ constexpr int odd_base(int k) {
    int b = 0;
    for (int q = 1; q < k; q += 2) b += region_floats(q);
    return b;
}
constexpr int kStageFloats = odd_base(17);

// Values P[m'k + o], o = 0 .. NV-1 (NV = ((15k + 8) >> 4) + 1) of factor K.
template <int K>
__device__ __forceinline__ void factor_values(float* v, const float* stage, const int* doff, const float* __restrict__ Pw,
                                              int64_t mp, int m) {
    constexpr int NV = ((15 * K + 8) >> 4) + 1;
    if constexpr (K % 2 == 1) {
        const float* r = stage + odd_base(K) + doff[K / 2] + m * K;
#pragma unroll
        for (int o = 0; o < NV; ++o) v[o] = r[o];
    } else {
        // even factors, direct threads only (add_factor loads edge threads itself)
        const float* g = Pw + mp * K;
        if constexpr (K % 4 == 0) {
            constexpr int NQ = (NV + 3) / 4;
#pragma unroll
            for (int q = 0; q < NQ; ++q) {
                const float4 x = __ldg(reinterpret_cast<const float4*>(g) + q);
                if (4 * q + 0 < NV) v[4 * q + 0] = x.x;
                if (4 * q + 1 < NV) v[4 * q + 1] = x.y;
                if (4 * q + 2 < NV) v[4 * q + 2] = x.z;
                if (4 * q + 3 < NV) v[4 * q + 3] = x.w;
            }
        } else {
            constexpr int NH = (NV + 1) / 2;
#pragma unroll
            for (int q = 0; q < NH; ++q) {
                const float2 x = __ldg(reinterpret_cast<const float2*>(g) + q);
                if (2 * q + 0 < NV) v[2 * q + 0] = x.x;
                if (2 * q + 1 < NV) v[2 * q + 1] = x.y;
            }
        }
    }
}

// s[r] += t[r] for the 16 trial bins, two bins per packed FP32 add (each lane
// the scalar IEEE add, so the sums are those of the fixed scalar order).
__device__ __forceinline__ void add_bins(float (&s)[16], const float (&t)[16]) {
#pragma unroll
    for (int r = 0; r < 16; r += 2) {
        const float2 y = __fadd2_rn(make_float2(s[r], s[r + 1]), make_float2(t[r], t[r + 1]));
        s[r] = y.x;
        s[r + 1] = y.y;
    }
}

// Adds factor K's values to t[r] (or sets them when SET) in the fixed order.
template <int K, bool SET>
__device__ __forceinline__ void add_factor(float (&t)[16], const float* stage, const int* doff,
                                           const float* __restrict__ Pw, int64_t mp, int m, bool direct,
                                           uint32_t M) {
    constexpr int NV = ((15 * K + 8) >> 4) + 1;
    float v[NV];
    if (K % 2 == 0 && !direct) {
#pragma unroll
        for (int o = 0; o < NV; ++o) {
            const int64_t gi = mp * K + o;
            v[o] = (gi >= 0 && gi < int64_t(M)) ? __ldg(Pw + gi) : 0.f;
        }
    } else {
        factor_values<K>(v, stage, doff, Pw, mp, m);
    }
    float x[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) x[r] = v[(r * K + 8) >> 4];
    if constexpr (SET) {
#pragma unroll
        for (int r = 0; r < 16; ++r) t[r] = x[r];
    } else {
        add_bins(t, x);
    }
}

struct LevelTail { float best, first; };

// Appends one candidate to the template's list.  The lanes of a warp that emit
// together take their slots with one atomic add of the leader (warp-aggregated
// compaction); the list order is arbitrary and sorted by (level, bin) later.
__device__ __forceinline__ void emit(uint32_t j, uint32_t h, float v, uint32_t* count, brp_candidate* out,
                                     uint32_t capacity, uint32_t* status) {
    namespace cg = cooperative_groups;
    const cg::coalesced_group active = cg::coalesced_threads();
    uint32_t base = 0;
    if (active.thread_rank() == 0) base = atomicAdd(count, active.size());
    const uint32_t slot = active.shfl(base, 0) + active.thread_rank();
    if (slot < capacity) {
        brp_candidate c;
        c.bin = j; c.level = h; c.power = v; c.reserved = 0;
        out[slot] = c;
    } else {
        atomicOr(status, BRP_STATUS_OVERFLOW);
    }
}

// Level h (W = 2^h) bookkeeping of one thread.  v[r] is the sum at trial bin
// i0 + r, or -1 for a bin outside [window, harmonic) when ALLV is false.
// Stores/emits the fully local fundamental bins (u >= 1); returns the head
// (first W/2 bins) and the tail (last W/2 bins) for the u = 0 bin.
template <int H, bool ALLV>
__device__ __forceinline__ void level_local(const float (&v)[16], uint32_t i0, bool own, uint32_t fundamental,
                                            uint32_t window, float thr, float* summed, uint32_t* count,
                                            brp_candidate* out, uint32_t capacity, uint32_t* status,
                                            LevelTail& head, LevelTail& tail) {
    constexpr int W = 1 << H, HALF = W / 2;
    // Without a summed-array snapshot only candidates matter, and a fundamental
    // bin is one only if its value exceeds thr: the largest sum when that exceeds
    // thr (the first sum never does then), else 0 for an empty range (only
    // when thr < 0).  So one maximum over the trial bins of the local
    // fundamentals [HALF, 16 - HALF) decides whether any of them needs a look.
    bool detail = true;
    if (16 / W > 1 && !summed) {
        float lm = v[HALF];
#pragma unroll
        for (int r = HALF + 1; r < 16 - HALF; ++r) lm = fmaxf(lm, v[r]);
        detail = lm > thr || (!ALLV && thr < 0.f);
    }
#pragma unroll
    for (int u = 1; u < 16 / W; ++u) {
        if (!detail) break;
        float best, first;
        if (ALLV) {
            first = v[u * W - HALF];
            best = first;
#pragma unroll
            for (int r = u * W - HALF + 1; r < u * W + HALF; ++r) best = fmaxf(best, v[r]);
        } else {
            best = -1.f; first = -1.f;
#pragma unroll
            for (int r = u * W - HALF; r < u * W + HALF; ++r) {
                best = fmaxf(best, v[r]);
                first = first < 0.f ? v[r] : first;
            }
        }
        const uint32_t j = (i0 >> H) + u;
        if (own && j < fundamental) {
            const float value = (!ALLV && best < 0.f) ? 0.f : (best > thr ? best : first);
            if (summed) summed[j] = value;
            // j is a fundamental bin (about i / 2^H): the window test stays even
            // when every trial bin of the thread lies above the window.
            if (j >= window && value > thr) emit(j, H, value, count, out, capacity, status);
        }
    }
    if (ALLV) {
        head.first = v[0]; head.best = v[0];
#pragma unroll
        for (int r = 1; r < HALF; ++r) head.best = fmaxf(head.best, v[r]);
        tail.first = v[16 - HALF]; tail.best = v[16 - HALF];
#pragma unroll
        for (int r = 16 - HALF + 1; r < 16; ++r) tail.best = fmaxf(tail.best, v[r]);
    } else {
        head.best = -1.f; head.first = -1.f;
#pragma unroll
        for (int r = 0; r < HALF; ++r) {
            head.best = fmaxf(head.best, v[r]);
            head.first = head.first < 0.f ? v[r] : head.first;
        }
        tail.best = -1.f; tail.first = -1.f;
#pragma unroll
        for (int r = 16 - HALF; r < 16; ++r) {
            tail.best = fmaxf(tail.best, v[r]);
            tail.first = tail.first < 0.f ? v[r] : tail.first;
        }
    }
}

struct HCtx {
    const float* stage;
    const int* doff;
    const float* Pw;
    int64_t mp;
    int m;
    bool direct;
    uint32_t M, i0, window, fundamental, harmonic;
    bool own;
    const float* thr;
    float* summed;
    uint32_t* count;
    brp_candidate* out;
    uint32_t cap;
    uint32_t* status;
};

// Masks the sums of the thread's trial bins for level bookkeeping: outside
// [window, harmonic) (and before bin 0) a bin takes the -1 sentinel.
template <bool ALLV>
__device__ __forceinline__ void masked(const HCtx& c, const float (&s)[16], float (&v)[16]) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
        if (ALLV) v[r] = s[r];
        else {
            const int64_t i = c.mp * 16 + r;
            v[r] = (c.mp >= 0 && i >= int64_t(c.window) && i < int64_t(c.harmonic)) ? s[r] : -1.f;
        }
    }
}

// Levels 1-3 (stages A-C): the even factors, read straight from global memory,
// so they run while the odd factors' staging copies are still in flight.
// Leaves s = s8 for stage D.
template <bool ALLV>
__device__ __forceinline__ void sums_abc(const HCtx& c, const float (&p16)[16], float (&s)[16], LevelTail (&head)[4],
                                         LevelTail (&tail)[4]) {
    float t[16], v[16];
    float* sm1 = c.summed ? c.summed + size_t(c.fundamental) : nullptr;
    float* sm2 = c.summed ? c.summed + size_t(2) * c.fundamental : nullptr;
    float* sm3 = c.summed ? c.summed + size_t(3) * c.fundamental : nullptr;
    // stage A: s2 = P16 + P8 (P16 = the level-0 values)
#pragma unroll
    for (int r = 0; r < 16; ++r) s[r] = p16[r];
    add_factor<8, false>(s, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    masked<ALLV>(c, s, v);
    level_local<1, ALLV>(v, c.i0, c.own, c.fundamental, c.window, c.thr[1], sm1, c.count, c.out, c.cap, c.status,
                         head[0], tail[0]);
    // stage B: s4 = s2 + (P12 + P4)
    add_factor<12, true>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<4, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_bins(s, t);
    masked<ALLV>(c, s, v);
    level_local<2, ALLV>(v, c.i0, c.own, c.fundamental, c.window, c.thr[2], sm2, c.count, c.out, c.cap, c.status,
                         head[1], tail[1]);
    // stage C: s8 = s4 + (((P14 + P10) + P6) + P2)
    add_factor<14, true>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<10, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<6, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<2, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_bins(s, t);
    masked<ALLV>(c, s, v);
    level_local<3, ALLV>(v, c.i0, c.own, c.fundamental, c.window, c.thr[3], sm3, c.count, c.out, c.cap, c.status,
                         head[2], tail[2]);
}

// Level 4 (stage D): s16 = s8 + (((((((P15 + P13) + P11) + P9) + P7) + P5) + P3) + P1)
// from the odd factors staged in shared memory.
template <bool ALLV>
__device__ __forceinline__ void sums_d(const HCtx& c, float (&s)[16], LevelTail& head, LevelTail& tail) {
    float t[16], v[16];
    float* sm4 = c.summed ? c.summed + size_t(4) * c.fundamental : nullptr;
    add_factor<15, true>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<13, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<11, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<9, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<7, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<5, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<3, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_factor<1, false>(t, c.stage, c.doff, c.Pw, c.mp, c.m, c.direct, c.M);
    add_bins(s, t);
    masked<ALLV>(c, s, v);
    level_local<4, ALLV>(v, c.i0, c.own, c.fundamental, c.window, c.thr[4], sm4, c.count, c.out, c.cap, c.status,
                         head, tail);
}

// Six CTAs per SM (80 registers per thread): the shared-memory staging allows
// six, and the extra warps hide the latency of the direct global loads.
__global__ void __launch_bounds__(kHThreads, 6) harmonic_fast_kernel(FusedArgs a) {
    extern __shared__ __align__(16) float stage[];
    __shared__ float xwarp[kHThreads / 32][8];
    __shared__ int doff[8];
    __shared__ __align__(8) uint64_t s_bar;
    const int g = blockIdx.y;
    const brp_params& P = a.params[g];
    const uint32_t window = P.window, fundamental = P.fundamental, harmonic = P.harmonic;
    const uint32_t M = a.M;
    const float* __restrict__ Pw = a.power + size_t(g) * a.power_stride;
    float* summed = (g == a.snap) ? a.snap_summed : nullptr;

    // 16-bin block of thread m: m' = first + m (first = blockIdx.x * kHBlocks - 1).
    const int64_t first = int64_t(blockIdx.x) * kHBlocks - 1;
    const int m = threadIdx.x;

    // ---- stage the odd factors.  Interior CTAs (every region inside [0, M)):
    // one bulk copy per region, issued by thread 0 and counted on an mbarrier.
    // Edge CTAs: 16-byte asynchronous copies from a 16-byte aligned start,
    // chunks reaching outside [0, M) copied element-wise with zero fill.  The
    // copies are only waited for before stage D, the first to read them.
    const uint32_t stage_sh = smem_u32(stage);
    const uint32_t bar = smem_u32(&s_bar);
    const bool bulk = first >= 0 && ((first * 15) & ~int64_t(3)) + region_floats(15) <= int64_t(M);
    if (bulk) {
        if (threadIdx.x == 0) {
            mbar_init(bar, 1);
            mbar_arrive_expect_tx(bar, uint32_t(kStageFloats) * 4u);
#pragma unroll
            for (int k = 1; k <= 15; k += 2) {
                const int64_t gs = first * k, ga = gs & ~int64_t(3);
                doff[k / 2] = int(gs - ga);
                bulk_copy_g2s(stage_sh + 4u * uint32_t(odd_base(k)), Pw + ga, 4u * uint32_t(region_floats(k)), bar);
            }
        }
        __syncthreads();  // the barrier is initialised before anyone polls it
    } else {
#pragma unroll 1
        for (int k = 1; k <= 15; k += 2) {
            const int64_t gs = first * k;
            const int64_t ga = gs >= 0 ? (gs & ~int64_t(3)) : -((-gs + 3) & ~int64_t(3));
            if (threadIdx.x == 0) doff[k / 2] = int(gs - ga);
            const int chunks = region_floats(k) / 4;
            const uint32_t reg = stage_sh + 4u * uint32_t(odd_base(k));
            for (int c = threadIdx.x; c < chunks; c += kHThreads) {
                const int64_t gi = ga + 4 * c;
                const uint32_t dst = reg + 16u * uint32_t(c);
                if (gi >= 0 && gi + 4 <= int64_t(M)) {
                    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(Pw + gi) : "memory");
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const bool in = gi + q >= 0 && gi + q < int64_t(M);
                        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst + 4u * q),
                                     "l"(Pw + (in ? gi + q : 0)), "r"(in ? 4 : 0)
                                     : "memory");
                    }
                }
            }
        }
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }

    HCtx c;
    c.stage = stage; c.doff = doff; c.Pw = Pw; c.m = m; c.M = M;
    c.mp = first + m;
    c.own = m > 0 && c.mp >= 0;
    c.i0 = c.mp >= 0 ? uint32_t(c.mp) * 16u : 0u;
    c.window = window; c.fundamental = fundamental; c.harmonic = harmonic;
    c.direct = c.mp >= 0 && uint64_t(c.mp + 1) * 16u <= M;
    c.thr = P.threshold;
    c.summed = summed; c.count = a.counts + g; c.out = a.cands + size_t(g) * a.capacity; c.cap = a.capacity;
    c.status = a.status + g;
    // Bins outside [window, harmonic) (and the halo before bin 0) take the -1 sentinel.
    const bool all_valid = c.direct && c.i0 >= window && c.i0 + 16 <= harmonic;

    // P[16 m' + r]: level 0 (P[j], j = i0 + r) and factor 16 of the sums ((16 i + 8) >> 4 = i)
    float p0[16];
    if (c.direct) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const float4 x = __ldg(reinterpret_cast<const float4*>(Pw + c.i0) + q);
            p0[4 * q] = x.x; p0[4 * q + 1] = x.y; p0[4 * q + 2] = x.z; p0[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const int64_t gi = c.mp * 16 + r;
            p0[r] = (gi >= 0 && gi < int64_t(M)) ? __ldg(Pw + gi) : 0.f;
        }
    }
    // level 0: only bins above threshold[0] are candidates, so without a
    // summed-array snapshot one maximum decides whether the bins need a look
    bool look = c.own;
    if (look && !summed) {
        float mx = p0[0];
#pragma unroll
        for (int r = 1; r < 16; ++r) mx = fmaxf(mx, p0[r]);
        look = mx > P.threshold[0];
    }
    if (look) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const uint32_t j = c.i0 + r;
            if (j < fundamental) {
                if (summed) summed[j] = p0[r];
                if (j >= window && p0[r] > P.threshold[0]) emit(j, 0, p0[r], c.count, c.out, c.cap, c.status);
            }
        }
    }

    LevelTail head[4], tail[4];
    float s8[16];
    if (all_valid) sums_abc<true>(c, p0, s8, head, tail);
    else sums_abc<false>(c, p0, s8, head, tail);

    // the odd factors' staging must have landed before stage D
    bool copied = true;
    if (bulk) copied = mbar_wait_bounded(bar, 0, a.wait_polls);
    else asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    if (__syncthreads_or(!copied)) {
        // A bulk copy did not complete within the bound: report it, give the
        // copies one more bounded wait (they write this CTA's shared memory) and leave.
        if (threadIdx.x == 0) atomicOr(a.status + g, BRP_STATUS_WAIT_TIMEOUT);
        mbar_wait_bounded(bar, 0, kDrainPolls);
        return;
    }
    if (all_valid) sums_d<true>(c, s8, head[3], tail[3]);
    else sums_d<false>(c, s8, head[3], tail[3]);

    // ---- u = 0 fundamental bins: previous thread's tail + own head
    const int lane = m & 31, warp = m >> 5;
    if (lane == 31) {
#pragma unroll
        for (int h = 0; h < 4; ++h) { xwarp[warp][2 * h] = tail[h].best; xwarp[warp][2 * h + 1] = tail[h].first; }
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 4; ++h) {
        float pb = __shfl_up_sync(0xffffffffu, tail[h].best, 1);
        float pf = __shfl_up_sync(0xffffffffu, tail[h].first, 1);
        if (lane == 0) {
            pb = warp > 0 ? xwarp[warp - 1][2 * h] : -1.f;
            pf = warp > 0 ? xwarp[warp - 1][2 * h + 1] : -1.f;
        }
        const uint32_t j = c.i0 >> (h + 1);
        if (c.own && j < fundamental) {
            const float best = fmaxf(pb, head[h].best);
            const float firstv = pf >= 0.f ? pf : head[h].first;
            const float thr = P.threshold[h + 1];
            const float value = best < 0.f ? 0.f : (best > thr ? best : firstv);
            if (summed) summed[size_t(h + 1) * fundamental + j] = value;
            if (j >= window && value > thr) emit(j, h + 1, value, c.count, c.out, c.cap, c.status);
        }
    }
}

}  // namespace

size_t harmonic_fast_smem() { return size_t(kStageFloats) * sizeof(float); }

cudaError_t set_harmonic_fast_attributes() {
    return cudaFuncSetAttribute(harmonic_fast_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(harmonic_fast_smem()));
}

void launch_harmonic_fast(const FusedArgs& a, uint32_t count, uint32_t max_span, cudaStream_t s) {
    const uint32_t blocks16 = (max_span + 15) / 16;
    const uint32_t ctas = (blocks16 + kHBlocks - 1) / kHBlocks;
    harmonic_fast_kernel<<<dim3(ctas ? ctas : 1, count), kHThreads, harmonic_fast_smem(), s>>>(a);
}

}  // namespace brp
