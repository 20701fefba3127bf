// Device building blocks shared by the compiled fused kernels (fused_fast.cu,
// fused_tc.cu): the padded shared-memory layout, the compile-time Stockham
// passes, the instruction-lean resampling index and the pass-1 gather.
//
// Resampling uses an instruction-lean form of the reference arithmetic that is
// bit-identical to it (src/science.cpp:20-40, :80):
//  * float(i) for i < 2^23 from the exponent trick 0x4B000000 | i;
//  * the table index int(x) for x in [0.5, 64.5] and float(int(x)) from one
//    add rounded toward -inf to 2^23 (its low mantissa bits are floor(x));
//  * (int)((double)index + 0.5) as trunc(fl_toward_zero(index + 0.5)): with
//    every integer below 2^24 representable, rounding toward zero never crosses
//    an integer, so truncating the rounded sum equals truncating the exact one.
// In the reference's FMA forms two samples go through packed FP32 instructions
// together (lean_index2), with the fractional part taken as y - floor(y).
// The reference-order function brp_resample_index (resample_math.h) remains the
// definition; tests compare both against the CPU resampler bit for bit.
#pragma once
#include "brp_internal.h"
#include "fft_device.cuh"
#include "resample_math.h"

namespace brp {
namespace {

// (sine, cosine) bit pairs: entry li is read as one 64-bit constant load
__constant__ __align__(8) uint32_t c_fast_lut_bits[130] = BRP_LUT_BITS;

// Gather modes: the low two bits select the index arithmetic (0: FP32
// reference order, 1: FP32 with the reference's FMA forms, 2: FP64 time
// index); kSmallIndex adds that every sample index is below 2^23, so float(i)
// needs no fallback for larger indices.
constexpr int kSmallIndex = 4;

// Shared-memory layout of the compiled kernels: element e of a sequence at
// e + e / 16 (one padding slot per 16 keeps radix-16 strided stores on distinct
// banks).  Sequences sit `stride` elements apart, stride = 16/G (mod 16)
// (G = sequences a warp touches side by side).
__host__ __device__ constexpr int ct_pos(int e) { return e + (e >> 4); }
__host__ __device__ constexpr int ct_stride(int L, int G) {
    int base = L + L / 16;
    int want = (G >= 16) ? 1 : 16 / G;
    int pad = ((want - base) % 16 + 16) % 16;
    return base + pad;
}

template <int R, bool PROD = false> struct TwStride {
    static constexpr int value = (pass_twiddle_powers(R, PROD) + 1) & ~1;
};

// v[r] *= W_{Ns R}^{r k} (r = 1..R-1).  The pass's table holds, for butterfly
// k, the twiddles of pass_twiddle_power, pair h at 16-byte entry h Ns + k.  In
// a product table (PROD, pass 2) radix 2, 4 and 8 load W^k, W^2k, W^4k and
// form W^3k, W^5k, W^6k, W^7k by one or two complex products, which trades
// table loads through L1 for FMA-pipe work; pass 1 (whose radix-8 pass ran
// faster with its table loads) and radix 3 and 16 load every twiddle.
template <int R, int Ns, bool PROD = false>
__device__ __forceinline__ void ct_twiddle(float2* v, const float2* __restrict__ tw, int k) {
    if constexpr (Ns > 1) {
        const float4* w4 = reinterpret_cast<const float4*>(tw) + k;
        if constexpr (pass_twiddle_products(R, PROD)) {
            const float4 a = __ldg(w4);
            const float2 w1 = make_float2(a.x, a.y), w2 = make_float2(a.z, a.w);
            if constexpr (R == 2) {
                v[1] = cmul(v[1], w1);
            } else if constexpr (R == 4) {
                v[3] = cmul(v[3], cmul(w1, w2));
                v[1] = cmul(v[1], w1);
                v[2] = cmul(v[2], w2);
            } else {
                const float4 b = __ldg(w4 + Ns);
                const float2 w4k = make_float2(b.x, b.y), w3 = cmul(w1, w2);
                v[7] = cmul(v[7], cmul(w3, w4k));
                v[6] = cmul(v[6], cmul(w2, w4k));
                v[5] = cmul(v[5], cmul(w1, w4k));
                v[4] = cmul(v[4], w4k);
                v[3] = cmul(v[3], w3);
                v[2] = cmul(v[2], w2);
                v[1] = cmul(v[1], w1);
            }
        } else {
#pragma unroll
            for (int r = 1; r < R; r += 2) {
                const float4 w = __ldg(w4 + ((r - 1) / 2) * Ns);
                v[r] = cmul(v[r], make_float2(w.x, w.y));
                if (r + 1 < R) v[r + 1] = cmul(v[r + 1], make_float2(w.z, w.w));
            }
        }
    }
}

// One Stockham pass: each thread loads its butterflies' inputs, the CTA
// synchronises, then each thread twiddles, transforms and stores in place.
template <int L, int STRIDE, int SEQ, int THREADS, int Ns, int R, bool PROD = false>
__device__ __forceinline__ void ct_pass(float2* buf, const float2* __restrict__ tw) {
    constexpr int NBF = L / R, TOTAL = NBF * SEQ, PER = (TOTAL + THREADS - 1) / THREADS;
    float2 v[PER][R];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int b = threadIdx.x + q * THREADS;
        if (TOTAL % THREADS == 0 || b < TOTAL) {
            const int c = b / NBF, j = b - c * NBF;
            const float2* src = buf + c * STRIDE;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = src[ct_pos(j + r * NBF)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int b = threadIdx.x + q * THREADS;
        if (TOTAL % THREADS == 0 || b < TOTAL) {
            const int c = b / NBF, j = b - c * NBF;
            const int k = j % Ns;
            ct_twiddle<R, Ns, PROD>(v[q], tw, k);
            dft<R>(v[q]);
            float2* dst = buf + c * STRIDE;
            const int base = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[ct_pos(base + r * Ns)] = v[q][r];
        }
    }
    __syncthreads();
}

template <bool PROD, int L, int STRIDE, int SEQ, int THREADS, int Ns, int R, int... Rest>
__device__ __forceinline__ void ct_fft(float2* buf, const float2* __restrict__ tw) {
    ct_pass<L, STRIDE, SEQ, THREADS, Ns, R, PROD>(buf, tw);
    if constexpr (sizeof...(Rest) > 0)
        ct_fft<PROD, L, STRIDE, SEQ, THREADS, Ns * R, Rest...>(buf, tw + (Ns > 1 ? Ns * TwStride<R, PROD>::value : 0));
}

// Number of float2 entries of the per-pass twiddle table of a radix sequence
// (PROD: a product table).
template <bool PROD, int Ns, int R, int... Rest>
__host__ __device__ constexpr int ct_table_size() {
    int here = Ns > 1 ? Ns * TwStride<R, PROD>::value : 0;
    if constexpr (sizeof...(Rest) > 0) return here + ct_table_size<PROD, Ns * R, Rest...>();
    else return here;
}

// ---- bit-identical lean resampling index (see the file comment) ----
template <bool SMALL>
__device__ __forceinline__ float u2f_exact(uint32_t i) {
    if (SMALL) return __fsub_rn(__int_as_float(0x4B000000 | int(i)), 8388608.0f);  // i < 2^23
    return i < (1u << 23) ? __fsub_rn(__int_as_float(0x4B000000 | int(i)), 8388608.0f) : __uint2float_rn(i);
}

template <bool FMA, bool SMALL = false>
__device__ __forceinline__ int lean_index(uint32_t i, const brp_resample_consts& p) {
    const float fi = u2f_exact<SMALL>(i);
    const float t = __fmul_rn(fi, p.dt);
    const float ph = FMA ? __fmaf_rn(p.omega, t, p.psi) : __fadd_rn(__fmul_rn(p.omega, t), p.psi);
    const float y = __fmul_rn(BRP_INV_TWO_PI_F, ph);
    float xt = __fsub_rn(y, truncf(y));
    if (xt < 0.f) xt = __fadd_rn(xt, 1.0f);
    const float x64 = FMA ? __fmaf_rn(xt, 64.0f, 0.5f) : __fadd_rn(__fmul_rn(xt, 64.0f), 0.5f);
    const float mg = __fadd_rd(x64, 8388608.0f);
    const int li = __float_as_int(mg) - 0x4B000000;
    const float fli = __fsub_rn(mg, 8388608.0f);
    const uint2 sc = reinterpret_cast<const uint2*>(c_fast_lut_bits)[li];
    const float s = __uint_as_float(sc.x), c = __uint_as_float(sc.y);
    float sn, off;
    if (FMA) {
        const float d = __fmul_rn(BRP_TWO_PI_F, __fmaf_rn(-fli, 0.015625f, xt));
        const float d2 = __fmul_rn(__fmul_rn(0.5f, d), d);
        sn = __fmaf_rn(-d2, s, __fmaf_rn(d, c, s));
        off = __fmaf_rn(__fmul_rn(p.tau, sn), p.step_inv, -p.s0);
    } else {
        const float d = __fmul_rn(BRP_TWO_PI_F, __fsub_rn(xt, __fmul_rn(0.015625f, fli)));
        const float d2 = __fmul_rn(d, __fmul_rn(0.5f, d));
        sn = __fsub_rn(__fadd_rn(s, __fmul_rn(d, c)), __fmul_rn(d2, s));
        off = __fsub_rn(__fmul_rn(__fmul_rn(p.tau, sn), p.step_inv), p.s0);
    }
    const float index = __fsub_rn(fi, off);
    return __float2int_rz(__fadd_rz(index, 0.5f));
}

// Packed FP32 operations of sm_100: two lanes per instruction, each lane the
// IEEE operation of the scalar form with the named rounding.
#define BRP_F2_OP2(name, op)                                                                      \
    __device__ __forceinline__ float2 name(float2 a, float2 b) {                                  \
        float2 r;                                                                                 \
        asm("{\n\t.reg .b64 a, b, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\t" op      \
            " d, a, b;\n\tmov.b64 {%0, %1}, d;\n\t}"                                                \
            : "=f"(r.x), "=f"(r.y)                                                                \
            : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));                                            \
        return r;                                                                                 \
    }
BRP_F2_OP2(add2_rn, "add.rn.f32x2")
BRP_F2_OP2(add2_rz, "add.rz.f32x2")
BRP_F2_OP2(add2_rm, "add.rm.f32x2")
BRP_F2_OP2(mul2_rn, "mul.rn.f32x2")
#undef BRP_F2_OP2

__device__ __forceinline__ float2 fma2_rn(float2 a, float2 b, float2 c) {
    float2 r;
    asm("{\n\t.reg .b64 a, b, c, d;\n\tmov.b64 a, {%2, %3};\n\tmov.b64 b, {%4, %5};\n\tmov.b64 c, {%6, %7};\n\t"
        "fma.rn.f32x2 d, a, b, c;\n\tmov.b64 {%0, %1}, d;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}

__device__ __forceinline__ float2 f2(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 neg2(float2 v) { return make_float2(-v.x, -v.y); }

// lean_index<true> (the reference's FMA forms) of two samples in packed
// operations, each step issued once for both samples.  The compiler fuses a
// packed multiply with a following packed add even when both carry an explicit
// rounding (CUDA 12.9), so this form is only bit-identical because none of its
// steps is such a pair: every product feeds an FMA as a factor, or (y, whose
// floor is taken too) has a second use.  The reference-order arithmetic has
// such pairs and stays scalar.  The bit-exact index tests run this form at
// n = 2^21 and 2^22 for every compiled pass-1 configuration.  Differences from
// the scalar form, each exact:
//  * a - b as a + (-b), and -(x y) as (-x) y;
//  * the fractional part y - trunc(y), plus 1 when negative, as
//    fl(y - floor(y)): y - trunc(y) is exact, and for y < 0 (not an integer)
//    y - floor(y) is that value plus 1, the same real number rounded once.
template <bool SMALL = false>
__device__ __forceinline__ int2 lean_index2(uint32_t i0, uint32_t i1, const brp_resample_consts& p) {
    float2 fi;
    if (SMALL)
        fi = add2_rn(make_float2(__int_as_float(0x4B000000 | int(i0)), __int_as_float(0x4B000000 | int(i1))),
                     f2(-8388608.0f));
    else
        fi = make_float2(u2f_exact<false>(i0), u2f_exact<false>(i1));
    const float2 t = mul2_rn(fi, f2(p.dt));
    const float2 ph = fma2_rn(f2(p.omega), t, f2(p.psi));
    const float2 y = mul2_rn(f2(BRP_INV_TWO_PI_F), ph);
    const float2 xt = add2_rn(y, make_float2(-floorf(y.x), -floorf(y.y)));
    const float2 x64 = fma2_rn(xt, f2(64.0f), f2(0.5f));
    const float2 mg = add2_rm(x64, f2(8388608.0f));
    const int li0 = __float_as_int(mg.x) - 0x4B000000, li1 = __float_as_int(mg.y) - 0x4B000000;
    const float2 fli = add2_rn(mg, f2(-8388608.0f));
    const uint2 sc0 = reinterpret_cast<const uint2*>(c_fast_lut_bits)[li0];
    const uint2 sc1 = reinterpret_cast<const uint2*>(c_fast_lut_bits)[li1];
    const float2 s = make_float2(__uint_as_float(sc0.x), __uint_as_float(sc1.x));
    const float2 c = make_float2(__uint_as_float(sc0.y), __uint_as_float(sc1.y));
    const float2 d = mul2_rn(f2(BRP_TWO_PI_F), fma2_rn(neg2(fli), f2(0.015625f), xt));
    const float2 d2 = mul2_rn(mul2_rn(f2(0.5f), d), d);
    const float2 sn = fma2_rn(neg2(d2), s, fma2_rn(d, c, s));
    const float2 off = fma2_rn(mul2_rn(f2(p.tau), sn), f2(p.step_inv), f2(-p.s0));
    const float2 r = add2_rz(add2_rn(fi, neg2(off)), f2(0.5f));
    return make_int2(__float2int_rz(r.x), __float2int_rz(r.y));
}

// Source indices j0, j1 of the adjacent samples ib and ib + 1 (the two reals of
// one complex point) in the index arithmetic MODE selects: -1 for a sample at
// or past the resampled length, and for one whose index falls outside the
// series, which also sets oob.
template <int MODE>
__device__ __forceinline__ void index_pair(uint32_t ib, const brp_resample_consts& rc, uint32_t steps,
                                           uint32_t unpadded, int& j0, int& j1, bool& oob) {
    constexpr bool SMALL = (MODE & kSmallIndex) != 0;
    j0 = j1 = -1;
    if (ib < steps) {
        int2 jj;
        if constexpr ((MODE & 3) == 2)
            jj = make_int2(brp_resample_index_fp64(ib, rc), brp_resample_index_fp64(ib + 1, rc));
        else if constexpr ((MODE & 3) == 1)
            jj = lean_index2<SMALL>(ib, ib + 1, rc);
        else
            jj = make_int2(lean_index<false, SMALL>(ib, rc), lean_index<false, SMALL>(ib + 1, rc));
        if (uint32_t(jj.x) < unpadded) j0 = jj.x;
        else oob = true;
        if (ib + 1 < steps) {
            if (uint32_t(jj.y) < unpadded) j1 = jj.y;
            else oob = true;
        }
    }
}

__device__ __forceinline__ brp_resample_consts consts_of(const brp_params& p) {
    brp_resample_consts c;
    c.tau = p.tau; c.omega = p.omega; c.psi = p.psi; c.dt = p.dt; c.step_inv = p.step_inv; c.s0 = p.s0;
    c.flags = p.flags;
    return c;
}

template <int THREADS>
__device__ __forceinline__ double block_sum_d(double v, double* scratch) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double r = 0;
    if (warp == 0) {
        r = lane < THREADS / 32 ? scratch[lane] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    }
    return r;
}

// Publishes this pass-1 CTA's FP64 sum of its samples (tot, valid in thread 0)
// and, in the CTA that completes the template's set (an atomic ticket taken
// after a fence), the template's padding value a.mean[g] = sum / steps, the
// partials summed in a fixed order.  That CTA re-arms the ticket, so the
// counters are zero again after every launch.  Every thread of the CTA calls
// this; it synchronises the CTA.
template <int THREADS>
__device__ __forceinline__ void publish_mean(const FusedArgs& a, int g, uint32_t steps, double tot, double* red) {
    __shared__ int s_last;
    double* pp = a.partial + size_t(g) * a.partial_stride;
    if (threadIdx.x == 0) {
        pp[blockIdx.x] = tot;
        __threadfence();
        s_last = atomicAdd(a.tickets + g, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double part = 0;
        for (uint32_t i = threadIdx.x; i < gridDim.x; i += THREADS) part += __ldcg(pp + i);
        const double all = block_sum_d<THREADS>(part, red);
        if (threadIdx.x == 0) {
            a.mean[g] = float(all / double(steps));
            a.tickets[g] = 0;
        }
    }
}

// Gathers this CTA's samples (rows n1 < L1, C complex points = 2C consecutive
// reals per row) into shared memory; returns the sum of the samples (FP32 per
// thread, a few dozen samples, then FP64 across threads).  Thread t handles
// column t % C of rows t / C + q THREADS / C: the two samples of a complex
// point, one 64-bit store; sample index and shared address advance by
// constants.
template <int L1, int C, int THREADS, int STRIDE, int MODE>
__device__ __forceinline__ double gather(float2* sm, const float* __restrict__ in, const brp_params& P,
                                         uint32_t L2, uint32_t c0, float* raw, bool& oob) {
    constexpr int TOTAL = L1 * C, PER = TOTAL / THREADS, ROWS_STEP = THREADS / C;
    static_assert(TOTAL % THREADS == 0 && THREADS % C == 0, "gather must tile the CTA");
    static_assert(ROWS_STEP % 16 == 0, "row step must keep the shared-memory padding periodic");
    const brp_resample_consts rc = consts_of(P);
    const uint32_t steps = P.steps, unpadded = P.unpadded;
    const int c = threadIdx.x % C, n1_0 = threadIdx.x / C;
    const uint32_t istep = 2u * L2 * ROWS_STEP;
    uint32_t i = 2u * (L2 * uint32_t(n1_0) + c0 + uint32_t(c));
    float2* dst = sm + c * STRIDE + ct_pos(n1_0);
    constexpr int DSTEP = ROWS_STEP + (ROWS_STEP / 16);
    float sum = 0.f;
    // Indices of a batch of points first, then all of the batch's loads, so each
    // thread keeps 2 BATCH gathers in flight.
    constexpr int BATCH = 4;
    static_assert(PER % BATCH == 0, "batch must divide the points per thread");
#pragma unroll 1
    for (int q0 = 0; q0 < PER; q0 += BATCH) {
        int j[2 * BATCH];
#pragma unroll
        for (int b = 0; b < BATCH; ++b)
            index_pair<MODE>(i + uint32_t(b) * istep, rc, steps, unpadded, j[2 * b], j[2 * b + 1], oob);
        float v[2 * BATCH];
#pragma unroll
        for (int b = 0; b < 2 * BATCH; ++b) v[b] = j[b] >= 0 ? __ldg(in + j[b]) : 0.f;
#pragma unroll
        for (int b = 0; b < BATCH; ++b) {
            if (raw) {
                const uint32_t ib = i + uint32_t(b) * istep;
                if (ib < steps) raw[ib] = v[2 * b];
                if (ib + 1 < steps) raw[ib + 1] = v[2 * b + 1];
            }
            sum += v[2 * b];
            sum += v[2 * b + 1];
            dst[b * DSTEP] = make_float2(v[2 * b], v[2 * b + 1]);
        }
        i += BATCH * istep;
        dst += BATCH * DSTEP;
    }
    return double(sum);
}

// Gather fused with the first Stockham pass (span 1, radix 16) when each
// thread owns exactly one of its butterflies (L1 C = 16 THREADS): thread
// t = j C + c gathers the 16 points n1 = j + r L1/16 of column c (the same
// points, sums and snapshot writes as gather; indices of eight points, then
// their 16 loads, twice), transforms them in registers and stores the 16
// outputs at 16 j + m, so the samples never take a shared-memory round trip
// before the first pass.
template <int L1, int C, int THREADS, int STRIDE, int MODE>
__device__ __forceinline__ double gather_dft16(float2* sm, const float* __restrict__ in, const brp_params& P,
                                               uint32_t L2, uint32_t c0, float* raw, bool& oob) {
    constexpr int NBF = L1 / 16;
    static_assert(L1 * C == 16 * THREADS, "one first-pass butterfly per thread");
    const brp_resample_consts rc = consts_of(P);
    const uint32_t steps = P.steps, unpadded = P.unpadded;
    const int t = threadIdx.x, c = t % C, j = t / C;
    const uint32_t istep = 2u * L2 * uint32_t(NBF);
    uint32_t i = 2u * (L2 * uint32_t(j) + c0 + uint32_t(c));
    float2 x[16];
    float sum = 0.f;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        int jx[16];
#pragma unroll
        for (int b = 0; b < 8; ++b)
            index_pair<MODE>(i + uint32_t(b) * istep, rc, steps, unpadded, jx[2 * b], jx[2 * b + 1], oob);
        float v[16];
#pragma unroll
        for (int b = 0; b < 16; ++b) v[b] = jx[b] >= 0 ? __ldg(in + jx[b]) : 0.f;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            if (raw) {
                const uint32_t ib = i + uint32_t(b) * istep;
                if (ib < steps) raw[ib] = v[2 * b];
                if (ib + 1 < steps) raw[ib + 1] = v[2 * b + 1];
            }
            sum += v[2 * b];
            sum += v[2 * b + 1];
            x[8 * q + b] = make_float2(v[2 * b], v[2 * b + 1]);
        }
        i += 8u * istep;
    }
    dft16(x);
    float2* dst = sm + c * STRIDE + ct_pos(16 * j);
#pragma unroll
    for (int m = 0; m < 16; ++m) dst[m] = x[m];
    return double(sum);
}

// Last Stockham pass of pass 1 (span Ns, radix R, Ns R = L) fused with the
// four-step twiddle and the store of the transformed columns:
//     T[k1][c0 + c] = Y[c][k1] W_M^{(c0 + c) k1}.
// Butterfly b of the pass takes column c = b % SEQ and j = b / SEQ, so a warp
// stores 32/SEQ rows of SEQ adjacent columns; its outputs are rows k1 = j + m Ns.
// The twiddle is W_M^{n2 j} W_M^{n2 m Ns} (n2 = c0 + c): one two-level table
// value per butterfly times the CTA's column factors, computed once into shared
// memory (rows padded by one entry, so the columns a warp reads sit on
// distinct banks).  Every thread of the CTA calls this; it synchronises the CTA.
template <int L, int STRIDE, int SEQ, int THREADS, int Ns, int R>
__device__ __forceinline__ void ct_last_pass_store(const float2* buf, const float2* __restrict__ tw,
                                                   float2* __restrict__ T, const float2* fs_hi, const float2* fs_lo,
                                                   uint32_t L2, uint32_t c0) {
    constexpr int NBF = L / R, TOTAL = NBF * SEQ, PER = (TOTAL + THREADS - 1) / THREADS;
    static_assert(Ns * R == L && THREADS % SEQ == 0, "last-pass tiling");
    __shared__ float2 s_fs[SEQ][R + 1];
    for (int t = threadIdx.x; t < SEQ * R; t += THREADS)
        s_fs[t / R][t % R] = twiddle2(fs_hi, fs_lo, kSplitLog2, (c0 + uint32_t(t / R)) * uint32_t((t % R) * Ns));
    __syncthreads();
    const int c = threadIdx.x % SEQ;
    const uint32_t n2 = c0 + uint32_t(c);
    const float2* src = buf + c * STRIDE;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        if (TOTAL % THREADS != 0 && threadIdx.x + q * THREADS >= TOTAL) break;
        const int j = threadIdx.x / SEQ + q * (THREADS / SEQ);
        float2 v[R];
#pragma unroll
        for (int r = 0; r < R; ++r) v[r] = src[ct_pos(j + r * NBF)];
        ct_twiddle<R, Ns>(v, tw, j);
        dft<R>(v);
        const float2 base = twiddle2(fs_hi, fs_lo, kSplitLog2, n2 * uint32_t(j));
#pragma unroll
        for (int m = 0; m < R; ++m) T[size_t(j + m * Ns) * L2 + n2] = cmul(v[m], cmul(base, s_fs[c][m]));
    }
}

// The shared-memory passes of pass 1 with the last one fused with the store.
template <int L, int STRIDE, int SEQ, int THREADS, int Ns, int R, int... Rest>
__device__ __forceinline__ void ct_fft_store(float2* buf, const float2* __restrict__ tw, float2* __restrict__ T,
                                             const float2* fs_hi, const float2* fs_lo, uint32_t L2, uint32_t c0) {
    if constexpr (sizeof...(Rest) == 0) {
        ct_last_pass_store<L, STRIDE, SEQ, THREADS, Ns, R>(buf, tw, T, fs_hi, fs_lo, L2, c0);
    } else {
        ct_pass<L, STRIDE, SEQ, THREADS, Ns, R>(buf, tw);
        ct_fft_store<L, STRIDE, SEQ, THREADS, Ns * R, Rest...>(buf, tw + (Ns > 1 ? Ns * TwStride<R>::value : 0), T,
                                                              fs_hi, fs_lo, L2, c0);
    }
}

// ct_last_pass_store with the outputs written as the CTA's L x SEQ tile of T
// ([row][column], at the first 128-byte boundary of buf) instead of to T: the
// butterflies of all of a thread's iterations are transformed into registers,
// the CTA synchronises (every read of buf done), the tile is written (a warp's
// 32 stores of one output are 256 contiguous bytes) and fenced for the
// asynchronous proxy, and after a second barrier the caller's one thread sends
// it to T by bulk tensor copies (tma_store.cuh).  Returns the tile's address.
template <int L, int STRIDE, int SEQ, int THREADS, int Ns, int R>
__device__ __forceinline__ uint32_t ct_last_pass_tile(float2* buf, const float2* __restrict__ tw,
                                                      const float2* fs_hi, const float2* fs_lo, uint32_t c0) {
    constexpr int NBF = L / R, TOTAL = NBF * SEQ, PER = TOTAL / THREADS;
    static_assert(Ns * R == L && THREADS % SEQ == 0 && TOTAL % THREADS == 0, "last-pass tiling");
    __shared__ float2 s_fs[SEQ][R + 1];
    for (int t = threadIdx.x; t < SEQ * R; t += THREADS)
        s_fs[t / R][t % R] = twiddle2(fs_hi, fs_lo, kSplitLog2, (c0 + uint32_t(t / R)) * uint32_t((t % R) * Ns));
    __syncthreads();
    const int c = threadIdx.x % SEQ;
    const uint32_t n2 = c0 + uint32_t(c);
    const float2* src = buf + c * STRIDE;
    float2 v[PER][R];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int j = threadIdx.x / SEQ + q * (THREADS / SEQ);
#pragma unroll
        for (int r = 0; r < R; ++r) v[q][r] = src[ct_pos(j + r * NBF)];
        ct_twiddle<R, Ns>(v[q], tw, j);
        dft<R>(v[q]);
        const float2 base = twiddle2(fs_hi, fs_lo, kSplitLog2, n2 * uint32_t(j));
#pragma unroll
        for (int m = 0; m < R; ++m) v[q][m] = cmul(v[q][m], cmul(base, s_fs[c][m]));
    }
    __syncthreads();
    const uint32_t buf_sh = static_cast<uint32_t>(__cvta_generic_to_shared(buf));
    const uint32_t tile_sh = (buf_sh + 127u) & ~127u;
    float2* tile = buf + (tile_sh - buf_sh) / 8;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const int j = threadIdx.x / SEQ + q * (THREADS / SEQ);
#pragma unroll
        for (int m = 0; m < R; ++m) tile[(j + m * Ns) * SEQ + c] = v[q][m];
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    return tile_sh;
}

// ct_fft_store with the last pass as ct_last_pass_tile; returns the tile's address.
template <int L, int STRIDE, int SEQ, int THREADS, int Ns, int R, int... Rest>
__device__ __forceinline__ uint32_t ct_fft_tile(float2* buf, const float2* __restrict__ tw, const float2* fs_hi,
                                                const float2* fs_lo, uint32_t c0) {
    if constexpr (sizeof...(Rest) == 0) {
        return ct_last_pass_tile<L, STRIDE, SEQ, THREADS, Ns, R>(buf, tw, fs_hi, fs_lo, c0);
    } else {
        ct_pass<L, STRIDE, SEQ, THREADS, Ns, R>(buf, tw);
        return ct_fft_tile<L, STRIDE, SEQ, THREADS, Ns * R, Rest...>(buf, tw + (Ns > 1 ? Ns * TwStride<R>::value : 0),
                                                                     fs_hi, fs_lo, c0);
    }
}

}  // namespace
}  // namespace brp
