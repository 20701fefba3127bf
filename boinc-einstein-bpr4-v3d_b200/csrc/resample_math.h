// Resampling arithmetic shared by the host (template set-up) and the device
// (resample kernels).  The index of output sample i is
//     j(i) = (int)((double)((float)i - offset(i)) + 0.5)
//     offset(i) = tau * sin(omega * float(i)*dt + psi) * step_inv - s0
// with the sine taken from a 65-point table, every FP32 operation rounded
// separately unless Params.flags bit 2 asks for fused multiply-adds.  This is
// the arithmetic of the reference's CPU resampler (src/science.cpp:20-40,
// :75-85); the resampled indices must match it bit for bit, so the order of
// operations below is fixed and must not be contracted or reassociated.
#pragma once
#include <stdint.h>
#include <math.h>

// The 65-point sine/cosine table of Einstein@Home erp_utilities.cpp, carried by
// the reference as include/brp/lut.hpp:4-5.  IEEE-754 bit patterns, interleaved
// (sin, cos).  Entry 64 repeats entry 0 (with the reference's -0.0 sine).
#define BRP_LUT_BITS { \
0x00000000, 0x3f800000, 0x3dc8bd23, 0x3f7ec472, 0x3e47c5ac, 0x3f7b14ba, 0x3e94a03c, 0x3f74fa05, \
    0x3ec3ef07, 0x3f6c8366, 0x3ef15af3, 0x3f61c593, 0x3f0e39d6, 0x3f54db38, 0x3f226794, 0x3f45e3fc, \
    0x3f3504f7, 0x3f3504f7, 0x3f45e3fc, 0x3f226794, 0x3f54db38, 0x3f0e39d6, 0x3f61c593, 0x3ef15af3, \
    0x3f6c8366, 0x3ec3ef07, 0x3f74fa05, 0x3e94a03c, 0x3f7b14ba, 0x3e47c5ac, 0x3f7ec472, 0x3dc8bd23, \
    0x3f800000, 0x00000000, 0x3f7ec472, 0xbdc8bd23, 0x3f7b14ba, 0xbe47c5ac, 0x3f74fa05, 0xbe94a03c, \
    0x3f6c8366, 0xbec3ef07, 0x3f61c593, 0xbef15af3, 0x3f54db38, 0xbf0e39d6, 0x3f45e3fc, 0xbf226794, \
    0x3f3504f7, 0xbf3504f7, 0x3f226794, 0xbf45e3fc, 0x3f0e39d6, 0xbf54db38, 0x3ef15af3, 0xbf61c593, \
    0x3ec3ef07, 0xbf6c8366, 0x3e94a03c, 0xbf74fa05, 0x3e47c5ef, 0xbf7b14ba, 0x3dc8bd23, 0xbf7ec472, \
    0x00000000, 0xbf800000, 0xbdc8bd23, 0xbf7ec472, 0xbe47c5ac, 0xbf7b14ba, 0xbe94a01b, 0xbf74fa05, \
    0xbec3ef07, 0xbf6c8366, 0xbef15af3, 0xbf61c593, 0xbf0e39d6, 0xbf54db38, 0xbf226794, 0xbf45e40d, \
    0xbf3504f7, 0xbf3504f7, 0xbf45e3fc, 0xbf226794, 0xbf54db27, 0xbf0e39d6, 0xbf61c593, 0xbef15af3, \
    0xbf6c8366, 0xbec3ef28, 0xbf74fa05, 0xbe94a03c, 0xbf7b14ba, 0xbe47c5ac, 0xbf7ec472, 0xbdc8bd23, \
    0xbf800000, 0x00000000, 0xbf7ec472, 0x3dc8bd23, 0xbf7b14ba, 0x3e47c5ac, 0xbf74fa05, 0x3e94a03c, \
    0xbf6c8366, 0x3ec3ef07, 0xbf61c593, 0x3ef15af3, 0xbf54db38, 0x3f0e39d6, 0xbf45e40d, 0x3f226794, \
    0xbf3504f7, 0x3f3504f7, 0xbf2267a5, 0x3f45e3fc, 0xbf0e39d6, 0x3f54db38, 0xbef15af3, 0x3f61c593, \
    0xbec3ef28, 0x3f6c8356, 0xbe94a03c, 0x3f74fa05, 0xbe47c5ef, 0x3f7b14ba, 0xbdc8bd23, 0x3f7ec472, \
    0x80000000, 0x3f800000 }

#if defined(__CUDACC__)
#define BRP_HD __host__ __device__ __forceinline__
#else
#define BRP_HD static inline
#endif

// Separately rounded FP32 operations.  On the device the _rn intrinsics are
// never fused by the compiler; host code is compiled with -ffp-contract=off.
#if defined(__CUDA_ARCH__)
#define BRP_MUL(a, b) __fmul_rn((a), (b))
#define BRP_ADD(a, b) __fadd_rn((a), (b))
#define BRP_SUB(a, b) __fsub_rn((a), (b))
#define BRP_FMA(a, b, c) __fmaf_rn((a), (b), (c))
#define BRP_TRUNC(a) truncf(a)
#else
#define BRP_MUL(a, b) ((float)(a) * (float)(b))
#define BRP_ADD(a, b) ((float)(a) + (float)(b))
#define BRP_SUB(a, b) ((float)(a) - (float)(b))
#define BRP_FMA(a, b, c) fmaf((a), (b), (c))
#define BRP_TRUNC(a) truncf(a)
#endif

// 1.0f/6.283185f and 6.283185f as the reference's compiler folds them.
#define BRP_INV_TWO_PI_F 0.15915495f
#define BRP_TWO_PI_F 6.283185f

#if defined(__CUDA_ARCH__)
#define BRP_BITS_TO_FLOAT(b) __uint_as_float(b)
#else
#include <string.h>
BRP_HD float brp_bits_to_float(uint32_t b) { float f; memcpy(&f, &b, 4); return f; }
#define BRP_BITS_TO_FLOAT(b) brp_bits_to_float(b)
#endif

// Fractional part with the sign of x, as modff: x - trunc(x) is exact in IEEE
// arithmetic.  The result may be +0 where modff gives -0; both take the same
// branch below and give the same table index and sine.
BRP_HD float brp_frac(float x) { return BRP_SUB(x, BRP_TRUNC(x)); }

// src/science.cpp:20-28.
BRP_HD float brp_lut_sin(float x, const uint32_t* lut) {
    float xt = brp_frac(BRP_MUL(BRP_INV_TWO_PI_F, x));
    if (xt < 0) xt = BRP_ADD(xt, 1.0f);
    int i = (int)BRP_ADD(BRP_MUL(xt, 64.0f), 0.5f);
    float d = BRP_MUL(BRP_TWO_PI_F, BRP_SUB(xt, BRP_MUL(0.015625f, (float)i)));
    float d2 = BRP_MUL(d, BRP_MUL(0.5f, d));
    float s = BRP_BITS_TO_FLOAT(lut[2 * i]), c = BRP_BITS_TO_FLOAT(lut[2 * i + 1]);
    return BRP_SUB(BRP_ADD(s, BRP_MUL(d, c)), BRP_MUL(d2, s));
}

// src/science.cpp:29-35.
BRP_HD float brp_fused_sin(float phase, const uint32_t* lut) {
    float xt = brp_frac(BRP_MUL(BRP_INV_TWO_PI_F, phase));
    if (xt < 0) xt = BRP_ADD(xt, 1.0f);
    int i = (int)BRP_FMA(xt, 64.0f, 0.5f);
    float d = BRP_MUL(BRP_TWO_PI_F, BRP_FMA(-(float)i, 0.015625f, xt));
    float d2 = BRP_MUL(BRP_MUL(0.5f, d), d);
    float s = BRP_BITS_TO_FLOAT(lut[2 * i]), c = BRP_BITS_TO_FLOAT(lut[2 * i + 1]);
    return BRP_FMA(-d2, s, BRP_FMA(d, c, s));
}

struct brp_resample_consts { float tau, omega, psi, dt, step_inv, s0; uint32_t flags; };

// src/science.cpp:36-40.
BRP_HD float brp_sample_offset(uint32_t i, const brp_resample_consts& p, const uint32_t* lut) {
    float t = BRP_MUL((float)i, p.dt);
    if (p.flags & 2u) return BRP_FMA(BRP_MUL(p.tau, brp_fused_sin(BRP_FMA(p.omega, t, p.psi), lut)), p.step_inv, -p.s0);
    return BRP_SUB(BRP_MUL(BRP_MUL(p.tau, brp_lut_sin(BRP_ADD(BRP_MUL(p.omega, t), p.psi), lut)), p.step_inv), p.s0);
}

// src/science.cpp:80: the +0.5 is a double addition (exact for any float) and
// the conversion truncates toward zero.
BRP_HD int brp_resample_index(uint32_t i, const brp_resample_consts& p, const uint32_t* lut) {
    float index = BRP_SUB((float)i, brp_sample_offset(i, p, lut));
    return (int)((double)index + 0.5);
}

// Extension (Params.flags bit 8): the time index in FP64 with an accurate sine,
// t + tau*sin(Omega*t + psi), relative to the same S0 reference point.
BRP_HD int brp_resample_index_fp64(uint32_t i, const brp_resample_consts& p) {
    double t = (double)i * (double)p.dt;
    double offset = (double)p.tau * (sin((double)p.omega * t + (double)p.psi) - sin((double)p.psi)) / (double)p.dt;
    return (int)((double)i - offset + 0.5);
}
