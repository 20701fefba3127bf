// Device building blocks of the FP32 Stockham FFTs: register DFTs of radix
// 2, 3, 4, 8 and 16 and a shared-memory Stockham pass over several
// independent sequences held in one CTA.
//
// Stockham autosort pass (radix R, span Ns = product of the radices already
// applied, L points): butterfly j in [0, L/R) with k = j mod Ns reads
// x_r = a[j + r L/R], multiplies by W_{Ns R}^{r k}, takes the R-point DFT y_m
// and writes y_m to a[(j / Ns) Ns R + k + m Ns].  Input and output are in
// natural order; radices may come in any order.  Twiddles come from a table
// W_L^e, e in [0, L), generated in FP64 and rounded once to FP32.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace brp {

struct cf { float x, y; };

// complex sum and difference as one packed FP32 add each (sm_100)
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return __fadd2_rn(a, make_float2(-b.x, -b.y)); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i
__device__ __forceinline__ float2 cmul_mi(float2 a) { return make_float2(a.y, -a.x); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// ---- register DFTs (forward, X_k = sum_n x_n e^{-2 pi i n k / R}) ----
__device__ __forceinline__ void dft2(float2& a, float2& b) {
    float2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

__device__ __forceinline__ void dft3(float2* v) {
    const float h = 0.866025403784438647f;  // sqrt(3)/2
    float2 t = cadd(v[1], v[2]), d = csub(v[1], v[2]);
    float2 c = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    float2 r = make_float2(h * d.y, -h * d.x);  // -i sqrt(3)/2 d
    v[0] = cadd(v[0], t);
    v[1] = cadd(c, r);
    v[2] = csub(c, r);
}

// in-place DFT of v[0], v[s], v[2s], v[3s]
template <int S>
__device__ __forceinline__ void dft4s(float2* v) {
    float2 a0 = v[0], a1 = v[S], a2 = v[2 * S], a3 = v[3 * S];
    float2 s02 = cadd(a0, a2), d02 = csub(a0, a2), s13 = cadd(a1, a3), d13 = cmul_mi(csub(a1, a3));
    v[0] = cadd(s02, s13);
    v[2 * S] = csub(s02, s13);
    v[S] = cadd(d02, d13);
    v[3 * S] = csub(d02, d13);
}

__device__ __forceinline__ void dft4(float2* v) { dft4s<1>(v); }

// v holds 8 inputs in natural order; on return the 8 outputs in natural order.
__device__ __forceinline__ void dft8(float2* v) {
    const float r = 0.707106781186547524f;
    float2 e[4] = {v[0], v[2], v[4], v[6]}, o[4] = {v[1], v[3], v[5], v[7]};
    dft4(e);
    dft4(o);
    o[1] = make_float2(r * (o[1].x + o[1].y), r * (o[1].y - o[1].x));   // * (1 - i)/sqrt2
    o[2] = cmul_mi(o[2]);                                                // * -i
    o[3] = make_float2(r * (o[3].y - o[3].x), -r * (o[3].x + o[3].y));  // * (-1 - i)/sqrt2
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        v[k] = cadd(e[k], o[k]);
        v[k + 4] = csub(e[k], o[k]);
    }
}

__device__ __forceinline__ void dft16(float2* v) {
    const float c1 = 0.923879532511286756f, s1 = 0.382683432365089772f, r = 0.707106781186547524f;
    float2 e[8], o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { e[k] = v[2 * k]; o[k] = v[2 * k + 1]; }
    dft8(e);
    dft8(o);
    // o[k] *= W16^k = cos(pi k/8) - i sin(pi k/8)
    o[1] = cmul(o[1], make_float2(c1, -s1));
    o[2] = make_float2(r * (o[2].x + o[2].y), r * (o[2].y - o[2].x));
    o[3] = cmul(o[3], make_float2(s1, -c1));
    o[4] = cmul_mi(o[4]);
    o[5] = cmul(o[5], make_float2(-s1, -c1));
    o[6] = make_float2(r * (o[6].y - o[6].x), -r * (o[6].x + o[6].y));
    o[7] = cmul(o[7], make_float2(-c1, -s1));
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        v[k] = cadd(e[k], o[k]);
        v[k + 8] = csub(e[k], o[k]);
    }
}

template <int R>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) dft2(v[0], v[1]);
    else if constexpr (R == 3) dft3(v);
    else if constexpr (R == 4) dft4(v);
    else if constexpr (R == 8) dft8(v);
    else if constexpr (R == 16) dft16(v);
}

// Shared-memory layout of one sequence: element e at e + e/16 (one padding
// slot per 16 elements keeps radix-16 strided stores conflict-free); sequences
// are `stride` elements apart (stride = L + L/16 + 1, the +1 staggers the banks
// of different sequences).
__device__ __forceinline__ int smem_pos(int e) { return e + (e >> 4); }
__host__ __device__ constexpr int smem_stride(int L) { return L + L / 16 + 1; }

// One Stockham pass over `count` sequences of length L in shared memory.
// MAXB bounds the butterflies one thread holds (count*L/R <= MAXB*blockDim.x).
template <int R, int MAXB>
__device__ __forceinline__ void stockham_pass(float2* buf, int L, int stride, int count, int Ns,
                                              const float2* __restrict__ tw) {
    const int nbf = L / R, total = nbf * count, tstep = L / (Ns * R);
    float2 v[MAXB][R];
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        int b = threadIdx.x + q * blockDim.x;
        if (b < total) {
            int c = b / nbf, j = b - c * nbf;
            const float2* src = buf + c * stride;
#pragma unroll
            for (int r = 0; r < R; ++r) v[q][r] = src[smem_pos(j + r * nbf)];
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXB; ++q) {
        int b = threadIdx.x + q * blockDim.x;
        if (b < total) {
            int c = b / nbf, j = b - c * nbf;
            int k = j % Ns;
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) v[q][r] = cmul(v[q][r], __ldg(tw + r * k * tstep));
            }
            dft<R>(v[q]);
            float2* dst = buf + c * stride;
            int base = (j / Ns) * Ns * R + k;
#pragma unroll
            for (int r = 0; r < R; ++r) dst[smem_pos(base + r * Ns)] = v[q][r];
        }
    }
    __syncthreads();
}

// A radix plan: up to 6 passes, radices from {16, 8, 4, 3, 2}.
struct RadixPlan {
    int count;
    int radix[6];
};

// Runs all passes of `plan` on `count` sequences of length L held in shared memory.
template <int MAXE>
__device__ __forceinline__ void fft_smem(float2* buf, int L, int stride, int count, const RadixPlan& plan,
                                         const float2* __restrict__ tw) {
    int Ns = 1;
    for (int p = 0; p < plan.count; ++p) {
        int R = plan.radix[p];
        switch (R) {
            case 16: stockham_pass<16, (MAXE + 15) / 16>(buf, L, stride, count, Ns, tw); break;
            case 8: stockham_pass<8, (MAXE + 7) / 8>(buf, L, stride, count, Ns, tw); break;
            case 4: stockham_pass<4, (MAXE + 3) / 4>(buf, L, stride, count, Ns, tw); break;
            case 3: stockham_pass<3, (MAXE + 2) / 3>(buf, L, stride, count, Ns, tw); break;
            default: stockham_pass<2, (MAXE + 1) / 2>(buf, L, stride, count, Ns, tw); break;
        }
        Ns *= R;
    }
}

// e^{-2 pi i e / P} from two tables: hi[e / split] = W_P^{split*(e/split)},
// lo[e % split] = W_P^{e % split} (both FP64-generated, rounded to FP32).
__device__ __forceinline__ float2 twiddle2(const float2* __restrict__ hi, const float2* __restrict__ lo,
                                           uint32_t split_log2, uint32_t e) {
    return cmul(__ldg(hi + (e >> split_log2)), __ldg(lo + (e & ((1u << split_log2) - 1))));
}

}  // namespace brp
