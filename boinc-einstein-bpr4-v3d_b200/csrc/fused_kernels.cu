// Fused per-template search pipeline: three kernels per group of templates.
//
//   pass 1  resample + pack + column FFTs + four-step twiddle
//           Each CTA owns C columns n2 of the packed series z[s] = r[2s] + i r[2s+1]
//           viewed as an L1 x L2 matrix (s = L2 n1 + n2).  It gathers the
//           resampled samples straight from the input series (no resampled
//           copy in HBM), transforms its columns (length L1) in shared memory
//           and writes T[k1][n2] = W_M^{n2 k1} Y_{n2}[k1].  Samples at or
//           beyond `steps` enter as zero; the mean padding is restored in the
//           spectrum by pass 2.  Per-CTA FP64 sums of the samples feed the mean.
//   pass 2  row FFTs + real post-process + padding term + power
//           Each CTA owns rows k1 in [qR, qR+R) and their mirrors L1-k1 (row 0
//           pairs with itself, and the CTA of q = 0 also takes row L1/2).  After
//           the row FFTs (length L2) it holds Z_k and Z_{M-k} for every bin k of
//           its rows, forms the real spectrum
//             X_k = 1/2 [(Z_k + Z*_{M-k}) - i W_N^k (Z_k - Z*_{M-k})] + mean G_k,
//           with G_k the closed-form DFT of the padding indicator [steps, n),
//           and writes P_k = |X_k|^2 / n (P_0 = 0).
//   harmonic dyadic harmonic sums, per-level maximum, threshold, compaction
//           (see harmonic_kernel below).
//
// HBM traffic per template: the series gather (4n bytes, shared by every
// template of a bank), T written and read (8n), P written and read (4n).
#include "brp_internal.h"
#include "fft_device.cuh"
#include "resample_math.h"

namespace brp {

__constant__ uint32_t c_lut_bits[130] = BRP_LUT_BITS;

namespace {

__device__ __forceinline__ RadixPlan load_plan(const int* p) {
    RadixPlan r;
    r.count = p[0];
#pragma unroll
    for (int i = 0; i < 6; ++i) r.radix[i] = p[1 + i];
    return r;
}

__device__ __forceinline__ brp_resample_consts resample_consts(const brp_params& p) {
    brp_resample_consts c;
    c.tau = p.tau; c.omega = p.omega; c.psi = p.psi; c.dt = p.dt; c.step_inv = p.step_inv; c.s0 = p.s0;
    c.flags = p.flags;
    return c;
}

// x mod n for n = 2^s or 3 * 2^s.
__device__ __forceinline__ uint32_t mod_n(uint64_t x, uint32_t n) {
    if ((n & (n - 1)) == 0) return uint32_t(x & (n - 1));
    uint32_t s = __ffs(n) - 1;
    return uint32_t((((x >> s) % 3ull) << s) | (x & ((1ull << s) - 1)));
}

// Shared-memory sequence stride: L + L/16 + pad with stride = 16/G (mod 16),
// G = number of sequences a warp touches side by side (keeps those accesses on
// distinct banks).
__host__ __device__ __forceinline__ int seq_stride(int L, int G) {
    int base = L + L / 16;
    int want = (G >= 16) ? 1 : 16 / G;
    int pad = ((want - base) % 16 + 16) % 16;
    return base + pad;
}

template <int THREADS>
__device__ __forceinline__ double block_sum(double v, double* scratch) {
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
    return r;  // valid in thread 0
}

template <int MAXE, int THREADS>
__global__ void __launch_bounds__(THREADS) pass1_kernel(FusedArgs a) {
    extern __shared__ float2 sm[];
    __shared__ double red[THREADS / 32];
    const int g = blockIdx.y;
    const brp_params& P = a.params[g];
    const uint32_t steps = P.steps, unpadded = P.unpadded;
    const brp_resample_consts rc = resample_consts(P);
    const bool fp64_index = (P.flags & BRP_FLAG_INDEX_FP64) != 0;
    const float* __restrict__ in = a.inputs[g];
    const int L1 = a.L1, L2 = a.L2, C = a.C;
    const int stride = seq_stride(L1, C);
    const int c0 = blockIdx.x * C;
    const int rowlen = 2 * C;
    float* smf = reinterpret_cast<float*>(sm);
    float* raw = (g == a.snap) ? a.snap_raw : nullptr;

    double sum = 0;
    bool oob = false;
    const int total = L1 * rowlen;
    for (int idx = threadIdx.x; idx < total; idx += THREADS) {
        const int n1 = idx / rowlen, rem = idx - n1 * rowlen;
        const uint32_t i = 2u * (uint32_t(L2) * n1 + c0) + rem;
        float v = 0.f;
        if (i < steps) {
            int j = fp64_index ? brp_resample_index_fp64(i, rc) : brp_resample_index(i, rc, c_lut_bits);
            if (j < 0 || uint32_t(j) >= unpadded) oob = true;
            else v = __ldg(in + j);
            if (raw) raw[i] = v;
        }
        sum += v;
        smf[2 * ((rem >> 1) * stride + smem_pos(n1)) + (rem & 1)] = v;
    }
    if (oob) atomicOr(a.status + g, BRP_STATUS_RESAMPLE_OOB);
    double total_sum = block_sum<THREADS>(sum, red);
    if (threadIdx.x == 0) a.partial[size_t(g) * a.partial_stride + blockIdx.x] = total_sum;
    __syncthreads();

    fft_smem<MAXE>(sm, L1, stride, C, load_plan(a.plan1), a.tw1);

    float2* __restrict__ T = a.work + size_t(g) * a.work_stride;
    for (int idx = threadIdx.x; idx < L1 * C; idx += THREADS) {
        const int k1 = idx / C, c = idx - k1 * C;
        float2 y = sm[c * stride + smem_pos(k1)];
        const uint32_t e = uint32_t(c0 + c) * uint32_t(k1);  // < M
        y = cmul(y, twiddle2(a.fs_hi, a.fs_lo, kSplitLog2, e));
        T[size_t(k1) * L2 + c0 + c] = y;
    }
}

// Real-spectrum bin from Z_k, Z_{M-k} (W = W_N^k) plus the padding term.
__device__ __forceinline__ float2 real_bin(float2 zk, float2 zm, float2 w, float2 pad) {
    float2 s = make_float2(zk.x + zm.x, zk.y - zm.y);   // Z_k + conj(Z_{M-k})
    float2 d = make_float2(zk.x - zm.x, zk.y + zm.y);   // Z_k - conj(Z_{M-k})
    float2 t = cmul(w, d);                              // W d
    // 1/2 [s - i t] = 1/2 [(s.x + t.y), (s.y - t.x)]
    return make_float2(0.5f * (s.x + t.y) + pad.x, 0.5f * (s.y - t.x) + pad.y);
}

template <int MAXE, int THREADS>
__global__ void __launch_bounds__(THREADS) pass2_kernel(FusedArgs a) {
    extern __shared__ float2 sm[];
    __shared__ double red[THREADS / 32];
    __shared__ float s_mean;
    const int g = blockIdx.y, q = blockIdx.x;
    const brp_params& P = a.params[g];
    const int L1 = a.L1, L2 = a.L2, R = a.R;
    const uint32_t n = a.n, M = a.M, steps = P.steps;
    const int stride = seq_stride(L2, R);
    const float2* __restrict__ T = a.work + size_t(g) * a.work_stride;

    // Rows: [0, R) = qR + r; [R, 2R) = mirror rows L1 - (qR + r), row L1/2 in place of row 0's mirror.
    for (int idx = threadIdx.x; idx < 2 * R * L2; idx += THREADS) {
        const int rr = idx / L2, k2 = idx - rr * L2;
        int row;
        if (rr < R) row = q * R + rr;
        else {
            int ar = q * R + (rr - R);
            row = ar == 0 ? L1 / 2 : L1 - ar;
        }
        sm[rr * stride + smem_pos(k2)] = T[size_t(row) * L2 + k2];
    }
    double part = 0;
    const double* pp = a.partial + size_t(g) * a.partial_stride;
    for (uint32_t i = threadIdx.x; i < uint32_t(L2 / a.C); i += THREADS) part += pp[i];
    double tot = block_sum<THREADS>(part, red);
    if (threadIdx.x == 0) {
        float mean = float(tot / double(steps));
        s_mean = mean;
        if (q == 0) a.mean[g] = mean;
    }
    __syncthreads();
    const float mean = s_mean;

    fft_smem<MAXE>(sm, L2, stride, 2 * R, load_plan(a.plan2), a.tw2);

    float* __restrict__ Pw = a.power + size_t(g) * a.power_stride;
    float2* fft = (g == a.snap) ? a.snap_fft : nullptr;
    const float inv_n = 1.0f / float(n);
    const bool pow2 = (n & (n - 1)) == 0;
    const bool a_odd = steps & 1u;
    const float pad0 = float(n - steps) * mean;

    for (int idx = threadIdx.x; idx < R * L2; idx += THREADS) {
        const int r = idx % R, k2 = idx / R;
        const int arow = q * R + r;
        if (arow == 0) {
            // Row 0 pairs with itself at (L2 - k2) mod L2; row L1/2 at L2-1-k2.
            for (int which = 0; which < 2; ++which) {
                const int rr = which == 0 ? 0 : R;
                const uint32_t k = which == 0 ? uint32_t(L1) * k2 : uint32_t(L1 / 2) + uint32_t(L1) * k2;
                const int m2 = which == 0 ? (L2 - k2) % L2 : L2 - 1 - k2;
                float2 zk = sm[rr * stride + smem_pos(k2)], zm = sm[rr * stride + smem_pos(m2)];
                float2 X;
                if (k == 0) {
                    X = make_float2(zk.x + zk.y + pad0, 0.f);
                    if (fft) fft[M] = make_float2(zk.x - zk.y - (a_odd ? mean : 0.f), 0.f);
                    Pw[0] = 0.f;
                } else {
                    float sv, cv;
                    sincospif(float(k) / float(n), &sv, &cv);
                    float2 wa = twiddle2(a.rl_hi, a.rl_lo, kSplitLog2, mod_n(uint64_t(k) * steps, n));
                    // G_k = -(1 - w^a) (s - i c) / (2 s)
                    float2 om = make_float2(1.f - wa.x, -wa.y);
                    float2 G = cmul(om, make_float2(sv, -cv));
                    float f = -0.5f / sv;
                    float2 pad = make_float2(G.x * f * mean, G.y * f * mean);
                    X = real_bin(zk, zm, twiddle2(a.rl_hi, a.rl_lo, kSplitLog2, k), pad);
                    float pw = X.x * X.x + X.y * X.y;
                    Pw[k] = pow2 ? pw * inv_n : pw / float(n);
                }
                if (fft) fft[k] = X;
            }
        } else {
            const int brow = L1 - arow;
            const uint32_t k = uint32_t(arow) + uint32_t(L1) * k2;
            const uint32_t km = uint32_t(brow) + uint32_t(L1) * uint32_t(L2 - 1 - k2);  // = M - k
            float2 zk = sm[r * stride + smem_pos(k2)], zm = sm[(R + r) * stride + smem_pos(L2 - 1 - k2)];
            float sv, cv;
            sincospif(float(k) / float(n), &sv, &cv);  // sin/cos(pi k/n); for M-k they swap
            float2 w = twiddle2(a.rl_hi, a.rl_lo, kSplitLog2, k);
            float2 wa = twiddle2(a.rl_hi, a.rl_lo, kSplitLog2, mod_n(uint64_t(k) * steps, n));
            // W_N^{M-k} = -conj(W_N^k); w^a at M-k = (-1)^a conj(w^a)
            float2 wm = make_float2(-w.x, w.y);
            float2 wam = a_odd ? make_float2(-wa.x, wa.y) : make_float2(wa.x, -wa.y);
            float2 G1 = cmul(make_float2(1.f - wa.x, -wa.y), make_float2(sv, -cv));
            float2 G2 = cmul(make_float2(1.f - wam.x, -wam.y), make_float2(cv, -sv));
            float f1 = -0.5f * mean / sv, f2 = -0.5f * mean / cv;
            float2 X1 = real_bin(zk, zm, w, make_float2(G1.x * f1, G1.y * f1));
            float2 X2 = real_bin(zm, zk, wm, make_float2(G2.x * f2, G2.y * f2));
            float p1 = X1.x * X1.x + X1.y * X1.y, p2 = X2.x * X2.x + X2.y * X2.y;
            Pw[k] = pow2 ? p1 * inv_n : p1 / float(n);
            Pw[km] = pow2 ? p2 * inv_n : p2 / float(n);
            if (fft) { fft[k] = X1; fft[km] = X2; }
        }
    }
}

// Warp-aggregated compaction of one candidate per predicated lane.
__device__ __forceinline__ void emit_candidate(bool pred, uint32_t bin, uint32_t level, float value, uint32_t* count,
                                               brp_candidate* out, uint32_t capacity, uint32_t* status) {
    const unsigned active = __activemask();
    const unsigned m = __ballot_sync(active, pred);
    if (!m) return;
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(count, uint32_t(__popc(m)));
    base = __shfl_sync(active, base, leader);
    if (pred) {
        uint32_t slot = base + __popc(m & ((1u << lane) - 1u));
        if (slot < capacity) {
            brp_candidate c;
            c.bin = bin; c.level = level; c.power = value; c.reserved = 0;
            out[slot] = c;
        } else {
            atomicOr(status, BRP_STATUS_OVERFLOW);
        }
    }
}

// Harmonic summing of shaders/harmonic.comp:5-35 in tile form.  A CTA owns the
// trial bins [I0, I0+T) (I0 a multiple of 16); it computes the dyadic sums of
// shaders/hs_sum.glsl for every trial bin in [I0-8, I0+T) once (16 power
// loads each) and keeps them in shared memory.  Level h >= 1 then owns the
// fundamental bins j in [I0/2^h, (I0+T)/2^h), whose trial ranges
// [j 2^h - 2^(h-1), j 2^h + 2^(h-1)) all lie inside the tile; level 0 owns
// j in [I0, I0+T).  Each j takes the maximum over its trial range when it
// exceeds the threshold, otherwise the sum at the first trial bin (0 for an
// empty range), and becomes a candidate when j >= window and it exceeds the
// threshold.
template <int T, int THREADS>
__global__ void __launch_bounds__(THREADS) harmonic_kernel(FusedArgs a) {
    __shared__ float sums[4][T + 8];
    const int g = blockIdx.y;
    const brp_params& P = a.params[g];
    const int64_t I0 = int64_t(blockIdx.x) * T, lo = I0 - 8;
    const uint32_t window = P.window, fundamental = P.fundamental, harmonic = P.harmonic;
    const float* __restrict__ Pw = a.power + size_t(g) * a.power_stride;
    float* summed = (g == a.snap) ? a.snap_summed : nullptr;
    uint32_t* count = a.counts + g;
    uint32_t* status = a.status + g;
    brp_candidate* out = a.cands + size_t(g) * a.capacity;

    for (int t = threadIdx.x; t < T + 8; t += THREADS) {
        const int64_t i64 = lo + t;
        if (i64 >= 0 && i64 < int64_t(harmonic)) {
            const uint32_t i = uint32_t(i64);
            float s = __ldg(Pw + i);
            s += __ldg(Pw + ((i * 8 + 8) >> 4));
            sums[0][t] = s;
            s += __ldg(Pw + ((i * 12 + 8) >> 4)) + __ldg(Pw + ((i * 4 + 8) >> 4));
            sums[1][t] = s;
            s += __ldg(Pw + ((i * 14 + 8) >> 4)) + __ldg(Pw + ((i * 10 + 8) >> 4)) + __ldg(Pw + ((i * 6 + 8) >> 4)) +
                 __ldg(Pw + ((i * 2 + 8) >> 4));
            sums[2][t] = s;
            s += __ldg(Pw + ((i * 15 + 8) >> 4)) + __ldg(Pw + ((i * 13 + 8) >> 4)) +
                 __ldg(Pw + ((i * 11 + 8) >> 4)) + __ldg(Pw + ((i * 9 + 8) >> 4)) + __ldg(Pw + ((i * 7 + 8) >> 4)) +
                 __ldg(Pw + ((i * 5 + 8) >> 4)) + __ldg(Pw + ((i * 3 + 8) >> 4)) + __ldg(Pw + ((i + 8) >> 4));
            sums[3][t] = s;
        }
    }
    __syncthreads();

    for (int t = threadIdx.x; t < T; t += THREADS) {
        const int64_t j = I0 + t;
        bool pred = false;
        float v = 0.f;
        if (j < int64_t(fundamental)) {
            v = __ldg(Pw + j);
            if (summed) summed[j] = v;
            pred = j >= int64_t(window) && v > P.threshold[0];
        }
        emit_candidate(pred, uint32_t(j), 0, v, count, out, a.capacity, status);
    }
#pragma unroll
    for (int h = 1; h <= 4; ++h) {
        const int64_t w = int64_t(1) << h;
        const int64_t jlo = I0 >> h;
        int64_t jhi = (I0 + T) >> h;
        if (jhi > int64_t(fundamental)) jhi = fundamental;
        const float thr = P.threshold[h];
        for (int64_t j = jlo + threadIdx.x; j < jlo + (T >> h); j += THREADS) {
            bool pred = false;
            float v = 0.f;
            if (j < jhi) {
                int64_t begin = j * w - w / 2, end = j * w + w / 2;
                if (begin < int64_t(window)) begin = window;
                if (end > int64_t(harmonic)) end = harmonic;
                if (begin < end) {
                    const float first = sums[h - 1][begin - lo];
                    float best = first;
                    for (int64_t i = begin + 1; i < end; ++i) {
                        float x = sums[h - 1][i - lo];
                        if (best < x) best = x;
                    }
                    v = best > thr ? best : first;
                }
                if (summed) summed[size_t(h) * fundamental + j] = v;
                pred = j >= int64_t(window) && v > thr;
            }
            emit_candidate(pred, uint32_t(j), uint32_t(h), v, count, out, a.capacity, status);
        }
    }
}

}  // namespace

size_t LengthPlan::smem1() const { return size_t(C) * seq_stride(L1, C) * sizeof(float2); }
size_t LengthPlan::smem2() const { return size_t(2 * R) * seq_stride(L2, R) * sizeof(float2); }

constexpr int kThreads = 512;

template <int MAXE>
static void launch_p1(const FusedArgs& a, const LengthPlan& lp, uint32_t count, cudaStream_t s) {
    pass1_kernel<MAXE, kThreads><<<dim3(lp.blocks1(), count), kThreads, lp.smem1(), s>>>(a);
}
template <int MAXE>
static void launch_p2(const FusedArgs& a, const LengthPlan& lp, uint32_t count, cudaStream_t s) {
    pass2_kernel<MAXE, kThreads><<<dim3(lp.blocks2(), count), kThreads, lp.smem2(), s>>>(a);
}

// Opts the fused kernels into the device's largest dynamic shared memory per
// block (done at plan creation, outside any stream capture).  The limit is a
// per-kernel maximum, so it is set once to the device limit rather than to one
// plan's need, which a later, smaller plan would otherwise lower.
cudaError_t set_fused_attributes(size_t max_dynamic_smem) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (size_t(optin) < max_dynamic_smem + 1024) return cudaErrorInvalidValue;
    int v = optin - 1024;  // static shared memory of the kernels (reduction scratch) fits in the rest
    cudaError_t e = cudaFuncSetAttribute(pass1_kernel<16, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pass1_kernel<24, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pass2_kernel<16, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(pass2_kernel<24, kThreads>, cudaFuncAttributeMaxDynamicSharedMemorySize, v);
    return e;
}

void launch_fused_pass1(const FusedArgs& a, const LengthPlan& lp, uint32_t count, cudaStream_t s) {
    if (lp.fp1) { lp.fp1->launch(a, lp.blocks1(), count, s); return; }
    if (lp.maxe <= 16) launch_p1<16>(a, lp, count, s);
    else launch_p1<24>(a, lp, count, s);
}
void launch_fused_pass2(const FusedArgs& a, const LengthPlan& lp, uint32_t count, cudaStream_t s) {
    if (lp.fp2) { lp.fp2->launch(a, lp.blocks2(), count, s); return; }
    if (lp.maxe <= 16) launch_p2<16>(a, lp, count, s);
    else launch_p2<24>(a, lp, count, s);
}
// max_span: the largest max(fundamental, harmonic + 8) of the templates; the
// top fundamental bin of level h may own trial bins up to harmonic + 2^(h-1).
void launch_fused_harmonic(const FusedArgs& a, const LengthPlan& lp, uint32_t count, uint32_t max_span,
                           cudaStream_t s) {
    if (lp.fused) { launch_harmonic_fast(a, count, max_span, s); return; }
    constexpr int T = 2048;
    uint32_t tiles = (max_span + T - 1) / T;
    if (!tiles) tiles = 1;
    harmonic_kernel<T, 256><<<dim3(tiles, count), 256, 0, s>>>(a);
}

void fill_fused_args(FusedArgs& a, const LengthPlan& lp) {
    a.n = lp.n; a.M = lp.M; a.L1 = lp.L1; a.L2 = lp.L2; a.C = lp.C; a.R = lp.R;
    a.plan1[0] = lp.plan1.count; a.plan2[0] = lp.plan2.count;
    for (int i = 0; i < 6; ++i) { a.plan1[1 + i] = lp.plan1.radix[i]; a.plan2[1 + i] = lp.plan2.radix[i]; }
    a.tw1 = lp.tw1; a.tw2 = lp.tw2; a.fs_hi = lp.fs_hi; a.fs_lo = lp.fs_lo; a.rl_hi = lp.rl_hi; a.rl_lo = lp.rl_lo;
    a.ptw1 = lp.ptw1; a.ptw2 = lp.ptw2;
    a.hf_hi = lp.hf_hi; a.hf_lo = lp.hf_lo; a.hq = lp.hq;
    a.wait_polls = kDefaultWaitPolls;
}

}  // namespace brp
