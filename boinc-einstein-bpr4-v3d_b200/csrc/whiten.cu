// Whitening and RFI zapping of an observation on the GPU: brp::preprocess
// (src/workload.cpp:58-95), optionally after the DD sample decoding of
// brp::load_observation (src/workload.cpp:48-56).
//
//   1. decode (optional): int8 or packed 4-bit samples, float(double(b) / scale);
//   2. forward real FFT of the series zero-padded to n (packed N/2-point complex
//      FFT by the global Stockham passes of the plain pipeline, then the real
//      post-process): X_k, k = 0..n/2;
//   3. power P_k = |X_k|^2 in FP64 rounded once to FP32, P_0 = 0;
//   4. running median of P over `window` bins (window even: the mean of the two
//      middle values; the historical rngmed.c is absent, this is its
//      definition as restated here) -- per CTA 1024 medians from one bitonic
//      sort of the 1024 + window - 1 (value, position) pairs in shared memory,
//      each thread then walks the sorted list counting the entries of its
//      window (all threads read the same entry: broadcasts);
//   5. X_{i + window/2} *= float(sqrt(ln 2 / median_i)) (FP64 square root);
//      a median that is not positive and finite is an error, as in the reference;
//   6. zapped bins take the host-generated Gaussian noise (brp_host_zap_noise);
//   7. the first and last window/2 bins are cleared;
//   8. inverse real FFT: 2 Z_k = (X_k + X*_{M-k}) + i W_n^{-k} (X_k - X*_{M-k})
//      (imaginary parts of X_0 and X_M ignored, as a C2R transform does), the
//      unnormalised inverse M-point DFT as conj(FFT(conj(2 Z))), even/odd
//      samples from its real/imaginary parts, times float(1 / sqrtf(n)).
// The window is limited to 4096 bins on the device (shared-memory sort).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "brp_internal.h"
#include "fft_device.cuh"

namespace brp {
namespace {

constexpr uint32_t kWhitenMaxWindow = 4096;
constexpr uint32_t kMedOut = 1024;  // medians per CTA
constexpr uint32_t kBlk = 256;

inline uint32_t blocks_of(uint64_t n, uint32_t b) { return uint32_t((n + b - 1) / b); }

__host__ __device__ constexpr uint32_t median_sort_size(uint32_t window) {
    uint32_t p = 2;
    while (p < kMedOut + window - 1) p <<= 1;
    return p;
}

__global__ void dd_decode(const uint8_t* __restrict__ bytes, uint32_t samples, int packed, double scale,
                          float* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= samples) return;
    if (packed) {
        const uint32_t b = bytes[i >> 1];
        out[i] = float(double((i & 1) ? (b & 15u) : (b >> 4)) / scale);
    } else {
        out[i] = float(double(int8_t(bytes[i])) / scale);
    }
}

// Zero-padded packed input in the decimated order of the plain FFT:
// a[blk B + j] = (x[2s], x[2s + 1]), s = j radix + blk.
__global__ void whiten_prepare(const float* __restrict__ x, uint32_t samples, float2* a, uint32_t M, uint32_t radix,
                               uint32_t B) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const uint32_t blk = t / B, j = t - blk * B, s = j * radix + blk;
    const uint32_t i0 = 2 * s, i1 = 2 * s + 1;
    a[t] = make_float2(i0 < samples ? x[i0] : 0.f, i1 < samples ? x[i1] : 0.f);
}

__global__ void whiten_power(const float2* __restrict__ X, float* P, uint32_t size) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= size) return;
    const double re = X[i].x, im = X[i].y;
    P[i] = i == 0 ? 0.f : float(__dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im)));
}

__global__ void __launch_bounds__(1024) whiten_median(const float* __restrict__ P, uint32_t size, uint32_t window,
                                                      float* med, uint32_t nmed) {
    extern __shared__ unsigned long long sk[];
    const uint32_t o0 = blockIdx.x * kMedOut;
    const uint32_t S = min(kMedOut + window - 1, size - o0);
    uint32_t P2 = 2;
    while (P2 < S) P2 <<= 1;
    // P >= 0, so the float bits order the values
    for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x)
        sk[i] = i < S ? (static_cast<unsigned long long>(__float_as_uint(P[o0 + i])) << 32) | i : ~0ull;
    __syncthreads();
    for (uint32_t w = 2; w <= P2; w <<= 1) {
        for (uint32_t j = w >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < P2 / 2; i += blockDim.x) {
                const uint32_t lo = ((i & ~(j - 1)) << 1) | (i & (j - 1)), hi = lo | j;
                const unsigned long long x = sk[lo], y = sk[hi];
                if ((x > y) == ((lo & w) == 0)) { sk[lo] = y; sk[hi] = x; }
            }
            __syncthreads();
        }
    }
    const uint32_t t = threadIdx.x;
    if (o0 + t >= nmed) return;
    const uint32_t lower = window / 2 - 1;
    uint32_t cnt = 0;
    float a = 0.f, b = 0.f;
    for (uint32_t e = 0; e < S; ++e) {
        const unsigned long long v = sk[e];
        const uint32_t pos = uint32_t(v);
        if (pos - t < window) {
            const float val = __uint_as_float(uint32_t(v >> 32));
            if (cnt == lower) a = val;
            if (cnt == lower + 1) { b = val; break; }
            ++cnt;
        }
    }
    med[o0 + t] = 0.5f * (a + b);
}

__global__ void whiten_scale(float2* X, const float* __restrict__ med, uint32_t nmed, uint32_t half_window,
                             uint32_t* bad) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nmed) return;
    const float m = med[i];
    if (!(m > 0.f) || !isfinite(m)) { atomicOr(bad, 1u); return; }
    const float f = float(sqrt(0.693147180559945309417232121458 / double(m)));
    float2 x = X[i + half_window];
    x.x *= f; x.y *= f;
    X[i + half_window] = x;
}

__global__ void whiten_zap(float2* X, const uint32_t* __restrict__ bins, const float2* __restrict__ vals,
                           uint32_t count) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < count) X[bins[k]] = vals[k];
}

__global__ void whiten_edges(float2* X, uint32_t size, uint32_t half_window) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= half_window) return;
    X[i] = make_float2(0.f, 0.f);
    X[size - 1 - i] = make_float2(0.f, 0.f);
}

// conj(2 Z_k) in the decimated input order of the plain FFT.
__global__ void whiten_inverse_pre(const float2* __restrict__ X, float2* a, uint32_t M, uint32_t radix, uint32_t B,
                                   const float2* rl_hi, const float2* rl_lo) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const uint32_t blk = t / B, j = t - blk * B, k = j * radix + blk;
    float2 p = X[k], q = X[M - k];
    if (k == 0) p.y = 0.f;
    if (k == 0) q.y = 0.f;  // X_M, real for a real series
    q.y = -q.y;             // conj(X_{M-k})
    const float2 e = cadd(p, q), d = csub(p, q);
    const float2 w = twiddle2(rl_hi, rl_lo, kSplitLog2, k);  // W_n^k
    const float2 cd = cmulc(d, w);                              // W_n^{-k} d
    const float2 z = make_float2(e.x - cd.y, e.y + cd.x);       // e + i W_n^{-k} d
    a[t] = make_float2(z.x, -z.y);
}

__global__ void whiten_output(const float2* __restrict__ w, uint32_t samples, float factor, float* out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= samples) return;
    const float2 v = w[i >> 1];
    out[i] = ((i & 1) ? -v.y : v.x) * factor;
}

thread_local std::string g_whiten_error;
int whiten_fail(int code, const std::string& m) { g_whiten_error = m; return code; }

struct DeviceBuffers {
    std::vector<void*> ptrs;
    template <class T>
    bool get(T** p, size_t count) {
        if (cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count * sizeof(T), 16)) != cudaSuccess) return false;
        ptrs.push_back(*p);
        return true;
    }
    ~DeviceBuffers() { for (void* p : ptrs) cudaFree(p); }
};

int preprocess_device(const float* d_decoded, float first_sample, uint32_t samples, uint32_t n, double sample_us,
                      double padding, uint32_t window, const double* zap_lower, const double* zap_upper,
                      uint32_t zap_count, float* preprocessed, cudaStream_t s, DeviceBuffers& mem) {
    const uint32_t M = n / 2, size = M + 1;
    if (!window || (window & 1) || window > n / 2) return whiten_fail(BRP_E_ARGUMENT, "unsupported whitening window");
    if (window > kWhitenMaxWindow)
        return whiten_fail(BRP_E_ARGUMENT, "whitening window above 4096 bins (the device median's limit)");
    // zap noise on the host, in the reference's order; the last write of a bin wins
    uint32_t zc = 0;
    uint32_t seed;
    std::memcpy(&seed, &first_sample, 4);
    if (brp_host_zap_noise(seed, n, sample_us, padding, zap_lower, zap_upper, zap_count, nullptr, nullptr, 0, &zc))
        return whiten_fail(BRP_E_ARGUMENT, brp_host_error());
    std::vector<uint32_t> bins(zc);
    std::vector<float2> vals(zc);
    if (zc && brp_host_zap_noise(seed, n, sample_us, padding, zap_lower, zap_upper, zap_count, bins.data(),
                                 reinterpret_cast<float*>(vals.data()), zc, &zc))
        return whiten_fail(BRP_E_ARGUMENT, brp_host_error());
    {
        // keep the last draw of each bin (overlapping ranges overwrite, as in the reference)
        std::vector<std::pair<uint32_t, uint32_t>> order(zc);
        for (uint32_t k = 0; k < zc; ++k) order[k] = {bins[k], k};
        std::sort(order.begin(), order.end());
        std::vector<uint32_t> keep_bins;
        std::vector<float2> keep_vals;
        for (uint32_t k = 0; k < zc; ++k)
            if (k + 1 == zc || order[k + 1].first != order[k].first) {
                keep_bins.push_back(order[k].first);
                keep_vals.push_back(vals[order[k].second]);
            }
        bins.swap(keep_bins);
        vals.swap(keep_vals);
        zc = uint32_t(bins.size());
    }
    LengthPlan lp;
    std::string e = make_length_plan(n, lp, s);
    struct Free { LengthPlan& p; ~Free() { free_length_plan(p); } } free_plan{lp};
    if (!e.empty()) return whiten_fail(BRP_E_ARGUMENT, e);
    float2 *a, *b, *X, *d_vals;
    float *P, *med, *d_out;
    uint32_t *d_bins, *d_bad;
    const uint32_t nmed = size - window + 1;
    if (!mem.get(&a, M) || !mem.get(&b, M) || !mem.get(&X, size) || !mem.get(&P, size) || !mem.get(&med, nmed) ||
        !mem.get(&d_out, samples) || !mem.get(&d_bins, zc) || !mem.get(&d_vals, zc) || !mem.get(&d_bad, 1))
        return whiten_fail(BRP_E_RUNTIME, "cudaMalloc failed (whitening buffers)");
    const size_t smem = size_t(median_sort_size(window)) * sizeof(unsigned long long);
    if (cudaFuncSetAttribute(whiten_median, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return whiten_fail(BRP_E_RUNTIME, "cannot enable the shared memory of the median kernel");
    if (cudaMemsetAsync(d_bad, 0, 4, s) != cudaSuccess ||
        (zc && (cudaMemcpyAsync(d_bins, bins.data(), zc * 4, cudaMemcpyHostToDevice, s) != cudaSuccess ||
                cudaMemcpyAsync(d_vals, vals.data(), zc * 8, cudaMemcpyHostToDevice, s) != cudaSuccess)))
        return whiten_fail(BRP_E_RUNTIME, "whitening upload failed");
    whiten_prepare<<<blocks_of(M, kBlk), kBlk, 0, s>>>(d_decoded, samples, a, M, lp.radix, lp.B);
    float2* z = plain_complex_fft(a, b, lp, s);
    launch_plain_realpost(z, X, nullptr, lp, s);
    whiten_power<<<blocks_of(size, kBlk), kBlk, 0, s>>>(X, P, size);
    whiten_median<<<blocks_of(nmed, kMedOut), kMedOut, smem, s>>>(P, size, window, med, nmed);
    whiten_scale<<<blocks_of(nmed, kBlk), kBlk, 0, s>>>(X, med, nmed, window / 2, d_bad);
    if (zc) whiten_zap<<<blocks_of(zc, kBlk), kBlk, 0, s>>>(X, d_bins, d_vals, zc);
    whiten_edges<<<blocks_of(window / 2, kBlk), kBlk, 0, s>>>(X, size, window / 2);
    whiten_inverse_pre<<<blocks_of(M, kBlk), kBlk, 0, s>>>(X, a, M, lp.radix, lp.B, lp.rl_hi, lp.rl_lo);
    float2* w = plain_complex_fft(a, b, lp, s);
    const float factor = float(1.0 / double(std::sqrt(float(n))));
    whiten_output<<<blocks_of(samples, kBlk), kBlk, 0, s>>>(w, samples, factor, d_out);
    uint32_t bad = 0;
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaMemcpyAsync(preprocessed, d_out, size_t(samples) * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return whiten_fail(BRP_E_RUNTIME, std::string("whitening failed: ") + cudaGetErrorString(cudaGetLastError()));
    if (bad) return whiten_fail(BRP_E_RESULT, "invalid whitening median");
    return BRP_OK;
}

int check_common(uint32_t samples, uint32_t n, double sample_us, double padding, const float* out) {
    if (!out || !samples || samples > n || !(sample_us > 0) || !(padding >= 1))
        return whiten_fail(BRP_E_ARGUMENT, "invalid observation");
    const bool pow2 = n && !(n & (n - 1)), pow3 = n % 3 == 0 && !((n / 3) & (n / 3 - 1));
    if (!(pow2 || pow3) || n < 8192 || n > 3u * (1u << 22))
        return whiten_fail(BRP_E_ARGUMENT, "whitening length must be 2^k or 3*2^k in 8192..3*2^22");
    return BRP_OK;
}

struct Device {
    int prev = -1;
    explicit Device(int32_t d) {
        cudaGetDevice(&prev);
        if (d >= 0) cudaSetDevice(d);
    }
    ~Device() { if (prev >= 0) cudaSetDevice(prev); }
};

}  // namespace
}  // namespace brp

using namespace brp;

extern "C" const char* brp_cuda_preprocess_error(void) { return g_whiten_error.c_str(); }

extern "C" int brp_cuda_preprocess(const float* decoded, uint32_t samples, uint32_t n, double sample_us,
                                   double padding, uint32_t window, const double* zap_lower, const double* zap_upper,
                                   uint32_t zap_count, float* preprocessed, int32_t device) {
    int st;
    if (!decoded) return whiten_fail(BRP_E_ARGUMENT, "null series");
    if ((st = check_common(samples, n, sample_us, padding, preprocessed))) return st;
    Device dev(device);
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return whiten_fail(BRP_E_RUNTIME, "no CUDA device");
    int rc;
    {
        DeviceBuffers mem;
        float* d_x;
        if (!mem.get(&d_x, samples)) rc = whiten_fail(BRP_E_RUNTIME, "cudaMalloc failed (series)");
        else if (cudaMemcpyAsync(d_x, decoded, size_t(samples) * 4, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = whiten_fail(BRP_E_RUNTIME, "series upload failed");
        else
            rc = preprocess_device(d_x, decoded[0], samples, n, sample_us, padding, window, zap_lower, zap_upper,
                                   zap_count, preprocessed, s, mem);
        cudaStreamSynchronize(s);
    }
    cudaStreamDestroy(s);
    return rc;
}

extern "C" int brp_cuda_preprocess_dd(const uint8_t* bytes, uint32_t samples, int32_t packed, double scale, uint32_t n,
                                      double sample_us, double padding, uint32_t window, const double* zap_lower,
                                      const double* zap_upper, uint32_t zap_count, float* decoded,
                                      float* preprocessed, int32_t device) {
    int st;
    if (!bytes) return whiten_fail(BRP_E_ARGUMENT, "null samples");
    if (!(scale > 0) || !std::isfinite(scale) || (packed && (samples & 1)))
        return whiten_fail(BRP_E_ARGUMENT, "invalid DD metadata");
    if ((st = check_common(samples, n, sample_us, padding, preprocessed))) return st;
    const uint32_t nbytes = packed ? samples / 2 : samples;
    const float first = packed ? float(double(bytes[0] >> 4) / scale) : float(double(int8_t(bytes[0])) / scale);
    Device dev(device);
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
        return whiten_fail(BRP_E_RUNTIME, "no CUDA device");
    int rc;
    {
        DeviceBuffers mem;
        uint8_t* d_bytes;
        float* d_x;
        if (!mem.get(&d_bytes, nbytes) || !mem.get(&d_x, samples)) rc = whiten_fail(BRP_E_RUNTIME, "cudaMalloc failed");
        else if (cudaMemcpyAsync(d_bytes, bytes, nbytes, cudaMemcpyHostToDevice, s) != cudaSuccess)
            rc = whiten_fail(BRP_E_RUNTIME, "sample upload failed");
        else {
            dd_decode<<<blocks_of(samples, kBlk), kBlk, 0, s>>>(d_bytes, samples, packed, scale, d_x);
            if (decoded && cudaMemcpyAsync(decoded, d_x, size_t(samples) * 4, cudaMemcpyDeviceToHost, s) != cudaSuccess)
                rc = whiten_fail(BRP_E_RUNTIME, "decoded download failed");
            else
                rc = preprocess_device(d_x, first, samples, n, sample_us, padding, window, zap_lower, zap_upper,
                                       zap_count, preprocessed, s, mem);
        }
        cudaStreamSynchronize(s);
    }
    cudaStreamDestroy(s);
    return rc;
}
