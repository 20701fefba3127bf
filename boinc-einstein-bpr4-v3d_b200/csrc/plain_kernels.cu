// Step-by-step per-template pipeline: one kernel per stage with global-memory
// FFT passes, the structure of the reference's recorded command sequence
// (src/vulkan.cpp:226-262): resample, mean, prepare, radix-8/4/2 Stockham
// passes, radix-3 combination, real post-process + power, harmonic summing
// with compaction.  It is the per-template comparator of the fused pipeline
// and a second, independent GPU implementation for cross-checks.
#include "brp_internal.h"
#include "fft_device.cuh"
#include "resample_math.h"

namespace brp {

__constant__ uint32_t c_plain_lut_bits[130] = BRP_LUT_BITS;

namespace {

constexpr int kBlock = 256;

__global__ void __launch_bounds__(kBlock) plain_resample(const float* __restrict__ in, brp_params p, float* raw,
                                                         double* partial, uint32_t* status) {
    __shared__ double red[kBlock / 32];
    const uint32_t i = blockIdx.x * kBlock + threadIdx.x;
    float v = 0.f;
    if (i < p.steps) {
        brp_resample_consts rc;
        rc.tau = p.tau; rc.omega = p.omega; rc.psi = p.psi; rc.dt = p.dt; rc.step_inv = p.step_inv; rc.s0 = p.s0;
        rc.flags = p.flags;
        int j = (p.flags & BRP_FLAG_INDEX_FP64) ? brp_resample_index_fp64(i, rc)
                                                : brp_resample_index(i, rc, c_plain_lut_bits);
        if (j < 0 || uint32_t(j) >= p.unpadded) atomicOr(status, BRP_STATUS_RESAMPLE_OOB);
        else v = __ldg(in + j);
        raw[i] = v;
    }
    double s = v;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < kBlock / 32 ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) partial[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(1024) plain_mean(const double* partial, uint32_t blocks, uint32_t steps,
                                                   float* mean) {
    __shared__ double red[32];
    double s = 0;
    for (uint32_t i = threadIdx.x; i < blocks; i += 1024) s += partial[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = red[threadIdx.x];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (threadIdx.x == 0) *mean = float(s / double(steps));
    }
}

// Packed complex input z[s] = r[2s] + i r[2s+1] with r[i] = raw[i] (i < steps)
// or the mean; for M = 3B the three decimated sub-series z[3j + b] go to
// block b (prepare.comp's source = j*radix + block).
__global__ void plain_prepare(const float* __restrict__ raw, const float* __restrict__ mean, float2* a, uint32_t steps,
                              uint32_t M, uint32_t radix, uint32_t B) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= M) return;
    const uint32_t blk = t / B, j = t - blk * B;
    const uint32_t s = j * radix + blk;
    const float m = *mean;
    const uint32_t i0 = 2 * s, i1 = 2 * s + 1;
    a[t] = make_float2(i0 < steps ? raw[i0] : m, i1 < steps ? raw[i1] : m);
}

// One global Stockham pass of radix R over `seqs` sequences of length B.
template <int R>
__global__ void plain_fft_pass(const float2* __restrict__ in, float2* __restrict__ out, uint32_t B, uint32_t seqs,
                               uint32_t Ns, const float2* __restrict__ tw) {
    const uint32_t nbf = B / R;
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nbf * seqs) return;
    const uint32_t sq = t / nbf, j = t - sq * nbf;
    const uint32_t k = j % Ns, tstep = B / (Ns * R);
    const float2* src = in + size_t(sq) * B;
    float2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[j + r * nbf];
    if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[r] = cmul(v[r], __ldg(tw + size_t(r) * k * tstep));
    }
    dft<R>(v);
    float2* dst = out + size_t(sq) * B;
    const uint32_t base = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];
}

// Radix-3 combination of three transformed blocks: X[k + m B] =
// sum_b W_M^{b k} W_3^{b m} A_b[k].
__global__ void plain_radix3(const float2* __restrict__ in, float2* __restrict__ out, uint32_t B,
                             const float2* __restrict__ hi, const float2* __restrict__ lo) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= B) return;
    float2 v[3];
    v[0] = in[k];
    v[1] = cmul(in[k + B], twiddle2(hi, lo, kSplitLog2, k));
    v[2] = cmul(in[k + 2 * B], twiddle2(hi, lo, kSplitLog2, 2 * k));
    dft3(v);
    out[k] = v[0];
    out[k + B] = v[1];
    out[k + 2 * B] = v[2];
}

// Real post-process (fft_real.comp's formula) and power (power.comp):
// X_k = 1/2 [(Z_k + Z*_{M-k}) - i W_N^k (Z_k - Z*_{M-k})], k = 0..M;
// P_k = |X_k|^2 / n for 1 <= k < M, P_0 = 0.
__global__ void plain_realpost(const float2* __restrict__ Z, float2* fft, float* power, uint32_t M, uint32_t n,
                               const float2* __restrict__ hi, const float2* __restrict__ lo) {
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > M) return;
    const uint32_t q = k == M ? 0 : k, rev = q == 0 ? 0 : M - q;
    const float2 x = Z[q], y = Z[rev];
    const float2 w = twiddle2(hi, lo, kSplitLog2, k);
    float2 s = make_float2(x.x + y.x, x.y - y.y), d = make_float2(x.x - y.x, x.y + y.y);
    float2 t = cmul(w, d);
    float2 X = make_float2(0.5f * (s.x + t.y), 0.5f * (s.y - t.x));
    fft[k] = X;
    if (power && k < M) power[k] = k == 0 ? 0.f : (X.x * X.x + X.y * X.y) / float(n);
}

// harmonic.comp:14-35 (gather form).  grid.y = level.
__global__ void plain_harmonic(const float* __restrict__ P, brp_params p, float* summed, uint32_t* count,
                               brp_candidate* cands, uint32_t* status) {
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x, h = blockIdx.y;
    if (j >= p.fundamental) return;
    float value = 0.f;
    if (h == 0) value = P[j];
    else {
        const int64_t w = int64_t(1) << h;
        int64_t begin = int64_t(j) * w - w / 2, end = int64_t(j) * w + w / 2;
        if (begin < int64_t(p.window)) begin = p.window;
        if (end > int64_t(p.harmonic)) end = p.harmonic;
        if (begin < end) {
            float first = 0.f, best = 0.f;
            for (int64_t ii = begin; ii < end; ++ii) {
                const uint32_t i = uint32_t(ii);
                float s = P[i];
                if (h >= 1) s += P[(i * 8 + 8) >> 4];
                if (h >= 2) s += P[(i * 12 + 8) >> 4] + P[(i * 4 + 8) >> 4];
                if (h >= 3) s += P[(i * 14 + 8) >> 4] + P[(i * 10 + 8) >> 4] + P[(i * 6 + 8) >> 4] + P[(i * 2 + 8) >> 4];
                if (h >= 4)
                    s += P[(i * 15 + 8) >> 4] + P[(i * 13 + 8) >> 4] + P[(i * 11 + 8) >> 4] + P[(i * 9 + 8) >> 4] +
                         P[(i * 7 + 8) >> 4] + P[(i * 5 + 8) >> 4] + P[(i * 3 + 8) >> 4] + P[(i + 8) >> 4];
                if (ii == begin) first = best = s;
                else if (best < s) best = s;
            }
            value = best > p.threshold[h] ? best : first;
        }
    }
    summed[size_t(h) * p.fundamental + j] = value;
    if (j >= p.window && value > p.threshold[h]) {
        uint32_t slot = atomicAdd(count, 1u);
        if (slot < p.capacity) {
            brp_candidate c;
            c.bin = j; c.level = h; c.power = value; c.reserved = 0;
            cands[slot] = c;
        } else {
            atomicOr(status, BRP_STATUS_OVERFLOW);
        }
    }
}

inline uint32_t blocks_for(uint64_t n, uint32_t b) { return uint32_t((n + b - 1) / b); }

}  // namespace

// Forward complex FFT of the M = radix * B packed points in `a` (in the
// decimated order of plain_prepare), by global Stockham passes: radix 8 while at
// least three factors of two remain, then 4 or 2, then the radix-3 combination.
// `b` is scratch; returns the buffer that holds Z (a or b).
float2* plain_complex_fft(float2* a, float2* b, const LengthPlan& lp, cudaStream_t s) {
    float2 *src = a, *dst = b;
    const uint32_t seqs = lp.radix;
    uint32_t Ns = 1;
    while (Ns < lp.B) {
        const uint32_t left = lp.B / Ns;
        if (left >= 8) {
            plain_fft_pass<8><<<blocks_for(uint64_t(lp.B / 8) * seqs, kBlock), kBlock, 0, s>>>(src, dst, lp.B, seqs, Ns, lp.twb);
            Ns *= 8;
        } else if (left == 4) {
            plain_fft_pass<4><<<blocks_for(uint64_t(lp.B / 4) * seqs, kBlock), kBlock, 0, s>>>(src, dst, lp.B, seqs, Ns, lp.twb);
            Ns *= 4;
        } else {
            plain_fft_pass<2><<<blocks_for(uint64_t(lp.B / 2) * seqs, kBlock), kBlock, 0, s>>>(src, dst, lp.B, seqs, Ns, lp.twb);
            Ns *= 2;
        }
        float2* t = src; src = dst; dst = t;
    }
    if (lp.radix == 3) {
        plain_radix3<<<blocks_for(lp.B, kBlock), kBlock, 0, s>>>(src, dst, lp.B, lp.fs_hi, lp.fs_lo);
        float2* t = src; src = dst; dst = t;
    }
    return src;
}

void launch_plain_realpost(const float2* z, float2* fft, float* power, const LengthPlan& lp, cudaStream_t s) {
    plain_realpost<<<blocks_for(uint64_t(lp.M) + 1, kBlock), kBlock, 0, s>>>(z, fft, power, lp.M, lp.n, lp.rl_hi,
                                                                         lp.rl_lo);
}

void launch_plain(const PlainArgs& a, cudaStream_t s, cudaEvent_t* ev) {
    const LengthPlan& lp = *a.lp;
    const brp_params& p = a.p;
    if (ev) cudaEventRecord(ev[0], s);
    const uint32_t rblocks = blocks_for(p.steps, kBlock);
    plain_resample<<<rblocks, kBlock, 0, s>>>(a.input, p, a.raw, a.partial, a.status);
    plain_mean<<<1, 1024, 0, s>>>(a.partial, rblocks, p.steps, a.mean);
    plain_prepare<<<blocks_for(lp.M, kBlock), kBlock, 0, s>>>(a.raw, a.mean, a.a, p.steps, lp.M, lp.radix, lp.B);
    if (ev) cudaEventRecord(ev[1], s);
    float2* z = plain_complex_fft(a.a, a.b, lp, s);
    launch_plain_realpost(z, a.fft, a.power, lp, s);
    if (ev) cudaEventRecord(ev[2], s);
    if (ev) cudaEventRecord(ev[3], s);
    plain_harmonic<<<dim3(blocks_for(p.fundamental, kBlock), 5), kBlock, 0, s>>>(a.power, p, a.summed, a.count,
                                                                                 a.cands, a.status);
    if (ev) cudaEventRecord(ev[4], s);
}

// Gathers the candidates of `count` result slots back to back in the caller's
// order, each slot's list sorted by (level, bin) -- the order the single-template
// read-out gives (src/vulkan.cpp:329-337 returns a slot's list; the lists here
// are sorted so that the result does not depend on the device's emission order).
// Slot k holds the caller's template rank[k]; offsets[t] = sum of
// min(counts[u], capacity) over the slots u with rank[u] < t, offsets[count] = total.
// One CTA per slot: it sums the clamped counts of the slots before its
// template, loads its list as 64-bit keys (level, bin, power bits; (level, bin)
// is unique within a slot, so the sorted order is unique), sorts them in shared
// memory (bitonic, padded to a power of two) and writes them out.  A list longer
// than the shared-memory sort (kCompactSortMax) is copied unsorted and sorted by
// the host.  With the toplist pre-filter (toplist_filter.cu) a slot writes only
// the candidates that pass it, and the offsets sum those kept counts.
__host__ __device__ constexpr uint32_t compact_sort_size(uint32_t capacity) {
    uint32_t p = 2;
    while (p < capacity && p < kCompactSortMax) p <<= 1;
    return p;
}

__device__ __forceinline__ unsigned long long compact_key(const brp_candidate& x) {
    return (static_cast<unsigned long long>(x.level) << 55) | (static_cast<unsigned long long>(x.bin) << 32) |
           __float_as_uint(x.power);
}

__global__ void __launch_bounds__(256) bank_compact_kernel(const uint32_t* counts, const brp_candidate* cands,
                                                           uint32_t capacity, uint32_t count, const uint32_t* rank,
                                                           brp_candidate* out, uint64_t out_cap, uint64_t* offsets,
                                                           FilterArgs f, bool filtered) {
    extern __shared__ unsigned long long keys[];
    __shared__ uint64_t s_part[8];
    __shared__ uint32_t s_fill;
    const uint32_t k = blockIdx.x, t = rank[k];
    // the slot's written count: all its candidates, or those that pass the filter
    auto written = [&](uint32_t u) { return filtered ? f.kept[u] : min(counts[u], capacity); };
    uint64_t acc = 0;
    for (uint32_t u = threadIdx.x; u < count; u += blockDim.x)
        if (rank[u] < t) acc += written(u);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s_part[threadIdx.x >> 5] = acc;
    if (threadIdx.x == 0) s_fill = 0u;
    __syncthreads();
    uint64_t off = 0;
#pragma unroll
    for (int w = 0; w < 8; ++w) off += s_part[w];
    const uint32_t all = min(counts[k], capacity), c = written(k);
    const uint32_t s = filtered ? f.slot_series[k] : 0u;
    if (threadIdx.x == 0) {
        offsets[t] = off;
        if (t + 1 == count) offsets[count] = off + c;
    }
    const brp_candidate* src = cands + size_t(k) * capacity;
    if (c > kCompactSortMax) {  // unsorted (the host sorts); filtered lists in any order
        for (uint32_t i = threadIdx.x; i < all; i += blockDim.x) {
            const brp_candidate x = src[i];
            if (filtered && !filter_keep(f, s, x)) continue;
            const uint32_t at = filtered ? atomicAdd(&s_fill, 1u) : i;
            if (off + at < out_cap) out[off + at] = x;
        }
        return;
    }
    uint32_t P = 2;
    while (P < c) P <<= 1;
    if (filtered) {
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) keys[i] = ~0ull;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < all; i += blockDim.x) {
            const brp_candidate x = src[i];
            if (filter_keep(f, s, x)) keys[atomicAdd(&s_fill, 1u)] = compact_key(x);
        }
    } else {
        for (uint32_t i = threadIdx.x; i < P; i += blockDim.x) keys[i] = i < c ? compact_key(src[i]) : ~0ull;
    }
    __syncthreads();
    for (uint32_t w = 2; w <= P; w <<= 1) {
        for (uint32_t j = w >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < P / 2; i += blockDim.x) {
                const uint32_t lo = ((i & ~(j - 1)) << 1) | (i & (j - 1)), hi = lo | j;
                const unsigned long long x = keys[lo], y = keys[hi];
                if ((x > y) == ((lo & w) == 0)) { keys[lo] = y; keys[hi] = x; }
            }
            __syncthreads();
        }
    }
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
        if (off + i >= out_cap) break;
        const unsigned long long key = keys[i];
        brp_candidate x;
        x.level = uint32_t(key >> 55); x.bin = uint32_t(key >> 32) & 0x7FFFFFu; x.power = __uint_as_float(uint32_t(key));
        x.reserved = 0;
        out[off + i] = x;
    }
}

cudaError_t set_bank_compact_attributes(uint32_t capacity) {
    return cudaFuncSetAttribute(bank_compact_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                int(compact_sort_size(capacity) * sizeof(unsigned long long)));
}

void launch_bank_compact(const uint32_t* counts, const brp_candidate* cands, uint32_t capacity, uint32_t count,
                         const uint32_t* rank, brp_candidate* out, uint64_t out_cap, uint64_t* offsets,
                         const FilterArgs* filter, cudaStream_t s) {
    if (count)
        bank_compact_kernel<<<count, 256, compact_sort_size(capacity) * sizeof(unsigned long long), s>>>(
            counts, cands, capacity, count, rank, out, out_cap, offsets, filter ? *filter : FilterArgs{},
            filter != nullptr);
}

}  // namespace brp
