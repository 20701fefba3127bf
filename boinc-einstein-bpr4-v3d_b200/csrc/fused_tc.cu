// Tensor-core form of the fused pass 1: the first radix-16 stage of the column
// FFTs runs as a matrix product on the fifth-generation tensor cores
// (tcgen05.mma kind::f16, BF16 operands, FP32 accumulation in tensor memory);
// the remaining Stockham passes, the last one fused with the four-step twiddle
// and the store, are those of pass1_fast (fused_fast.cu).
//
// A CTA transforms C columns of L1 points.  The first Stockham pass (span 1,
// radix 16) of a column is L1/16 independent 16-point DFTs: butterfly j takes
// x[j + r L1/16], r < 16, and writes y[16 j + m], m < 16.  With the 16 complex
// inputs of a butterfly as one row of 32 reals (re, im interleaved), the
// outputs of all C L1/16 butterflies of the CTA are one product
//     Y (rows x 32) = X (rows x 32) . F^T,
// F[2m + p][2r + q] the real 32 x 32 form of W_16^{rm} (angle a = 2 pi (rm mod 16) / 16):
//     F[2m][2r] = cos a, F[2m][2r+1] = sin a, F[2m+1][2r] = -sin a, F[2m+1][2r+1] = cos a.
// BF16 keeps 8 significant bits, so every FP32 operand is split into TERMS
// BF16 parts, v = v_0 + v_1 (+ v_2), v_{i+1} the BF16 rounding of what the
// earlier parts leave.  The product keeps the part products X_i F_j with
// i + j < TERMS, smallest first, in one FP32 accumulator: TERMS = 2 is the
// hi/lo split (3 of 4 products, 16 bits of each operand); TERMS = 3 carries
// all 24 bits of an FP32 operand (6 of 9 products).
//
// Data path: the CTA's rows are enumerated as row = j C + c = threadIdx.x, so
// each thread gathers exactly one butterfly row (L1 C / THREADS = 16 resampled
// complex points) and writes its BF16 parts straight into the operand tiles in
// shared memory, in the tensor core's K-major layout without swizzle: 128-row
// tiles of 8 x 16-byte core matrices, element k of row i at
//     (i / 8) 512 + (k / 8) 128 + (i % 8) 16 + (k % 8) 2 bytes
// (descriptor: leading-dimension offset 128 B between the core matrices along
// K, stride offset 512 B between 8-row groups).  F lives in the same layout
// (32 rows).  One thread issues TILES x products x 2 MMAs (M = 128, N = 32,
// K = 16) into a tensor-memory accumulator of 32 columns per tile and commits
// them to an mbarrier; every thread waits with an iteration bound.  Warp w
// reads lanes 32 (w % 4) .. +31 of tile w / 4 (tcgen05.ld 32x32b, one row of
// 32 FP32 per thread) and stores the 16 complex outputs into the padded FP32
// layout of the CUDA-core passes, which overlays the operand tiles (the MMAs
// have completed when the mbarrier phase flips).  A wait that reaches its
// bound sets BRP_STATUS_WAIT_TIMEOUT for the template, frees the tensor memory
// and leaves the CTA.
#include <cuda_bf16.h>
#include "async_device.cuh"
#include "fast_common.cuh"

namespace brp {
namespace {

constexpr int kTileRows = 128;              // MMA M
constexpr int kTileBytes = kTileRows * 64;  // 128 rows x 32 BF16
constexpr int kFBytes = 32 * 64;            // F: 32 rows x 32 BF16
constexpr int kSmPerSm = 233472;            // shared memory of one SM (228 KiB)

// Shared-memory matrix descriptor, K-major, no swizzle: start address, leading
// byte offset 128, stride byte offset 512 (all in 16-byte units), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr) {
    return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t(128 >> 4) << 16) | (uint64_t(512 >> 4) << 32) |
           (uint64_t(1) << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = 32, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(32 >> 3) << 17) |
                            (uint32_t(128 >> 4) << 24);

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
        : "memory");
}

// Part products X_i F_j (i + j < terms), smallest first: (1,1) (0,2) (2,0)
// (0,1) (1,0) (0,0) for three parts, (0,1) (1,0) (0,0) for two.
__host__ __device__ constexpr int part_a(int terms, int k) {
    return terms == 3 ? (k == 0 ? 1 : k == 2 ? 2 : k == 4 ? 1 : 0) : (k == 1 ? 1 : 0);
}
__host__ __device__ constexpr int part_b(int terms, int k) {
    return terms == 3 ? (k == 0 ? 1 : k == 1 ? 2 : k == 3 ? 1 : 0) : (k == 0 ? 1 : 0);
}

// cos(2 pi t / 16), from the FP32 roundings of cos(pi v / 8), v <= 4.
__device__ __forceinline__ float cos16(int t) {
    t &= 15;
    const int u = t <= 8 ? t : 16 - t, v = u <= 4 ? u : 8 - u;
    const float x = v == 0 ? 1.0f : v == 1 ? 0.923879532511286756f : v == 2 ? 0.707106781186547524f
                  : v == 3 ? 0.382683432365089772f : 0.0f;
    return u <= 4 ? x : -x;
}

__device__ __forceinline__ uint32_t bf16_bits(__nv_bfloat16 h) {
    return static_cast<uint32_t>(__bfloat16_as_ushort(h));
}

// Splits a pair of FP32 values into TERMS BF16 parts (exact remainders), one
// packed word per part: low half the first value, high half the second.
template <int TERMS>
__device__ __forceinline__ void split_pair(float a, float b, uint32_t* w) {
#pragma unroll
    for (int p = 0; p < TERMS; ++p) {
        const __nv_bfloat16 ha = __float2bfloat16_rn(a), hb = __float2bfloat16_rn(b);
        w[p] = bf16_bits(ha) | (bf16_bits(hb) << 16);
        a = __fsub_rn(a, __bfloat162float(ha));
        b = __fsub_rn(b, __bfloat162float(hb));
    }
}

// Gathers the 16 complex inputs of butterfly row threadIdx.x (column c =
// threadIdx.x % C, j = threadIdx.x / C: points n1 = j + r L1/16) and writes
// their BF16 parts into the operand tiles, four points (one 16-byte row chunk
// of a core matrix per part) at a time.  Returns the sum of the samples, added
// in the order of the CUDA-core gather.
template <int L1, int C, int THREADS, int MODE, int TERMS>
__device__ __forceinline__ double gather_rows(unsigned char* A, const float* __restrict__ in, const brp_params& P,
                                              uint32_t L2, uint32_t c0, float* raw, bool& oob) {
    constexpr int NBF = L1 / 16, TILES = THREADS / kTileRows, PART = TILES * kTileBytes;
    static_assert(L1 * C == 16 * THREADS && THREADS % kTileRows == 0, "one butterfly row per thread");
    const brp_resample_consts rc = consts_of(P);
    const uint32_t steps = P.steps, unpadded = P.unpadded;
    const int t = threadIdx.x, c = t % C, j = t / C;
    const uint32_t istep = 2u * L2 * uint32_t(NBF);
    uint32_t i = 2u * (L2 * uint32_t(j) + c0 + uint32_t(c));
    const int ri = t & (kTileRows - 1);
    unsigned char* dst = A + (t / kTileRows) * kTileBytes + (ri >> 3) * 512 + (ri & 7) * 16;
    float sum = 0.f;
#pragma unroll 1
    for (int q = 0; q < 4; ++q) {
        int jx[8];
#pragma unroll
        for (int b = 0; b < 4; ++b)
            index_pair<MODE>(i + uint32_t(b) * istep, rc, steps, unpadded, jx[2 * b], jx[2 * b + 1], oob);
        float v[8];
#pragma unroll
        for (int b = 0; b < 8; ++b) v[b] = jx[b] >= 0 ? __ldg(in + jx[b]) : 0.f;
        uint32_t w[4][TERMS];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            if (raw) {
                const uint32_t ib = i + uint32_t(b) * istep;
                if (ib < steps) raw[ib] = v[2 * b];
                if (ib + 1 < steps) raw[ib + 1] = v[2 * b + 1];
            }
            sum += v[2 * b];
            sum += v[2 * b + 1];
            split_pair<TERMS>(v[2 * b], v[2 * b + 1], w[b]);
        }
#pragma unroll
        for (int p = 0; p < TERMS; ++p)
            *reinterpret_cast<uint4*>(dst + p * PART + q * 128) = make_uint4(w[0][p], w[1][p], w[2][p], w[3][p]);
        i += 4u * istep;
    }
    return double(sum);
}

// Writes the BF16 parts of F (32 x 32, K-major) into shared memory.
template <int THREADS, int TERMS>
__device__ __forceinline__ void fill_dft16_operand(unsigned char* Fm) {
    for (int e = threadIdx.x; e < 32 * 16; e += THREADS) {
        const int n = e >> 4, r = e & 15, m = n >> 1;
        const int t = (r * m) & 15;
        const float cs = cos16(t), sn = cos16(t + 12);
        const float x0 = (n & 1) ? -sn : cs, x1 = (n & 1) ? cs : sn;
        uint32_t w[TERMS];
        split_pair<TERMS>(x0, x1, w);
        const int off = (n >> 3) * 512 + (r >> 2) * 128 + (n & 7) * 16 + (r & 3) * 4;
#pragma unroll
        for (int p = 0; p < TERMS; ++p) *reinterpret_cast<uint32_t*>(Fm + p * kFBytes + off) = w[p];
    }
}

template <int L1, int C, int THREADS, int TERMS>
struct TcLayout {
    static constexpr int TILES = THREADS / kTileRows;
    static constexpr int STRIDE = ct_stride(L1, C);
    static constexpr int SM_BYTES = C * STRIDE * 8;  // FP32 layout of the CUDA-core passes
    static constexpr int A_BYTES = TERMS * TILES * kTileBytes;
    static constexpr int F_OFF = ((SM_BYTES > A_BYTES ? SM_BYTES : A_BYTES) + 1023) & ~1023;
    static constexpr int SMEM = F_OFF + TERMS * kFBytes;
    static constexpr uint32_t COLS = TILES * 32 <= 32 ? 32 : TILES * 32 <= 64 ? 64 : TILES * 32 <= 128 ? 128
                                     : TILES * 32 <= 256 ? 256 : 512;
    // Tensor memory is allocated without a retry bound, so every CTA that can
    // be resident on an SM (shared memory decides) must fit in its 512 columns.
    static_assert((kSmPerSm / (SMEM + 1024)) * COLS <= 512, "tensor memory of resident CTAs");
    static_assert(TILES * 32 <= 512 && THREADS / 32 >= 4 * TILES, "one warp per 32 accumulator lanes");
};

template <int L1, int C, int THREADS, int MINB, int TERMS, int... Rest>
__global__ void __launch_bounds__(THREADS, MINB) pass1_tc(FusedArgs a) {
    using Lay = TcLayout<L1, C, THREADS, TERMS>;
    constexpr int STRIDE = Lay::STRIDE, TILES = Lay::TILES, PART = TILES * kTileBytes;
    constexpr int NP = TERMS == 3 ? 6 : 3;
    extern __shared__ __align__(1024) unsigned char dsm[];
    __shared__ double red[THREADS / 32];
    __shared__ uint32_t s_tmem;
    __shared__ __align__(8) uint64_t s_bar;
    unsigned char* A = dsm;
    unsigned char* Fm = dsm + Lay::F_OFF;
    float2* sm = reinterpret_cast<float2*>(dsm);  // overlays A once the MMAs have completed
    const int g = blockIdx.y, warp = threadIdx.x >> 5;
    const brp_params& P = a.params[g];
    const float* __restrict__ in = a.inputs[g];
    const uint32_t L2 = a.L2, c0 = blockIdx.x * C;
    const uint32_t bar = smem_u32(&s_bar);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(Lay::COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
    }
    fill_dft16_operand<THREADS, TERMS>(Fm);

    float* raw = (g == a.snap) ? a.snap_raw : nullptr;
    bool oob = false;
    double sum;
    if (P.flags & BRP_FLAG_INDEX_FP64) sum = gather_rows<L1, C, THREADS, 2, TERMS>(A, in, P, L2, c0, raw, oob);
    else if (P.flags & 2u) sum = gather_rows<L1, C, THREADS, 1, TERMS>(A, in, P, L2, c0, raw, oob);
    else sum = gather_rows<L1, C, THREADS, 0, TERMS>(A, in, P, L2, c0, raw, oob);
    if (oob) atomicOr(a.status + g, BRP_STATUS_RESAMPLE_OOB);
    // Operand writes (generic proxy) become visible to the tensor core (async proxy).
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    const double tot = block_sum_d<THREADS>(sum, red);  // synchronises the CTA
    publish_mean<THREADS>(a, g, P.steps, tot, red);      // before any early exit below
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (threadIdx.x == 0) {
        const uint32_t a0 = smem_u32(A), f0 = smem_u32(Fm);
#pragma unroll 1
        for (int tile = 0; tile < TILES; ++tile) {
            uint32_t acc = 0;
#pragma unroll
            for (int k = 0; k < NP; ++k) {
                const int ia = part_a(TERMS, k), ib = part_b(TERMS, k);
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    umma_bf16(tmem + uint32_t(tile * 32), umma_desc(a0 + ia * PART + tile * kTileBytes + ks * 256),
                              umma_desc(f0 + ib * kFBytes + ks * 256), acc);
                    acc = 1;
                }
            }
        }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                     : "memory");
    }
    const bool done = mbar_wait_bounded(bar, 0, a.wait_polls);
    const int timed_out = __syncthreads_or(!done);
    // On expiry the MMAs may still write this CTA's tensor memory and read its
    // operand tiles: drain them (full bound) before the memory is freed.
    if (timed_out) mbar_wait_bounded(bar, 0, kDrainPolls);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!timed_out && warp < 4 * TILES) {
        const int quad = warp & 3, tile = warp >> 2;
        uint32_t d[32];
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
            "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
            : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
              "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]), "=r"(d[14]),
              "=r"(d[15]), "=r"(d[16]), "=r"(d[17]), "=r"(d[18]), "=r"(d[19]), "=r"(d[20]), "=r"(d[21]),
              "=r"(d[22]), "=r"(d[23]), "=r"(d[24]), "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]),
              "=r"(d[29]), "=r"(d[30]), "=r"(d[31])
            : "r"(tmem + (uint32_t(quad * 32) << 16) + uint32_t(tile * 32)));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const int row = tile * kTileRows + quad * 32 + (threadIdx.x & 31);
        const int c = row % C, j = row / C;
        float2* dst = sm + c * STRIDE + ct_pos(16 * j);
#pragma unroll
        for (int m = 0; m < 16; ++m) dst[m] = make_float2(__uint_as_float(d[2 * m]), __uint_as_float(d[2 * m + 1]));
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Lay::COLS)
                     : "memory");
    }
    if (timed_out) {
        if (threadIdx.x == 0) atomicOr(a.status + g, BRP_STATUS_WAIT_TIMEOUT);
        return;
    }

    ct_fft_store<L1, STRIDE, C, THREADS, 16, Rest...>(sm, a.ptw1, a.work + size_t(g) * a.work_stride, a.fs_hi, a.fs_lo,
                                                    L2, c0);
}

template <int L1, int C, int THREADS, int MINB, int TERMS, int... Rest>
struct P1T {
    static constexpr int smem = TcLayout<L1, C, THREADS, TERMS>::SMEM;
    static void launch(const FusedArgs& a, uint32_t blocks, uint32_t count, cudaStream_t s) {
        pass1_tc<L1, C, THREADS, MINB, TERMS, Rest...><<<dim3(blocks, count), THREADS, smem, s>>>(a);
    }
    static cudaError_t attr() {
        return cudaFuncSetAttribute(pass1_tc<L1, C, THREADS, MINB, TERMS, Rest...>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    }
    static FastPass info(int id) {
        FastPass f;
        f.id = id; f.L = L1; f.group = C; f.threads = THREADS; f.smem = smem; f.launch = &launch; f.attr = &attr;
        int r[] = {16, Rest...};
        f.plan.count = int(1 + sizeof...(Rest));
        for (int i = 0; i < f.plan.count; ++i) f.plan.radix[i] = r[i];
        f.table = ct_table_size<false, 1, 16, Rest...>();
        f.tensor = TERMS;
        return f;
    }
};

}  // namespace

// Tensor-core pass-1 configurations, each the tuned CUDA-core decomposition
// with its first radix-16 stage on the tensor cores: 111/112 columns of 2048
// (n = 2^22) as 16 x 8 x 16 like 110, 113/114 columns of 1536 (n = 3 2^21 with
// rows of 2048) as 16 x 4 x 3 x 8 like 119; the odd ids carry three BF16 parts
// per operand, the even ids two.
void append_pass1_tc_configs(std::vector<FastPass>& v) {
    v.push_back(P1T<2048, 4, 512, 2, 3, 8, 16>::info(111));
    v.push_back(P1T<2048, 4, 512, 2, 2, 8, 16>::info(112));
    v.push_back(P1T<1536, 4, 384, 2, 3, 4, 3, 8>::info(113));
    v.push_back(P1T<1536, 4, 384, 2, 2, 4, 3, 8>::info(114));
}

}  // namespace brp
