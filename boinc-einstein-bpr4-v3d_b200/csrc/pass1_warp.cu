// Pass 1 with warp-local exchanges (compiled pass-1 configurations 124-127).
//
// Same transform as pass1_fast with the radix sequence (16, R2, 16) over
// L1 = 256 R2 and C = 32 / R2 columns per CTA (512 threads): resampling gather
// of 16 points per thread, first radix-16 pass in registers, a radix-R2 pass,
// a last radix-16 pass fused with the four-step twiddle and the store of T.
// Only the thread assignment and the shared-memory layout differ, chosen so
// that the exchange between the first and the middle pass stays inside a warp:
//
//  * warp w (0..15), lane l: column c = l % C, q = l / C (0..R2-1) gathers and
//    transforms the first-pass butterfly j = w + 16 q of column c;
//  * the middle butterflies b = 16 w + m (m = 0..15) of column c need the first
//    pass's output m of the butterflies w + 16 r (r = 0..R2-1): exactly the R2
//    lanes of warp w with that column.  They exchange through the warp's own
//    region S[w][c][r][m] (rows of 16 values, row stride 18 float2 so that
//    16-byte accesses of a quarter warp hit distinct banks) with a __syncwarp,
//    and each lane transforms its butterflies m = (16/R2) q .. in place: it
//    writes its outputs to exactly the slots it read, so no other lane's data
//    is overwritten and no barrier is needed;
//  * output r' of middle butterfly (w, m) is element 128 w + m + 16 r' of the
//    Stockham sequence; the last pass's butterfly j' needs elements j' + 16 R2 r
//    (r = 0..15), i.e. S[r][c][j'/16][j'%16] from every warp: one block barrier.
//
// So a CTA synchronises once between the gather and the store (plus the
// publication of its FP64 sum at the end), and a warp runs its gather, first
// and middle passes independently of the other warps of its CTA.
//
// Configurations 126 and 127 are 124 and 125 with the store of T done by the
// tensor-memory accelerator: the CTA's outputs form one L1 x C tile of T (rows
// of C complex values, 8 C bytes, at a row pitch of L2), which the threads
// write into shared memory (a warp's stores are 256 contiguous bytes there)
// and one thread sends to T as R2 boxes of 256 rows (cp.async.bulk.tensor,
// no multicast).  A row of the tile is 32 or 64 bytes, so every st.global of
// the plain store touches 32/C lines; the bulk store moves the tile without
// the load/store unit.  The tile reuses the exchange buffer after a barrier.
#include "fast_common.cuh"
#include "tma_store.cuh"

namespace brp {
namespace {

constexpr int kRowStride = 18;  // float2 per row of 16 values in a warp region

template <int R2, int C>
struct WarpLayout {
    static_assert(R2 * C == 32, "one first-pass butterfly per lane");
    static constexpr int L1 = 256 * R2;
    // float2 per (warp, column) region: at least its R2 rows, and = 16 / C
    // (mod 16), so that region (w, c) starts (16 / C) c float2 = (8 / C) c
    // 16-byte granules past a bank-aligned offset (16 C REG = 0 mod 16 per warp).
    static constexpr int SHIFT = 16 / C;
    static constexpr int REG = R2 * kRowStride + ((SHIFT - R2 * kRowStride) % 16 + 16) % 16;
    static constexpr int SLOTS = 16 * C * REG;
    __host__ __device__ static constexpr int base(int w, int c) { return (w * C + c) * REG; }
    static_assert(REG % 16 == SHIFT % 16 && REG >= R2 * kRowStride && REG % 2 == 0, "region layout");
};

// The 16 points x[j + (L1/16) r] (r = 0..15) of column c as in gather_dft16
// (indices of eight points, then their 16 loads, twice); returns the FP32 sum.
template <int L1, int MODE>
__device__ __forceinline__ float gather16(float2 (&x)[16], const float* __restrict__ in, const brp_params& P,
                                          uint32_t L2, uint32_t c0, int j, int c, float* raw, bool& oob) {
    constexpr int NBF = L1 / 16;
    const brp_resample_consts rc = consts_of(P);
    const uint32_t steps = P.steps, unpadded = P.unpadded;
    const uint32_t istep = 2u * L2 * uint32_t(NBF);
    uint32_t i = 2u * (L2 * uint32_t(j) + c0 + uint32_t(c));
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
    return sum;
}

// The kernel body; TMA: the store of T as bulk tensor copies through the
// tensor map *tm (3-D: L2 complex values as 8-byte elements, L1 rows, the
// launch's templates; box C x 256 x 1).
template <int R2, int C, bool TMA>
__device__ __forceinline__ void pass1_warp_body(const FusedArgs& a, const CUtensorMap* tm) {
    using Lay = WarpLayout<R2, C>;
    constexpr int L1 = Lay::L1, NBF = L1 / 16, MB = 16 / R2;  // MB middle butterflies per lane
    extern __shared__ __align__(16) float2 sm[];
    __shared__ double red[16];
    __shared__ float2 s_fs[C][17];  // W_M^{n2 m NBF}, n2 = c0 + column, m = 0..15 (rows padded: columns on distinct banks)
    const int g = blockIdx.y;
    const brp_params& P = a.params[g];
    const float* __restrict__ in = a.inputs[g];
    const uint32_t L2 = a.L2, c0 = blockIdx.x * C;
    float* raw = (g == a.snap) ? a.snap_raw : nullptr;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the column factors of the four-step twiddle (read after the block barrier)
    if (threadIdx.x < 16 * C) {
        const int col = threadIdx.x / 16, mm = threadIdx.x % 16;
        s_fs[col][mm] = twiddle2(a.fs_hi, a.fs_lo, kSplitLog2, (c0 + uint32_t(col)) * uint32_t(mm * NBF));
    }
    const int c = lane % C, q = lane / C;

    // ---- gather + first radix-16 pass (butterfly j = w + 16 q of column c)
    float2 x[16];
    bool oob = false;
    float sum;
    const int j = w + 16 * q;
    const bool small = P.unpadded <= (1u << 23);  // every sample index below 2^23
    if (P.flags & BRP_FLAG_INDEX_FP64) sum = gather16<L1, 2>(x, in, P, L2, c0, j, c, raw, oob);
    else if ((P.flags & 2u) && small) sum = gather16<L1, 1 | kSmallIndex>(x, in, P, L2, c0, j, c, raw, oob);
    else if (P.flags & 2u) sum = gather16<L1, 1>(x, in, P, L2, c0, j, c, raw, oob);
    else if (small) sum = gather16<L1, kSmallIndex>(x, in, P, L2, c0, j, c, raw, oob);
    else sum = gather16<L1, 0>(x, in, P, L2, c0, j, c, raw, oob);
    if (oob) atomicOr(a.status + g, BRP_STATUS_RESAMPLE_OOB);
    double dsum = double(sum);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dsum += __shfl_down_sync(0xffffffffu, dsum, o);
    if (lane == 0) red[w] = dsum;
    dft16(x);
    float2* reg = sm + Lay::base(w, c);
    {
        float4* row = reinterpret_cast<float4*>(reg + kRowStride * q);
#pragma unroll
        for (int m = 0; m < 16; m += 2) row[m / 2] = make_float4(x[m].x, x[m].y, x[m + 1].x, x[m + 1].y);
    }
    __syncwarp();

    // ---- middle radix-R2 pass (span 16): butterflies m = MB q .. MB q + MB - 1
    {
        float2 v[MB][R2];
#pragma unroll
        for (int r = 0; r < R2; ++r) {
            const float4* src = reinterpret_cast<const float4*>(reg + kRowStride * r + MB * q);
#pragma unroll
            for (int h = 0; h < MB / 2; ++h) {
                const float4 t = src[h];
                v[2 * h][r] = make_float2(t.x, t.y);
                v[2 * h + 1][r] = make_float2(t.z, t.w);
            }
        }
#pragma unroll
        for (int u = 0; u < MB; ++u) {
            ct_twiddle<R2, 16>(v[u], a.ptw1, MB * q + u);
            dft<R2>(v[u]);
        }
#pragma unroll
        for (int r = 0; r < R2; ++r) {
            float4* dst = reinterpret_cast<float4*>(reg + kRowStride * r + MB * q);
#pragma unroll
            for (int h = 0; h < MB / 2; ++h)
                dst[h] = make_float4(v[2 * h][r].x, v[2 * h][r].y, v[2 * h + 1][r].x, v[2 * h + 1][r].y);
        }
    }
    __syncthreads();

    // ---- last radix-16 pass (span NBF) fused with the four-step twiddle and the
    // store: thread t = C j' + cc takes butterfly j' of column cc, so a warp
    // stores 32/C rows of C adjacent columns.
    const int cc = threadIdx.x % C, jp = threadIdx.x / C;
    const uint32_t n2 = c0 + uint32_t(cc);
    {
        float2 v[16];
        const int off = kRowStride * (jp / 16) + (jp % 16);
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = sm[Lay::base(r, cc) + off];
        ct_twiddle<16, NBF>(v, a.ptw1 + 16 * TwStride<R2>::value, jp);
        dft16(v);
        // W_M^{n2 (jp + m NBF)} = W_M^{n2 jp} W_M^{n2 m NBF}: one table value per
        // thread and the CTA's column factors from shared memory
        const float2 base = twiddle2(a.fs_hi, a.fs_lo, kSplitLog2, n2 * uint32_t(jp));
        if constexpr (!TMA) {
            float2* __restrict__ T = a.work + size_t(g) * a.work_stride;
#pragma unroll
            for (int m = 0; m < 16; ++m)
                T[size_t(jp + m * NBF) * L2 + n2] = cmul(v[m], cmul(base, s_fs[cc][m]));
        } else {
#pragma unroll
            for (int m = 0; m < 16; ++m) v[m] = cmul(v[m], cmul(base, s_fs[cc][m]));
            __syncthreads();  // every thread has read its last-pass inputs from the exchange buffer
            // the tile [row][column] at the first 128-byte boundary of the buffer
            // (L1 C 8 = 64 KiB; the buffer has at least 128 bytes more)
            const uint32_t tile_sh = tile_address(sm);
            float2* tile = sm + (tile_sh - smem_u32(sm)) / 8;
#pragma unroll
            for (int m = 0; m < 16; ++m) tile[(jp + m * NBF) * C + cc] = v[m];
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the bulk copies
            __syncthreads();
            if (threadIdx.x == 0) store_tile_bulk<L1, C>(tm, tile_sh, c0, g);
        }
    }

    // ---- this CTA's FP64 sum of its samples; the template's mean from its last CTA
    double tot = 0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int k = 0; k < 16; ++k) tot += red[k];
    }
    publish_mean<512>(a, g, P.steps, tot, red);
    // the tile stays in shared memory until the bulk copies have read it
    if constexpr (TMA)
        if (threadIdx.x == 0) wait_tile_read();
}

template <int R2, int C, int MINB>
__global__ void __launch_bounds__(512, MINB) pass1_warp(FusedArgs a) {
    pass1_warp_body<R2, C, false>(a, nullptr);
}

template <int R2, int C, int MINB>
__global__ void __launch_bounds__(512, MINB) pass1_warp_tma(FusedArgs a, const __grid_constant__ CUtensorMap tm) {
    pass1_warp_body<R2, C, true>(a, &tm);
}

template <int R2, int C, int MINB, bool TMA = false>
struct P1W {
    using Lay = WarpLayout<R2, C>;
    static constexpr int smem = Lay::SLOTS * 8;
    static_assert(!TMA || smem >= Lay::L1 * C * 8 + 128, "the tile and its alignment fit the exchange buffer");
    static void launch(const FusedArgs& a, uint32_t blocks, uint32_t count, cudaStream_t s) {
        if constexpr (!TMA) {
            pass1_warp<R2, C, MINB><<<dim3(blocks, count), 512, smem, s>>>(a);
        } else {
            CUtensorMap tm{};
            const bool ok = encode_tile_map(&tm, a, uint32_t(Lay::L1), uint32_t(C), blocks, count);
            // without a tensor map nothing is launched, and the empty grid makes
            // the caller's launch check report cudaErrorInvalidConfiguration
            pass1_warp_tma<R2, C, MINB><<<ok ? dim3(blocks, count) : dim3(0, 0), 512, smem, s>>>(a, tm);
        }
    }
    static cudaError_t attr() {
        if constexpr (!TMA)
            return cudaFuncSetAttribute(pass1_warp<R2, C, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        else
            return cudaFuncSetAttribute(pass1_warp_tma<R2, C, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    }
    static FastPass info(int id) {
        FastPass f;
        f.id = id; f.L = Lay::L1; f.group = C; f.threads = 512; f.smem = smem; f.launch = &launch; f.attr = &attr;
        f.plan.count = 3;
        f.plan.radix[0] = 16; f.plan.radix[1] = R2; f.plan.radix[2] = 16;
        f.table = ct_table_size<false, 1, 16, R2, 16>();
        return f;
    }
};

}  // namespace

void append_pass1_warp_configs(std::vector<FastPass>& v) {
    v.push_back(P1W<8, 4, 2>::info(124));  // L1 = 2048 = 16 x 8 x 16, 4 columns (the layout of 110)
    v.push_back(P1W<4, 8, 2>::info(125));  // L1 = 1024 = 16 x 4 x 16, 8 columns (the layout of 118)
    v.push_back(P1W<8, 4, 2, true>::info(126));  // 124 with the bulk tensor store of T
    v.push_back(P1W<4, 8, 2, true>::info(127));  // 125 with the bulk tensor store of T
}

}  // namespace brp
