// Length plans: the FFT decomposition chosen for one series length n and its
// twiddle tables.  Every table entry is computed in FP64 (cos/sin of an exact
// rational angle) and rounded once to FP32; no recurrences.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>
#include "brp_internal.h"

namespace brp {

static bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }
static uint32_t ilog2(uint32_t x) { uint32_t r = 0; while (x > 1) { x >>= 1; ++r; } return r; }

// Radix plan of a shared-memory FFT of length L = 2^a or 3*2^a: ceil(a/4)
// power-of-two passes with the bits spread evenly (radix 16, 8, 4, 2), and a
// radix-3 pass last when L has the factor 3.
RadixPlanHost radix_plan(uint32_t L) {
    RadixPlanHost p;
    uint32_t three = (L % 3 == 0) ? 1 : 0;
    uint32_t a = ilog2(L / (three ? 3 : 1));
    uint32_t passes = (a + 3) / 4;
    for (uint32_t i = 0; i < passes; ++i) {
        uint32_t bits = a / passes + (i < a % passes ? 1 : 0);
        p.radix[p.count++] = 1 << bits;
    }
    if (three) p.radix[p.count++] = 3;
    return p;
}

static void fill_twiddles(float2* out, uint32_t count, uint64_t period, uint64_t first, uint64_t step) {
    for (uint32_t i = 0; i < count; ++i) {
        // angle = -2 pi e / period with e reduced exactly in integers
        uint64_t e = (first + uint64_t(i) * step) % period;
        double ang = -2.0 * M_PI * (double(e) / double(period));
        out[i] = make_float2(float(std::cos(ang)), float(std::sin(ang)));
    }
}

size_t plan_smem_limit() { return 110 * 1024; }

static const FastPass* find_fast(const std::vector<FastPass>& v, uint32_t L, int want) {
    if (want < 0) return nullptr;
    for (auto& f : v)
        if (f.L == L && (want == 0 || f.id == want)) return &f;
    return nullptr;
}

// Per-pass twiddle table of a radix sequence: pass p (span Ns = product of the
// earlier radices, radix R) holds, for butterfly k, the twiddles W_{Ns R}^{q k}
// of the powers q = pass_twiddle_power(R, s), s < pass_twiddle_powers(R) (W^0
// in a padding slot to an even count RS), pair h = s / 2 as one 16-byte entry at
// [h Ns + k]: the butterflies of a warp read adjacent k of one pair, so their
// loads are contiguous.  The first pass (Ns = 1) needs none.  prod: a product
// table (pass 2).
static void fill_pass_tables(float2* out, const RadixPlanHost& plan, bool prod) {
    uint64_t Ns = 1;
    size_t at = 0;
    for (int p = 0; p < plan.count; ++p) {
        const int R = plan.radix[p], NP = pass_twiddle_powers(R, prod);
        const uint64_t RS = (uint64_t(NP) + 1) & ~uint64_t(1);
        if (Ns > 1)
            for (uint64_t k = 0; k < Ns; ++k)
                for (uint64_t r = 0; r < RS; ++r) {
                    const uint64_t e = (int(r) < NP) ? (uint64_t(pass_twiddle_power(R, int(r), prod)) * k) % (Ns * R) : 0;
                    const double ang = -2.0 * M_PI * (double(e) / double(Ns * R));
                    out[at + 2 * ((r / 2) * Ns + k) + (r % 2)] = make_float2(float(std::cos(ang)), float(std::sin(ang)));
                }
        if (Ns > 1) at += Ns * RS;
        Ns *= R;
    }
}

// The compiled pass pair a length takes when the caller names none and the
// plan cache has no tuned plan for it: the pairs the autotuner chose on one
// B200 for bank workloads of these lengths (n = 2^20, 3*2^20, 2^22, 3*2^21).
// Other lengths take the first compiled pair that fits.
static void preferred_pair(uint32_t M, int& id1, int& id2) {
    id1 = id2 = 0;
    if (M == (1u << 19)) { id1 = 120; id2 = 202; }
    if (M == (3u << 19)) { id1 = 119; id2 = 202; }
    if (M == (1u << 21)) { id1 = 126; id2 = 202; }
    if (M == (3u << 20)) { id1 = 119; id2 = 207; }
}

std::string choose_length_plan(uint32_t n, LengthPlan& lp, int fast1, int fast2, bool use_cache) {
    const bool radix3 = !is_pow2(n);
    if (n < 64 || n > 3u * (1u << 22) || (radix3 && !(n % 3 == 0 && is_pow2(n / 3))))
        return "series length must be 2^k or 3*2^k in 64..3*2^22";
    lp = LengthPlan();
    lp.n = n;
    lp.M = n / 2;
    lp.radix = radix3 ? 3 : 1;
    lp.B = lp.M / lp.radix;
    lp.planB = radix_plan(lp.B);
    // Fused two-pass decomposition for M >= 4096: L2 = 2^min(10, a/2) (a = log2 of
    // the power-of-two part of M), L1 = M / L2 <= 4096.
    // Compiled two-pass decomposition when one exists (rows of 1024 preferred).
    if (lp.M >= 4096 && fast1 >= 0 && fast2 >= 0) {
        int want1[2] = {fast1, fast1}, want2[2] = {fast2, fast2};
        CachedPlan cp;
        if (!fast1 && !fast2) {
            // the autotuner's plan for this length and device, else the pairs it chose on one B200
            if (use_cache && cached_plan(n, cp)) { want1[0] = cp.pass1; want2[0] = cp.pass2; }
            else preferred_pair(lp.M, want1[0], want2[0]);
        }
        for (int attempt = 0; attempt < 2 && !lp.fp1; ++attempt)
            for (uint32_t l2 : {1024u, 512u, 2048u, 256u}) {
                if (lp.M % l2 || lp.M / l2 > 4096) continue;
                const FastPass* f1 = find_fast(fast_pass1_configs(), lp.M / l2, want1[attempt]);
                const FastPass* f2 = find_fast(fast_pass2_configs(), l2, want2[attempt]);
                if (!f1 || !f2 || l2 % f1->group || (lp.M / l2) % (2 * f2->group)) continue;
                lp.fp1 = f1; lp.fp2 = f2;
                lp.L1 = lp.M / l2; lp.L2 = l2; lp.C = f1->group; lp.R = f2->group;
                lp.plan1 = f1->plan; lp.plan2 = f2->plan;
                lp.fused = true;
                if (f1->attr() != cudaSuccess || f2->attr() != cudaSuccess)
                    return "cannot enable the shared memory of the compiled fused kernels";
                break;
            }
    }
    if (lp.M >= 4096 && !lp.fp1) {
        uint32_t a = ilog2(lp.B);
        uint32_t l2 = 1u << std::min<uint32_t>(10, a / 2);
        while (lp.M / l2 > 4096) l2 <<= 1;
        lp.L2 = l2;
        lp.L1 = lp.M / l2;
        // Elements held per thread (512 threads): 16, or 24 for the longest columns.
        lp.maxe = lp.L1 * 4 <= 16 * 512 ? 16 : 24;
        uint32_t cap = lp.maxe * 512;
        uint32_t C = 16;
        while (C > 1 && (C * lp.L1 > cap || C > lp.L2 || C * (lp.L1 + lp.L1 / 16 + 16) * 8 > plan_smem_limit())) C >>= 1;
        uint32_t R = 8;
        while (R > 1 && (2 * R * lp.L2 > cap || R > lp.L1 / 2 || 2 * R * (lp.L2 + lp.L2 / 16 + 16) * 8 > plan_smem_limit()))
            R >>= 1;
        lp.C = C;
        lp.R = R;
        lp.plan1 = radix_plan(lp.L1);
        lp.plan2 = radix_plan(lp.L2);
        lp.fused = C >= 2 && (lp.L1 / (2 * R)) * 2 * R == lp.L1;
        if (lp.fused && set_fused_attributes(std::max(lp.smem1(), lp.smem2())) != cudaSuccess)
            return "cannot enable the shared memory of the fused kernels";
    }
    if (lp.fused && set_harmonic_fast_attributes() != cudaSuccess)
        return "cannot enable the shared memory of the harmonic kernel";
    return "";
}

// Table layout of a chosen plan: offsets (float2 entries) of tw1, tw2, fs_hi,
// fs_lo, rl_hi, rl_lo, twb, ptw1, ptw2, hf_hi, hf_lo, hq and the total.  Tables:
// tw1[L1] tw2[L2] fs_hi[ceil(M/2048)] fs_lo[2048] rl_hi[ceil(n/2048)] rl_lo[2048]
// twb[B] (only with_plain) ptw1 ptw2 (per-pass tables of the compiled passes)
// hf_hi[ceil((M+1)/2048)] hf_lo[2048] (W_{2n}^e = cos(pi e/n) - i sin(pi e/n),
// e <= M) hq[L2] (W_{4 L2}^e); each block 16-byte aligned.
size_t length_plan_layout(const LengthPlan& lp, bool with_plain, size_t off[kPlanTableBlocks + 1]) {
    const uint32_t split = 1u << kSplitLog2, n = lp.n;
    const uint32_t fs_hi_n = (lp.M + split - 1) / split, rl_hi_n = (n + split - 1) / split;
    const uint32_t hf_hi_n = (lp.M + 1 + split - 1) / split;
    const uint32_t counts[kPlanTableBlocks] = {lp.L1, lp.L2, fs_hi_n, split, rl_hi_n, split, with_plain ? lp.B : 0u,
                                               uint32_t(lp.fp1 ? lp.fp1->table : 0),
                                               uint32_t(lp.fp2 ? lp.fp2->table : 0), hf_hi_n, split, lp.L2};
    size_t total = 0;
    for (int i = 0; i < kPlanTableBlocks; ++i) { off[i] = total; total += (counts[i] + 1) & ~1u; }
    off[kPlanTableBlocks] = total;
    return total;
}

// Fills the tables of lp into host[] (laid out by length_plan_layout) and
// points lp's table views at dev (the device copy of host[]).
void fill_length_plan_tables(LengthPlan& lp, bool with_plain, float2* host, float2* dev) {
    size_t off[kPlanTableBlocks + 1];
    length_plan_layout(lp, with_plain, off);
    const uint32_t split = 1u << kSplitLog2, n = lp.n;
    if (lp.L1) fill_twiddles(host + off[0], lp.L1, lp.L1, 0, 1);
    if (lp.L2) fill_twiddles(host + off[1], lp.L2, lp.L2, 0, 1);
    fill_twiddles(host + off[2], uint32_t(off[3] - off[2]) & ~0u, lp.M, 0, split);
    fill_twiddles(host + off[3], split, lp.M, 0, 1);
    fill_twiddles(host + off[4], uint32_t(off[5] - off[4]), n, 0, split);
    fill_twiddles(host + off[5], split, n, 0, 1);
    if (with_plain) fill_twiddles(host + off[6], lp.B, lp.B, 0, 1);
    if (lp.fp1) fill_pass_tables(host + off[7], lp.plan1, false);
    if (lp.fp2) fill_pass_tables(host + off[8], lp.plan2, true);
    fill_twiddles(host + off[9], uint32_t(off[10] - off[9]), 2ull * n, 0, split);
    fill_twiddles(host + off[10], split, 2ull * n, 0, 1);
    if (lp.L2) fill_twiddles(host + off[11], lp.L2, 4ull * lp.L2, 0, 1);
    lp.tw1 = dev + off[0];
    lp.tw2 = dev + off[1];
    lp.fs_hi = dev + off[2];
    lp.fs_lo = dev + off[3];
    lp.rl_hi = dev + off[4];
    lp.rl_lo = dev + off[5];
    lp.twb = with_plain ? dev + off[6] : nullptr;
    lp.ptw1 = dev + off[7];
    lp.ptw2 = dev + off[8];
    lp.hf_hi = dev + off[9];
    lp.hf_lo = dev + off[10];
    lp.hq = dev + off[11];
}

std::string make_length_plan(uint32_t n, LengthPlan& lp, cudaStream_t stream, int fast1, int fast2) {
    std::string e = choose_length_plan(n, lp, fast1, fast2);
    if (!e.empty()) return e;
    size_t off[kPlanTableBlocks + 1];
    const size_t total = length_plan_layout(lp, true, off);
    lp.tables_bytes = total * sizeof(float2);
    if (cudaMalloc(&lp.d_tables, lp.tables_bytes) != cudaSuccess) return "cudaMalloc of twiddle tables failed";
    std::vector<float2> host(total);
    fill_length_plan_tables(lp, true, host.data(), lp.d_tables);
    if (cudaMemcpyAsync(lp.d_tables, host.data(), lp.tables_bytes, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return "upload of twiddle tables failed";
    return "";
}

void free_length_plan(LengthPlan& lp) {
    if (lp.d_tables) cudaFree(lp.d_tables);
    lp.d_tables = nullptr;
}

}  // namespace brp
