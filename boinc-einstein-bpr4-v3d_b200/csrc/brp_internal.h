// Internal interfaces of the CUDA backend: length plans, kernel argument
// blocks and kernel launchers.  Not part of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include "../../include/brp_cuda.h"

namespace brp {

// Twiddles a compiled Stockham pass of radix R keeps per butterfly k in its
// table.  In a product table (pass 2) radix 2, 4 and 8 keep W^{p k} for the
// powers p = 1, 2, 4 below R and the kernels form the other twiddles as
// products of these; otherwise (pass 1; radix 3 and 16 in either) the table
// holds every twiddle p = 1 .. R - 1.
__host__ __device__ constexpr bool pass_twiddle_products(int R, bool prod) {
    return prod && (R == 2 || R == 4 || R == 8);
}
__host__ __device__ constexpr int pass_twiddle_powers(int R, bool prod) {
    return pass_twiddle_products(R, prod) ? (R == 8 ? 3 : R == 4 ? 2 : 1) : R - 1;
}
__host__ __device__ constexpr int pass_twiddle_power(int R, int s, bool prod) {
    return pass_twiddle_products(R, prod) ? 1 << s : s + 1;
}

// Radix plan of one shared-memory FFT (mirrors the device struct in fft_device.cuh).
struct RadixPlanHost {
    int count = 0;
    int radix[6] = {0, 0, 0, 0, 0, 0};
};
RadixPlanHost radix_plan(uint32_t length);

struct FastPass;

// Tables of one FFT length class, all FP64-generated and rounded once to FP32.
//   tw1[L1], tw2[L2]       : W_L^e for the two shared-memory passes
//   fs_hi/fs_lo (split 2^11): W_M^e, e < M (four-step twiddles)
//   rl_hi/rl_lo (split 2^11): W_N^e, e < N (real post-process and padding term)
//   twb[B]                  : W_B^e, B = M or M/3 (global passes of the plain pipeline)
struct LengthPlan {
    uint32_t n = 0, M = 0;     // series length and packed complex length M = n/2
    uint32_t radix = 1, B = 0; // M = radix * B (radix 1 or 3), for the plain pipeline
    bool fused = false;        // fused two-pass pipeline available for this length
    uint32_t L1 = 0, L2 = 0;   // M = L1 * L2; pass 1 transforms columns of L1, pass 2 rows of L2
    uint32_t C = 0;            // pass 1: columns per CTA
    uint32_t R = 0;            // pass 2: row pairs per CTA
    uint32_t maxe = 16;        // elements per thread held during a shared-memory pass
    uint32_t harm_tile = 2048; // harmonic kernel: trial bins per CTA
    RadixPlanHost plan1, plan2, planB;
    const FastPass* fp1 = nullptr;  // compiled pass 1 / pass 2 (nullptr: generic kernels)
    const FastPass* fp2 = nullptr;
    const float2 *ptw1 = nullptr, *ptw2 = nullptr;
    const float2 *hf_hi = nullptr, *hf_lo = nullptr;  // W_{2n}^e (cos, -sin of pi e / n)
    const float2* hq = nullptr;  // W_{4 L2}^e, e < L2: W_{2n}^{L1 e}, the row factor of pass 2's W_{2n}^k
    float2* d_tables = nullptr;
    size_t tables_bytes = 0;
    const float2 *tw1 = nullptr, *tw2 = nullptr, *fs_hi = nullptr, *fs_lo = nullptr, *rl_hi = nullptr,
                 *rl_lo = nullptr, *twb = nullptr;
    uint32_t blocks1() const { return L2 / C; }        // pass-1 CTAs per template
    uint32_t blocks2() const { return L1 / (2 * R); }  // pass-2 CTAs per template
    size_t smem1() const;
    size_t smem2() const;
};
// Chooses the decomposition for length n and uploads its tables.  Returns an
// error message or empty.  fast1/fast2 (optional) force compiled pass
// configurations by id (0: default choice, -1: generic kernels).
std::string make_length_plan(uint32_t n, LengthPlan& plan, cudaStream_t stream, int fast1 = 0, int fast2 = 0);
// The tuned plan of length n for the current device from the plan cache
// (autotune.cu): the entry tuned on the largest bank of that length.
struct CachedPlan { int pass1 = 0, pass2 = 0; uint32_t group = 0, chains = 1; };
bool cached_plan(uint32_t n, CachedPlan& out);
// The parts of make_length_plan: the decomposition and kernel choice (no
// allocation), the table layout (offsets[12], returns the float2 count;
// with_plain adds the table of the step-by-step pipeline) and the table fill
// (host[] laid out by the layout, lp's views pointed at dev).
std::string choose_length_plan(uint32_t n, LengthPlan& plan, int fast1 = 0, int fast2 = 0, bool use_cache = true);
constexpr int kPlanTableBlocks = 12;  // table blocks of a length plan (length_plan_layout)
size_t length_plan_layout(const LengthPlan& lp, bool with_plain, size_t offsets[kPlanTableBlocks + 1]);
void fill_length_plan_tables(LengthPlan& lp, bool with_plain, float2* host, float2* dev);
void free_length_plan(LengthPlan& plan);

constexpr uint32_t kSplitLog2 = 11;

// Device views passed to the fused kernels.  Per-template arrays are indexed
// by blockIdx.y (the template within the launch).
struct FusedArgs;
// A compiled specialisation of pass 1 (L = L1, group = columns per CTA) or
// pass 2 (L = L2, group = row pairs per CTA) with its radix sequence and the
// size of its per-pass twiddle table.
struct FastPass {
    int id = 0;
    uint32_t L = 0, group = 0, threads = 0;
    size_t smem = 0;
    void (*launch)(const FusedArgs&, uint32_t blocks, uint32_t count, cudaStream_t) = nullptr;
    cudaError_t (*attr)() = nullptr;
    RadixPlanHost plan;
    int table = 0;
    int tensor = 0;  // pass 1 only: BF16 parts per operand of the tensor-core first stage (0: CUDA cores)
};
// Compiled pass configurations.  Pass-1 configurations with tensor != 0 (the
// tensor-core form, fused_tc.cu) follow the CUDA-core ones and are chosen only
// by id.
const std::vector<FastPass>& fast_pass1_configs();
void append_pass1_warp_configs(std::vector<FastPass>& v);
void append_pass1_tc_configs(std::vector<FastPass>& v);
const std::vector<FastPass>& fast_pass2_configs();
size_t harmonic_fast_smem();
cudaError_t set_harmonic_fast_attributes();

struct FusedArgs {
    const float* const* inputs;  // per template: series (unpadded floats)
    const brp_params* params;    // per template
    uint32_t n, M, L1, L2, C, R;
    int plan1[7], plan2[7];      // count followed by radices
    const float2 *tw1, *tw2, *fs_hi, *fs_lo, *rl_hi, *rl_lo;
    const float2 *ptw1, *ptw2;  // per-pass twiddle tables of the compiled passes
    const float2 *hf_hi, *hf_lo;  // W_{2n}^e: (cos(pi e/n), -sin(pi e/n)), e <= M
    const float2* hq;             // W_{4 L2}^e = W_{2n}^{L1 e}, e < L2
    float2* work;     // per template: M complex (four-step intermediate)
    size_t work_stride;
    float* power;     // per template: M floats (P[k] = |X_k|^2 / n, P[0] = 0)
    size_t power_stride;
    double* partial;  // per template: blocks1 partial sums of the resampled series
    uint32_t partial_stride;
    float* mean;      // per template: padding value (compiled kernels: pass 1's last CTA; generic: pass 2)
    uint32_t* tickets;  // per template: pass-1 CTAs done (compiled kernels; zero between launches)
    uint32_t* status; // per template: BRP_STATUS_* bits
    uint32_t* counts; // per template: candidate count
    brp_candidate* cands;  // per template: capacity candidates
    uint32_t capacity;
    // Snapshot outputs, written for template `snap` of the launch only (-1: none).
    int snap;
    float* snap_raw;     // resampled series (first steps values)
    float2* snap_fft;    // X[0..M]
    float* snap_summed;  // 5*fundamental
    // Poll bound of a kernel's first wait for its own asynchronous work (the
    // harmonic kernel's staging copies, the tensor-core pass 1's MMAs); on
    // expiry the template's status gets BRP_STATUS_WAIT_TIMEOUT and the kernel
    // drains that work with the full bound before the CTA leaves.
    uint32_t wait_polls;
};
// Default of FusedArgs::wait_polls and of the per-context / per-bank device
// wait limit; default host deadline of a run (seconds).
constexpr uint32_t kDefaultWaitPolls = 1u << 22;
constexpr double kDefaultWaitSeconds = 300.0;

cudaError_t set_fused_attributes(size_t max_dynamic_smem);
void launch_fused_pass1(const FusedArgs& a, const LengthPlan& lp, uint32_t count, cudaStream_t s);
void launch_fused_pass2(const FusedArgs& a, const LengthPlan& lp, uint32_t count, cudaStream_t s);
void launch_fused_harmonic(const FusedArgs& a, const LengthPlan& lp, uint32_t count, uint32_t max_span,
                           cudaStream_t s);
void launch_harmonic_fast(const FusedArgs& a, uint32_t count, uint32_t max_span, cudaStream_t s);
// Fills the FFT description and tables of lp into a.
void fill_fused_args(FusedArgs& a, const LengthPlan& lp);

// Step-by-step pipeline (one template; buffers sized for the length class).
struct PlainArgs {
    const float* input;
    brp_params p;
    const LengthPlan* lp;
    float* raw;       // steps floats
    double* partial;  // ceil(steps/256) partial sums
    float* mean;      // 1 float
    float2* a;        // M complex
    float2* b;        // M complex
    float2* fft;      // M+1 complex (X)
    float* power;     // M floats
    float* summed;    // 5*fundamental floats
    uint32_t* status; // 1 word
    uint32_t* count;  // 1 word
    brp_candidate* cands;
};
// Records the plain pipeline on stream s; ev (optional, 5 events) brackets the 4 stages.
void launch_plain(const PlainArgs& a, cudaStream_t s, cudaEvent_t* ev);
// Its FFT stages: the forward complex FFT of the packed series (returns the
// buffer holding Z, a or b) and the real post-process X_k, k = 0..M (power, if
// given, |X_k|^2 / n for 0 < k < M and 0 at k = 0).
float2* plain_complex_fft(float2* a, float2* b, const LengthPlan& lp, cudaStream_t s);
void launch_plain_realpost(const float2* z, float2* fft, float* power, const LengthPlan& lp, cudaStream_t s);

// Device toplist pre-filter of a bank run (toplist_filter.cu).  Per series s
// the per-bin arrays of level h start at base[s] + h * half[s] (half = n/2).
struct FilterArgs {
    const uint32_t* counts;       // per slot: candidate count (may exceed capacity)
    const brp_candidate* cands;   // per slot: capacity candidates
    uint32_t capacity, count;     // slots
    const uint32_t* slot_series;  // per slot: series index
    uint32_t series, rows;        // series count; toplist rows per level
    const uint64_t* base;         // per series
    const uint32_t* half;         // per series
    uint32_t* maxkey;             // per (series, level, bin): highest power key
    uint32_t* flag;               // per (series, level, bin)
    uint32_t* owners;             // per (series, level): keys of the per-bin maxima
    uint32_t* owner_count;        // per (series, level)
    uint32_t* threshold_key;      // per (series, level): the rows-th largest per-bin maximum
    uint32_t* kept;               // per slot: candidates that pass
};
void launch_toplist_filter(const FilterArgs& f, cudaStream_t s);

#ifdef __CUDACC__
// Order-preserving unsigned image of an FP32 power.
__device__ __forceinline__ uint32_t power_key(float x) {
    const uint32_t b = __float_as_uint(x);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
// Whether candidate x of a slot of series s passes the filter (out-of-range
// candidates pass, so that the host sees and rejects them).
__device__ __forceinline__ bool filter_keep(const FilterArgs& f, uint32_t s, const brp_candidate& x) {
    if (x.level >= 5 || x.bin >= f.half[s]) return true;
    return power_key(x.power) >= f.threshold_key[s * 5 + x.level];
}
#endif

// Candidate compaction of a bank run (plain_kernels.cu): slot k's list goes,
// sorted by (level, bin), to the caller's position rank[k]; lists longer than
// kCompactSortMax are copied unsorted (the host sorts them).  With `filter`
// only the candidates that pass the toplist pre-filter are written.
constexpr uint32_t kCompactSortMax = 16384;
cudaError_t set_bank_compact_attributes(uint32_t capacity);
void launch_bank_compact(const uint32_t* counts, const brp_candidate* cands, uint32_t capacity, uint32_t count,
                         const uint32_t* rank, brp_candidate* out, uint64_t out_cap, uint64_t* offsets,
                         const FilterArgs* filter, cudaStream_t s);

}  // namespace brp
