/*
 * brp_cuda.h -- C ABI of the B200 (sm_100a) backend for the BRP4 per-template
 * search path: orbital resampling, mean padding, packed real FFT, normalized
 * power spectrum, 1/2/4/8/16-harmonic summing, candidate compaction.
 *
 * The entry points replace the Vulkan backend src/vulkan.cpp of
 * void-512/boinc-einstein-bpr4-v3d behind its unchanged C++ interface
 * include/brp/vulkan.hpp (class brp::GPU).  The package's
 * csrc/brp_gpu_adapter.cpp implements brp::GPU on top of these functions, so
 * the reference's brp_bench (src/main.cpp) and brp_workunit
 * (src/workunit_main.cpp) link against this library unmodified.
 *
 * Conventions: every function returns an int status (BRP_OK, or a BRP_E* code),
 * never throws, never exits; brp_cuda_last_error() gives the message of the
 * last failure of a context (or of the calling thread for a NULL context).
 * Plain pointers and sizes only; all host buffers are caller owned.
 */
#ifndef BRP_CUDA_H
#define BRP_CUDA_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define BRP_CUDA_ABI_VERSION 1

/* Status codes.  BRP_E_RUNTIME maps to the reference's std::runtime_error
 * (exit code 1 of src/main.cpp:118); BRP_E_RESULT is a device error word set by
 * a kernel (resample index outside the observation, candidate overflow;
 * src/vulkan.cpp:333); BRP_E_TIMEOUT a host wait that reached its deadline. */
enum { BRP_OK = 0, BRP_E_RUNTIME = 1, BRP_E_RESULT = 2, BRP_E_TIMEOUT = 3, BRP_E_ARGUMENT = 4 };

/* Per-template device error word bits (shaders/resample.comp:18,
 * shaders/harmonic.comp:34).  BRP_STATUS_WAIT_TIMEOUT has no reference
 * counterpart: a kernel gave up a bounded wait for its own asynchronous work
 * (the bulk copies that stage the harmonic kernel's power values, the matrix
 * multiplies of the tensor-core pass-1 form, configurations 111-114). */
enum { BRP_STATUS_OVERFLOW = 1u, BRP_STATUS_RESAMPLE_OOB = 2u, BRP_STATUS_WAIT_TIMEOUT = 4u };

/* Byte-identical to brp::Params (include/brp/science.hpp:8-17, 108 bytes). */
typedef struct brp_params {
    uint32_t n, unpadded, steps, logn;
    float tau, omega, psi, dt, step_inv, s0;
    uint32_t fundamental, harmonic, window, stage;
    float threshold[5];
    uint32_t capacity;
    uint32_t fft_n, fft_base, fft_radix, flags, twiddle3, twiddle_real;
    uint32_t result_slot;
} brp_params;

/* Params.flags bits the backend honours.  Bit 2 selects the FMA resampling
 * arithmetic of src/science.cpp:29-38 (bit 4, the V3D FMA emulation of
 * shaders/common.glsl:43-58, is the same correctly rounded FMA here).
 * BRP_FLAG_INDEX_FP64 is an extension: the time index t + tau*sin(Omega*t+psi)
 * in FP64 with a libm-accurate sine instead of the FP32 LUT (it does not match
 * the reference's indices bit for bit and reports its own mismatch count). */
enum { BRP_FLAG_PACKED = 1u, BRP_FLAG_FMA = 2u, BRP_FLAG_FMA_EMULATED = 4u, BRP_FLAG_INDEX_FP64 = 256u };

/* brp::Candidate (include/brp/science.hpp:18). */
typedef struct brp_candidate { uint32_t bin, level; float power; uint32_t reserved; } brp_candidate;

/* The constructor options of brp::GPU (include/brp/vulkan.hpp:13;
 * src/vulkan.cpp:278-284).  The reference's algorithm switches (stockham,
 * radix4, radix8, ...) are validated with the reference's rules and recorded;
 * the results do not depend on them here. */
enum {
    BRP_OPT_SOFTWARE = 1u, BRP_OPT_STOCKHAM = 2u, BRP_OPT_RADIX4 = 4u, BRP_OPT_PACKED = 8u,
    BRP_OPT_SCATTER = 16u, BRP_OPT_RADIX8 = 32u, BRP_OPT_FUSED_POWER = 64u, BRP_OPT_RADIX8_STORE = 128u,
    /* Extension: run the step-by-step per-template pipeline (one kernel per
     * stage, global-memory FFT passes) instead of the fused pipeline. */
    BRP_OPT_PLAIN = 1u << 16
};
typedef struct brp_options {
    uint32_t workgroup; /* 1..256, as src/vulkan.cpp:121 */
    uint32_t tile;      /* 0 or a power of two in 64..4096 (src/vulkan.cpp:121) */
    uint32_t batch;     /* 1..64 templates per run (src/vulkan.cpp:121) */
    uint32_t flags;     /* BRP_OPT_* */
    int32_t device;     /* CUDA device ordinal; -1 = the calling thread's current device */
    /* reserved[0], reserved[1]: compiled pass-1 / pass-2 configuration ids
     * (brp_cuda_fast_configs); 0 = default, UINT32_MAX = generic kernels. */
    uint32_t reserved[3];
} brp_options;

/* brp::Timings (include/brp/vulkan.hpp:6).  stage_ms: resample+pad, FFT,
 * power, harmonic+candidates, summed over the templates of the run. */
typedef struct brp_timings { double wall_ms, cpu_ms, submit_ms; double stage_ms[4]; } brp_timings;

typedef struct brp_ctx brp_ctx;

/* Replaces brp::GPU::GPU / GPU::Impl::init (src/vulkan.cpp:109-214, :278-284).
 * Copies input[unpadded] to the device. */
int brp_cuda_create(const brp_params* params, const float* input, uint32_t unpadded, const brp_options* options,
                    brp_ctx** out);
/* Replaces GPU::~GPU (src/vulkan.cpp:38-56). */
void brp_cuda_destroy(brp_ctx* ctx);
/* Replaces GPU::set_templates / set_template (src/vulkan.cpp:286-295, :270-276):
 * 1..batch templates with the constructor's n, unpadded, fundamental, harmonic,
 * capacity and arithmetic flags. */
int brp_cuda_set_templates(brp_ctx* ctx, const brp_params* templates, uint32_t count);
/* Replaces GPU::run (src/vulkan.cpp:296-318): runs every template set, blocks
 * until done.  template_stage_ms (optional) receives count*4 doubles. */
int brp_cuda_run(brp_ctx* ctx, brp_timings* timings, double* template_stage_ms);
/* Replaces GPU::snapshot (src/vulkan.cpp:319-328) for the last template of the
 * last run.  Any pointer may be NULL.  resampled: n floats (steps values then
 * the mean); fft: 2*(n/2+1) floats; power: n/2 floats; summed: 5*fundamental. */
int brp_cuda_snapshot(brp_ctx* ctx, float* resampled, float* fft, float* power, float* summed);
/* Replaces GPU::candidates (src/vulkan.cpp:329-337): the candidates of one
 * result slot sorted by (level, bin); slot UINT32_MAX = the last template.
 * *count receives the full count even when it exceeds cap.  Returns
 * BRP_E_RESULT when the slot's error word is set (overflow or resample OOB). */
int brp_cuda_candidates(brp_ctx* ctx, uint32_t slot, brp_candidate* out, uint32_t cap, uint32_t* count);
/* Replaces GPU::device_info / allocated_bytes / profile_counters
 * (src/vulkan.cpp:338-346).  Counters are a JSON string of per-stage event times. */
int brp_cuda_device_info(brp_ctx* ctx, char* buffer, size_t length);
uint64_t brp_cuda_allocated_bytes(const brp_ctx* ctx);
int brp_cuda_profile_counters(brp_ctx* ctx, char* buffer, size_t length);
const char* brp_cuda_last_error(const brp_ctx* ctx);
/* Replaces the unbounded fence wait of GPU::run (src/vulkan.cpp:306,
 * vkWaitForFences with UINT64_MAX).  host_seconds (0..86400, default 300) is
 * the deadline of brp_cuda_run's wait: past it the run returns BRP_E_TIMEOUT
 * while the GPU finishes the work, and the next call on the context first
 * waits (again bounded) for that work before it reuses the buffers.
 * device_polls (default 4194304) bounds a kernel's first wait for its own
 * asynchronous work (the harmonic kernel's staging copies, the tensor-core
 * pass-1 MMAs); on expiry the template's status gets BRP_STATUS_WAIT_TIMEOUT,
 * the kernel drains that work with the full bound and the run reports
 * BRP_E_RESULT.  device_polls = 0 gives up at once (tests use it to exercise
 * that path). */
int brp_cuda_set_wait_limits(brp_ctx* ctx, uint32_t device_polls, double host_seconds);

/* ---- Bank extension: a whole orbital bank over series of different lengths,
 * run as one captured CUDA graph (the batched form of src/workunit_main.cpp:77-93).
 * No reference counterpart beyond that loop; candidates per template are those
 * GPU::candidates would return. ---- */
typedef struct brp_bank brp_bank;
/* series_count series; series s has unpadded[s] samples padded to n[s]
 * (a power of two or 3*2^k, 64..3*2^22).  max_templates bounds one run;
 * capacity is the candidate capacity of each template's result slot. */
int brp_cuda_bank_create(uint32_t series_count, const uint32_t* n, const uint32_t* unpadded, uint32_t max_templates,
                         uint32_t capacity, int32_t device, brp_bank** out);
void brp_cuda_bank_destroy(brp_bank* bank);
/* Copies one series (unpadded[s] floats, host memory) to the device,
 * asynchronously on the bank's copy stream; the next submitted run waits for
 * it.  From page-locked memory the copy overlaps the device's work, and the
 * host buffer must then stay unchanged until the next run has completed; from
 * pageable memory the call returns once the data is staged. */
int brp_cuda_bank_set_series(brp_bank* bank, uint32_t series, const float* input);
/* Runs count templates; template t searches series series_of[t] with
 * templates[t] (whose n/unpadded must equal that series').  Writes the
 * candidates of all templates back to back into out (sorted by (level, bin)
 * within a template), counts[t] per template and status[t] (BRP_STATUS_* bits).
 * out_cap bounds the total; BRP_E_RESULT if a template's status is non-zero or
 * out_cap is too small.  Blocks until done. */
int brp_cuda_bank_run(brp_bank* bank, const brp_params* templates, const uint32_t* series_of, uint32_t count,
                      brp_candidate* out, uint64_t out_cap, uint32_t* counts, uint32_t* status);
/* brp_cuda_bank_run in two halves, so a caller can overlap its own work with
 * the device's (the reference's bank loop, src/workunit_main.cpp:77-93, waits
 * on every batch): brp_cuda_bank_submit enqueues the run (templates are copied
 * at the call) and returns; brp_cuda_bank_wait blocks until it is done and
 * returns its results as brp_cuda_bank_run does.  One run at a time: a second
 * submit, configure, toplist filter, profile, launch or wait-limit change
 * before the wait is refused (BRP_E_ARGUMENT).  brp_cuda_bank_set_series is
 * allowed meanwhile: each series has two device buffers, and an upload while
 * a run is in flight goes to the buffer that run does not read (the next
 * submit reads it), so the next step's series can cross PCIe while this step
 * runs. */
int brp_cuda_bank_submit(brp_bank* bank, const brp_params* templates, const uint32_t* series_of, uint32_t count);
int brp_cuda_bank_wait(brp_bank* bank, brp_candidate* out, uint64_t out_cap, uint32_t* counts, uint32_t* status);
/* Selects the kernels of one length class: compiled pass-1 / pass-2
 * configuration ids (0 = default, -1 = generic kernels), templates per
 * launch and independent launch chains in the graph (1 or 2; 0 = keep).
 * Used by the autotuner; the next run re-captures.  Buffers that a larger
 * group replaces are freed. */
int brp_cuda_bank_configure(brp_bank* bank, uint32_t n, int32_t pass1, int32_t pass2, uint32_t group,
                            uint32_t chains);
/* Device pre-filter for the bank-wide toplist (src/workload.cpp:126-159, rows
 * per harmonic level, one row per bin).  With rows > 0 brp_cuda_bank_run returns, per template, only
 * the candidates whose power reaches the rows-th highest per-bin maximum power
 * of their level among all candidates of the templates of the same series, and
 * counts[t] is that kept count (overflow is still decided on the full count).
 * Folding the kept candidates of a series into a toplist of `rows` rows per
 * level in bank order gives the same final rows as folding all of them.
 * rows = 0 (the default) returns every candidate.  The next run re-captures. */
int brp_cuda_bank_set_toplist_filter(brp_bank* bank, uint32_t rows);
/* Lists the compiled configurations: ids, sequence length L (pass 1: column
 * length L1, pass 2: row length L2) and kind (1 = pass 1, 2 = pass 2,
 * 3 = pass 1 whose first radix-16 stage runs on the tensor cores as split
 * BF16 DFT products; kind 3 is never a default and is selected by id).
 * Returns the total count; writes at most cap entries. */
int brp_cuda_fast_configs(int32_t* ids, uint32_t* lengths, uint32_t* kinds, uint32_t cap);
/* Autotuner for C callers.  The reference fixes its kernel variant by
 * command-line options (workgroup, tile, radix and store variants of
 * src/main.cpp and src/workunit_main.cpp:70); here, for every length class of
 * the templates, each compiled pass-1 / pass-2 pair covering n (CUDA-core
 * forms), each group size (groups[group_count], NULL: 16, 32, 64, 128) and 1 or
 * 2 launch chains is timed over `reps` replays of the bank's captured graph of
 * these templates with L2 flushed before each (CUDA events on the bank's
 * stream); the bank is left configured with the fastest.  cache_path (NULL:
 * none) is a JSON plan file shared with the Python tuner, keyed by device,
 * n and template count: with BRP_TUNE_USE_CACHE an entry there is used without
 * timing; new results are merged into it.  Every result also becomes the
 * default plan of that length for brp::GPU contexts and banks created later in
 * the process.  results[cap] receives one entry per length, *found their
 * number.  Allocates an L2 flush buffer (512 MiB) while it runs. */
typedef struct brp_tune_result {
    double ms;  /* device time of one replay of the bank with this plan */
    uint32_t n;
    int32_t pass1, pass2;
    uint32_t group, chains, tried, cached, reserved;
} brp_tune_result;
enum { BRP_TUNE_USE_CACHE = 1u };
int brp_cuda_bank_autotune(brp_bank* bank, const brp_params* templates, const uint32_t* series_of, uint32_t count,
                           uint32_t reps, const uint32_t* groups, uint32_t group_count, const char* cache_path,
                           uint32_t flags, brp_tune_result* results, uint32_t cap, uint32_t* found);
/* Merges a plan file (written by brp_cuda_bank_autotune or the Python tuner)
 * into the plans that default choices consult: for a length with a plan for
 * the current device, brp_cuda_create, brp_cuda_bank_create and the static
 * search take its pass pair (banks also its group and chains) instead of the
 * built-in pairs.  NULL: $BRP_PLAN_CACHE, else ~/.cache/brp_b200/plans.json
 * (which the library also reads by itself before its first default choice);
 * "" forgets every plan (the built-in pairs again) and reads no file later. */
int brp_cuda_load_plan_cache(const char* path);
/* Message of the calling thread's last failed autotune / plan-cache call. */
const char* brp_cuda_autotune_error(void);
/* Device-only replay of the last brp_cuda_bank_run's graph (no host copies,
 * no wait): the throughput kernel time is measured around this by the caller
 * with events on brp_cuda_bank_stream().  brp_cuda_bank_configure and
 * brp_cuda_bank_set_toplist_filter drop the graph: until the next run this
 * returns BRP_E_ARGUMENT. */
int brp_cuda_bank_launch(brp_bank* bank);
void* brp_cuda_bank_stream(brp_bank* bank);
/* Replays the last run's kernels eagerly with an event pair around each launch
 * and sums the device time per kernel kind: kernel_ms[0] pass 1 (resample +
 * column FFTs), [1] pass 2 (row FFTs + real spectrum + power), [2] harmonic
 * summing + compaction, [3] candidate gather.  launches (optional) gets the
 * launch count per kind. */
int brp_cuda_bank_profile(brp_bank* bank, double* kernel_ms, uint32_t* launches);
/* Kernels launched by one replay (for launch accounting). */
uint32_t brp_cuda_bank_kernels_per_run(const brp_bank* bank);
const char* brp_cuda_bank_last_error(const brp_bank* bank);
/* brp_cuda_set_wait_limits for a bank (the same replacement of
 * src/vulkan.cpp:306): host_seconds bounds brp_cuda_bank_run's and
 * brp_cuda_bank_profile's waits, device_polls is a launch argument of the
 * captured kernels (a change re-captures at the next run). */
int brp_cuda_bank_set_wait_limits(brp_bank* bank, uint32_t device_polls, double host_seconds);
/* No counterpart in the reference; a test aid for the error paths.  The
 * `after`-th device allocation from now on (1 = the next one) made by a context
 * or a bank reports failure without calling cudaMalloc; 0 turns it off.
 * Process-wide. */
void brp_cuda_debug_fail_allocation(uint32_t after);

/* ---- Search without device allocation ----
 * No counterpart in the reference.  For callers that may not allocate device
 * memory while they run (a plugin limited to the buffers its host hands it, a
 * process whose device memory belongs to another framework's pool, a
 * real-time loop that must not block in the allocator): one template through
 * the fused search (resampling, packed real FFT, power spectrum, harmonic
 * summing, candidate compaction) with all working memory in a static device
 * array inside this library (about 4.2 MiB, held by every GPU that loads the
 * library until the process exits).  It calls no cudaMalloc or cudaFree.
 *   input      device, params->unpadded floats (the series), 4-byte aligned
 *   power      device, n/2 floats (P[k] = |X_k|^2 / n, P[0] = 0), 16-byte aligned
 *   candidates device, capacity entries, 16-byte aligned; *count (device,
 *              4-byte aligned) the number found, which may exceed capacity;
 *              *status (device, 4-byte aligned) BRP_STATUS_* bits
 *   stream     cudaStream_t (NULL: legacy default stream)
 * Series lengths 8192..1048576 (2^k or 3*2^k); longer ones, and misaligned
 * buffers, are rejected with BRP_E_ARGUMENT before any device work.  The call
 * is asynchronous on `stream`; results are valid once the stream has
 * completed.  The first call on a device (and the first call with a new series
 * length) does set-up -- the scratch array's device address, kernel
 * attributes, the twiddle tables copied into the array -- so that first call
 * should come before any stream capture.  Every call shares the one array,
 * which keeps the last call's contents: calls that overlap on the GPU (other
 * streams, other threads) race and must be serialised by the caller.  The
 * set-up belongs to the device's context: do not call this again on a device
 * after cudaDeviceReset in the same process.
 * brp_cuda_search_static_error() gives the calling thread's last message. */
int brp_cuda_search_static(const brp_params* params, const float* input, float* power, brp_candidate* candidates,
                           uint32_t capacity, uint32_t* count, uint32_t* status, void* stream);
const char* brp_cuda_search_static_error(void);

/* ---- Host helpers (the reference's host code around the path) ---- */
/* src/science.cpp:46-65 (brp::parameters). */
int brp_host_parameters(uint32_t n, uint32_t unpadded, float tau, float period, float psi, float dt,
                        brp_params* out);
/* src/science.cpp:41-45 (brp::resampling_steps). */
int brp_host_resampling_steps(brp_params* p);
/* src/workload.cpp:108-125 (brp::search_parameters); n, samples and sample_us
 * describe the observation. */
int brp_host_search_parameters(uint32_t n, uint32_t samples, double sample_us, double period, double tau,
                               double psi, double f0, double false_alarm, uint32_t window, brp_params* out);

/* src/workload.cpp:126-159 (brp::Toplist). */
typedef struct brp_bank_candidate {
    double power, period, tau, psi, significance;
    uint32_t harmonics, bin;
} brp_bank_candidate;
typedef struct brp_toplist brp_toplist;
brp_toplist* brp_toplist_create(void);
void brp_toplist_destroy(brp_toplist* t);
void brp_toplist_thresholds(const brp_toplist* t, brp_params* p);
int brp_toplist_retain(brp_toplist* t, const brp_candidate* candidates, uint32_t count, double period, double tau,
                       double psi, const brp_params* p);
/* Writes up to 100 final candidates; returns how many. */
uint32_t brp_toplist_final(const brp_toplist* t, brp_bank_candidate* out);
/* The bank loop after the search (src/workunit_main.cpp:77-124): for each of
 * count templates in bank order, raise its thresholds to the toplist's current
 * rows (thresholds) and retain its candidates (retain).  candidates: the
 * templates' lists back to back, counts[t] each; orbits: 3 doubles (period,
 * tau, psi) per template. */
int brp_toplist_fold(brp_toplist* t, const brp_params* templates, const double* orbits,
                     const brp_candidate* candidates, const uint32_t* counts, uint32_t count);

/* ---- Whitening and RFI zapping of an observation (brp::preprocess,
 * src/workload.cpp:58-95) on the GPU ----
 * decoded[samples] (host) is zero-padded to n (2^k or 3*2^k, 8192..3*2^22), real
 * FFT, power, running median over `window` bins (even, <= n/2 and <= 4096 on
 * the device), scaling of bin i + window/2 by sqrt(ln 2 / median_i), zapped
 * bins (ranges zap_lower[z]..zap_upper[z] in the reference's units, x the
 * observation length n * sample_us) replaced by Gaussian noise of sigma
 * sqrt(padding / 2) drawn as the reference draws it (taus2 seeded with the bits
 * of decoded[0], ziggurat), the first and last window/2 bins cleared, inverse
 * real FFT and scaling by 1/sqrt(n); preprocessed[samples] (host) receives the
 * result.  Errors follow the reference: BRP_E_ARGUMENT for an unsupported
 * window, an invalid zap range or a zap beyond Nyquist, BRP_E_RESULT for an
 * invalid median; brp_cuda_preprocess_error() gives the message. */
int brp_cuda_preprocess(const float* decoded, uint32_t samples, uint32_t n, double sample_us, double padding,
                        uint32_t window, const double* zap_lower, const double* zap_upper, uint32_t zap_count,
                        float* preprocessed, int32_t device);
/* As brp_cuda_preprocess from the DD sample bytes of brp::load_observation
 * (src/workload.cpp:48-56): int8 samples, or (packed != 0) two 4-bit samples
 * per byte, high nibble first, each float(double(b) / scale); decoded on the
 * device (decoded[samples], host, optional, receives the decoded series). */
int brp_cuda_preprocess_dd(const uint8_t* bytes, uint32_t samples, int32_t packed, double scale, uint32_t n,
                           double sample_us, double padding, uint32_t window, const double* zap_lower,
                           const double* zap_upper, uint32_t zap_count, float* decoded, float* preprocessed,
                           int32_t device);
const char* brp_cuda_preprocess_error(void);
/* The zap list of src/workload.cpp:77-88: whitespace-separated (lower, upper)
 * pairs; invalid ranges and trailing garbage are errors.  Writes at most cap
 * pairs, *count = all pairs. */
int brp_host_read_zap(const char* path, double* lower, double* upper, uint32_t cap, uint32_t* count);
/* The zap noise of src/workload.cpp:73-87 for `ranges` zap ranges: per zapped
 * bin (in the reference's order) bins[k] and values[2k], values[2k+1] (real,
 * imaginary); at most cap written, *count = all. */
int brp_host_zap_noise(uint32_t seed, uint32_t n, double sample_us, double padding, const double* lower,
                       const double* upper, uint32_t ranges, uint32_t* bins, float* values, uint32_t cap,
                       uint32_t* count);
/* Message of the last failed brp_host_* call of this thread. */
const char* brp_host_error(void);

#ifdef __cplusplus
}
#endif
#endif
