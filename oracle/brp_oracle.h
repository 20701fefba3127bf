/*
 * CPU oracle for the BRP4 per-template search path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the smoke
 * entry point and bench.py's cpu_baseline leg call it to produce the expected
 * results of the search path on the CPU.  Nothing in the product path links
 * it, and the CUDA extension never falls back to it.
 *
 * Every function restates the reference's own CPU code (void-512/
 * boinc-einstein-bpr4-v3d, src/science.cpp and src/workload.cpp) or, where the
 * reference's CPU code calls sources absent from its snapshot (the historical
 * hs_common.c harmonic summing), the reference's GPU shader that was validated
 * against it (shaders/harmonic.comp, shaders/hs_sum.glsl).  Each function names
 * the file:line it follows.  It is compiled with -ffp-contract=off, like the
 * reference's science library (CMakeLists.txt:14), so FP32 operations round
 * exactly where the reference's do.
 */
#ifndef BRP_ORACLE_H
#define BRP_ORACLE_H
#include <stdint.h>
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Byte-identical to brp::Params (include/brp/science.hpp:8-17, 108 bytes). */
typedef struct oracle_params {
    uint32_t n, unpadded, steps, logn;
    float tau, omega, psi, dt, step_inv, s0;
    uint32_t fundamental, harmonic, window, stage;
    float threshold[5];
    uint32_t capacity;
    uint32_t fft_n, fft_base, fft_radix, flags, twiddle3, twiddle_real;
    uint32_t result_slot;
} oracle_params;

/* brp::Candidate (include/brp/science.hpp:18). */
typedef struct oracle_candidate { uint32_t bin, level; float power; uint32_t reserved; } oracle_candidate;

/* brp::BankCandidate (include/brp/workload.hpp:14). */
typedef struct oracle_bank_candidate {
    double power, period, tau, psi, significance;
    uint32_t harmonics, bin;
} oracle_bank_candidate;

/* Status codes: 0 ok, 1 invalid argument / runtime error (the reference throws). */
float oracle_lut_sin(float x);                          /* science.cpp:20-28 */
float oracle_fused_sin(float x);                        /* science.cpp:29-35 */
float oracle_sample_offset(uint32_t i, const oracle_params* p); /* science.cpp:36-40 */
int oracle_resampling_steps(oracle_params* p);          /* science.cpp:41-45 */
int oracle_parameters(uint32_t n, uint32_t unpadded, float tau, float period, float psi,
                      float dt, oracle_params* out);    /* science.cpp:46-65 */
/* science.cpp:75-85.  out has p->n floats; index (optional, p->steps ints) receives j(i). */
int oracle_resample(const float* input, size_t input_len, const oracle_params* p,
                    float* out, int32_t* index);
/* Mean of out[0..steps) accumulated in FP64 and rounded once (the CUDA path's padding value). */
float oracle_exact_mean(const float* resampled, uint32_t steps);
/* science.cpp:114-118: power[i] = float(double(1.0f/n)*(re^2+im^2)), power[0] = 0. */
void oracle_power_from_fft(const double* fft_re, const double* fft_im, uint32_t n, float* power);
/* shaders/harmonic.comp:5-30 with shaders/hs_sum.glsl:2-9 ordering.  summed has 5*fundamental floats. */
int oracle_harmonic(const float* power, size_t power_len, const oracle_params* p, float* summed);
/* science.cpp:106-112.  Returns the count; writes at most cap candidates. */
size_t oracle_select(const float* summed, const oracle_params* p, oracle_candidate* out, size_t cap);

/* Chi-square tail for even degrees of freedom and its inverse (GSL stand-ins, see oracle.c). */
double oracle_chisq_Q(double x, double nu);
double oracle_chisq_Qinv(double q, double nu);
/* workload.cpp:108-125.  n, samples and sample_us describe the Observation. */
int oracle_search_parameters(uint32_t n, uint32_t samples, double sample_us, double period,
                             double tau, double psi, double f0, double false_alarm,
                             uint32_t window, oracle_params* out);

/* workload.cpp:126-159: the bank-wide toplist (5 levels x 100 rows). */
typedef struct oracle_toplist { oracle_bank_candidate rows[500]; } oracle_toplist;
void oracle_toplist_init(oracle_toplist* t);
void oracle_toplist_thresholds(const oracle_toplist* t, oracle_params* p);
int oracle_toplist_retain(oracle_toplist* t, const oracle_candidate* c, size_t count,
                          double period, double tau, double psi, const oracle_params* p);
size_t oracle_toplist_final(const oracle_toplist* t, oracle_bank_candidate* out /* 100 */);

/* FP64 reference DFT of a real float series of length n (2^k or 3*2^k); writes n/2+1 bins. */
int oracle_rfft64(const float* x, uint32_t n, double* re, double* im);

/* ---- whitening (src/workload.cpp:58-95) and DD decoding (:48-56) ----
 * Parity notes: FFTW (FP32 r2c/c2r) is absent, the oracle transforms in FP64
 * (the r2c output rounded to float, as the reference's std::complex<float>
 * spectrum holds it); the historical rngmed.c is absent, oracle_rngmed defines
 * the running median restated here (even window: 0.5f * (a + b) of the two
 * middle values); GSL is absent, its taus2 generator and ziggurat Gaussian are
 * restated from the published algorithms (L'Ecuyer 1996 with the taus2
 * seeding; Marsaglia and Tsang 2000, 128 layers).  Those three are
 * "parity unpinned"; the rest of the whitening is pinned against the
 * reference's own preprocess compiled with these stand-ins (oracle/_ref). */
int oracle_cfft64(double* re, double* im, uint32_t n, int inverse); /* in place, unnormalised */
int oracle_c2r64(const float* x_re, const float* x_im, uint32_t n, double* out); /* sum over all n bins */
int oracle_rngmed(const float* data, uint32_t length, uint32_t window, float* medians);
typedef struct oracle_taus2 { uint32_t s1, s2, s3; } oracle_taus2;
void oracle_taus2_seed(oracle_taus2* r, uint32_t seed);
uint32_t oracle_taus2_get(oracle_taus2* r);
double oracle_gaussian_ziggurat(oracle_taus2* r, double sigma);
float oracle_dd_sample(const uint8_t* bytes, uint32_t i, int packed, double scale); /* workload.cpp:53-54 */
int oracle_preprocess(const float* decoded, uint32_t samples, uint32_t n, double sample_us, double padding,
                      uint32_t window, const double* zap_lower, const double* zap_upper, uint32_t zap_count,
                      float* preprocessed);

const char* oracle_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
