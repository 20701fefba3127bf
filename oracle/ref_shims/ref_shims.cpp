// Link-time stand-ins that let the reference's own CPU sources
// (src/science.cpp, src/workload.cpp) compile and run here, where FFTW, GSL and
// the historical Einstein@Home sources are absent.  TEST INFRASTRUCTURE ONLY:
// built into oracle/_ref as the checker, never into the product library.
//
//  * fftwf_plan_dft_r2c_1d / fftwf_execute / fftwf_destroy_plan: an FP64 DFT
//    (oracle_rfft64) rounded to float.  This makes brp::fft_reference the
//    "FP64 FFT oracle"; parity with FFTW itself is unpinned.
//  * harmonic_summing: the restatement of shaders/harmonic.comp (the historical
//    hs_common.c is absent; the reference validated the shader against it,
//    src/main.cpp:63-64).
//  * gsl_cdf_chisq_Q / Qinv: closed form for even degrees of freedom.
//  * rngmed / gsl_rng_*: whitening is outside the search path; these report failure.
#include "hs_common.h"
#include "rngmed.h"
#include "gsl/gsl_cdf.h"
#include "gsl/gsl_randist.h"
#include "../brp_oracle.h"
#include <cstdlib>
#include <vector>

extern "C" {
struct fftwf_plan_s { int n; float* in; float (*out)[2]; bool forward; };
typedef fftwf_plan_s* fftwf_plan;

fftwf_plan fftwf_plan_dft_r2c_1d(int n, float* in, float (*out)[2], unsigned) {
    if (n < 2) return nullptr;
    return new fftwf_plan_s{n, in, out, true};
}
fftwf_plan fftwf_plan_dft_c2r_1d(int, float (*)[2], float*, unsigned) { return nullptr; }
void fftwf_execute(fftwf_plan p) {
    if (!p || !p->forward) return;
    std::vector<double> re(p->n / 2 + 1), im(p->n / 2 + 1);
    if (oracle_rfft64(p->in, uint32_t(p->n), re.data(), im.data())) std::abort();
    for (int k = 0; k <= p->n / 2; ++k) { p->out[k][0] = float(re[k]); p->out[k][1] = float(im[k]); }
}
void fftwf_destroy_plan(fftwf_plan p) { delete p; }

double gsl_cdf_chisq_Q(double x, double nu) { return oracle_chisq_Q(x, nu); }
double gsl_cdf_chisq_Qinv(double q, double nu) { return oracle_chisq_Qinv(q, nu); }
const gsl_rng_type* gsl_rng_taus2 = nullptr;
gsl_rng* gsl_rng_alloc(const gsl_rng_type*) { return nullptr; }
void gsl_rng_free(gsl_rng*) {}
void gsl_rng_set(const gsl_rng*, unsigned long) {}
double gsl_ran_gaussian_ziggurat(const gsl_rng*, double) { return 0; }
}

int rngmed(const float*, unsigned int, unsigned int, float*) { return 1; }

// Signature follows the call at src/science.cpp:103.  sums[1..4] receive the
// harmonic levels; sums[0] and the dirty-page flags are not written.
int harmonic_summing(float** sums, int32_t**, const float* power, uint32_t window, uint32_t fundamental,
                     uint32_t harmonic, const float* thresholds) {
    oracle_params p{};
    p.window = window; p.fundamental = fundamental; p.harmonic = harmonic;
    for (int h = 0; h < 5; ++h) p.threshold[h] = thresholds[h];
    std::vector<float> summed(size_t(5) * fundamental);
    size_t len = harmonic > fundamental ? harmonic : fundamental;
    if (oracle_harmonic(power, len, &p, summed.data())) return 1;
    for (int h = 1; h < 5; ++h)
        for (uint32_t j = 0; j < fundamental; ++j) sums[h][j] = summed[size_t(h) * fundamental + j];
    return 0;
}
