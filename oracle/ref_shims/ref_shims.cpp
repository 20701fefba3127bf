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
//  * fftwf_plan_dft_c2r_1d: the FP64 inverse (oracle_c2r64) rounded to float.
//  * rngmed: the running median restated by the oracle (oracle_rngmed; the
//    historical rngmed.c is absent).
//  * gsl_rng_taus2 / gsl_ran_gaussian_ziggurat: the oracle's restatements of
//    the published algorithms (GSL is absent).  With these the reference's own
//    brp::preprocess runs here; parity with FFTW, rngmed.c and GSL is unpinned.
#include "hs_common.h"
#include "rngmed.h"
#include "gsl/gsl_cdf.h"
#include "gsl/gsl_randist.h"
#include "../brp_oracle.h"
#include <cstdlib>
#include <vector>

extern "C" {
struct fftwf_plan_s { int n; float* real; float (*cplx)[2]; bool forward; };
typedef fftwf_plan_s* fftwf_plan;

fftwf_plan fftwf_plan_dft_r2c_1d(int n, float* in, float (*out)[2], unsigned) {
    if (n < 2) return nullptr;
    return new fftwf_plan_s{n, in, out, true};
}
fftwf_plan fftwf_plan_dft_c2r_1d(int n, float (*in)[2], float* out, unsigned) {
    if (n < 2) return nullptr;
    return new fftwf_plan_s{n, out, in, false};
}
void fftwf_execute(fftwf_plan p) {
    if (!p) return;
    const uint32_t n = uint32_t(p->n);
    if (p->forward) {
        std::vector<double> re(n / 2 + 1), im(n / 2 + 1);
        if (oracle_rfft64(p->real, n, re.data(), im.data())) std::abort();
        for (uint32_t k = 0; k <= n / 2; ++k) { p->cplx[k][0] = float(re[k]); p->cplx[k][1] = float(im[k]); }
    } else {
        std::vector<float> re(n / 2 + 1), im(n / 2 + 1);
        for (uint32_t k = 0; k <= n / 2; ++k) { re[k] = p->cplx[k][0]; im[k] = p->cplx[k][1]; }
        std::vector<double> out(n);
        if (oracle_c2r64(re.data(), im.data(), n, out.data())) std::abort();
        for (uint32_t j = 0; j < n; ++j) p->real[j] = float(out[j]);
    }
}
void fftwf_destroy_plan(fftwf_plan p) { delete p; }

double gsl_cdf_chisq_Q(double x, double nu) { return oracle_chisq_Q(x, nu); }
double gsl_cdf_chisq_Qinv(double q, double nu) { return oracle_chisq_Qinv(q, nu); }
struct gsl_rng_type { int unused; };
struct gsl_rng { oracle_taus2 state; };
static const gsl_rng_type k_taus2{0};
const gsl_rng_type* gsl_rng_taus2 = &k_taus2;
gsl_rng* gsl_rng_alloc(const gsl_rng_type*) { return new gsl_rng{}; }
void gsl_rng_free(gsl_rng* r) { delete r; }
void gsl_rng_set(const gsl_rng* r, unsigned long seed) {
    oracle_taus2_seed(&const_cast<gsl_rng*>(r)->state, uint32_t(seed));
}
double gsl_ran_gaussian_ziggurat(const gsl_rng* r, double sigma) {
    return oracle_gaussian_ziggurat(&const_cast<gsl_rng*>(r)->state, sigma);
}
}

int rngmed(const float* data, unsigned int length, unsigned int window, float* medians) {
    return oracle_rngmed(data, length, window, medians);
}

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
