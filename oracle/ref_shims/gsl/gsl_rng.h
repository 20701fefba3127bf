/* Stand-in GSL declarations (GSL is not installed here).  Random numbers are
 * only used by whitening, outside the search path; gsl_rng_alloc returns NULL
 * so that path reports "GSL allocation failed".  TEST INFRASTRUCTURE ONLY. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
typedef struct gsl_rng_type gsl_rng_type;
typedef struct gsl_rng gsl_rng;
extern const gsl_rng_type* gsl_rng_taus2;
gsl_rng* gsl_rng_alloc(const gsl_rng_type* type);
void gsl_rng_free(gsl_rng* r);
void gsl_rng_set(const gsl_rng* r, unsigned long seed);
#ifdef __cplusplus
}
#endif
