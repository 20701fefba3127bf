/* Stand-in GSL declarations (GSL is not installed here).  The generator behind
 * them is the oracle's restatement of taus2 (ref_shims.cpp).  TEST
 * INFRASTRUCTURE ONLY. */
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
