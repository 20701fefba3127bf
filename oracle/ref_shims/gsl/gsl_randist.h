/* Stand-in GSL declarations.  TEST INFRASTRUCTURE ONLY. */
#pragma once
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
double gsl_ran_gaussian_ziggurat(const gsl_rng* r, double sigma);
#ifdef __cplusplus
}
#endif
