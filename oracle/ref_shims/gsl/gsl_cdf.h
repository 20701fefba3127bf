/* Stand-in GSL declarations (GSL is not installed here).  TEST INFRASTRUCTURE ONLY. */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
double gsl_cdf_chisq_Q(double x, double nu);
double gsl_cdf_chisq_Qinv(double q, double nu);
#ifdef __cplusplus
}
#endif
