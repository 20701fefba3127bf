/* Stand-in declaration for the historical rngmed.h (absent from the reference
 * snapshot); ref_shims.cpp forwards it to the oracle's running median
 * (oracle_rngmed).  TEST INFRASTRUCTURE ONLY. */
#pragma once
int rngmed(const float* data, unsigned int length, unsigned int window, float* medians);
