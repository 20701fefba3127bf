/* Stand-in declaration for the historical rngmed.h (absent from the reference
 * snapshot).  Whitening (src/workload.cpp:58-95) is outside the search path;
 * the stand-in lets workload.cpp compile and reports failure if called.
 * TEST INFRASTRUCTURE ONLY. */
#pragma once
int rngmed(const float* data, unsigned int length, unsigned int window, float* medians);
