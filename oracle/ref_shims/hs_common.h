/* Stand-in declaration for the historical Einstein@Home hs_common.h, which the
 * reference snapshot does not contain (CMakeLists.txt:8-11).  Declares the one
 * function src/science.cpp:103 and the reference adapter call.  TEST
 * INFRASTRUCTURE ONLY: used to compile the reference's own CPU sources into
 * oracle/_ref. */
#pragma once
#include <stdint.h>
int harmonic_summing(float** sums, int32_t** dirty, const float* power, uint32_t window,
                     uint32_t fundamental, uint32_t harmonic, const float* thresholds);
