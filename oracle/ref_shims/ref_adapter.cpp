// Stand-in for the reference's src/reference_adapter.cpp, whose historical
// sources (demod_binary_resamp_cpu.c, demod_binary_fft_fftw.c, hs_common.c) are
// absent from the snapshot.  TEST INFRASTRUCTURE ONLY: it lets the reference's
// unmodified src/main.cpp (brp_bench) link into oracle/_ref.
//  * historical_resample: the oracle's independent C restatement of the
//    resampler, so src/main.cpp:46 checks science.cpp against it bit for bit.
//  * historical_power: FP64 FFT rounded to float, then the power formula of
//    src/science.cpp:115-118 (src/main.cpp:47 requires equality).
//  * benchmark_cpu: the loop of src/reference_adapter.cpp:30-56 over the
//    reference's own science.cpp functions.
#include "brp/science.hpp"
#include "../brp_oracle.h"
#include <algorithm>
#include <chrono>
#include <cstring>
#include <ctime>
#include <stdexcept>
extern "C" int boinc_resolve_filename(const char*, char*, int) { return -1; }
namespace brp {
std::vector<float> historical_resample(std::span<const float> input, const Params& p) {
    std::vector<float> out(p.n);
    oracle_params q;
    static_assert(sizeof(q) == sizeof(p));
    std::memcpy(&q, &p, sizeof q);
    if (oracle_resample(input.data(), input.size(), &q, out.data(), nullptr))
        throw std::runtime_error(oracle_last_error());
    return out;
}
std::vector<float> historical_power(std::span<const float> resampled, const Params& p) {
    auto fft = fft_reference(resampled);
    std::vector<float> power(p.n / 2);
    for (uint32_t i = 1; i < p.n / 2; ++i) {
        double re = fft[i].real(), im = fft[i].imag();
        power[i] = float(double(1.0f / p.n) * (re * re + im * im));
    }
    return power;
}
CPUStats benchmark_cpu(std::span<const float> input, const Params& p, uint32_t reps) {
    std::vector<double> walls, cpus;
    auto cpu_now = [] { timespec t{}; clock_gettime(CLOCK_PROCESS_CPUTIME_ID, &t); return t.tv_sec * 1000.0 + t.tv_nsec / 1e6; };
    for (uint32_t r = 0; r <= reps; ++r) {
        auto start = std::chrono::steady_clock::now();
        double cpu = cpu_now();
        auto result = reference(input, p);
        if (r) {
            cpus.push_back(cpu_now() - cpu);
            walls.push_back(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count());
        }
    }
    std::sort(walls.begin(), walls.end());
    std::sort(cpus.begin(), cpus.end());
    return {walls[walls.size() / 2], cpus[cpus.size() / 2]};
}
}
