// C entry points over the reference's own CPU code (src/science.cpp,
// src/workload.cpp) compiled into oracle/_ref/libbrp_ref.so.  TEST
// INFRASTRUCTURE ONLY: tests/golden/make_golden.py and the bench's reference
// arm call these through ctypes to run the reference's CPU path.
#include "brp/science.hpp"
#include "brp/workload.hpp"
#include <cstring>
#include <exception>
#include <string>
static thread_local std::string g_error;
template <class F> static int guard(F&& f) {
    try { f(); return 0; } catch (const std::exception& e) { g_error = e.what(); return 1; }
}
extern "C" {
const char* ref_last_error() { return g_error.c_str(); }
float ref_lut_sin(float x) { return brp::lut_sin(x); }
float ref_sample_offset(uint32_t i, const brp::Params* p) { return brp::sample_offset(i, *p); }
int ref_parameters(uint32_t n, uint32_t unpadded, float tau, float period, float psi, float dt, brp::Params* out) {
    return guard([&] { *out = brp::parameters(n, unpadded, tau, period, psi, dt); });
}
int ref_resampling_steps(brp::Params* p) { return guard([&] { brp::resampling_steps(*p); }); }
int ref_resample(const float* input, uint32_t len, const brp::Params* p, float* out) {
    return guard([&] { auto r = brp::resample({input, len}, *p); std::memcpy(out, r.data(), r.size() * 4); });
}
// Full reference pipeline (src/science.cpp:113-120).  Buffers: resampled n,
// fft 2*(n/2+1), power n/2, summed 5*fundamental, candidates up to cap.
int ref_reference(const float* input, uint32_t len, const brp::Params* p, float* resampled, float* fft, float* power,
                  float* summed, brp::Candidate* cands, uint32_t cap, uint32_t* count) {
    return guard([&] {
        auto r = brp::reference({input, len}, *p);
        if (resampled) std::memcpy(resampled, r.resampled.data(), r.resampled.size() * 4);
        if (fft) std::memcpy(fft, r.fft.data(), r.fft.size() * 8);
        if (power) std::memcpy(power, r.power.data(), r.power.size() * 4);
        if (summed) std::memcpy(summed, r.summed.data(), r.summed.size() * 4);
        *count = uint32_t(r.candidates.size());
        std::memcpy(cands, r.candidates.data(), std::min<size_t>(cap, r.candidates.size()) * sizeof(brp::Candidate));
    });
}
int ref_harmonic(const float* power, uint32_t len, const brp::Params* p, float* summed) {
    return guard([&] { auto s = brp::harmonic_reference({power, len}, *p); std::memcpy(summed, s.data(), s.size() * 4); });
}
int ref_search_parameters(uint32_t n, uint32_t samples, double sample_us, double period, double tau, double psi,
                          double f0, double fa, uint32_t window, brp::Params* out) {
    return guard([&] {
        brp::Observation o;
        o.n = n; o.samples = samples; o.sample_us = sample_us;
        *out = brp::search_parameters(o, brp::Orbit{period, tau, psi}, f0, fa, window);
    });
}
void* ref_toplist_new() { return new brp::Toplist(); }
void ref_toplist_free(void* t) { delete static_cast<brp::Toplist*>(t); }
void ref_toplist_thresholds(void* t, brp::Params* p) { static_cast<brp::Toplist*>(t)->thresholds(*p); }
int ref_toplist_retain(void* t, const brp::Candidate* c, uint32_t count, double period, double tau, double psi,
                       const brp::Params* p) {
    return guard([&] { static_cast<brp::Toplist*>(t)->retain({c, count}, brp::Orbit{period, tau, psi}, *p); });
}
uint32_t ref_toplist_final(void* t, brp::BankCandidate* out) {
    auto r = static_cast<brp::Toplist*>(t)->final();
    std::memcpy(out, r.data(), r.size() * sizeof(brp::BankCandidate));
    return uint32_t(r.size());
}
// brp::load_observation (src/workload.cpp:29-57) of a gzip DD file: metadata
// meta[4] = {sample_us, scale, samples, n}, decoded samples up to cap.
int ref_load_observation(const char* path, double padding, double* meta, float* decoded, uint32_t cap) {
    return guard([&] {
        auto o = brp::load_observation(path, padding);
        meta[0] = o.sample_us; meta[1] = o.scale; meta[2] = o.samples; meta[3] = o.n;
        if (decoded) std::memcpy(decoded, o.decoded.data(), std::min<size_t>(cap, o.decoded.size()) * 4);
    });
}
// brp::preprocess (src/workload.cpp:58-95) of a decoded series with a zap-list file.
int ref_preprocess(const float* decoded, uint32_t samples, uint32_t n, double sample_us, double padding,
                   const char* zap_path, uint32_t window, float* out) {
    return guard([&] {
        brp::Observation o;
        o.sample_us = sample_us; o.padding = padding; o.samples = samples; o.n = n;
        o.decoded.assign(decoded, decoded + samples);
        brp::preprocess(o, zap_path, window);
        std::memcpy(out, o.preprocessed.data(), size_t(samples) * 4);
    });
}
}
