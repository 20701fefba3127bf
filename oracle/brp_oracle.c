/*
 * CPU oracle for the BRP4 per-template search path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker used by tests/, the smoke entry point and bench.py's
 * cpu_baseline leg.  It is never linked into the product library and the CUDA
 * path never falls back to it.  Each function restates the reference
 * (void-512/boinc-einstein-bpr4-v3d) at the cited file:line.  Compile with
 * -ffp-contract=off (the reference's science library uses the same flag,
 * CMakeLists.txt:14) so every FP32 product and sum rounds separately unless the
 * reference calls fma explicitly.
 *
 * Parity pins: the restatement is checked against the reference's own
 * science.cpp / workload.cpp compiled from its sources (oracle/Makefile,
 * target `ref`) and against golden vectors generated from that build
 * (tests/golden/make_golden.py).  The reference snapshot has no golden vectors
 * of its own.  Harmonic summing restates shaders/harmonic.comp because the
 * historical hs_common.c it was validated against is absent from the snapshot.
 * The chi-square functions stand in for GSL (absent here): parity with GSL is
 * unpinned; the closed form used is exact mathematics for even degrees of
 * freedom.
 */
#include "brp_oracle.h"
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

static __thread char g_error[256];
static int fail(const char* msg) { snprintf(g_error, sizeof g_error, "%s", msg); return 1; }
const char* oracle_last_error(void) { return g_error; }

/* The 65-entry sine/cosine table of Einstein@Home erp_utilities.cpp, as carried
 * by include/brp/lut.hpp:4-5.  Stored as IEEE-754 bit patterns, interleaved
 * (sin, cos), because the resampled indices depend on every bit. */
static const uint32_t k_lut_bits[130] = {
    0x00000000, 0x3f800000, 0x3dc8bd23, 0x3f7ec472, 0x3e47c5ac, 0x3f7b14ba, 0x3e94a03c, 0x3f74fa05,
    0x3ec3ef07, 0x3f6c8366, 0x3ef15af3, 0x3f61c593, 0x3f0e39d6, 0x3f54db38, 0x3f226794, 0x3f45e3fc,
    0x3f3504f7, 0x3f3504f7, 0x3f45e3fc, 0x3f226794, 0x3f54db38, 0x3f0e39d6, 0x3f61c593, 0x3ef15af3,
    0x3f6c8366, 0x3ec3ef07, 0x3f74fa05, 0x3e94a03c, 0x3f7b14ba, 0x3e47c5ac, 0x3f7ec472, 0x3dc8bd23,
    0x3f800000, 0x00000000, 0x3f7ec472, 0xbdc8bd23, 0x3f7b14ba, 0xbe47c5ac, 0x3f74fa05, 0xbe94a03c,
    0x3f6c8366, 0xbec3ef07, 0x3f61c593, 0xbef15af3, 0x3f54db38, 0xbf0e39d6, 0x3f45e3fc, 0xbf226794,
    0x3f3504f7, 0xbf3504f7, 0x3f226794, 0xbf45e3fc, 0x3f0e39d6, 0xbf54db38, 0x3ef15af3, 0xbf61c593,
    0x3ec3ef07, 0xbf6c8366, 0x3e94a03c, 0xbf74fa05, 0x3e47c5ef, 0xbf7b14ba, 0x3dc8bd23, 0xbf7ec472,
    0x00000000, 0xbf800000, 0xbdc8bd23, 0xbf7ec472, 0xbe47c5ac, 0xbf7b14ba, 0xbe94a01b, 0xbf74fa05,
    0xbec3ef07, 0xbf6c8366, 0xbef15af3, 0xbf61c593, 0xbf0e39d6, 0xbf54db38, 0xbf226794, 0xbf45e40d,
    0xbf3504f7, 0xbf3504f7, 0xbf45e3fc, 0xbf226794, 0xbf54db27, 0xbf0e39d6, 0xbf61c593, 0xbef15af3,
    0xbf6c8366, 0xbec3ef28, 0xbf74fa05, 0xbe94a03c, 0xbf7b14ba, 0xbe47c5ac, 0xbf7ec472, 0xbdc8bd23,
    0xbf800000, 0x00000000, 0xbf7ec472, 0x3dc8bd23, 0xbf7b14ba, 0x3e47c5ac, 0xbf74fa05, 0x3e94a03c,
    0xbf6c8366, 0x3ec3ef07, 0xbf61c593, 0x3ef15af3, 0xbf54db38, 0x3f0e39d6, 0xbf45e40d, 0x3f226794,
    0xbf3504f7, 0x3f3504f7, 0xbf2267a5, 0x3f45e3fc, 0xbf0e39d6, 0x3f54db38, 0xbef15af3, 0x3f61c593,
    0xbec3ef28, 0x3f6c8356, 0xbe94a03c, 0x3f74fa05, 0xbe47c5ef, 0x3f7b14ba, 0xbdc8bd23, 0x3f7ec472,
    0x80000000, 0x3f800000};

static float lut_sin_at(int i) { float f; memcpy(&f, &k_lut_bits[2 * i], 4); return f; }
static float lut_cos_at(int i) { float f; memcpy(&f, &k_lut_bits[2 * i + 1], 4); return f; }

/* science.cpp:20-28 (non-FMA LUT sine). */
float oracle_lut_sin(float x) {
    float dummy;
    float xt = modff((1.0f / 6.283185f) * x, &dummy);
    if (xt < 0) xt += 1;
    int i = (int)(xt * 64.0f + 0.5f);
    float d = 6.283185f * (xt - (1.0f / 64) * i);
    float d2 = d;
    d2 *= 0.5f * d;
    return lut_sin_at(i) + d * lut_cos_at(i) - d2 * lut_sin_at(i);
}

/* science.cpp:29-35 (FMA LUT sine used when Params.flags has bit 2). */
float oracle_fused_sin(float phase) {
    float whole;
    float xt = modff((1.0f / 6.283185f) * phase, &whole);
    if (xt < 0) xt += 1;
    int i = (int)fmaf(xt, 64.0f, 0.5f);
    float d = 6.283185f * fmaf(-(float)i, 1.0f / 64, xt);
    float d2 = (0.5f * d) * d;
    return fmaf(-d2, lut_sin_at(i), fmaf(d, lut_cos_at(i), lut_sin_at(i)));
}

/* science.cpp:36-40. */
float oracle_sample_offset(uint32_t i, const oracle_params* p) {
    float t = (float)i * p->dt;
    if (p->flags & 2) return fmaf(p->tau * oracle_fused_sin(fmaf(p->omega, t, p->psi)), p->step_inv, -p->s0);
    return p->tau * oracle_lut_sin(p->omega * t + p->psi) * p->step_inv - p->s0;
}

/* science.cpp:41-45. */
int oracle_resampling_steps(oracle_params* p) {
    p->steps = p->unpadded - 1;
    while (p->steps && (float)p->steps - oracle_sample_offset(p->steps, p) >= (float)(p->unpadded - 1)) --p->steps;
    if (!p->steps) return fail("template produces empty series");
    return 0;
}

static int single_bit(uint32_t x) { return x && !(x & (x - 1)); }
static uint32_t ctz32(uint32_t x) { uint32_t c = 0; while (!(x & 1u)) { x >>= 1; ++c; } return c; }

/* science.cpp:46-65. */
int oracle_parameters(uint32_t n, uint32_t unpadded, float tau, float period, float psi, float dt,
                      oracle_params* out) {
    uint32_t radix = single_bit(n) ? 1 : ((n % 3 == 0 && single_bit(n / 3)) ? 3 : 0);
    if (!radix || n < 64 || n > 3 * (1u << 22) || unpadded < 32 || unpadded > n || dt <= 0 || period <= 0 ||
        tau < 0 || !isfinite(tau + period + psi + dt))
        return fail("invalid observation/template");
    oracle_params p;
    memset(&p, 0, sizeof p);
    p.n = n; p.unpadded = unpadded; p.fft_n = n; p.fft_radix = radix; p.fft_base = n / radix;
    p.logn = ctz32(p.fft_base); p.tau = tau;
    p.omega = (float)(2.0 * 3.14159265358979323846 / (double)period);
    p.psi = psi; p.dt = dt; p.step_inv = 1.0f / dt;
    /* The historical main computes S0 with the double sine (science.cpp:54-55). */
    p.s0 = (float)((double)tau * sin((double)psi) * (double)p.step_inv);
    if (!isfinite(p.omega) || !isfinite(p.step_inv) || !isfinite(p.s0) || !isfinite(p.tau * p.step_inv) ||
        !isfinite((float)unpadded * p.dt) || !isfinite(p.omega * ((float)unpadded * p.dt) + p.psi))
        return fail("template exceeds finite FP32 arithmetic domain");
    if (oracle_resampling_steps(&p)) return 1;
    p.harmonic = n / 2; p.fundamental = n / 2; p.window = 8;
    static const float thresholds[5] = {20, 30, 45, 70, 110};
    memcpy(p.threshold, thresholds, sizeof thresholds);
    p.capacity = 65536;
    *out = p;
    return 0;
}

/* science.cpp:75-85.  The +0.5 is added in double and the sum truncates toward
 * zero (int conversion), exactly as the reference's CPU loop does. */
int oracle_resample(const float* input, size_t input_len, const oracle_params* p, float* out, int32_t* index) {
    if (input_len != p->unpadded) return fail("input length mismatch");
    float sum = 0;
    for (uint32_t i = 0; i < p->steps; ++i) {
        int j = (int)((double)((float)i - oracle_sample_offset(i, p)) + 0.5);
        if (j < 0 || (uint32_t)j >= p->unpadded) return fail("resample index outside observation");
        if (index) index[i] = j;
        sum += out[i] = input[j];
    }
    float mean = sum / (float)p->steps;
    for (uint32_t i = p->steps; i < p->n; ++i) out[i] = mean;
    return 0;
}

float oracle_exact_mean(const float* x, uint32_t steps) {
    double s = 0;
    for (uint32_t i = 0; i < steps; ++i) s += x[i];
    return (float)(s / (double)steps);
}

/* science.cpp:114-118. */
void oracle_power_from_fft(const double* re, const double* im, uint32_t n, float* power) {
    power[0] = 0;
    double scale = (double)(1.0f / (float)n);
    for (uint32_t i = 1; i < n / 2; ++i) {
        double r = re[i], m = im[i];
        power[i] = (float)(scale * (r * r + m * m));
    }
}

/* Dyadic sums in the historical order of shaders/hs_sum.glsl:2-9 (identical to
 * the sum_at order of shaders/harmonic.comp:5-13).  s[0..3] = 2,4,8,16 harmonics. */
static void dyadic_sums(const float* P, uint32_t i, float s[4]) {
    float t = P[i];
    t += P[(i * 8 + 8) >> 4]; s[0] = t;
    t += P[(i * 12 + 8) >> 4] + P[(i * 4 + 8) >> 4]; s[1] = t;
    t += P[(i * 14 + 8) >> 4] + P[(i * 10 + 8) >> 4] + P[(i * 6 + 8) >> 4] + P[(i * 2 + 8) >> 4]; s[2] = t;
    t += P[(i * 15 + 8) >> 4] + P[(i * 13 + 8) >> 4] + P[(i * 11 + 8) >> 4] + P[(i * 9 + 8) >> 4] +
         P[(i * 7 + 8) >> 4] + P[(i * 5 + 8) >> 4] + P[(i * 3 + 8) >> 4] + P[(i + 8) >> 4];
    s[3] = t;
}

/* shaders/harmonic.comp:14-30: for level h (width w = 2^h) and fundamental bin j the
 * trial bins are i in [max(window, j*w - w/2), min(harmonic, j*w + w/2)); the stored
 * value is the maximum dyadic sum when it exceeds threshold[h], otherwise the sum at
 * the first trial bin, otherwise 0 when the range is empty.  Level 0 is the power. */
int oracle_harmonic(const float* P, size_t power_len, const oracle_params* p, float* summed) {
    if (power_len < p->harmonic || power_len < p->fundamental) return fail("power length mismatch");
    for (uint32_t j = 0; j < p->fundamental; ++j) summed[j] = P[j];
    for (int h = 1; h <= 4; ++h) {
        int64_t w = 1 << h;
        for (uint32_t j = 0; j < p->fundamental; ++j) {
            int64_t begin = (int64_t)j * w - w / 2, end = (int64_t)j * w + w / 2;
            if (begin < (int64_t)p->window) begin = p->window;
            if (end > (int64_t)p->harmonic) end = p->harmonic;
            float value = 0;
            if (begin < end) {
                float s[4];
                dyadic_sums(P, (uint32_t)begin, s);
                float first = s[h - 1], best = first;
                for (int64_t i = begin + 1; i < end; ++i) {
                    dyadic_sums(P, (uint32_t)i, s);
                    if (best < s[h - 1]) best = s[h - 1];
                }
                value = best > p->threshold[h] ? best : first;
            }
            summed[(size_t)h * p->fundamental + j] = value;
        }
    }
    return 0;
}

/* science.cpp:106-112: candidates come out ordered by (level, bin). */
size_t oracle_select(const float* summed, const oracle_params* p, oracle_candidate* out, size_t cap) {
    size_t count = 0;
    for (uint32_t h = 0; h < 5; ++h)
        for (uint32_t j = p->window; j < p->fundamental; ++j) {
            float x = summed[(size_t)h * p->fundamental + j];
            if (x > p->threshold[h]) {
                if (count < cap) { out[count].bin = j; out[count].level = h; out[count].power = x; out[count].reserved = 0; }
                ++count;
            }
        }
    return count;
}

/* Chi-square upper tail for nu = 2k: Q = exp(-x/2) * sum_{i<k} (x/2)^i / i!.
 * Stands in for gsl_cdf_chisq_Q (workload.cpp:146); only even nu occur there. */
double oracle_chisq_Q(double x, double nu) {
    if (!(x >= 0) || nu < 2 || fmod(nu, 2.0) != 0) return NAN;
    double y = 0.5 * x;
    int k = (int)(nu / 2);
    if (y <= 600) {
        double term = 1, sum = 1;
        for (int i = 1; i < k; ++i) { term *= y / i; sum += term; }
        return exp(-y) * sum;
    }
    double ly = log(y), m = (k - 1) * ly - lgamma((double)k), acc = 0;
    for (int i = 0; i < k; ++i) acc += exp(i * ly - lgamma((double)i + 1) - m);
    return exp(-y + m + log(acc));
}

/* Inverse of oracle_chisq_Q in x, to full double precision by safeguarded
 * Newton iteration on log Q.  Stands in for gsl_cdf_chisq_Qinv (workload.cpp:122). */
double oracle_chisq_Qinv(double q, double nu) {
    if (!(q > 0 && q < 1) || nu < 2 || fmod(nu, 2.0) != 0) return NAN;
    double lo = 0, hi = nu + 10;
    while (oracle_chisq_Q(hi, nu) > q) { lo = hi; hi *= 2; }
    double x = 0.5 * (lo + hi), lq = log(q);
    int k = (int)(nu / 2);
    for (int it = 0; it < 200; ++it) {
        double Q = oracle_chisq_Q(x, nu);
        if (Q > q) lo = x; else hi = x;
        /* d log Q / dx = -pdf / Q, pdf = (x/2)^(k-1) e^(-x/2) / (2 (k-1)!). */
        double lpdf = (k - 1) * log(0.5 * x) - 0.5 * x - log(2.0) - lgamma((double)k);
        double next = x + (log(Q) - lq) / exp(lpdf - log(Q));
        if (!(next > lo && next < hi)) next = 0.5 * (lo + hi);
        if (fabs(next - x) <= 1e-16 * x || hi - lo <= 4e-16 * x) { x = next; break; }
        x = next;
    }
    return x;
}

/* workload.cpp:108-125. */
int oracle_search_parameters(uint32_t n, uint32_t samples, double sample_us, double period, double tau,
                             double psi, double f0, double false_alarm, uint32_t window, oracle_params* out) {
    if (!isfinite(f0 + false_alarm) || f0 <= 0 || false_alarm <= 0 || false_alarm >= 1 || !window)
        return fail("invalid search parameters");
    oracle_params p;
    if (oracle_parameters(n, samples, (float)tau, (float)period, (float)psi, (float)(sample_us * 1e-6), &p)) return 1;
    p.flags = 2 | 4;
    p.s0 = (p.tau * sinf(p.psi)) * p.step_inv;
    if (oracle_resampling_steps(&p)) return 1;
    double seconds = n * sample_us * 1e-6;
    p.window = (uint32_t)(window * 0.5 + 0.5);
    if (p.window >= p.n / 2 + 1) return fail("search window exceeds spectrum");
    double limit = p.n / 2 + 1 - p.window;
    double f = f0 * seconds + 0.5, hf = 16 * f0 * seconds + 0.5;
    p.fundamental = (uint32_t)(limit < f ? limit : f);
    p.harmonic = (uint32_t)(limit < hf ? limit : hf);
    float probability = (float)(1.0 - pow(1.0 - false_alarm, 1.0 / (p.n / 2 + 1)));
    if (!(probability > 0 && probability < 1)) return fail("false-alarm probability outside representable domain");
    for (uint32_t h = 0; h < 5; ++h) p.threshold[h] = (float)(0.5 * oracle_chisq_Qinv(probability, 2.0 * (1u << h)));
    if (p.fundamental <= p.window) return fail("empty frequency search");
    *out = p;
    return 0;
}

void oracle_toplist_init(oracle_toplist* t) { memset(t, 0, sizeof *t); }

/* workload.cpp:126. */
void oracle_toplist_thresholds(const oracle_toplist* t, oracle_params* p) {
    for (uint32_t h = 0; h < 5; ++h) {
        float row = (float)t->rows[(h + 1) * 100 - 1].power;
        if (p->threshold[h] < row) p->threshold[h] = row;
    }
}

/* workload.cpp:127-128 comparators, used with the C library's qsort exactly as the reference does. */
static int by_power(const void* x, const void* y) {
    const oracle_bank_candidate *a = x, *b = y;
    return a->power < b->power ? 1 : (a->power > b->power ? -1 : 0);
}
static int by_significance(const void* x, const void* y) {
    const oracle_bank_candidate *a = x, *b = y;
    return a->significance < b->significance ? 1 : (a->significance > b->significance ? -1 : 0);
}

/* workload.cpp:129-141. */
int oracle_toplist_retain(oracle_toplist* t, const oracle_candidate* cands, size_t count, double period,
                          double tau, double psi, const oracle_params* p) {
    for (size_t k = 0; k < count; ++k) {
        oracle_candidate c = cands[k];
        if (c.level >= 5 || c.bin < p->window || c.bin >= p->fundamental || !isfinite(c.power))
            return fail("invalid compact candidate");
        uint32_t first = c.level * 100, last = first + 99;
        if (c.power <= p->threshold[c.level] || c.power <= t->rows[last].power) continue;
        int place = (int)last;
        for (uint32_t i = first; i <= last; ++i)
            if (t->rows[i].bin == c.bin) { place = t->rows[i].power < c.power ? (int)i : -1; break; }
        if (place >= (int)first) {
            oracle_bank_candidate r;
            r.power = c.power; r.period = (float)period; r.tau = (float)tau; r.psi = (float)psi;
            r.significance = 0; r.harmonics = 1u << c.level; r.bin = c.bin;
            t->rows[place] = r;
            qsort(t->rows + first, 100, sizeof(oracle_bank_candidate), by_power);
        }
    }
    return 0;
}

/* workload.cpp:142-159. */
size_t oracle_toplist_final(const oracle_toplist* t, oracle_bank_candidate* out) {
    oracle_bank_candidate copy[500];
    memcpy(copy, t->rows, sizeof copy);
    for (int i = 0; i < 500; ++i) {
        oracle_bank_candidate* c = &copy[i];
        if (!c->harmonics) { c->significance = -10; continue; }
        double probability = oracle_chisq_Q(2 * c->power, 2.0 * c->harmonics);
        c->significance = probability > 0 ? -log10(probability) : 320;
        c->power /= (double)(float)sqrtf((float)c->harmonics);
    }
    qsort(copy, 500, sizeof(oracle_bank_candidate), by_significance);
    size_t count = 0;
    while (count < 100 && copy[0].significance > 0) {
        out[count++] = copy[0];
        uint32_t bin = copy[0].bin;
        for (int i = 0; i < 500; ++i) if (copy[i].bin == bin) copy[i].significance = -10;
        qsort(copy, 500, sizeof(oracle_bank_candidate), by_significance);
    }
    return count;
}

/* ---- FP64 reference DFT ---------------------------------------------------
 * Iterative radix-2 decimation-in-time FFT in double precision with twiddles
 * evaluated directly by cos/sin (no recurrences); lengths 3*2^k add one radix-3
 * combination of three interleaved 2^k transforms.  Only used as the FP64
 * oracle of the power spectrum. */
static void fft2_inplace(double* re, double* im, uint32_t m, const double* cr, const double* ci, uint32_t stride) {
    /* m a power of two; cr/ci hold exp(-2 pi i k / (m*stride)) at index k*stride... for k < m/2. */
    for (uint32_t i = 1, j = 0; i < m; ++i) {
        uint32_t bit = m >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) { double t = re[i]; re[i] = re[j]; re[j] = t; t = im[i]; im[i] = im[j]; im[j] = t; }
    }
    for (uint32_t len = 2; len <= m; len <<= 1) {
        uint32_t half = len >> 1, step = (m / len) * stride;
        for (uint32_t s = 0; s < m; s += len)
            for (uint32_t k = 0; k < half; ++k) {
                double wr = cr[k * step], wi = ci[k * step];
                uint32_t a = s + k, b = a + half;
                double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
                re[b] = re[a] - xr; im[b] = im[a] - xi;
                re[a] += xr; im[a] += xi;
            }
    }
}

int oracle_rfft64(const float* x, uint32_t n, double* out_re, double* out_im) {
    uint32_t radix = single_bit(n) ? 1 : ((n % 3 == 0 && single_bit(n / 3)) ? 3 : 0);
    if (!radix || n < 2) return fail("unsupported FFT length");
    uint32_t m = n / radix;
    double* re = malloc(sizeof(double) * n);
    double* im = malloc(sizeof(double) * n);
    double* cr = malloc(sizeof(double) * (n / 2 + 1));
    double* ci = malloc(sizeof(double) * (n / 2 + 1));
    if (!re || !im || !cr || !ci) { free(re); free(im); free(cr); free(ci); return fail("allocation failed"); }
    for (uint32_t k = 0; k <= n / 2; ++k) {
        double a = -2.0 * 3.14159265358979323846 * (double)k / (double)n;
        cr[k] = cos(a); ci[k] = sin(a);
    }
    /* Split into radix interleaved sub-series, transform each (twiddle stride = radix). */
    for (uint32_t r = 0; r < radix; ++r)
        for (uint32_t i = 0; i < m; ++i) { re[r * m + i] = x[i * radix + r]; im[r * m + i] = 0; }
    for (uint32_t r = 0; r < radix; ++r) fft2_inplace(re + r * m, im + r * m, m, cr, ci, radix);
    for (uint32_t k = 0; k <= n / 2; ++k) {
        double sr = 0, si = 0;
        for (uint32_t r = 0; r < radix; ++r) {
            uint32_t q = k % m;
            uint64_t e = ((uint64_t)k * r) % n;
            double wr, wi;
            if (e <= n / 2) { wr = cr[e]; wi = ci[e]; } else { wr = cr[n - e]; wi = -ci[n - e]; }
            double ar = re[r * m + q], ai = im[r * m + q];
            sr += ar * wr - ai * wi; si += ar * wi + ai * wr;
        }
        out_re[k] = sr; out_im[k] = si;
    }
    free(re); free(im); free(cr); free(ci);
    return 0;
}

/* ---------------------------------------------------------------- whitening */
/* In-place unnormalised complex DFT of length n = 2^k or 3*2^k in FP64:
 * X_k = sum_j x_j exp(-+2 pi i jk / n) (minus for forward, plus for inverse). */
int oracle_cfft64(double* re, double* im, uint32_t n, int inverse) {
    uint32_t radix = single_bit(n) ? 1 : ((n % 3 == 0 && single_bit(n / 3)) ? 3 : 0);
    if (!radix || n < 2) return fail("unsupported FFT length");
    uint32_t m = n / radix;
    double* cr = malloc(sizeof(double) * n);
    double* ci = malloc(sizeof(double) * n);
    double* tr = malloc(sizeof(double) * n);
    double* ti = malloc(sizeof(double) * n);
    if (!cr || !ci || !tr || !ti) { free(cr); free(ci); free(tr); free(ti); return fail("allocation failed"); }
    for (uint32_t k = 0; k < n; ++k) {
        double a = -2.0 * 3.14159265358979323846 * (double)k / (double)n;
        cr[k] = cos(a); ci[k] = sin(a);
    }
    if (inverse) for (uint32_t j = 0; j < n; ++j) im[j] = -im[j];
    for (uint32_t r = 0; r < radix; ++r)
        for (uint32_t i = 0; i < m; ++i) { tr[r * m + i] = re[i * radix + r]; ti[r * m + i] = im[i * radix + r]; }
    for (uint32_t r = 0; r < radix; ++r) fft2_inplace(tr + r * m, ti + r * m, m, cr, ci, radix);
    for (uint32_t k = 0; k < n; ++k) {
        double sr = 0, si = 0;
        for (uint32_t r = 0; r < radix; ++r) {
            uint32_t q = k % m;
            uint64_t e = ((uint64_t)k * r) % n;
            double ar = tr[r * m + q], ai = ti[r * m + q];
            sr += ar * cr[e] - ai * ci[e]; si += ar * ci[e] + ai * cr[e];
        }
        re[k] = sr; im[k] = si;
    }
    if (inverse) for (uint32_t j = 0; j < n; ++j) im[j] = -im[j];
    free(cr); free(ci); free(tr); free(ti);
    return 0;
}

/* FFTW-style c2r: x_j = sum over all n bins of the Hermitian extension of
 * X[0..n/2], imaginary parts of X_0 and X_{n/2} ignored; unnormalised. */
int oracle_c2r64(const float* x_re, const float* x_im, uint32_t n, double* out) {
    double* re = malloc(sizeof(double) * n);
    double* im = malloc(sizeof(double) * n);
    if (!re || !im) { free(re); free(im); return fail("allocation failed"); }
    for (uint32_t k = 0; k <= n / 2; ++k) {
        re[k] = x_re[k];
        im[k] = (k == 0 || 2 * k == n) ? 0.0 : x_im[k];
        if (k && k < n - k) { re[n - k] = x_re[k]; im[n - k] = -(double)x_im[k]; }
    }
    int st = oracle_cfft64(re, im, n, 1);
    if (!st) for (uint32_t j = 0; j < n; ++j) out[j] = re[j];
    free(re); free(im);
    return st;
}

/* Running median: medians[i] = median of data[i .. i + window), i <= length -
 * window; for an even window the mean of the two middle values, 0.5f * (a + b).
 * The window's sorted copy is updated by one removal and one insertion per step. */
int oracle_rngmed(const float* data, uint32_t length, uint32_t window, float* medians) {
    if (!window || window > length) return fail("invalid running-median window");
    float* w = malloc(sizeof(float) * window);
    if (!w) return fail("allocation failed");
    for (uint32_t i = 0; i < window; ++i) {  /* insertion sort of the first window */
        uint32_t j = i;
        while (j > 0 && w[j - 1] > data[i]) { w[j] = w[j - 1]; --j; }
        w[j] = data[i];
    }
    for (uint32_t i = 0;; ++i) {
        medians[i] = (window & 1) ? w[window / 2] : 0.5f * (w[window / 2 - 1] + w[window / 2]);
        if (i + window >= length) break;
        float out = data[i], in = data[i + window];
        uint32_t j = 0;
        while (j < window && !(w[j] == out || (w[j] != w[j] && out != out))) ++j; /* the leaving value */
        if (j == window) { free(w); return fail("running median lost a value"); }
        for (; j + 1 < window; ++j) w[j] = w[j + 1];
        j = window - 1;
        while (j > 0 && w[j - 1] > in) { w[j] = w[j - 1]; --j; }
        w[j] = in;
    }
    free(w);
    return 0;
}

void oracle_taus2_seed(oracle_taus2* r, uint32_t seed) {
    if (!seed) seed = 1;
    r->s1 = 69069u * seed; if (r->s1 < 2) r->s1 += 2;
    r->s2 = 69069u * r->s1; if (r->s2 < 8) r->s2 += 8;
    r->s3 = 69069u * r->s2; if (r->s3 < 16) r->s3 += 16;
    for (int i = 0; i < 6; ++i) oracle_taus2_get(r);
}

uint32_t oracle_taus2_get(oracle_taus2* r) {
    r->s1 = ((r->s1 & 4294967294u) << 12) ^ (((r->s1 << 13) ^ r->s1) >> 19);
    r->s2 = ((r->s2 & 4294967288u) << 4) ^ (((r->s2 << 2) ^ r->s2) >> 25);
    r->s3 = ((r->s3 & 4294967280u) << 17) ^ (((r->s3 << 3) ^ r->s3) >> 11);
    return r->s1 ^ r->s2 ^ r->s3;
}

static double taus2_uniform(oracle_taus2* r) { return oracle_taus2_get(r) / 4294967296.0; }

/* Marsaglia-Tsang ziggurat tables: 128 layers of area V, base layer plus tail
 * beyond R, a 24-bit integer uniform. */
static double zig_k[128], zig_w[128], zig_f[128];
static int zig_ready = 0;
static const double ZIG_R = 3.442619855899, ZIG_V = 9.91256303526217e-3, ZIG_M = 16777216.0;
static void zig_init(void) {
    double dn = ZIG_R, tn = ZIG_R, q = ZIG_V / exp(-0.5 * dn * dn);
    zig_k[0] = dn / q * ZIG_M; zig_k[1] = 0;
    zig_w[0] = q / ZIG_M; zig_w[127] = dn / ZIG_M;
    zig_f[0] = 1.0; zig_f[127] = exp(-0.5 * dn * dn);
    for (int i = 126; i >= 1; --i) {
        dn = sqrt(-2.0 * log(ZIG_V / dn + exp(-0.5 * dn * dn)));
        zig_k[i + 1] = dn / tn * ZIG_M;
        tn = dn;
        zig_f[i] = exp(-0.5 * dn * dn);
        zig_w[i] = dn / ZIG_M;
    }
    zig_ready = 1;
}

double oracle_gaussian_ziggurat(oracle_taus2* r, double sigma) {
    if (!zig_ready) zig_init();
    for (;;) {
        uint32_t bits = oracle_taus2_get(r);
        int i = (int)(bits & 0x7Fu);
        double sign = (bits & 0x80u) ? 1.0 : -1.0;
        uint32_t j = bits >> 8;
        double x = j * zig_w[i];
        if (j < zig_k[i]) return sign * sigma * x;
        if (i == 0) {
            double y;
            do {
                x = -log(1.0 - taus2_uniform(r)) / ZIG_R;
                y = -log(1.0 - taus2_uniform(r));
            } while (y + y < x * x);
            return sign * sigma * (ZIG_R + x);
        }
        if (zig_f[i] + taus2_uniform(r) * (zig_f[i - 1] - zig_f[i]) < exp(-0.5 * x * x)) return sign * sigma * x;
    }
}

float oracle_dd_sample(const uint8_t* bytes, uint32_t i, int packed, double scale) {
    /* src/workload.cpp:52-54 */
    if (packed) return (float)((double)((i & 1) ? (bytes[i / 2] & 15) : (bytes[i / 2] >> 4)) / scale);
    return (float)((double)(int8_t)bytes[i] / scale);
}

/* src/workload.cpp:58-95. */
int oracle_preprocess(const float* decoded, uint32_t samples, uint32_t n, double sample_us, double padding,
                      uint32_t window, const double* zap_lower, const double* zap_upper, uint32_t zap_count,
                      float* preprocessed) {
    if (!window || (window & 1) || window > n / 2) return fail("unsupported whitening window");
    uint32_t size = n / 2 + 1;
    float* time = calloc(n, sizeof(float));
    double* xr = malloc(sizeof(double) * size);
    double* xi = malloc(sizeof(double) * size);
    float* fr = malloc(sizeof(float) * size);
    float* fi = malloc(sizeof(float) * size);
    float* power = malloc(sizeof(float) * size);
    float* median = malloc(sizeof(float) * (size - window + 1));
    double* back = malloc(sizeof(double) * n);
    int st = 0;
    if (!time || !xr || !xi || !fr || !fi || !power || !median || !back) { st = fail("allocation failed"); goto done; }
    memcpy(time, decoded, sizeof(float) * samples);
    if ((st = oracle_rfft64(time, n, xr, xi))) goto done;
    for (uint32_t k = 0; k < size; ++k) { fr[k] = (float)xr[k]; fi[k] = (float)xi[k]; }
    power[0] = 0;
    for (uint32_t k = 1; k < size; ++k) { double re = fr[k], im = fi[k]; power[k] = (float)(re * re + im * im); }
    if ((st = oracle_rngmed(power, size, window, median))) goto done;
    for (uint32_t i = 0; i < size - window + 1; ++i) {
        if (!(median[i] > 0) || !isfinite(median[i])) { st = fail("invalid whitening median"); goto done; }
        float factor = (float)sqrt(0.693147180559945309417232121458 / median[i]);
        fr[i + window / 2] *= factor;
        fi[i + window / 2] *= factor;
    }
    {
        uint32_t seed;
        memcpy(&seed, &decoded[0], 4);
        oracle_taus2 rng;
        oracle_taus2_seed(&rng, seed);
        double seconds = n * sample_us * 1e-6;
        for (uint32_t z = 0; z < zap_count; ++z) {
            double lower = zap_lower[z], upper = zap_upper[z];
            if (!isfinite(lower + upper) || lower < 0 || upper < lower) { st = fail("invalid zap range"); goto done; }
            double first = lower * seconds + 0.5, last = upper * seconds + 0.5;
            if (last >= size) { st = fail("zap exceeds Nyquist"); goto done; }
            for (uint32_t i = (uint32_t)first; i <= (uint32_t)last; ++i) {
                double sigma = sqrt(2.0) / 2 * sqrt(padding);
                float re = (float)oracle_gaussian_ziggurat(&rng, sigma), im = (float)oracle_gaussian_ziggurat(&rng, sigma);
                fr[i] = re; fi[i] = im;
            }
        }
    }
    for (uint32_t i = 0; i < window / 2; ++i) fr[i] = fi[i] = fr[size - i - 1] = fi[size - i - 1] = 0;
    if ((st = oracle_c2r64(fr, fi, n, back))) goto done;
    {
        float factor = (float)(1.0 / sqrtf((float)n));
        for (uint32_t i = 0; i < samples; ++i) preprocessed[i] = (float)back[i] * factor;
    }
done:
    free(time); free(xr); free(xi); free(fr); free(fi); free(power); free(median); free(back);
    return st;
}
