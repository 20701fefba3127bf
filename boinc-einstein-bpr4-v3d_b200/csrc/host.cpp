// Host-side code around the search path: template constants, the chi-square
// thresholds and the bank-wide toplist.  These restate the reference's host
// functions (src/science.cpp:41-65, src/workload.cpp:108-159) so that a bank
// search through this library produces the reference's thresholds, candidate
// filtering and final ranking.  Compiled with -ffp-contract=off: the FP32
// expressions round exactly where the reference's do.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include "../../include/brp_cuda.h"
#include "resample_math.h"

namespace {
thread_local std::string g_host_error;
int host_fail(const char* msg) { g_host_error = msg; return BRP_E_ARGUMENT; }
const uint32_t k_lut[130] = BRP_LUT_BITS;
bool single_bit(uint32_t x) { return x && !(x & (x - 1)); }

brp_resample_consts consts_of(const brp_params& p) {
    brp_resample_consts c;
    c.tau = p.tau; c.omega = p.omega; c.psi = p.psi; c.dt = p.dt; c.step_inv = p.step_inv; c.s0 = p.s0;
    c.flags = p.flags;
    return c;
}
}  // namespace

const char* brp_host_last_error() { return g_host_error.c_str(); }
extern "C" const char* brp_host_error(void) { return g_host_error.c_str(); }

extern "C" int brp_host_resampling_steps(brp_params* p) {
    // src/science.cpp:41-45: the largest steps with steps - offset(steps) < unpadded - 1.
    if (!p || p->unpadded < 2) return host_fail("invalid template");
    const brp_resample_consts c = consts_of(*p);
    p->steps = p->unpadded - 1;
    while (p->steps && float(p->steps) - brp_sample_offset(p->steps, c, k_lut) >= float(p->unpadded - 1)) --p->steps;
    if (!p->steps) return host_fail("template produces empty series");
    return BRP_OK;
}

extern "C" int brp_host_parameters(uint32_t n, uint32_t unpadded, float tau, float period, float psi, float dt,
                                   brp_params* out) {
    // src/science.cpp:46-65.
    if (!out) return host_fail("null output");
    uint32_t radix = single_bit(n) ? 1 : ((n % 3 == 0 && single_bit(n / 3)) ? 3 : 0);
    if (!radix || n < 64 || n > 3 * (1u << 22) || unpadded < 32 || unpadded > n || dt <= 0 || period <= 0 || tau < 0 ||
        !std::isfinite(tau + period + psi + dt))
        return host_fail("invalid observation/template");
    brp_params p;
    std::memset(&p, 0, sizeof p);
    p.n = n; p.unpadded = unpadded; p.fft_n = n; p.fft_radix = radix; p.fft_base = n / radix;
    p.logn = uint32_t(__builtin_ctz(p.fft_base));
    p.tau = tau;
    p.omega = float(2.0 * M_PI / double(period));
    p.psi = psi; p.dt = dt; p.step_inv = 1.0f / dt;
    p.s0 = float(double(tau) * std::sin(double(psi)) * double(p.step_inv));
    if (!std::isfinite(p.omega) || !std::isfinite(p.step_inv) || !std::isfinite(p.s0) ||
        !std::isfinite(p.tau * p.step_inv) || !std::isfinite(float(unpadded) * p.dt) ||
        !std::isfinite(p.omega * (float(unpadded) * p.dt) + p.psi))
        return host_fail("template exceeds finite FP32 arithmetic domain");
    int st = brp_host_resampling_steps(&p);
    if (st) return st;
    p.harmonic = n / 2; p.fundamental = n / 2; p.window = 8;
    const float thresholds[5] = {20, 30, 45, 70, 110};
    std::memcpy(p.threshold, thresholds, sizeof thresholds);
    p.capacity = 65536;
    *out = p;
    return BRP_OK;
}

// Chi-square upper tail Q(x; nu) for even nu = 2k: exp(-x/2) sum_{i<k} (x/2)^i / i!.
// Closed form of the regularized incomplete gamma function at integer order,
// standing in for gsl_cdf_chisq_Q (src/workload.cpp:146).
static double chisq_Q(double x, double nu) {
    if (!(x >= 0) || nu < 2 || std::fmod(nu, 2.0) != 0) return NAN;
    double y = 0.5 * x;
    int k = int(nu / 2);
    if (y <= 600) {
        double term = 1, sum = 1;
        for (int i = 1; i < k; ++i) { term *= y / i; sum += term; }
        return std::exp(-y) * sum;
    }
    double ly = std::log(y), m = (k - 1) * ly - std::lgamma(double(k)), acc = 0;
    for (int i = 0; i < k; ++i) acc += std::exp(i * ly - std::lgamma(double(i) + 1) - m);
    return std::exp(-y + m + std::log(acc));
}

// Inverse of chisq_Q in x by safeguarded Newton iteration on log Q, standing in
// for gsl_cdf_chisq_Qinv (src/workload.cpp:122).
static double chisq_Qinv(double q, double nu) {
    if (!(q > 0 && q < 1) || nu < 2 || std::fmod(nu, 2.0) != 0) return NAN;
    double lo = 0, hi = nu + 10;
    while (chisq_Q(hi, nu) > q) { lo = hi; hi *= 2; }
    double x = 0.5 * (lo + hi), lq = std::log(q);
    int k = int(nu / 2);
    for (int it = 0; it < 200; ++it) {
        double Q = chisq_Q(x, nu);
        if (Q > q) lo = x; else hi = x;
        double lpdf = (k - 1) * std::log(0.5 * x) - 0.5 * x - std::log(2.0) - std::lgamma(double(k));
        double next = x + (std::log(Q) - lq) / std::exp(lpdf - std::log(Q));
        if (!(next > lo && next < hi)) next = 0.5 * (lo + hi);
        if (std::fabs(next - x) <= 1e-16 * x || hi - lo <= 4e-16 * x) { x = next; break; }
        x = next;
    }
    return x;
}

extern "C" double brp_host_chisq_Q(double x, double nu) { return chisq_Q(x, nu); }
extern "C" double brp_host_chisq_Qinv(double q, double nu) { return chisq_Qinv(q, nu); }

extern "C" int brp_host_search_parameters(uint32_t n, uint32_t samples, double sample_us, double period, double tau,
                                          double psi, double f0, double false_alarm, uint32_t window,
                                          brp_params* out) {
    // src/workload.cpp:108-125.
    if (!out) return host_fail("null output");
    if (!std::isfinite(f0 + false_alarm) || f0 <= 0 || false_alarm <= 0 || false_alarm >= 1 || !window)
        return host_fail("invalid search parameters");
    brp_params p;
    int st = brp_host_parameters(n, samples, float(tau), float(period), float(psi), float(sample_us * 1e-6), &p);
    if (st) return st;
    p.flags = 2 | 4;  // production FMA arithmetic
    p.s0 = (p.tau * std::sin(p.psi)) * p.step_inv;
    st = brp_host_resampling_steps(&p);
    if (st) return st;
    double seconds = n * sample_us * 1e-6;
    p.window = uint32_t(window * 0.5 + 0.5);
    if (p.window >= p.n / 2 + 1) return host_fail("search window exceeds spectrum");
    double limit = p.n / 2 + 1 - p.window;
    p.fundamental = uint32_t(std::min(limit, f0 * seconds + 0.5));
    p.harmonic = uint32_t(std::min(limit, 16 * f0 * seconds + 0.5));
    float probability = 1.0 - std::pow(1.0 - false_alarm, 1.0 / (p.n / 2 + 1));
    if (!(probability > 0 && probability < 1)) return host_fail("false-alarm probability outside representable domain");
    for (uint32_t h = 0; h < 5; ++h) p.threshold[h] = 0.5 * chisq_Qinv(probability, 2.0 * (1u << h));
    if (p.fundamental <= p.window) return host_fail("empty frequency search");
    *out = p;
    return BRP_OK;
}

// ---- bank-wide toplist: 5 harmonic levels x 100 rows (src/workload.cpp:126-159) ----
struct brp_toplist { brp_bank_candidate rows[500]; };

extern "C" brp_toplist* brp_toplist_create(void) {
    auto* t = new (std::nothrow) brp_toplist;
    if (t) std::memset(t, 0, sizeof *t);
    return t;
}
extern "C" void brp_toplist_destroy(brp_toplist* t) { delete t; }

extern "C" void brp_toplist_thresholds(const brp_toplist* t, brp_params* p) {
    for (uint32_t h = 0; h < 5; ++h) p->threshold[h] = std::max(p->threshold[h], float(t->rows[(h + 1) * 100 - 1].power));
}

// The reference sorts with the C library's qsort and these comparators; equal
// keys keep whatever order that qsort gives, so the same call is made here.
static int by_power(const void* x, const void* y) {
    auto a = static_cast<const brp_bank_candidate*>(x), b = static_cast<const brp_bank_candidate*>(y);
    return a->power < b->power ? 1 : (a->power > b->power ? -1 : 0);
}
static int by_significance(const void* x, const void* y) {
    auto a = static_cast<const brp_bank_candidate*>(x), b = static_cast<const brp_bank_candidate*>(y);
    return a->significance < b->significance ? 1 : (a->significance > b->significance ? -1 : 0);
}

// Re-sorts a level's 100 rows after row i was replaced by a row of higher
// power (the reference calls qsort with by_power here).  The rows were sorted
// before, so moving row i up to its place gives a sorted array; when no two
// filled rows of the result have equal power (unfilled rows are all-zero and
// interchangeable), that sorted order is the only one, so it is exactly what
// qsort produces.  With a tie the order of equal rows is qsort's to decide, and
// qsort is called as in the reference.
static void resort_level(brp_bank_candidate* r, int i) {
    const brp_bank_candidate row = r[i];
    int j = i;
    while (j > 0 && r[j - 1].power < row.power) --j;
    // Equal powers among filled rows of the result: pairs already adjacent
    // (those without row i), the pair that closes up where row i leaves (when
    // it moves), and the moved row with its new upper neighbour.  Its new lower
    // neighbour has lower power (it was below row i's old or new place).
    bool tie = j > 0 && r[j - 1].power == row.power;
    for (int m = 0; m + 1 < 100 && !tie; ++m)
        if (m != i && m + 1 != i && r[m].harmonics && r[m + 1].harmonics && r[m].power == r[m + 1].power) tie = true;
    if (!tie && j < i && i + 1 < 100 && i > 0 && r[i - 1].harmonics && r[i + 1].harmonics &&
        r[i - 1].power == r[i + 1].power)
        tie = true;
    if (tie) {
        std::qsort(r, 100, sizeof(brp_bank_candidate), by_power);
        return;
    }
    std::memmove(r + j + 1, r + j, size_t(i - j) * sizeof(brp_bank_candidate));
    r[j] = row;
}

extern "C" int brp_toplist_retain(brp_toplist* t, const brp_candidate* cands, uint32_t count, double period,
                                  double tau, double psi, const brp_params* p) {
    for (uint32_t k = 0; k < count; ++k) {
        const brp_candidate c = cands[k];
        if (c.level >= 5 || c.bin < p->window || c.bin >= p->fundamental || !std::isfinite(c.power))
            return host_fail("invalid compact candidate");
        uint32_t first = c.level * 100, last = first + 99;
        if (c.power <= p->threshold[c.level] || c.power <= t->rows[last].power) continue;
        int place = int(last);
        for (uint32_t i = first; i <= last; ++i)
            if (t->rows[i].bin == c.bin) { place = t->rows[i].power < c.power ? int(i) : -1; break; }
        if (place >= int(first)) {
            t->rows[place] = {c.power, float(period), float(tau), float(psi), 0, 1u << c.level, c.bin};
            resort_level(t->rows + first, place - int(first));
        }
    }
    return BRP_OK;
}

extern "C" uint32_t brp_toplist_final(const brp_toplist* t, brp_bank_candidate* out) {
    brp_bank_candidate copy[500];
    std::memcpy(copy, t->rows, sizeof copy);
    for (auto& c : copy) {
        if (!c.harmonics) { c.significance = -10; continue; }
        double probability = chisq_Q(2 * c.power, 2.0 * c.harmonics);
        c.significance = probability > 0 ? -std::log10(probability) : 320;
        c.power /= float(std::sqrt(float(c.harmonics)));
    }
    std::qsort(copy, 500, sizeof(brp_bank_candidate), by_significance);
    uint32_t count = 0;
    while (count < 100 && copy[0].significance > 0) {
        out[count++] = copy[0];
        uint32_t bin = copy[0].bin;
        for (auto& c : copy) if (c.bin == bin) c.significance = -10;
        std::qsort(copy, 500, sizeof(brp_bank_candidate), by_significance);
    }
    return count;
}

// The bank loop of src/workunit_main.cpp:77-124 after the search: for each
// template in bank order, raise its thresholds to the toplist's current row
// 100 (Toplist::thresholds) and retain its candidates (Toplist::retain).
// candidates holds the templates' lists back to back; counts[t] per template;
// orbits[t] = (period, tau, psi).
extern "C" int brp_toplist_fold(brp_toplist* t, const brp_params* templates, const double* orbits,
                                const brp_candidate* candidates, const uint32_t* counts, uint32_t count) {
    if (!t || !templates || !orbits || !counts || (!candidates && count)) return host_fail("null argument");
    uint64_t off = 0;
    for (uint32_t k = 0; k < count; ++k) {
        brp_params p = templates[k];
        brp_toplist_thresholds(t, &p);
        const int st = brp_toplist_retain(t, candidates + off, counts[k], orbits[3 * k], orbits[3 * k + 1],
                                          orbits[3 * k + 2], &p);
        if (st) return st;
        off += counts[k];
    }
    return BRP_OK;
}

// ---- RFI zap list and zap noise of the whitening step (src/workload.cpp:72-88) ----
namespace {
// The generator pair the reference takes from GSL (absent here): gsl_rng_taus2
// and gsl_ran_gaussian_ziggurat.  Restated from the published algorithms:
// L'Ecuyer's maximally equidistributed three-component Tausworthe generator
// (Math. Comp. 65 (1996) 203-213) with the taus2 seeding (a 69069 LCG chain,
// components raised to their minima 2, 8, 16, six warm-up draws), and Marsaglia
// and Tsang's ziggurat (J. Stat. Softw. 5(8), 2000) for the normal with 128
// layers, a 24-bit uniform and the sign and layer from the low byte.
struct Taus2 {
    uint32_t s1, s2, s3;
    uint32_t next() {
        s1 = ((s1 & 0xFFFFFFFEu) << 12) ^ (((s1 << 13) ^ s1) >> 19);
        s2 = ((s2 & 0xFFFFFFF8u) << 4) ^ (((s2 << 2) ^ s2) >> 25);
        s3 = ((s3 & 0xFFFFFFF0u) << 17) ^ (((s3 << 3) ^ s3) >> 11);
        return s1 ^ s2 ^ s3;
    }
    double uniform() { return next() / 4294967296.0; }
    explicit Taus2(uint32_t seed) {
        if (!seed) seed = 1;
        s1 = 69069u * seed;
        if (s1 < 2) s1 += 2;
        s2 = 69069u * s1;
        if (s2 < 8) s2 += 8;
        s3 = 69069u * s2;
        if (s3 < 16) s3 += 16;
        for (int i = 0; i < 6; ++i) next();
    }
};

struct ZigguratTables {
    static constexpr double R = 3.442619855899, V = 9.91256303526217e-3, M = 16777216.0;
    double k[128], w[128], f[128];
    ZigguratTables() {
        double dn = R, tn = R;
        const double q = V / std::exp(-0.5 * dn * dn);
        k[0] = dn / q * M; k[1] = 0;
        w[0] = q / M; w[127] = dn / M;
        f[0] = 1.0; f[127] = std::exp(-0.5 * dn * dn);
        for (int i = 126; i >= 1; --i) {
            dn = std::sqrt(-2.0 * std::log(V / dn + std::exp(-0.5 * dn * dn)));
            k[i + 1] = dn / tn * M;
            tn = dn;
            f[i] = std::exp(-0.5 * dn * dn);
            w[i] = dn / M;
        }
    }
};

double gaussian(Taus2& r, double sigma) {
    static const ZigguratTables z;
    for (;;) {
        const uint32_t bits = r.next();
        const int i = int(bits & 0x7Fu);
        const double sign = (bits & 0x80u) ? 1.0 : -1.0;
        const uint32_t j = bits >> 8;
        double x = j * z.w[i];
        if (j < z.k[i]) return sign * sigma * x;
        if (i == 0) {  // the tail beyond R
            double y;
            do {
                x = -std::log(1.0 - r.uniform()) / ZigguratTables::R;
                y = -std::log(1.0 - r.uniform());
            } while (y + y < x * x);
            return sign * sigma * (ZigguratTables::R + x);
        }
        if (z.f[i] + r.uniform() * (z.f[i - 1] - z.f[i]) < std::exp(-0.5 * x * x)) return sign * sigma * x;
    }
}
}  // namespace

extern "C" int brp_host_read_zap(const char* path, double* lower, double* upper, uint32_t cap, uint32_t* count) {
    // src/workload.cpp:77-81, :88: whitespace-separated (lower, upper) pairs in Hz/seconds-normalised units.
    if (!path || !count) return host_fail("null argument");
    FILE* fp = std::fopen(path, "r");
    if (!fp) return host_fail("cannot open zap list");
    uint32_t k = 0;
    double lo, hi;
    int got;
    while ((got = std::fscanf(fp, "%lf %lf", &lo, &hi)) == 2) {
        if (!std::isfinite(lo + hi) || lo < 0 || hi < lo) { std::fclose(fp); return host_fail("invalid zap range"); }
        if (k < cap) { if (lower) lower[k] = lo; if (upper) upper[k] = hi; }
        ++k;
    }
    const bool clean = got == EOF && !std::ferror(fp);
    std::fclose(fp);
    if (!clean) return host_fail("malformed zap list");
    *count = k;
    return BRP_OK;
}

extern "C" int brp_host_zap_noise(uint32_t seed, uint32_t n, double sample_us, double padding, const double* lower,
                                  const double* upper, uint32_t ranges, uint32_t* bins, float* values, uint32_t cap,
                                  uint32_t* count) {
    // src/workload.cpp:73-87: one taus2 stream seeded with the bits of the
    // first decoded sample; per zapped bin a real then an imaginary Gaussian
    // of sigma sqrt(2)/2 sqrt(padding), in the order of the ranges.
    if (!count || (ranges && (!lower || !upper))) return host_fail("null argument");
    Taus2 rng(seed);
    const double seconds = double(n) * sample_us * 1e-6;
    const uint64_t size = uint64_t(n) / 2 + 1;
    const double sigma = std::sqrt(2.0) / 2 * std::sqrt(padding);
    uint32_t k = 0;
    for (uint32_t r = 0; r < ranges; ++r) {
        if (!std::isfinite(lower[r] + upper[r]) || lower[r] < 0 || upper[r] < lower[r]) return host_fail("invalid zap range");
        const double first = lower[r] * seconds + 0.5, last = upper[r] * seconds + 0.5;
        if (last >= double(size)) return host_fail("zap exceeds Nyquist");
        for (uint32_t i = uint32_t(first); i <= uint32_t(last); ++i) {
            const float re = float(gaussian(rng, sigma)), im = float(gaussian(rng, sigma));
            if (k < cap) {
                if (bins) bins[k] = i;
                if (values) { values[2 * k] = re; values[2 * k + 1] = im; }
            }
            ++k;
        }
    }
    *count = k;
    return BRP_OK;
}
