// Autotuner of the bank search and its plan cache, for every host language.
//
// brp_cuda_bank_autotune times, on the device, each compatible pair of compiled
// pass-1 / pass-2 configurations with each number of templates per launch and
// each number of launch chains, by replaying the bank's captured graph of the
// caller's own templates with L2 flushed between replays (CUDA events on the
// bank's stream), keeps the fastest per length class and configures the bank
// with it.  It is a client of the bank's C ABI (configure / run / launch).
//
// Plans are kept in a JSON file shared with the Python tuner (brp_b200.tune):
//     {"<device>|n=<n>|templates=<count>": {"pass1": id, "pass2": id,
//      "group": g, "chains": c, "ms": t}, ...}
// with <device> = "<name>/sm<major><minor>/<SMs>".  The library also reads
// that file (BRP_PLAN_CACHE, else ~/.cache/brp_b200/plans.json) when it first
// chooses a plan with no configuration named by the caller, so brp::GPU and a
// new bank take the tuned kernels for any tuned length.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include <sys/stat.h>
#include "brp_internal.h"

namespace brp {
namespace {

struct PlanEntry {
    int pass1 = 0, pass2 = 0;
    uint32_t group = 0, chains = 1;
    double ms = 0;
};
using PlanMap = std::map<std::string, PlanEntry>;

// ---- a small JSON reader for the plan file (objects, strings, numbers;
// other values are skipped) and its writer
struct Json {
    const char* p;
    const char* e;
    void ws() { while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p; }
    bool eat(char c) { ws(); if (p < e && *p == c) { ++p; return true; } return false; }
    bool str(std::string& out) {
        ws();
        if (p >= e || *p != '"') return false;
        ++p;
        out.clear();
        while (p < e && *p != '"') {
            if (*p == '\\') {
                if (++p >= e) return false;
                switch (*p) {
                    case 'n': out += '\n'; break;
                    case 't': out += '\t'; break;
                    case 'u': if (e - p < 5) return false; out += '?'; p += 4; break;  // not in plan keys
                    default: out += *p;
                }
                ++p;
            } else {
                out += *p++;
            }
        }
        if (p >= e) return false;
        ++p;
        return true;
    }
    bool num(double& v) {
        ws();
        char* end = nullptr;
        std::string tok;
        while (p < e && *p && std::strchr("+-0123456789.eE", *p)) tok += *p++;
        if (tok.empty()) return false;
        v = std::strtod(tok.c_str(), &end);
        return end && *end == 0;
    }
    bool skip() {
        ws();
        if (p >= e) return false;
        if (*p == '"') { std::string s; return str(s); }
        if (*p == '{' || *p == '[') {
            const char close = *p == '{' ? '}' : ']';
            const bool obj = *p == '{';
            ++p;
            if (eat(close)) return true;
            do {
                if (obj) { std::string k; if (!str(k) || !eat(':')) return false; }
                if (!skip()) return false;
            } while (eat(','));
            return eat(close);
        }
        if (!std::strncmp(p, "true", 4) && e - p >= 4) { p += 4; return true; }
        if (!std::strncmp(p, "false", 5) && e - p >= 5) { p += 5; return true; }
        if (!std::strncmp(p, "null", 4) && e - p >= 4) { p += 4; return true; }
        double v;
        return num(v);
    }
};

bool parse_plans(const std::string& text, PlanMap& out) {
    Json j{text.data(), text.data() + text.size()};
    if (!j.eat('{')) return false;
    if (j.eat('}')) return true;
    do {
        std::string key;
        if (!j.str(key) || !j.eat(':') || !j.eat('{')) return false;
        PlanEntry pe;
        bool has1 = false, has2 = false;
        if (!j.eat('}')) {
            do {
                std::string f;
                if (!j.str(f) || !j.eat(':')) return false;
                double v = 0;
                const bool numeric = f == "pass1" || f == "pass2" || f == "group" || f == "chains" || f == "ms";
                if (numeric) {
                    if (!j.num(v)) return false;
                } else if (!j.skip()) {
                    return false;
                }
                if (f == "pass1") { pe.pass1 = int(v); has1 = true; }
                if (f == "pass2") { pe.pass2 = int(v); has2 = true; }
                if (f == "group") pe.group = uint32_t(v);
                if (f == "chains") pe.chains = uint32_t(v);
                if (f == "ms") pe.ms = v;
            } while (j.eat(','));
            if (!j.eat('}')) return false;
        }
        if (has1 && has2) out[key] = pe;
    } while (j.eat(','));
    return j.eat('}');
}

std::string json_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

bool read_file(const std::string& path, std::string& text) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    char buf[65536];
    size_t n;
    text.clear();
    while ((n = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, n);
    std::fclose(f);
    return true;
}

bool write_plans(const std::string& path, const PlanMap& m) {
    // the directories of the path, then a temporary file renamed over the plan file
    for (size_t k = 1; k < path.size(); ++k)
        if (path[k] == '/') mkdir(path.substr(0, k).c_str(), 0755);
    const std::string tmp = path + ".tmp";
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return false;
    std::fprintf(f, "{");
    bool first = true;
    for (const auto& kv : m) {
        std::fprintf(f,
                     "%s\n \"%s\": {\n  \"chains\": %u,\n  \"group\": %u,\n  \"ms\": %.17g,\n  \"pass1\": %d,\n"
                     "  \"pass2\": %d\n }",
                     first ? "" : ",", json_escape(kv.first).c_str(), kv.second.chains, kv.second.group, kv.second.ms,
                     kv.second.pass1, kv.second.pass2);
        first = false;
    }
    std::fprintf(f, "\n}\n");
    const bool ok = std::fclose(f) == 0;
    return ok && std::rename(tmp.c_str(), path.c_str()) == 0;
}

std::string default_cache_path() {
    if (const char* env = std::getenv("BRP_PLAN_CACHE")) return env;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : ".") + "/.cache/brp_b200/plans.json";
}

// "<name>/sm<major><minor>/<SMs>" of the current device (the Python tuner's key).
std::string device_key() {
    int dev = 0;
    cudaDeviceProp prop{};
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&prop, dev) != cudaSuccess) return "cuda";
    char buf[512];
    std::snprintf(buf, sizeof buf, "%s/sm%d%d/%d", prop.name, prop.major, prop.minor, prop.multiProcessorCount);
    return buf;
}

std::string plan_key(const std::string& dev, uint32_t n, uint32_t templates) {
    return dev + "|n=" + std::to_string(n) + "|templates=" + std::to_string(templates);
}

// The process-wide plan table that default plan choices consult.
std::mutex g_plan_mutex;
PlanMap g_plans;
bool g_plans_loaded = false;

void merge_plan_file_locked(const std::string& path) {
    std::string text;
    PlanMap m;
    if (read_file(path, text) && parse_plans(text, m))
        for (auto& kv : m) g_plans[kv.first] = kv.second;
}

// Polls an event with a deadline (seconds).
bool wait_done(cudaEvent_t ev, double seconds) {
    const auto t0 = std::chrono::steady_clock::now();
    for (int spin = 0;; ++spin) {
        const cudaError_t e = cudaEventQuery(ev);
        if (e == cudaSuccess) return true;
        if (e != cudaErrorNotReady) return false;
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() > seconds) return false;
        if (spin > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

thread_local std::string g_tune_error;

int tune_fail(int code, const std::string& m) {
    g_tune_error = m;
    return code;
}

}  // namespace

bool cached_plan(uint32_t n, CachedPlan& out) {
    std::lock_guard<std::mutex> lock(g_plan_mutex);
    if (!g_plans_loaded) {
        merge_plan_file_locked(default_cache_path());
        g_plans_loaded = true;
    }
    const std::string prefix = device_key() + "|n=" + std::to_string(n) + "|templates=";
    uint32_t best_templates = 0;
    bool found = false;
    for (auto it = g_plans.lower_bound(prefix); it != g_plans.end() && it->first.compare(0, prefix.size(), prefix) == 0;
         ++it) {
        // the entry tuned on the largest bank of this length
        const uint32_t t = uint32_t(std::strtoul(it->first.c_str() + prefix.size(), nullptr, 10));
        if (!found || t > best_templates) {
            out.pass1 = it->second.pass1; out.pass2 = it->second.pass2;
            out.group = it->second.group; out.chains = it->second.chains;
            best_templates = t;
            found = true;
        }
    }
    return found;
}

}  // namespace brp

using namespace brp;

extern "C" const char* brp_cuda_autotune_error(void) { return g_tune_error.c_str(); }

extern "C" int brp_cuda_load_plan_cache(const char* path) {
    std::lock_guard<std::mutex> lock(g_plan_mutex);
    if (path && !*path) {  // "": forget every plan, read no file by itself any more
        g_plans.clear();
        g_plans_loaded = true;
        return BRP_OK;
    }
    const std::string p = path ? std::string(path) : default_cache_path();
    std::string text;
    PlanMap m;
    if (!read_file(p, text)) return tune_fail(BRP_E_ARGUMENT, "cannot read plan cache " + p);
    if (!parse_plans(text, m)) return tune_fail(BRP_E_ARGUMENT, "invalid plan cache " + p);
    for (auto& kv : m) g_plans[kv.first] = kv.second;
    g_plans_loaded = true;  // the default file is not read over an explicitly loaded one
    return BRP_OK;
}

extern "C" int brp_cuda_bank_autotune(brp_bank* bank, const brp_params* templates, const uint32_t* series_of,
                                      uint32_t count, uint32_t reps, const uint32_t* groups, uint32_t group_count,
                                      const char* cache_path, uint32_t flags, brp_tune_result* results, uint32_t cap,
                                      uint32_t* found) {
    if (!bank || !templates || !series_of || !count || !found)
        return tune_fail(BRP_E_ARGUMENT, "null argument or empty bank");
    *found = 0;
    reps = std::max<uint32_t>(reps, 1);
    std::vector<uint32_t> grp = groups && group_count ? std::vector<uint32_t>(groups, groups + group_count)
                                                      : std::vector<uint32_t>{16, 32, 64, 128};
    std::vector<uint32_t> lengths;
    for (uint32_t t = 0; t < count; ++t) lengths.push_back(templates[t].n);
    std::sort(lengths.begin(), lengths.end());
    lengths.erase(std::unique(lengths.begin(), lengths.end()), lengths.end());
    const std::string dev = device_key();
    PlanMap cache;
    if (cache_path) {
        std::string text;
        if (read_file(cache_path, text) && !parse_plans(text, cache)) cache.clear();
    }
    // compiled CUDA-core configurations (the tensor-core forms are chosen by id only)
    const int total = brp_cuda_fast_configs(nullptr, nullptr, nullptr, 0);
    std::vector<int32_t> ids(total);
    std::vector<uint32_t> lens(total), kinds(total);
    brp_cuda_fast_configs(ids.data(), lens.data(), kinds.data(), uint32_t(total));

    cudaStream_t s = static_cast<cudaStream_t>(brp_cuda_bank_stream(bank));
    const size_t flush_bytes = size_t(512) << 20;  // larger than L2: every replay starts cold
    void* flush = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (cudaMalloc(&flush, flush_bytes) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        if (flush) cudaFree(flush);
        if (e0) cudaEventDestroy(e0);
        return tune_fail(BRP_E_RUNTIME, "autotune: cannot allocate the L2 flush buffer or events");
    }
    std::vector<uint32_t> counts(count), status(count);
    int rc = BRP_OK;
    for (uint32_t n : lengths) {
        const std::string key = plan_key(dev, n, count);
        brp_tune_result r{};
        r.n = n;
        auto hit = cache.find(key);
        if ((flags & BRP_TUNE_USE_CACHE) && hit != cache.end()) {
            const PlanEntry& pe = hit->second;
            if (brp_cuda_bank_configure(bank, n, pe.pass1, pe.pass2, pe.group, pe.chains) == BRP_OK) {
                r.pass1 = pe.pass1; r.pass2 = pe.pass2; r.group = pe.group; r.chains = pe.chains; r.ms = pe.ms;
                r.cached = 1;
                if (*found < cap && results) results[*found] = r;
                ++*found;
                continue;
            }
        }
        double best = INFINITY;
        PlanEntry be;
        for (int a = 0; a < total; ++a) {
            if (kinds[a] != 1) continue;
            for (int b = 0; b < total; ++b) {
                if (kinds[b] != 2 || uint64_t(lens[a]) * lens[b] != n / 2) continue;
                for (uint32_t g : grp)
                    for (uint32_t ch = 1; ch <= 2; ++ch) {
                        if (brp_cuda_bank_configure(bank, n, ids[a], ids[b], g, ch) != BRP_OK) continue;
                        const int st = brp_cuda_bank_run(bank, templates, series_of, count, nullptr, 0, counts.data(),
                                                         status.data());
                        if (st != BRP_OK && st != BRP_E_RESULT) continue;  // a result error still timed the kernels
                        double sum = 0;
                        bool ok = true;
                        for (uint32_t k = 0; k < reps && ok; ++k) {
                            ok = cudaMemsetAsync(flush, k & 1, flush_bytes, s) == cudaSuccess &&
                                 cudaEventRecord(e0, s) == cudaSuccess && brp_cuda_bank_launch(bank) == BRP_OK &&
                                 cudaEventRecord(e1, s) == cudaSuccess && wait_done(e1, 300.0);
                            float ms = 0;
                            if (ok) ok = cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
                            sum += ms;
                        }
                        ++r.tried;
                        if (!ok) continue;
                        const double ms = sum / reps;
                        if (ms < best) {
                            best = ms;
                            be.pass1 = ids[a]; be.pass2 = ids[b]; be.group = g; be.chains = ch; be.ms = ms;
                        }
                    }
            }
        }
        if (!std::isfinite(best)) {
            brp_cuda_bank_configure(bank, n, 0, 0, 0, 0);
            rc = tune_fail(BRP_E_RUNTIME, "autotune: no configuration ran for n = " + std::to_string(n));
            continue;
        }
        brp_cuda_bank_configure(bank, n, be.pass1, be.pass2, be.group, be.chains);
        r.pass1 = be.pass1; r.pass2 = be.pass2; r.group = be.group; r.chains = be.chains; r.ms = be.ms;
        cache[key] = be;
        {
            std::lock_guard<std::mutex> lock(g_plan_mutex);
            g_plans[key] = be;  // later default choices in this process take it too
        }
        if (*found < cap && results) results[*found] = r;
        ++*found;
    }
    cudaFree(flush);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cache_path && !write_plans(cache_path, cache) && rc == BRP_OK)
        rc = tune_fail(BRP_E_RUNTIME, std::string("autotune: cannot write the plan cache ") + cache_path);
    return rc;
}
