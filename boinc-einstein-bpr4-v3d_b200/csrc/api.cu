// C ABI of the CUDA backend (include/brp_cuda.h): the per-template context that
// replaces src/vulkan.cpp behind brp::GPU, and the bank extension that runs a
// whole orbital bank as one captured CUDA graph.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <map>
#include <string>
#include <thread>
#include <vector>
#include "brp_internal.h"

using namespace brp;

namespace {

thread_local std::string g_thread_error;

double cpu_ms_now() {
    timespec t{};
    clock_gettime(CLOCK_PROCESS_CPUTIME_ID, &t);
    return t.tv_sec * 1000.0 + t.tv_nsec / 1e6;
}

// Waits for `ev` with a deadline instead of an unbounded blocking wait.
cudaError_t wait_event(cudaEvent_t ev, double seconds, bool* timed_out) {
    *timed_out = false;
    auto start = std::chrono::steady_clock::now();
    for (int spin = 0;; ++spin) {
        cudaError_t e = cudaEventQuery(ev);
        if (e != cudaErrorNotReady) return e;
        if (std::chrono::duration<double>(std::chrono::steady_clock::now() - start).count() > seconds) {
            *timed_out = true;
            return cudaErrorNotReady;
        }
        if (spin > 64) std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
}

bool is_pow2(uint32_t x) { return x && !(x & (x - 1)); }

// Host-side fake of a failing cudaMalloc for tests of the error paths
// (brp_cuda_debug_fail_allocation): when the countdown reaches the allocation
// it names, that allocation reports failure without calling cudaMalloc.
std::atomic<uint32_t> g_alloc_countdown{0};
bool alloc_fault_due() {
    uint32_t c = g_alloc_countdown.load();
    while (c)
        if (g_alloc_countdown.compare_exchange_weak(c, c - 1)) return c == 1;
    return false;
}

std::string validate_wait_limits(double seconds) {
    if (!(seconds >= 0.0) || seconds > 86400.0) return "host deadline must be within 0..86400 seconds";
    return "";
}

}  // namespace

struct brp_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    brp_params base{};
    uint32_t wg = 0, tile = 0, batch = 0, opt = 0;
    bool fused = false;
    std::vector<brp_params> templates;
    LengthPlan lp;
    std::vector<void*> allocations;
    uint64_t allocated = 0;
    // device buffers
    float* d_input = nullptr;
    const float** d_inputs = nullptr;
    brp_params* d_params = nullptr;
    float2* d_work = nullptr;
    float* d_power = nullptr;
    double* d_partial = nullptr;
    float* d_mean = nullptr;
    uint32_t* d_tickets = nullptr;  // pass-1 CTA tickets per template (zero between runs)
    uint32_t* d_status = nullptr;
    uint32_t* d_counts = nullptr;
    brp_candidate* d_cands = nullptr;
    float* d_raw = nullptr;
    float2* d_fft = nullptr;
    float* d_summed = nullptr;
    float2* d_a = nullptr;
    float2* d_b = nullptr;
    std::vector<cudaEvent_t> events;
    uint32_t last_count = 0;
    double last_stage_ms[4] = {0, 0, 0, 0};
    uint32_t wait_polls = kDefaultWaitPolls;   // device: first-wait poll bound of the kernels
    double wait_seconds = kDefaultWaitSeconds; // host: deadline of a run
    cudaEvent_t pending = nullptr;             // completion of a run that passed its deadline
    std::string error;

    void run_finished() {}
    int fail(int code, const std::string& msg) {
        error = msg;
        g_thread_error = msg;
        return code;
    }
    int cuda(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return BRP_OK;
        return fail(BRP_E_RUNTIME, std::string(what) + ": " + cudaGetErrorString(e));
    }
    template <class T>
    int alloc(T** p, size_t count, const char* what) {
        size_t bytes = std::max<size_t>(count * sizeof(T), 16);
        if (alloc_fault_due() || cudaMalloc(reinterpret_cast<void**>(p), bytes) != cudaSuccess)
            return fail(BRP_E_RUNTIME, std::string("cudaMalloc failed: ") + what);
        allocations.push_back(*p);
        allocated += bytes;
        return BRP_OK;
    }
    ~brp_ctx() {
        if (device >= 0) cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (auto e : events) cudaEventDestroy(e);
        for (auto p : allocations) cudaFree(p);
        free_length_plan(lp);
        if (stream) cudaStreamDestroy(stream);
    }
};

static int set_thread_error(int code, const std::string& m) {
    g_thread_error = m;
    return code;
}

// Validation of src/vulkan.cpp:110-122 and :278-284 (flag combinations, limits).
static std::string validate_options(const brp_params& p, const brp_options& o) {
    const bool stockham = o.flags & BRP_OPT_STOCKHAM, packed = o.flags & BRP_OPT_PACKED;
    const bool radix8 = o.flags & BRP_OPT_RADIX8, fused_power = o.flags & BRP_OPT_FUSED_POWER;
    const bool radix8_store = o.flags & BRP_OPT_RADIX8_STORE;
    if (fused_power && !packed) return "fused power requires packed real FFT";
    if (radix8_store && !radix8) return "paired-store radix 8 requires radix 8";
    if (radix8 && (!stockham || o.tile)) return "radix8 requires Stockham without a shared tile";
    uint32_t fft_n = packed ? p.n / 2 : p.n;
    uint32_t base = is_pow2(fft_n) ? fft_n : fft_n / 3;
    if (o.tile > base) return "FFT tile exceeds radix-2 block";
    if (stockham && o.tile) return "Stockham requires --tile 0";
    if (!o.workgroup || o.workgroup > 256 || !o.batch || o.batch > 64 ||
        (o.tile && (!is_pow2(o.tile) || o.tile < 64 || o.tile > 4096 || o.tile > p.n)))
        return "invalid workgroup, FFT tile, or batch";
    return "";
}

static std::string validate_template(const brp_params& base, const brp_params& next) {
    // src/vulkan.cpp:271-273.
    if ((next.flags & 6u) != (base.flags & 6u)) return "arithmetic specialization changed; rebuild pipelines";
    if (next.n != base.n || next.unpadded != base.unpadded || next.fundamental != base.fundamental ||
        next.harmonic != base.harmonic || next.capacity != base.capacity || !next.steps || next.steps > next.unpadded)
        return "template dimensions changed; rebuild resources";
    return "";
}

static std::string validate_dims(const brp_params& p) {
    if (p.n < 64 || p.n > 3u * (1u << 22) || !(is_pow2(p.n) || (p.n % 3 == 0 && is_pow2(p.n / 3))))
        return "series length must be 2^k or 3*2^k in 64..3*2^22";
    if (p.unpadded < 2 || p.unpadded > p.n) return "invalid unpadded length";
    if (!p.steps || p.steps > p.unpadded) return "invalid resampled length";
    if (p.fundamental > p.n / 2 || p.harmonic > p.n / 2) return "harmonic search range exceeds the spectrum";
    if (!p.capacity) return "zero candidate capacity";
    return "";
}

extern "C" const char* brp_cuda_last_error(const brp_ctx* ctx) {
    return ctx ? ctx->error.c_str() : g_thread_error.c_str();
}

extern "C" int brp_cuda_create(const brp_params* params, const float* input, uint32_t unpadded,
                               const brp_options* options, brp_ctx** out) {
    if (!params || !input || !options || !out) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    *out = nullptr;
    brp_params p = *params;
    std::string v = validate_options(p, *options);
    if (v.empty()) v = validate_dims(p);
    if (v.empty() && unpadded != p.unpadded) v = "input length mismatch";
    if (!v.empty()) return set_thread_error(BRP_E_RUNTIME, v);
    auto* c = new (std::nothrow) brp_ctx;
    if (!c) return set_thread_error(BRP_E_RUNTIME, "out of host memory");
    c->device = options->device;
    if (c->device < 0) cudaGetDevice(&c->device);
    int st;
    if ((st = c->cuda(cudaSetDevice(c->device), "cudaSetDevice"))) { std::string m = c->error; delete c; return set_thread_error(st, m); }
    if ((st = c->cuda(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate"))) {
        std::string m = c->error; delete c; return set_thread_error(st, m);
    }
    c->base = p;
    if (options->flags & BRP_OPT_PACKED) c->base.flags |= BRP_FLAG_PACKED;
    c->wg = options->workgroup; c->tile = options->tile; c->batch = options->batch; c->opt = options->flags;
    // reserved[0] / reserved[1]: compiled pass-1 / pass-2 configuration ids
    // (0 = default choice, UINT32_MAX = generic kernels).
    const int f1 = options->reserved[0] == UINT32_MAX ? -1 : int(options->reserved[0]);
    const int f2 = options->reserved[1] == UINT32_MAX ? -1 : int(options->reserved[1]);
    std::string e = make_length_plan(p.n, c->lp, c->stream, f1, f2);
    if (!e.empty()) { delete c; return set_thread_error(BRP_E_RUNTIME, e); }
    c->fused = c->lp.fused && !(options->flags & BRP_OPT_PLAIN);
    const uint32_t B = c->batch, M = c->lp.M, cap = p.capacity;
    const uint32_t slots = c->fused ? B : 1;
    auto cleanup = [&](int code) { std::string m = c->error; delete c; return set_thread_error(code, m); };
    if ((st = c->alloc(&c->d_input, unpadded, "input")) || (st = c->alloc(&c->d_inputs, B, "input table")) ||
        (st = c->alloc(&c->d_params, B, "params")) || (st = c->alloc(&c->d_work, size_t(slots) * M, "work")) ||
        (st = c->alloc(&c->d_power, size_t(slots) * M, "power")) ||
        (st = c->alloc(&c->d_partial, size_t(slots) * std::max<uint32_t>(c->fused ? c->lp.blocks1() : (p.unpadded + 255) / 256, 1), "partial")) ||
        (st = c->alloc(&c->d_mean, B, "mean")) || (st = c->alloc(&c->d_tickets, B, "tickets")) ||
        (st = c->alloc(&c->d_status, B, "status")) ||
        (st = c->alloc(&c->d_counts, B, "counts")) || (st = c->alloc(&c->d_cands, size_t(B) * cap, "candidates")) ||
        (st = c->alloc(&c->d_raw, p.unpadded, "resampled")) || (st = c->alloc(&c->d_fft, size_t(M) + 1, "fft")) ||
        (st = c->alloc(&c->d_summed, size_t(5) * p.fundamental, "summed")))
        return cleanup(st);
    if (!c->fused && ((st = c->alloc(&c->d_a, M, "fft a")) || (st = c->alloc(&c->d_b, M, "fft b")))) return cleanup(st);
    c->allocated += c->lp.tables_bytes;
    if ((st = c->cuda(cudaMemcpy(c->d_input, input, size_t(unpadded) * 4, cudaMemcpyHostToDevice), "input upload")) ||
        (st = c->cuda(cudaMemset(c->d_tickets, 0, size_t(B) * 4), "tickets clear")))
        return cleanup(st);
    std::vector<const float*> ptrs(B, c->d_input);
    if ((st = c->cuda(cudaMemcpy(c->d_inputs, ptrs.data(), B * sizeof(void*), cudaMemcpyHostToDevice), "input table")))
        return cleanup(st);
    c->events.resize(5 * B);
    for (auto& ev : c->events)
        if ((st = c->cuda(cudaEventCreate(&ev), "cudaEventCreate"))) { ev = nullptr; return cleanup(st); }
    c->templates.assign(1, c->base);
    *out = c;
    return BRP_OK;
}

extern "C" void brp_cuda_destroy(brp_ctx* ctx) { delete ctx; }

extern "C" int brp_cuda_set_templates(brp_ctx* c, const brp_params* t, uint32_t count) {
    if (!c || !t) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    if (!count || count > c->batch) return c->fail(BRP_E_RUNTIME, "template batch exceeds retained result capacity");
    std::vector<brp_params> next(t, t + count);
    for (auto& p : next) {
        std::string v = validate_template(c->base, p);
        if (!v.empty()) return c->fail(BRP_E_RUNTIME, v);
        // Dimensions stay the constructor's; the remaining fields follow the template
        // (src/vulkan.cpp:274-275).
        brp_params q = c->base;
        q.steps = p.steps; q.tau = p.tau; q.omega = p.omega; q.psi = p.psi; q.dt = p.dt; q.step_inv = p.step_inv;
        q.s0 = p.s0; q.window = p.window;
        std::memcpy(q.threshold, p.threshold, sizeof q.threshold);
        p = q;
    }
    c->templates = next;
    return BRP_OK;
}

static FusedArgs fused_args(brp_ctx* c, uint32_t count) {
    FusedArgs a{};
    const LengthPlan& lp = c->lp;
    a.inputs = c->d_inputs;
    a.params = c->d_params;
    fill_fused_args(a, lp);
    a.work = c->d_work; a.work_stride = lp.M;
    a.power = c->d_power; a.power_stride = lp.M;
    a.partial = c->d_partial; a.partial_stride = lp.blocks1();
    a.mean = c->d_mean; a.tickets = c->d_tickets;
    a.status = c->d_status; a.counts = c->d_counts; a.cands = c->d_cands;
    a.capacity = c->base.capacity;
    a.snap = int(count) - 1;
    a.snap_raw = c->d_raw; a.snap_fft = c->d_fft; a.snap_summed = c->d_summed;
    a.wait_polls = c->wait_polls;
    return a;
}

// A run that passed its host deadline may still be executing: before the next
// run reuses the context's buffers, wait for it (bounded by the deadline).
template <class Obj>
static int settle_pending(Obj* o) {
    if (!o->pending) return BRP_OK;
    bool timed_out = false;
    cudaError_t e = wait_event(o->pending, o->wait_seconds, &timed_out);
    if (timed_out) return o->fail(BRP_E_TIMEOUT, "the previous run is still executing after the deadline");
    o->pending = nullptr;
    o->run_finished();
    return o->cuda(e, "previous run");
}

extern "C" int brp_cuda_run(brp_ctx* c, brp_timings* timings, double* template_stage_ms) {
    if (!c) return set_thread_error(BRP_E_ARGUMENT, "null context");
    int st;
    if ((st = c->cuda(cudaSetDevice(c->device), "cudaSetDevice"))) return st;
    if ((st = settle_pending(c))) return st;
    auto start = std::chrono::steady_clock::now();
    double cpu0 = cpu_ms_now();
    const uint32_t count = uint32_t(c->templates.size());
    const brp_params& last = c->templates.back();
    cudaStream_t s = c->stream;
    auto submit0 = std::chrono::steady_clock::now();
    if ((st = c->cuda(cudaMemcpyAsync(c->d_params, c->templates.data(), count * sizeof(brp_params),
                                      cudaMemcpyHostToDevice, s), "params upload")))
        return st;
    cudaMemsetAsync(c->d_counts, 0, count * sizeof(uint32_t), s);
    cudaMemsetAsync(c->d_status, 0, count * sizeof(uint32_t), s);
    cudaMemsetAsync(c->d_summed, 0, size_t(5) * last.fundamental * sizeof(float), s);
    cudaEvent_t* ev = c->events.data();
    if (c->fused) {
        FusedArgs a = fused_args(c, count);
        uint32_t span = 0;
        for (auto& p : c->templates) span = std::max(span, std::max(p.fundamental, p.harmonic + 8));
        cudaEventRecord(ev[0], s);
        launch_fused_pass1(a, c->lp, count, s);
        cudaEventRecord(ev[1], s);
        launch_fused_pass2(a, c->lp, count, s);
        cudaEventRecord(ev[2], s);
        cudaEventRecord(ev[3], s);
        launch_fused_harmonic(a, c->lp, count, span, s);
        cudaEventRecord(ev[4], s);
    } else {
        for (uint32_t t = 0; t < count; ++t) {
            PlainArgs a{};
            a.input = c->d_input; a.p = c->templates[t]; a.lp = &c->lp;
            a.raw = c->d_raw; a.partial = c->d_partial; a.mean = c->d_mean; a.a = c->d_a; a.b = c->d_b;
            a.fft = c->d_fft; a.power = c->d_power; a.summed = c->d_summed;
            a.status = c->d_status + t; a.count = c->d_counts + t; a.cands = c->d_cands + size_t(t) * c->base.capacity;
            launch_plain(a, s, ev + 5 * t);
        }
    }
    if ((st = c->cuda(cudaGetLastError(), "kernel launch"))) return st;
    double submit_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - submit0).count();
    bool timed_out = false;
    cudaEvent_t done = c->fused ? ev[4] : ev[5 * (count - 1) + 4];
    cudaError_t e = wait_event(done, c->wait_seconds, &timed_out);
    if (timed_out) {
        c->pending = done;
        return c->fail(BRP_E_TIMEOUT, "GPU run exceeded its deadline");
    }
    if ((st = c->cuda(e, "GPU run"))) return st;
    brp_timings t{};
    t.submit_ms = submit_ms;
    for (int k = 0; k < 4; ++k) c->last_stage_ms[k] = 0;
    const uint32_t groups = c->fused ? 1 : count;
    for (uint32_t g = 0; g < groups; ++g)
        for (int k = 0; k < 4; ++k) {
            float ms = 0;
            cudaEventElapsedTime(&ms, ev[5 * g + k], ev[5 * g + k + 1]);
            t.stage_ms[k] += ms;
            c->last_stage_ms[k] += ms;
            if (template_stage_ms) {
                if (c->fused) for (uint32_t r = 0; r < count; ++r) template_stage_ms[4 * r + k] = ms / count;
                else template_stage_ms[4 * g + k] = ms;
            }
        }
    c->last_count = count;
    t.cpu_ms = cpu_ms_now() - cpu0;
    t.wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - start).count();
    if (timings) *timings = t;
    return BRP_OK;
}

extern "C" int brp_cuda_snapshot(brp_ctx* c, float* resampled, float* fft, float* power, float* summed) {
    if (!c) return set_thread_error(BRP_E_ARGUMENT, "null context");
    if (!c->last_count) return c->fail(BRP_E_RUNTIME, "snapshot before run");
    int st;
    if ((st = c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) || (st = settle_pending(c))) return st;
    const uint32_t g = c->last_count - 1;
    const brp_params& p = c->templates[g];
    const uint32_t slot = c->fused ? g : 0;
    if (resampled) {
        float mean = 0;
        if ((st = c->cuda(cudaMemcpy(resampled, c->d_raw, size_t(p.steps) * 4, cudaMemcpyDeviceToHost), "snapshot")) ||
            (st = c->cuda(cudaMemcpy(&mean, c->d_mean + (c->fused ? g : 0), 4, cudaMemcpyDeviceToHost), "snapshot")))
            return st;
        std::fill(resampled + p.steps, resampled + p.n, mean);
    }
    if (fft && (st = c->cuda(cudaMemcpy(fft, c->d_fft, (size_t(c->lp.M) + 1) * 8, cudaMemcpyDeviceToHost), "snapshot")))
        return st;
    if (power && (st = c->cuda(cudaMemcpy(power, c->d_power + size_t(slot) * c->lp.M, size_t(c->lp.M) * 4,
                                          cudaMemcpyDeviceToHost), "snapshot")))
        return st;
    if (summed && (st = c->cuda(cudaMemcpy(summed, c->d_summed, size_t(5) * p.fundamental * 4, cudaMemcpyDeviceToHost),
                                "snapshot")))
        return st;
    return BRP_OK;
}

static void sort_candidates(brp_candidate* c, size_t n) {
    std::sort(c, c + n, [](const brp_candidate& a, const brp_candidate& b) {
        return a.level != b.level ? a.level < b.level : a.bin < b.bin;
    });
}

extern "C" int brp_cuda_candidates(brp_ctx* c, uint32_t slot, brp_candidate* out, uint32_t cap, uint32_t* count) {
    if (!c || !count) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    if (slot == UINT32_MAX) slot = c->last_count ? c->last_count - 1 : 0;
    if (slot >= c->last_count) return c->fail(BRP_E_RUNTIME, "candidate slot outside executed batch");
    int st;
    if ((st = c->cuda(cudaSetDevice(c->device), "cudaSetDevice")) || (st = settle_pending(c))) return st;
    uint32_t hdr[2];
    if ((st = c->cuda(cudaMemcpy(&hdr[0], c->d_counts + slot, 4, cudaMemcpyDeviceToHost), "candidates")) ||
        (st = c->cuda(cudaMemcpy(&hdr[1], c->d_status + slot, 4, cudaMemcpyDeviceToHost), "candidates")))
        return st;
    *count = hdr[0];
    if (hdr[1] || hdr[0] > c->base.capacity)
        return c->fail(BRP_E_RESULT, "GPU invalid resample index or candidate overflow; no valid result");
    std::vector<brp_candidate> tmp(hdr[0]);
    if (hdr[0] && (st = c->cuda(cudaMemcpy(tmp.data(), c->d_cands + size_t(slot) * c->base.capacity,
                                           size_t(hdr[0]) * sizeof(brp_candidate), cudaMemcpyDeviceToHost),
                                "candidates")))
        return st;
    sort_candidates(tmp.data(), tmp.size());
    if (out) std::memcpy(out, tmp.data(), std::min<size_t>(cap, tmp.size()) * sizeof(brp_candidate));
    return BRP_OK;
}

extern "C" int brp_cuda_device_info(brp_ctx* c, char* buffer, size_t length) {
    if (!c || !buffer || !length) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    cudaDeviceProp prop{};
    int st;
    if ((st = c->cuda(cudaGetDeviceProperties(&prop, c->device), "cudaGetDeviceProperties"))) return st;
    int rt = 0, drv = 0;
    cudaRuntimeGetVersion(&rt);
    cudaDriverGetVersion(&drv);
    snprintf(buffer, length,
             "%s; CUDA sm_%d%d; SMs=%d; runtime=%d; driver=%d; shared_per_block_optin=%zu; L2=%d; pipeline=%s; "
             "decomposition=%ux%u; pass1=%d; pass2=%d",
             prop.name, prop.major, prop.minor, prop.multiProcessorCount, rt, drv, prop.sharedMemPerBlockOptin,
             prop.l2CacheSize, c->fused ? "fused" : "plain", c->lp.L1, c->lp.L2, c->lp.fp1 ? c->lp.fp1->id : -1,
             c->lp.fp2 ? c->lp.fp2->id : -1);
    return BRP_OK;
}

extern "C" uint64_t brp_cuda_allocated_bytes(const brp_ctx* c) { return c ? c->allocated : 0; }

extern "C" int brp_cuda_profile_counters(brp_ctx* c, char* buffer, size_t length) {
    if (!c || !buffer || !length) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    snprintf(buffer, length,
             "{\"source\": \"cuda events\", \"templates\": %u, \"stage_ms\": {\"resample\": %.6f, \"fft\": %.6f, "
             "\"power\": %.6f, \"harmonic_candidate\": %.6f}}",
             c->last_count, c->last_stage_ms[0], c->last_stage_ms[1], c->last_stage_ms[2], c->last_stage_ms[3]);
    return BRP_OK;
}

// ===================================================================== bank
struct brp_bank {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t side = nullptr;  // second chain of the graph
    cudaEvent_t fork = nullptr, join = nullptr;
    std::vector<uint32_t> n, unpadded;
    // Two device buffers per series: an upload while a submitted run is in
    // flight goes to the buffer that run does not read (on the copy stream,
    // ordered before the next run by an event).
    std::vector<float*> d_series[2];
    std::vector<int> latest;              // per series: buffer holding the latest upload
    std::vector<int> in_use;              // per series: buffer the in-flight run reads (-1: none)
    std::vector<cudaEvent_t> series_ready;
    cudaStream_t copy = nullptr;
    bool inflight = false;                // a submitted run awaits brp_cuda_bank_wait
    std::vector<uint32_t> run_order;      // the in-flight run's slot -> caller index
    std::map<uint32_t, LengthPlan> plans;  // by n
    struct ClassBuffers {
        float2* work = nullptr;
        float* power = nullptr;
        double* partial = nullptr;
        uint32_t group = 0;                 // templates per launch
        uint32_t chains = 1;                // independent launch chains (streams) in the graph
        uint32_t capacity = 0;              // templates the buffers hold (group * chains)
        uint32_t partial_per_template = 0;  // pass-1 partial sums per template
    };
    std::map<uint32_t, ClassBuffers> classes;
    uint32_t max_templates = 0, capacity = 0;
    std::vector<void*> allocations;
    brp_params* d_params = nullptr;
    const float** d_inputs = nullptr;
    uint32_t *d_counts = nullptr, *d_status = nullptr;
    float* d_mean = nullptr;
    uint32_t* d_tickets = nullptr;  // pass-1 CTA tickets per template (zero between runs)
    brp_candidate* d_cands = nullptr;
    brp_candidate* d_compact = nullptr;
    uint64_t* d_offsets = nullptr;
    uint32_t* d_rank = nullptr;  // per result slot: the caller's index of its template
    uint64_t compact_cap = 0;
    // toplist pre-filter (off while filter_rows == 0)
    uint32_t filter_rows = 0;
    uint32_t *d_slot_series = nullptr, *h_slot_series = nullptr, *h_kept = nullptr;
    FilterArgs filter{};
    brp_params* h_params = nullptr;
    const float** h_inputs = nullptr;
    uint32_t* h_counts = nullptr;
    uint64_t* h_offsets = nullptr;
    uint32_t* h_rank = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<uint64_t> graph_key;
    uint32_t kernels_per_run = 0;
    std::vector<uint32_t> last_sorted_n, last_spans;
    uint32_t last_count = 0;
    cudaEvent_t done = nullptr;
    uint32_t wait_polls = kDefaultWaitPolls;   // device: first-wait poll bound of the kernels
    double wait_seconds = kDefaultWaitSeconds; // host: deadline of a run or profile replay
    cudaEvent_t pending = nullptr;             // completion of a run that passed its deadline
    std::string error;

    // A run has finished on the device: its series buffers may be written again.
    void run_finished() { std::fill(in_use.begin(), in_use.end(), -1); }
    int fail(int code, const std::string& msg) {
        error = msg;
        g_thread_error = msg;
        return code;
    }
    int cuda(cudaError_t e, const char* what) {
        if (e == cudaSuccess) return BRP_OK;
        return fail(BRP_E_RUNTIME, std::string(what) + ": " + cudaGetErrorString(e));
    }
    template <class T>
    int alloc(T** p, size_t count, const char* what) {
        if (alloc_fault_due() ||
            cudaMalloc(reinterpret_cast<void**>(p), std::max<size_t>(count * sizeof(T), 16)) != cudaSuccess)
            return fail(BRP_E_RUNTIME, std::string("cudaMalloc failed: ") + what);
        allocations.push_back(*p);
        return BRP_OK;
    }
    // Frees one buffer of alloc() (the caller has synchronised the stream and
    // dropped every graph that references it).
    void release(void* p) {
        auto it = std::find(allocations.begin(), allocations.end(), p);
        if (it == allocations.end()) return;
        cudaFree(p);
        allocations.erase(it);
    }
    // The captured graph references the class buffers, plan tables and filter
    // state of the last run; a change to any of them drops it, so that
    // brp_cuda_bank_launch cannot replay a stale graph and the next run captures.
    void drop_graph() {
        if (exec) { cudaGraphExecDestroy(exec); exec = nullptr; }
        if (graph) { cudaGraphDestroy(graph); graph = nullptr; }
        graph_key.clear();
    }
    ~brp_bank() {
        cudaSetDevice(device);
        if (copy) cudaStreamSynchronize(copy);
        if (stream) cudaStreamSynchronize(stream);
        for (auto e : series_ready) cudaEventDestroy(e);
        if (copy) cudaStreamDestroy(copy);
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (done) cudaEventDestroy(done);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        if (side) cudaStreamDestroy(side);
        for (auto p : allocations) cudaFree(p);
        for (auto& kv : plans) free_length_plan(kv.second);
        if (h_params) cudaFreeHost(h_params);
        if (h_inputs) cudaFreeHost(h_inputs);
        if (h_counts) cudaFreeHost(h_counts);
        if (h_offsets) cudaFreeHost(h_offsets);
        if (h_rank) cudaFreeHost(h_rank);
        if (h_slot_series) cudaFreeHost(h_slot_series);
        if (h_kept) cudaFreeHost(h_kept);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" const char* brp_cuda_bank_last_error(const brp_bank* b) { return b ? b->error.c_str() : g_thread_error.c_str(); }

// Templates of one length class run in groups of `group` templates per launch;
// the class's intermediate buffers hold one group.
static uint32_t default_group(uint32_t n) {
    // Templates per launch when the caller does not configure the class: long
    // launches amortise each kernel's partial last wave (the autotuner picks
    // 64-128 on one B200).  Intermediates take 6n bytes per template: 3 GiB
    // for 128 templates at n = 2^22.
    return n >= (1u << 22) ? 128 : 64;
}

extern "C" int brp_cuda_bank_create(uint32_t series_count, const uint32_t* n, const uint32_t* unpadded,
                                    uint32_t max_templates, uint32_t capacity, int32_t device, brp_bank** out) {
    if (!n || !unpadded || !out || !series_count || !max_templates || !capacity)
        return set_thread_error(BRP_E_ARGUMENT, "invalid bank arguments");
    *out = nullptr;
    auto* b = new (std::nothrow) brp_bank;
    if (!b) return set_thread_error(BRP_E_RUNTIME, "out of host memory");
    auto cleanup = [&](int code) { std::string m = b->error; delete b; return set_thread_error(code, m); };
    b->device = device;
    if (b->device < 0) cudaGetDevice(&b->device);
    int st;
    if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice"))) return cleanup(st);
    if ((st = b->cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate"))) return cleanup(st);
    if ((st = b->cuda(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "cudaEventCreate"))) return cleanup(st);
    if ((st = b->cuda(cudaStreamCreateWithFlags(&b->copy, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (st = b->cuda(cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking), "cudaStreamCreate")) ||
        (st = b->cuda(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "cudaEventCreate")) ||
        (st = b->cuda(cudaEventCreateWithFlags(&b->join, cudaEventDisableTiming), "cudaEventCreate")))
        return cleanup(st);
    b->n.assign(n, n + series_count);
    b->unpadded.assign(unpadded, unpadded + series_count);
    b->max_templates = max_templates;
    b->capacity = capacity;
    for (uint32_t s = 0; s < series_count; ++s) {
        if (unpadded[s] < 2 || unpadded[s] > n[s]) return b->fail(BRP_E_ARGUMENT, "invalid series length"), cleanup(BRP_E_ARGUMENT);
        float *d0 = nullptr, *d1 = nullptr;
        cudaEvent_t ev = nullptr;
        if ((st = b->alloc(&d0, unpadded[s], "series")) || (st = b->alloc(&d1, unpadded[s], "series")) ||
            (st = b->cuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate")))
            return cleanup(st);
        b->d_series[0].push_back(d0);
        b->d_series[1].push_back(d1);
        b->series_ready.push_back(ev);
        b->latest.push_back(0);
        b->in_use.push_back(-1);
        if (!b->plans.count(n[s])) {
            std::string e = make_length_plan(n[s], b->plans[n[s]], b->stream);
            if (!e.empty()) { b->fail(BRP_E_ARGUMENT, e); return cleanup(BRP_E_ARGUMENT); }
            if (!b->plans[n[s]].fused) { b->fail(BRP_E_ARGUMENT, "bank search needs n >= 8192"); return cleanup(BRP_E_ARGUMENT); }
        }
    }
    for (auto& kv : b->plans) {
        const LengthPlan& lp = kv.second;
        brp_bank::ClassBuffers cb;
        cb.group = std::min(default_group(lp.n), max_templates);
        CachedPlan cp;  // a tuned plan of this length: its templates per launch and chains too
        if (lp.fp1 && lp.fp2 && cached_plan(lp.n, cp) && cp.pass1 == lp.fp1->id && cp.pass2 == lp.fp2->id &&
            cp.group > 0) {
            cb.group = std::min(cp.group, max_templates);
            cb.chains = std::min<uint32_t>(std::max<uint32_t>(cp.chains, 1), 2);
        }
        cb.capacity = cb.group * cb.chains;  // every chain has its own intermediates
        cb.partial_per_template = std::max<uint32_t>(lp.blocks1(), lp.M / 64);
        if ((st = b->alloc(&cb.work, size_t(cb.capacity) * lp.M, "work")) ||
            (st = b->alloc(&cb.power, size_t(cb.capacity) * lp.M, "power")) ||
            (st = b->alloc(&cb.partial, size_t(cb.capacity) * cb.partial_per_template, "partial")))
            return cleanup(st);
        b->classes[kv.first] = cb;
    }
    b->compact_cap = uint64_t(max_templates) * capacity;
    if ((st = b->alloc(&b->d_params, max_templates, "params")) || (st = b->alloc(&b->d_inputs, max_templates, "inputs")) ||
        (st = b->alloc(&b->d_counts, max_templates, "counts")) || (st = b->alloc(&b->d_status, max_templates, "status")) ||
        (st = b->alloc(&b->d_mean, max_templates, "mean")) || (st = b->alloc(&b->d_tickets, max_templates, "tickets")) ||
        (st = b->cuda(cudaMemset(b->d_tickets, 0, size_t(max_templates) * 4), "tickets clear")) ||
        (st = b->alloc(&b->d_cands, size_t(max_templates) * capacity, "candidates")) ||
        (st = b->alloc(&b->d_compact, b->compact_cap, "compact")) ||
        (st = b->alloc(&b->d_offsets, size_t(max_templates) + 1, "offsets")) ||
        (st = b->alloc(&b->d_rank, max_templates, "rank")) ||
        (st = b->cuda(set_bank_compact_attributes(capacity), "compaction shared memory")))
        return cleanup(st);
    if ((st = b->cuda(cudaMallocHost(&b->h_params, max_templates * sizeof(brp_params)), "cudaMallocHost")) ||
        (st = b->cuda(cudaMallocHost(&b->h_inputs, max_templates * sizeof(void*)), "cudaMallocHost")) ||
        (st = b->cuda(cudaMallocHost(&b->h_counts, 2 * max_templates * sizeof(uint32_t)), "cudaMallocHost")) ||
        (st = b->cuda(cudaMallocHost(&b->h_offsets, (max_templates + 1) * sizeof(uint64_t)), "cudaMallocHost")) ||
        (st = b->cuda(cudaMallocHost(&b->h_rank, max_templates * sizeof(uint32_t)), "cudaMallocHost")))
        return cleanup(st);
    *out = b;
    return BRP_OK;
}

extern "C" void brp_cuda_bank_destroy(brp_bank* b) { delete b; }

extern "C" int brp_cuda_bank_set_series(brp_bank* b, uint32_t s, const float* input) {
    if (!b || !input) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    if (s >= b->latest.size()) return b->fail(BRP_E_ARGUMENT, "series index out of range");
    int st;
    if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice"))) return st;
    // Into the buffer no in-flight run reads; runs submitted later read it.
    const int target = b->in_use[s] >= 0 ? 1 - b->in_use[s] : b->latest[s];
    if ((st = b->cuda(cudaMemcpyAsync(b->d_series[target][s], input, size_t(b->unpadded[s]) * 4,
                                      cudaMemcpyHostToDevice, b->copy),
                      "series upload")) ||
        (st = b->cuda(cudaEventRecord(b->series_ready[s], b->copy), "series upload")))
        return st;
    b->latest[s] = target;
    return BRP_OK;
}

// Records the whole bank search on b->stream (captured into the graph).  With
// `prof` (eager replay only) each kernel is bracketed by events: prof->push_back
// gets (kind, start, end) with kind 0 = pass 1, 1 = pass 2, 2 = harmonic, 3 = compaction.
struct KernelEvents { std::vector<int> kind; std::vector<cudaEvent_t> ev; };
static void record_bank(brp_bank* b, const std::vector<uint32_t>& sorted_n, const std::vector<uint32_t>& spans,
                        uint32_t count, KernelEvents* prof = nullptr) {
    cudaStream_t s = b->stream;
    auto mark = [&](int kind, bool start) {
        if (!prof) return;
        cudaEvent_t e;
        cudaEventCreate(&e);
        cudaEventRecord(e, s);
        prof->ev.push_back(e);
        if (start) prof->kind.push_back(kind);
    };
    cudaMemsetAsync(b->d_counts, 0, count * sizeof(uint32_t), s);
    cudaMemsetAsync(b->d_status, 0, count * sizeof(uint32_t), s);
    // Groups of a class alternate between the chains (the main stream and the
    // side stream), each chain with its own intermediate buffers, so that one
    // group's kernels overlap another's.  Profiling replays use one chain.
    bool forked = false;
    uint32_t kernels = 0;
    uint32_t t = 0;
    std::map<uint32_t, uint32_t> groups_done;
    while (t < count) {
        const uint32_t n = sorted_n[t];
        const LengthPlan& lp = b->plans.at(n);
        const brp_bank::ClassBuffers& cb = b->classes.at(n);
        uint32_t end = t;
        while (end < count && sorted_n[end] == n && end - t < cb.group) ++end;
        const uint32_t g = end - t;
        const uint32_t chain = prof ? 0 : groups_done[n]++ % cb.chains;
        cudaStream_t cs = s;
        if (chain == 1) {
            if (!forked) {
                cudaEventRecord(b->fork, s);
                cudaStreamWaitEvent(b->side, b->fork, 0);
                forked = true;
            }
            cs = b->side;
        }
        FusedArgs a{};
        a.inputs = b->d_inputs + t;
        a.params = b->d_params + t;
        fill_fused_args(a, lp);
        a.work = cb.work + size_t(chain) * cb.group * lp.M; a.work_stride = lp.M;
        a.power = cb.power + size_t(chain) * cb.group * lp.M; a.power_stride = lp.M;
        a.partial = cb.partial + size_t(chain) * cb.group * cb.partial_per_template;
        a.partial_stride = lp.blocks1();
        a.mean = b->d_mean + t; a.tickets = b->d_tickets + t;
        a.status = b->d_status + t; a.counts = b->d_counts + t;
        a.cands = b->d_cands + size_t(t) * b->capacity;
        a.capacity = b->capacity;
        a.snap = -1;
        a.wait_polls = b->wait_polls;
        uint32_t span = 0;
        for (uint32_t u = t; u < end; ++u) span = std::max(span, spans[u]);
        mark(0, true);
        launch_fused_pass1(a, lp, g, cs);
        mark(0, false);
        mark(1, true);
        launch_fused_pass2(a, lp, g, cs);
        mark(1, false);
        mark(2, true);
        launch_fused_harmonic(a, lp, g, span, cs);
        mark(2, false);
        kernels += 3;
        t = end;
    }
    if (forked) {
        cudaEventRecord(b->join, b->side);
        cudaStreamWaitEvent(s, b->join, 0);
    }
    mark(3, true);
    const FilterArgs* filter = nullptr;
    if (b->filter_rows) {
        b->filter.counts = b->d_counts; b->filter.cands = b->d_cands; b->filter.capacity = b->capacity;
        b->filter.count = count; b->filter.slot_series = b->d_slot_series;
        launch_toplist_filter(b->filter, s);
        filter = &b->filter;
        kernels += 4;
    }
    launch_bank_compact(b->d_counts, b->d_cands, b->capacity, count, b->d_rank, b->d_compact, b->compact_cap,
                        b->d_offsets, filter, s);
    mark(3, false);
    b->kernels_per_run = kernels + 1;
}

extern "C" int brp_cuda_bank_submit(brp_bank* b, const brp_params* templates, const uint32_t* series_of,
                                    uint32_t count) {
    if (!b || !templates || !series_of) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    if (!count || count > b->max_templates) return b->fail(BRP_E_ARGUMENT, "template count outside 1..max_templates");
    if (b->inflight) return b->fail(BRP_E_ARGUMENT, "a submitted run awaits brp_cuda_bank_wait");
    int st;
    if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice"))) return st;
    // The pinned staging buffers below are the sources and targets of the
    // previous run's copies: a run past its deadline must have finished first.
    if ((st = settle_pending(b))) return st;
    // Order templates by length class (stable), remembering the caller's order.
    std::vector<uint32_t> order(count);
    for (uint32_t t = 0; t < count; ++t) {
        order[t] = t;
        const uint32_t s = series_of[t];
        if (s >= b->n.size()) return b->fail(BRP_E_ARGUMENT, "series index out of range");
        const brp_params& p = templates[t];
        if (p.n != b->n[s] || p.unpadded != b->unpadded[s]) return b->fail(BRP_E_ARGUMENT, "template does not match its series");
        std::string v = validate_dims(p);
        if (!v.empty()) return b->fail(BRP_E_ARGUMENT, v);
    }
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t x, uint32_t y) { return b->n[series_of[x]] > b->n[series_of[y]]; });
    // every chain of a class writes its own group of intermediates
    for (const auto& kv : b->classes)
        if (uint64_t(kv.second.group) * kv.second.chains > kv.second.capacity)
            return b->fail(BRP_E_RUNTIME, "bank class buffers smaller than its groups and chains");
    std::vector<uint32_t> sorted_n(count), spans(count);
    std::vector<uint64_t> key;
    key.push_back(count);
    key.push_back(b->filter_rows);
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t t = order[k];
        b->h_rank[k] = t;
        if (b->h_slot_series) b->h_slot_series[k] = series_of[t];
        b->h_params[k] = templates[t];
        b->h_params[k].capacity = b->capacity;
        b->h_inputs[k] = b->d_series[b->latest[series_of[t]]][series_of[t]];
        sorted_n[k] = b->n[series_of[t]];
        spans[k] = std::max(templates[t].fundamental, templates[t].harmonic + 8);
        key.push_back((uint64_t(sorted_n[k]) << 32) | spans[k]);
    }
    cudaStream_t s = b->stream;
    // the series uploads (copy stream) before the run
    std::vector<char> used(b->latest.size(), 0);
    for (uint32_t t = 0; t < count; ++t) used[series_of[t]] = 1;
    for (size_t q = 0; q < used.size(); ++q)
        if (used[q] && (st = b->cuda(cudaStreamWaitEvent(s, b->series_ready[q], 0), "series upload wait")))
            return st;
    if ((st = b->cuda(cudaMemcpyAsync(b->d_params, b->h_params, count * sizeof(brp_params), cudaMemcpyHostToDevice, s),
                      "params upload")) ||
        (st = b->cuda(cudaMemcpyAsync(b->d_inputs, b->h_inputs, count * sizeof(void*), cudaMemcpyHostToDevice, s),
                      "inputs upload")) ||
        (st = b->cuda(cudaMemcpyAsync(b->d_rank, b->h_rank, count * sizeof(uint32_t), cudaMemcpyHostToDevice, s),
                      "rank upload")) ||
        (b->filter_rows &&
         (st = b->cuda(cudaMemcpyAsync(b->d_slot_series, b->h_slot_series, count * sizeof(uint32_t),
                                       cudaMemcpyHostToDevice, s),
                       "slot series upload"))))
        return st;
    b->last_sorted_n = sorted_n;
    b->last_spans = spans;
    b->last_count = count;
    if (key != b->graph_key || !b->exec) {
        if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
        if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
        if ((st = b->cuda(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal), "begin capture"))) return st;
        record_bank(b, sorted_n, spans, count);
        cudaError_t e = cudaStreamEndCapture(s, &b->graph);
        if ((st = b->cuda(e, "end capture"))) return st;
        if ((st = b->cuda(cudaGraphInstantiate(&b->exec, b->graph, 0), "graph instantiate"))) return st;
        b->graph_key = key;
    }
    if ((st = b->cuda(cudaGraphLaunch(b->exec, s), "graph launch"))) return st;
    uint32_t* h_status = b->h_counts + b->max_templates;
    cudaMemcpyAsync(b->h_counts, b->d_counts, count * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_status, b->d_status, count * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(b->h_offsets, b->d_offsets, (count + 1) * 8, cudaMemcpyDeviceToHost, s);
    if (b->filter_rows) cudaMemcpyAsync(b->h_kept, b->filter.kept, count * 4, cudaMemcpyDeviceToHost, s);
    if ((st = b->cuda(cudaEventRecord(b->done, s), "bank search"))) return st;
    for (size_t q = 0; q < used.size(); ++q) b->in_use[q] = used[q] ? b->latest[q] : -1;
    b->run_order = order;
    b->inflight = true;
    return BRP_OK;
}

extern "C" int brp_cuda_bank_wait(brp_bank* b, brp_candidate* out, uint64_t out_cap, uint32_t* counts,
                                  uint32_t* status) {
    if (!b || !counts || !status) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    if (!b->inflight) return b->fail(BRP_E_ARGUMENT, "no submitted run to wait for");
    int st;
    if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice"))) return st;
    // The run is over for the caller whatever the outcome.  Its series buffers
    // stay marked in use until it has finished on the device (below, or when
    // the next call settles a run that passed its deadline).
    b->inflight = false;
    const std::vector<uint32_t>& order = b->run_order;
    const uint32_t count = uint32_t(order.size());
    uint32_t* h_status = b->h_counts + b->max_templates;
    bool timed_out = false;
    cudaError_t e = wait_event(b->done, b->wait_seconds, &timed_out);
    if (timed_out) {
        b->pending = b->done;  // the next submit waits for it before it reuses the staging buffers
        return b->fail(BRP_E_TIMEOUT, "bank search exceeded its deadline");
    }
    std::fill(b->in_use.begin(), b->in_use.end(), -1);
    if ((st = b->cuda(e, "bank search"))) return st;
    // The compaction wrote the lists in the caller's order, each sorted by
    // (level, bin); offsets are by caller index.
    const uint64_t total = b->h_offsets[count];
    if (out && total && (st = b->cuda(cudaMemcpy(out, b->d_compact, std::min<uint64_t>(total, out_cap) *
                                                 sizeof(brp_candidate), cudaMemcpyDeviceToHost),
                                      "candidates download")))
        return st;
    bool bad = false;
    for (uint32_t k = 0; k < count; ++k) {
        const uint32_t t = order[k];
        const uint32_t kept = b->filter_rows ? b->h_kept[k] : std::min(b->h_counts[k], b->capacity);
        counts[t] = b->filter_rows ? kept : b->h_counts[k];
        status[t] = h_status[k] | (b->h_counts[k] > b->capacity ? uint32_t(BRP_STATUS_OVERFLOW) : 0u);
        if (status[t]) bad = true;
        const uint64_t first = b->h_offsets[t];
        if (out && kept > kCompactSortMax && first + kept <= out_cap) sort_candidates(out + first, kept);
    }
    if (total > out_cap) return b->fail(BRP_E_RESULT, "candidate output buffer too small");
    if (bad) return b->fail(BRP_E_RESULT, "GPU invalid resample index or candidate overflow; no valid result");
    return BRP_OK;
}

extern "C" int brp_cuda_bank_run(brp_bank* b, const brp_params* templates, const uint32_t* series_of, uint32_t count,
                                 brp_candidate* out, uint64_t out_cap, uint32_t* counts, uint32_t* status) {
    if (!b || !templates || !series_of || !counts || !status) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    const int st = brp_cuda_bank_submit(b, templates, series_of, count);
    return st ? st : brp_cuda_bank_wait(b, out, out_cap, counts, status);
}

// Calls that change or read the bank's buffers wait until a submitted run is collected.
static int refuse_inflight(brp_bank* b) {
    return b->inflight ? b->fail(BRP_E_ARGUMENT, "a submitted run awaits brp_cuda_bank_wait") : BRP_OK;
}

extern "C" int brp_cuda_bank_configure(brp_bank* b, uint32_t n, int32_t pass1, int32_t pass2, uint32_t group,
                                       uint32_t chains) {
    if (!b) return set_thread_error(BRP_E_ARGUMENT, "null bank");
    if (refuse_inflight(b)) return BRP_E_ARGUMENT;
    auto it = b->plans.find(n);
    if (it == b->plans.end()) return b->fail(BRP_E_ARGUMENT, "no series of that length");
    int st;
    if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice"))) return st;
    if ((st = b->cuda(cudaStreamSynchronize(b->stream), "bank configure"))) return st;
    LengthPlan lp;
    std::string e = make_length_plan(n, lp, b->stream, pass1, pass2);
    if (!e.empty()) { free_length_plan(lp); return b->fail(BRP_E_ARGUMENT, e); }
    if (!lp.fused) { free_length_plan(lp); return b->fail(BRP_E_ARGUMENT, "no fused plan for that configuration"); }
    brp_bank::ClassBuffers& cb = b->classes.at(n);
    const uint32_t g = group ? std::min(group, b->max_templates) : cb.group;
    const uint32_t ch = chains ? std::min(chains, 2u) : cb.chains;
    b->drop_graph();  // it references the plan tables freed below
    if (g * ch > cb.capacity || lp.blocks1() > cb.partial_per_template) {
        // grow the class buffers; the old ones are freed once the new ones exist
        brp_bank::ClassBuffers nb;
        nb.capacity = std::max(g * ch, cb.capacity);
        nb.partial_per_template = std::max(lp.blocks1(), cb.partial_per_template);
        if ((st = b->alloc(&nb.work, size_t(nb.capacity) * lp.M, "work")) ||
            (st = b->alloc(&nb.power, size_t(nb.capacity) * lp.M, "power")) ||
            (st = b->alloc(&nb.partial, size_t(nb.capacity) * nb.partial_per_template, "partial"))) {
            b->release(nb.work); b->release(nb.power); b->release(nb.partial);
            free_length_plan(lp);
            return st;
        }
        b->release(cb.work); b->release(cb.power); b->release(cb.partial);
        cb.work = nb.work; cb.power = nb.power; cb.partial = nb.partial;
        cb.capacity = nb.capacity; cb.partial_per_template = nb.partial_per_template;
    }
    cb.group = g;
    cb.chains = ch;
    free_length_plan(it->second);
    it->second = lp;
    return BRP_OK;
}

extern "C" int brp_cuda_bank_set_toplist_filter(brp_bank* b, uint32_t rows) {
    if (!b) return set_thread_error(BRP_E_ARGUMENT, "null bank");
    if (refuse_inflight(b)) return BRP_E_ARGUMENT;
    int st;
    if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice"))) return st;
    if ((st = b->cuda(cudaStreamSynchronize(b->stream), "toplist filter"))) return st;
    if (rows && !b->filter.maxkey) {
        // Per series the per-bin arrays of its five levels, n/2 bins each.
        const uint32_t S = uint32_t(b->n.size());
        std::vector<uint64_t> base(S);
        std::vector<uint32_t> half(S);
        uint64_t total = 0;
        for (uint32_t s = 0; s < S; ++s) { base[s] = total; half[s] = b->n[s] / 2; total += 5ull * half[s]; }
        if (total >= (1ull << 32)) return b->fail(BRP_E_ARGUMENT, "toplist filter: series too long");
        // Everything is allocated and initialised into locals first and committed
        // to the bank only when all of it succeeded, so a failed set-up leaves
        // the filter off and a later call starts it afresh.
        FilterArgs f = b->filter;
        uint32_t* slot_series = nullptr;
        uint64_t* d_base = nullptr;
        uint32_t* d_half = nullptr;
        uint32_t *h_slot = nullptr, *h_kept = nullptr;
        if ((st = b->alloc(&f.maxkey, total, "filter")) || (st = b->alloc(&f.flag, total, "filter")) ||
            (st = b->alloc(&f.owners, total, "filter")) || (st = b->alloc(&f.owner_count, size_t(S) * 5, "filter")) ||
            (st = b->alloc(&f.threshold_key, size_t(S) * 5, "filter")) ||
            (st = b->alloc(&f.kept, b->max_templates, "filter")) ||
            (st = b->alloc(&slot_series, b->max_templates, "filter")) || (st = b->alloc(&d_base, S, "filter")) ||
            (st = b->alloc(&d_half, S, "filter")) ||
            (st = b->cuda(cudaMemset(f.maxkey, 0, total * 4), "filter clear")) ||
            (st = b->cuda(cudaMemset(f.flag, 0, total * 4), "filter clear")) ||
            (st = b->cuda(cudaMemset(f.owner_count, 0, size_t(S) * 5 * 4), "filter clear")) ||
            (st = b->cuda(cudaMemcpy(d_base, base.data(), S * 8, cudaMemcpyHostToDevice), "filter upload")) ||
            (st = b->cuda(cudaMemcpy(d_half, half.data(), S * 4, cudaMemcpyHostToDevice), "filter upload")) ||
            (st = b->cuda(cudaMallocHost(&h_slot, b->max_templates * sizeof(uint32_t)), "cudaMallocHost")) ||
            (st = b->cuda(cudaMallocHost(&h_kept, b->max_templates * sizeof(uint32_t)), "cudaMallocHost"))) {
            for (void* p : {(void*)f.maxkey, (void*)f.flag, (void*)f.owners, (void*)f.owner_count,
                            (void*)f.threshold_key, (void*)f.kept, (void*)slot_series, (void*)d_base, (void*)d_half})
                if (p) b->release(p);
            if (h_slot) cudaFreeHost(h_slot);
            if (h_kept) cudaFreeHost(h_kept);
            return st;
        }
        f.base = d_base;
        f.half = d_half;
        f.series = S;
        b->filter = f;
        b->d_slot_series = slot_series;
        b->h_slot_series = h_slot;
        b->h_kept = h_kept;
    }
    b->filter_rows = rows;
    b->filter.rows = rows;
    b->drop_graph();
    return BRP_OK;
}

extern "C" int brp_cuda_fast_configs(int32_t* ids, uint32_t* lengths, uint32_t* kinds, uint32_t cap) {
    uint32_t k = 0;
    for (int kind = 1; kind <= 2; ++kind)
        for (auto& f : kind == 1 ? fast_pass1_configs() : fast_pass2_configs()) {
            if (k < cap) {
                if (ids) ids[k] = f.id;
                if (lengths) lengths[k] = f.L;
                if (kinds) kinds[k] = uint32_t(kind == 1 && f.tensor ? 3 : kind);
            }
            ++k;
        }
    return int(k);
}

extern "C" int brp_cuda_bank_launch(brp_bank* b) {
    if (!b) return set_thread_error(BRP_E_ARGUMENT, "null bank");
    if (refuse_inflight(b)) return BRP_E_ARGUMENT;
    if (!b->exec) return b->fail(BRP_E_ARGUMENT, "no captured bank graph (run the bank after configuring it)");
    return b->cuda(cudaGraphLaunch(b->exec, b->stream), "graph launch");
}

extern "C" int brp_cuda_bank_profile(brp_bank* b, double* kernel_ms, uint32_t* launches) {
    if (!b || !kernel_ms) return set_thread_error(BRP_E_ARGUMENT, "null argument");
    if (refuse_inflight(b)) return BRP_E_ARGUMENT;
    if (!b->last_count) return b->fail(BRP_E_ARGUMENT, "no bank run to profile");
    int st;
    if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) || (st = settle_pending(b))) return st;
    KernelEvents prof;
    record_bank(b, b->last_sorted_n, b->last_spans, b->last_count, &prof);
    cudaEventRecord(b->done, b->stream);
    bool timed_out = false;
    cudaError_t e = wait_event(b->done, b->wait_seconds, &timed_out);
    if (timed_out) {
        b->pending = b->done;
        for (auto ev : prof.ev) cudaEventDestroy(ev);  // released once the replay reaches them
        return b->fail(BRP_E_TIMEOUT, "bank profile exceeded its deadline");
    }
    if ((st = b->cuda(e, "bank profile"))) return st;
    for (int k = 0; k < 4; ++k) { kernel_ms[k] = 0; if (launches) launches[k] = 0; }
    for (size_t i = 0; i < prof.kind.size(); ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, prof.ev[2 * i], prof.ev[2 * i + 1]);
        kernel_ms[prof.kind[i]] += ms;
        if (launches) launches[prof.kind[i]] += 1;
    }
    for (auto ev : prof.ev) cudaEventDestroy(ev);
    return BRP_OK;
}

extern "C" void* brp_cuda_bank_stream(brp_bank* b) { return b ? static_cast<void*>(b->stream) : nullptr; }
extern "C" uint32_t brp_cuda_bank_kernels_per_run(const brp_bank* b) { return b ? b->kernels_per_run : 0; }

// ============================================================ wait limits
template <class Obj>
static int set_wait_limits(Obj* o, uint32_t device_polls, double host_seconds) {
    std::string v = validate_wait_limits(host_seconds);
    if (!v.empty()) return o->fail(BRP_E_ARGUMENT, v);
    o->wait_polls = device_polls;
    o->wait_seconds = host_seconds;
    return BRP_OK;
}

extern "C" int brp_cuda_set_wait_limits(brp_ctx* c, uint32_t device_polls, double host_seconds) {
    if (!c) return set_thread_error(BRP_E_ARGUMENT, "null context");
    return set_wait_limits(c, device_polls, host_seconds);
}

extern "C" int brp_cuda_bank_set_wait_limits(brp_bank* b, uint32_t device_polls, double host_seconds) {
    if (!b) return set_thread_error(BRP_E_ARGUMENT, "null bank");
    if (refuse_inflight(b)) return BRP_E_ARGUMENT;
    const uint32_t before = b->wait_polls;
    int st = set_wait_limits(b, device_polls, host_seconds);
    if (!st && before != device_polls) {
        // the poll bound is a launch argument of the captured kernels
        if ((st = b->cuda(cudaSetDevice(b->device), "cudaSetDevice")) ||
            (st = b->cuda(cudaStreamSynchronize(b->stream), "wait limits")))
            return st;
        b->drop_graph();
    }
    return st;
}

extern "C" void brp_cuda_debug_fail_allocation(uint32_t after) { g_alloc_countdown.store(after); }
