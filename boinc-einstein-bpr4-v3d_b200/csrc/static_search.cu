// brp_cuda_search_static: the per-template fused search (resampling, packed
// real FFT, power spectrum, harmonic summing, candidate compaction) for callers
// that cannot allocate device memory.  Some hosts forbid cudaMalloc once they
// are running -- a plugin that may only use the buffers its host hands it, a
// process whose device memory is owned by another framework's pool, a
// real-time loop that must not block in the allocator.  This entry point takes
// the series, the power-spectrum buffer and the candidate buffers from the
// caller and keeps all of its own working memory (the four-step FFT
// intermediate, the per-CTA partial sums, the twiddle tables and the launch
// arguments) in one file-scope device array, g_scratch, of fixed size.
//
// The array is part of the module: every GPU that loads the library holds it
// (kScratchBytes, about 4.2 MiB) until the process exits.  Host code only sees
// a stand-in for it; its device address comes from cudaGetSymbolAddress, once
// per device, with that device current.  The cached address and the tables
// copied into the array belong to the device's context: after a
// cudaDeviceReset in the same process the entry point must not be called
// again on that device.
//
// Per call, the template constants and the series pointer reach the array
// through one single-thread kernel that takes them by value (no host staging
// buffer), so a call after set-up only enqueues kernels on the caller's
// stream and returns.
#include <cstdint>
#include <cstring>
#include <mutex>
#include "brp_internal.h"

namespace brp {
namespace {

constexpr uint32_t kStaticMaxN = 1u << 20;   // longest series (samples after padding)
constexpr uint32_t kStaticMinN = 8192;       // shortest series with a fused plan
constexpr size_t kWorkBytes = size_t(kStaticMaxN / 2) * sizeof(float2);  // four-step intermediate
constexpr size_t kTableEntries = 16384;                                  // twiddle tables (float2)
constexpr size_t kTableBytes = kTableEntries * sizeof(float2);
constexpr uint32_t kMaxPartials = 4096;                                  // pass-1 CTAs of one template
constexpr size_t kPartialBytes = kMaxPartials * sizeof(double);
constexpr size_t kMiscBytes = 512;  // brp_params, the input pointer, the padding value, the pass-1 ticket
constexpr size_t kScratchBytes = kWorkBytes + kTableBytes + kPartialBytes + kMiscBytes;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

struct StaticDevice {
    bool ready = false;
    unsigned char* base = nullptr;  // device address of g_scratch on this device
    uint32_t table_n = 0;           // series length whose tables g_scratch holds
    LengthPlan lp;
};

std::mutex g_static_mutex;
StaticDevice g_static_devices[64];
float2 g_static_host_tables[kTableEntries];  // host staging of the tables (no heap)
thread_local char g_static_error[256];

int static_fail(int code, const char* msg) {
    std::strncpy(g_static_error, msg, sizeof g_static_error - 1);
    return code;
}

// Writes one call's arguments into the array and clears the caller's count
// and status words.
__global__ void static_args_kernel(brp_params p, const float* input, brp_params* d_params, const float** d_input,
                                   uint32_t* count, uint32_t* status) {
    *d_params = p;
    *d_input = input;
    *count = 0;
    *status = 0;
}

bool misaligned(const void* ptr, uintptr_t bytes) { return (reinterpret_cast<uintptr_t>(ptr) & (bytes - 1)) != 0; }

}  // namespace
}  // namespace brp

using namespace brp;

extern "C" const char* brp_cuda_search_static_error(void) { return g_static_error; }

extern "C" int brp_cuda_search_static(const brp_params* params, const float* input, float* power,
                                      brp_candidate* candidates, uint32_t capacity, uint32_t* count,
                                      uint32_t* status, void* stream) {
    if (!params || !input || !power || !candidates || !count || !status || !capacity)
        return static_fail(BRP_E_ARGUMENT, "null buffer or zero capacity");
    // The harmonic kernel stages the power spectrum with 16-byte bulk and
    // vector copies; candidates are 16-byte records; the series, the count and
    // the status word are read and updated as 32-bit words.
    if (misaligned(power, 16) || misaligned(candidates, 16))
        return static_fail(BRP_E_ARGUMENT, "power and candidates must be 16-byte aligned");
    if (misaligned(input, 4) || misaligned(count, 4) || misaligned(status, 4))
        return static_fail(BRP_E_ARGUMENT, "input, count and status must be 4-byte aligned");
    const brp_params& p = *params;
    const bool pow2 = p.n && !(p.n & (p.n - 1));
    if (!(pow2 || (p.n % 3 == 0 && !((p.n / 3) & (p.n / 3 - 1)))))
        return static_fail(BRP_E_ARGUMENT, "series length must be 2^k or 3*2^k");
    if (p.n < kStaticMinN || p.n > kStaticMaxN)
        return static_fail(BRP_E_ARGUMENT, "series length outside 8192..1048576 (the static scratch bound)");
    if (p.unpadded < 2 || p.unpadded > p.n || !p.steps || p.steps > p.unpadded || p.fundamental > p.n / 2 ||
        p.harmonic > p.n / 2)
        return static_fail(BRP_E_ARGUMENT, "invalid template dimensions");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return static_fail(BRP_E_RUNTIME, "no CUDA device");

    std::lock_guard<std::mutex> lock(g_static_mutex);
    StaticDevice& d = g_static_devices[dev];
    if (!d.ready) {
        // Set-up, once per device: the device address of the scratch array.
        void* addr = nullptr;
        if (cudaGetSymbolAddress(&addr, g_scratch) != cudaSuccess || !addr)
            return static_fail(BRP_E_RUNTIME, "cudaGetSymbolAddress of the static scratch failed");
        d.base = static_cast<unsigned char*>(addr);
        d.ready = true;
    }
    float2* work = reinterpret_cast<float2*>(d.base);
    float2* tables = reinterpret_cast<float2*>(d.base + kWorkBytes);
    double* partial = reinterpret_cast<double*>(d.base + kWorkBytes + kTableBytes);
    unsigned char* misc = d.base + kWorkBytes + kTableBytes + kPartialBytes;
    brp_params* d_params = reinterpret_cast<brp_params*>(misc);
    const float** d_input = reinterpret_cast<const float**>(misc + 128);
    float* d_mean = reinterpret_cast<float*>(misc + 136);
    // pass-1 CTA ticket: zero in the module image, re-armed by every launch's last CTA
    uint32_t* d_ticket = reinterpret_cast<uint32_t*>(misc + 144);

    if (d.table_n != p.n) {
        // New length: choose the kernels and refill the tables (the tables of
        // the previous length are overwritten; set-up calls are not capturable).
        LengthPlan lp;
        std::string e = choose_length_plan(p.n, lp, 0, 0, false);  // the built-in plan: no plan file read here
        if (!e.empty()) return static_fail(BRP_E_RUNTIME, e.c_str());
        if (!lp.fused) return static_fail(BRP_E_ARGUMENT, "no fused plan for this length");
        size_t off[kPlanTableBlocks + 1];
        if (length_plan_layout(lp, false, off) > kTableEntries || lp.blocks1() > kMaxPartials)
            return static_fail(BRP_E_ARGUMENT, "plan exceeds the static scratch");
        fill_length_plan_tables(lp, false, g_static_host_tables, tables);
        if (cudaMemcpyAsync(tables, g_static_host_tables, off[kPlanTableBlocks] * sizeof(float2),
                            cudaMemcpyHostToDevice, s) != cudaSuccess)
            return static_fail(BRP_E_RUNTIME, "upload of the twiddle tables failed");
        d.lp = lp;
        d.table_n = p.n;
    }
    const LengthPlan& lp = d.lp;
    static_args_kernel<<<1, 1, 0, s>>>(p, input, d_params, d_input, count, status);
    if (cudaGetLastError() != cudaSuccess) return static_fail(BRP_E_RUNTIME, "argument kernel launch failed");

    FusedArgs a{};
    a.inputs = d_input;
    a.params = d_params;
    fill_fused_args(a, lp);
    a.work = work; a.work_stride = lp.M;
    a.power = power; a.power_stride = lp.M;
    a.partial = partial; a.partial_stride = lp.blocks1();
    a.mean = d_mean; a.tickets = d_ticket; a.status = status; a.counts = count; a.cands = candidates;
    a.capacity = capacity;
    a.snap = -1;
    const uint32_t span = p.fundamental > p.harmonic + 8 ? p.fundamental : p.harmonic + 8;
    launch_fused_pass1(a, lp, 1, s);
    launch_fused_pass2(a, lp, 1, s);
    launch_fused_harmonic(a, lp, 1, span, s);
    if (cudaGetLastError() != cudaSuccess) return static_fail(BRP_E_RUNTIME, "kernel launch failed");
    return BRP_OK;
}
