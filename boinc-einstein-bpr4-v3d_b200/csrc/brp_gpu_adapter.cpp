// brp::GPU on the CUDA backend: the drop-in replacement of the reference's
// src/vulkan.cpp.  It implements the class declared by the reference's
// unchanged include/brp/vulkan.hpp (GPU at :12-29) on top of the C ABI of
// include/brp_cuda.h, so src/main.cpp (brp_bench) and src/workunit_main.cpp
// (brp_workunit) link against libbrp_cuda.so without source changes.  Build it
// with the reference's include directory on the include path (see
// oracle/Makefile, target dropin).
//
// Error behaviour follows the reference: every failure throws
// std::runtime_error with the backend's message (src/vulkan.cpp:17-19, :333).
#include <cstring>
#include <stdexcept>
#include <vector>
#include "brp/vulkan.hpp"
#include "brp_cuda.h"

namespace brp {

static_assert(sizeof(Params) == sizeof(brp_params), "brp::Params and brp_params must share one layout");
static_assert(sizeof(Candidate) == sizeof(brp_candidate), "brp::Candidate and brp_candidate must share one layout");

struct GPU::Impl {
    brp_ctx* ctx = nullptr;
    std::vector<Params> templates;
    ~Impl() { brp_cuda_destroy(ctx); }
};

static void check(int status, const brp_ctx* ctx) {
    if (status) throw std::runtime_error(brp_cuda_last_error(ctx));
}

GPU::GPU(const Params& p, std::span<const float> input, uint32_t workgroup, uint32_t tile, uint32_t batch,
         bool software, bool stockham, bool radix4, bool packed, bool scatter, bool radix8, bool fused_power,
         bool radix8_store)
    : impl(std::make_unique<Impl>()) {
    brp_options o{};
    o.workgroup = workgroup;
    o.tile = tile;
    o.batch = batch;
    o.flags = (software ? BRP_OPT_SOFTWARE : 0u) | (stockham ? BRP_OPT_STOCKHAM : 0u) | (radix4 ? BRP_OPT_RADIX4 : 0u) |
              (packed ? BRP_OPT_PACKED : 0u) | (scatter ? BRP_OPT_SCATTER : 0u) | (radix8 ? BRP_OPT_RADIX8 : 0u) |
              (fused_power ? BRP_OPT_FUSED_POWER : 0u) | (radix8_store ? BRP_OPT_RADIX8_STORE : 0u);
    o.device = -1;
    brp_params bp;
    std::memcpy(&bp, &p, sizeof bp);
    check(brp_cuda_create(&bp, input.data(), uint32_t(input.size()), &o, &impl->ctx), nullptr);
    impl->templates.assign(1, p);
}

GPU::~GPU() = default;

void GPU::set_template(const Params& next) { set_templates(std::span<const Params>(&next, 1)); }

void GPU::set_templates(std::span<const Params> next) {
    check(brp_cuda_set_templates(impl->ctx, reinterpret_cast<const brp_params*>(next.data()), uint32_t(next.size())),
          impl->ctx);
    impl->templates.assign(next.begin(), next.end());
}

Timings GPU::run() {
    brp_timings t{};
    std::vector<double> per(4 * impl->templates.size());
    check(brp_cuda_run(impl->ctx, &t, per.data()), impl->ctx);
    Timings out{};
    out.wall_ms = t.wall_ms;
    out.cpu_ms = t.cpu_ms;
    out.submit_ms = t.submit_ms;
    for (int s = 0; s < 4; ++s) out.stage_ms[s] = t.stage_ms[s];
    out.template_stage_ms.resize(impl->templates.size());
    for (size_t r = 0; r < impl->templates.size(); ++r)
        for (int s = 0; s < 4; ++s) out.template_stage_ms[r][s] = per[4 * r + s];
    return out;
}

Snapshot GPU::snapshot() const {
    const Params& p = impl->templates.back();
    Snapshot s;
    s.resampled.resize(p.n);
    s.fft.resize(p.n / 2 + 1);
    s.power.resize(p.n / 2);
    s.summed.resize(size_t(5) * p.fundamental);
    check(brp_cuda_snapshot(impl->ctx, s.resampled.data(), reinterpret_cast<float*>(s.fft.data()), s.power.data(),
                            s.summed.data()),
          impl->ctx);
    s.candidates = candidates();
    return s;
}

std::vector<Candidate> GPU::candidates(uint32_t slot) const {
    uint32_t count = 0;
    check(brp_cuda_candidates(impl->ctx, slot, nullptr, 0, &count), impl->ctx);
    std::vector<Candidate> out(count);
    check(brp_cuda_candidates(impl->ctx, slot, reinterpret_cast<brp_candidate*>(out.data()), count, &count),
          impl->ctx);
    return out;
}

std::string GPU::device_info() const {
    char buf[1024];
    check(brp_cuda_device_info(impl->ctx, buf, sizeof buf), impl->ctx);
    return buf;
}

uint64_t GPU::allocated_bytes() const { return brp_cuda_allocated_bytes(impl->ctx); }

std::string GPU::profile_counters() {
    char buf[4096];
    check(brp_cuda_profile_counters(impl->ctx, buf, sizeof buf), impl->ctx);
    return buf;
}

}  // namespace brp
