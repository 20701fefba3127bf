// Device pre-filter of a bank run's candidates for the host toplist
// (src/workload.cpp:126-159: per harmonic level `rows` rows, one row per bin,
// a bin's row keeps its highest power, the lowest row gives way to a higher
// candidate).
//
// Over a series' templates in any order the toplist ends holding, per level,
// the `rows` bins of highest per-bin maximum power: the lowest row's power
// never decreases, so a bin once evicted can only come back with a power above
// the one it was evicted with.  A candidate whose power is below V, the
// rows-th highest per-bin maximum of its level among all candidates of its
// series, therefore never reaches the final rows, and dropping it leaves the
// per-bin maxima of the kept bins, and so the final toplist, unchanged
// (candidates equal to V are kept).  Per (series, level) V comes from:
//   1. filter_max:    per bin the maximum power key (atomicMax) and a flag;
//   2. filter_owners: the one candidate per bin that holds the maximum claims
//                     the flag (atomicExch) and appends the key to the level's
//                     list of per-bin maxima;
//   3. filter_select: the rows-th largest key of that list by a three-pass
//                     radix select (11, 11, 10 bits) in shared memory;
//   4. filter_count:  per slot the number of candidates >= V; it also clears
//                     the per-bin arrays it touched for the next run.
// The compaction (plain_kernels.cu) then writes only the kept candidates.
// Power keys are the order-preserving unsigned images of the FP32 powers.
#include "brp_internal.h"

namespace brp {
namespace {

__device__ __forceinline__ uint32_t cand_index(const FilterArgs& f, uint32_t s, const brp_candidate& c, bool& ok) {
    ok = c.level < 5 && c.bin < f.half[s];
    return uint32_t(f.base[s] + uint64_t(c.level) * f.half[s] + c.bin);
}

__global__ void __launch_bounds__(256) filter_max(FilterArgs f) {
    const uint32_t k = blockIdx.x, s = f.slot_series[k];
    const uint32_t c = min(f.counts[k], f.capacity);
    const brp_candidate* src = f.cands + size_t(k) * f.capacity;
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
        const brp_candidate x = src[i];
        bool ok;
        const uint32_t at = cand_index(f, s, x, ok);
        if (!ok) continue;
        atomicMax(f.maxkey + at, power_key(x.power));
        f.flag[at] = 1u;
    }
}

__global__ void __launch_bounds__(256) filter_owners(FilterArgs f) {
    const uint32_t k = blockIdx.x, s = f.slot_series[k];
    const uint32_t c = min(f.counts[k], f.capacity);
    const brp_candidate* src = f.cands + size_t(k) * f.capacity;
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
        const brp_candidate x = src[i];
        bool ok;
        const uint32_t at = cand_index(f, s, x, ok);
        if (!ok) continue;
        const uint32_t key = power_key(x.power);
        if (key == f.maxkey[at] && atomicExch(f.flag + at, 0u) == 1u) {
            const uint32_t pos = atomicAdd(f.owner_count + s * 5 + x.level, 1u);
            f.owners[f.base[s] + uint64_t(x.level) * f.half[s] + pos] = key;
        }
    }
}

// One CTA per (series, level): the rows-th largest of the level's per-bin maxima.
__global__ void __launch_bounds__(1024) filter_select(FilterArgs f) {
    __shared__ uint32_t hist[2048];
    __shared__ uint32_t s_prefix, s_mask, s_remaining;
    const uint32_t s = blockIdx.x / 5, level = blockIdx.x % 5;
    const uint32_t cnt = f.owner_count[blockIdx.x];
    const uint32_t* keys = f.owners + f.base[s] + uint64_t(level) * f.half[s];
    if (cnt < f.rows) {  // fewer bins than rows: every candidate stays
        if (threadIdx.x == 0) { f.threshold_key[blockIdx.x] = 0u; f.owner_count[blockIdx.x] = 0u; }
        return;
    }
    if (threadIdx.x == 0) { s_prefix = 0u; s_mask = 0u; s_remaining = f.rows; }
    const int shifts[3] = {21, 10, 0}, widths[3] = {11, 11, 10};
    for (int pass = 0; pass < 3; ++pass) {
        const uint32_t shift = shifts[pass], nb = 1u << widths[pass];
        for (uint32_t b = threadIdx.x; b < 2048; b += blockDim.x) hist[b] = 0u;
        __syncthreads();
        const uint32_t prefix = s_prefix, mask = s_mask;
        for (uint32_t i = threadIdx.x; i < cnt; i += blockDim.x) {
            const uint32_t key = keys[i];
            if ((key & mask) == prefix) atomicAdd(hist + ((key >> shift) & (nb - 1)), 1u);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            // Walk the buckets from the highest down, 32 at a time: the bucket
            // holding the remaining-th largest key is the first whose running
            // count reaches `remaining`.
            const uint32_t lane = threadIdx.x;
            uint32_t remaining = s_remaining;
            int found = 0;
            for (int top = int(nb) - 1; top >= 0; top -= 32) {
                const uint32_t h = hist[top - int(lane)];
                uint32_t incl = h;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= uint32_t(o)) incl += v;
                }
                const uint32_t excl = incl - h;
                const uint32_t hit = __ballot_sync(0xffffffffu, excl < remaining && incl >= remaining);
                if (hit) {
                    const int l = __ffs(hit) - 1;
                    found = top - l;
                    remaining -= __shfl_sync(0xffffffffu, excl, l);
                    break;
                }
                remaining -= __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) {
                s_prefix = prefix | (uint32_t(found) << shift);
                s_mask = mask | ((nb - 1) << shift);
                s_remaining = remaining;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        f.threshold_key[blockIdx.x] = s_prefix;
        f.owner_count[blockIdx.x] = 0u;
    }
}

__global__ void __launch_bounds__(256) filter_count(FilterArgs f) {
    __shared__ uint32_t s_kept;
    const uint32_t k = blockIdx.x, s = f.slot_series[k];
    const uint32_t c = min(f.counts[k], f.capacity);
    const brp_candidate* src = f.cands + size_t(k) * f.capacity;
    if (threadIdx.x == 0) s_kept = 0u;
    __syncthreads();
    uint32_t kept = 0;
    for (uint32_t i = threadIdx.x; i < c; i += blockDim.x) {
        const brp_candidate x = src[i];
        bool ok;
        const uint32_t at = cand_index(f, s, x, ok);
        if (!ok) { ++kept; continue; }  // invalid candidates go to the host, which rejects them
        if (power_key(x.power) >= f.threshold_key[s * 5 + x.level]) ++kept;
        f.maxkey[at] = 0u;
        f.flag[at] = 0u;
    }
    atomicAdd(&s_kept, kept);
    __syncthreads();
    if (threadIdx.x == 0) f.kept[k] = s_kept;
}

}  // namespace

void launch_toplist_filter(const FilterArgs& f, cudaStream_t s) {
    if (!f.count) return;
    filter_max<<<f.count, 256, 0, s>>>(f);
    filter_owners<<<f.count, 256, 0, s>>>(f);
    filter_select<<<f.series * 5, 1024, 0, s>>>(f);
    filter_count<<<f.count, 256, 0, s>>>(f);
}

}  // namespace brp
