// Bulk tensor store of a pass-1 tile of T (the tensor-memory accelerator),
// shared by the pass-1 kernels that take it (pass1_warp.cu, fused_fast.cu).
//
// A pass-1 CTA's outputs are one L1 x C tile of T: rows of C complex values
// (8 C bytes) at a row pitch of L2 complex values.  With C = 4 every plain
// st.global of a warp touches 8 lines (32-byte row segments); staged in shared
// memory as [row][column] the tile leaves the SM as L1/256 boxes of 256 rows
// (cp.async.bulk.tensor, no multicast), off the load/store pipe.
#pragma once
#include <cuda.h>  // CUtensorMap; encoded through the runtime's driver entry point (no libcuda link)
#include <cudaTypedefs.h>
#include "async_device.cuh"
#include "brp_internal.h"

namespace brp {
namespace {

// cuTensorMapEncodeTiled from the driver the runtime has loaded (null if absent).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// The tensor map of T for one pass-1 launch: 8-byte elements, L2 columns x L1
// rows x the launch's templates (a.work + g work_stride), box C x 256 x 1.
// Every box of the launch lies inside T (rows 256 b.. < L1, columns c0 .. c0 +
// C - 1 < L2 with c0 = C blockIdx.x, so c0 8 bytes is a multiple of 16 for even
// C).  Returns false, with nothing to launch, when the shape does not allow it.
inline bool encode_tile_map(CUtensorMap* tm, const FusedArgs& a, uint32_t L1, uint32_t C, uint32_t blocks,
                            uint32_t count) {
    const PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || a.L1 != L1 || L1 % 256 || C % 2 || blocks * C != a.L2 || count == 0 ||
        (reinterpret_cast<uintptr_t>(a.work) & 15u) != 0)
        return false;
    const cuuint64_t dim[3] = {a.L2, a.L1, count};
    const cuuint64_t stride[2] = {cuuint64_t(a.L2) * 8u, cuuint64_t(a.work_stride) * 8u};
    const cuuint32_t box[3] = {C, 256u, 1u}, estride[3] = {1u, 1u, 1u};
    return enc(tm, CU_TENSOR_MAP_DATA_TYPE_UINT64, 3, a.work, dim, stride, box, estride,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Shared-memory address of the tile: the first 128-byte boundary of buf (the
// caller's buffer holds L1 C 8 + 128 bytes at least).
__device__ __forceinline__ uint32_t tile_address(const float2* buf) { return (smem_u32(buf) + 127u) & ~127u; }

// Issued by one thread after the tile is written, fenced for the asynchronous
// proxy (fence.proxy.async.shared::cta by every writer) and the CTA
// synchronised: the L1/256 boxes of template g's columns c0.., then the commit.
template <int L1, int C>
__device__ __forceinline__ void store_tile_bulk(const CUtensorMap* tm, uint32_t tile_sh, uint32_t c0, int g) {
#pragma unroll
    for (int b = 0; b < L1 / 256; ++b)
        asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(tm),
                     "r"(int(c0)), "r"(256 * b), "r"(g), "r"(tile_sh + uint32_t(b) * 256u * C * 8u)
                     : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}

// The issuing thread, before the CTA leaves: the tile stays in shared memory
// until the bulk copies have read it.
__device__ __forceinline__ void wait_tile_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

}  // namespace
}  // namespace brp
