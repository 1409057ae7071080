// amx_mm_common.cuh -- tile shape and tcgen05 building blocks shared by the two packed-matrix
// multiply paths (amx_matmul.cu: operands unpacked to the workspace, then a TMA-fed GEMM;
// amx_mm_fused.cuh: operands unpacked by warps of the GEMM kernel into its shared memory).
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>

#include "amx_pipeline.cuh"

namespace amx {

constexpr uint32_t kMmBM = 128;   // output rows per tile (TMEM lanes)
constexpr uint32_t kMmBN = 256;   // output columns per tile (TMEM columns of one accumulator)
constexpr uint32_t kMmBK = 128;   // K bytes per stage = one 128-byte swizzle row
constexpr uint32_t kMmStages = 4;
constexpr uint32_t kMmStageA = kMmBM * kMmBK;  // 16 KB
constexpr uint32_t kMmStageB = kMmBN * kMmBK;  // 32 KB
constexpr uint32_t kMmThreads = 192;           // TMA warp, MMA warp, 4 epilogue warps
constexpr uint32_t kMmTmemCols = 2 * kMmBN;    // two accumulators
constexpr uint32_t kMmSmem = 1024 + kMmStages * (kMmStageA + kMmStageB) + 256;
constexpr uint32_t kMmMaxBits = 8;


// ---------------------------------------------------------------------------------------------
// TMA (2-D tiled loads, no multicast) and tcgen05 building blocks (inline PTX)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int32_t x, int32_t y, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}


// shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart
__device__ __forceinline__ uint64_t sdesc_sw128(const void* p)
{
    const uint32_t a = smem_u32(p);
    return (uint64_t)((a & 0x3FFFFu) >> 4) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ void umma_i8(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t addr, uint32_t (&r)[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// instruction descriptor of kind::i8: D s32, A u8, B u8, both K-major, M = 128, N = 256
constexpr uint32_t kMmIdesc = (2u << 4) | (0u << 7) | (0u << 10) | ((kMmBN >> 3) << 17) | ((kMmBM >> 4) << 24);

// cuTensorMapEncodeTiled through the runtime's driver entry point (null when unavailable)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// the fused path (amx_mm_fused.cu): slab operands of one width 1..8 when amx_tuning.policy is 2
// (packed stages by TMA) or 3 (packed words read from global memory); the automatic choice is
// the two-pass path, measured faster at every shape tried
bool mf_applicable(const amx_column* a, const amx_column* b);
amx_status mf_run(const amx_column* a, const amx_column* b, uint32_t M, uint32_t N, uint32_t K, const amx_column* out,
                  uint32_t* d_out_bits, uint32_t* hdr, unsigned long long* colsq, void* scratch, cudaStream_t s);

}  // namespace amx
