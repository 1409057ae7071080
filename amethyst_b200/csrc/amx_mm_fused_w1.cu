// amx_mm_fused_w1.cu -- mf_gemm_kernel<W> for slab widths W = 5..8 (split for build parallelism).
#include "amx_dispatch.h"
#include "amx_mm_fused.cuh"

namespace amx {

template amx_status mf_launch_w<5>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);
template amx_status mf_launch_w<6>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);
template amx_status mf_launch_w<7>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);
template amx_status mf_launch_w<8>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);

}  // namespace amx
