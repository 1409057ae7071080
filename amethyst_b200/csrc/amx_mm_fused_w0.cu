// amx_mm_fused_w0.cu -- mf_gemm_kernel<W> for slab widths W = 1..4 (split for build parallelism).
#include "amx_dispatch.h"
#include "amx_mm_fused.cuh"

namespace amx {

template amx_status mf_launch_w<1>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);
template amx_status mf_launch_w<2>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);
template amx_status mf_launch_w<3>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);
template amx_status mf_launch_w<4>(const CUtensorMap&, const CUtensorMap&, const MfParams&, cudaStream_t);

}  // namespace amx
