// amx_swar_w0.cu -- pipe_kernel<SwarPol<B>> for slab widths B = 1..8.
#include "amx_launch.cuh"

namespace amx {

template <int B>
amx_status launch_swar_w(PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream)
{
    if (!p.has_out && !p.has_agg && p.mask_out)  // the filter alone
        return launch<SwarPol<B, false, true>>(p, ws, ws_bytes, stream);
    if (!p.has_out && !p.mask_out) {  // a count and at most one aggregate
        // at 1-4 bits a count or a sum with no input mask takes runs of 8 slabs
        if constexpr (B <= kSwarPlaneMax)
            if (!p.has_mask_in && (!p.has_agg || p.agg == AMX_AGG_SUM))
                return launch<SwarPol<B, false, false, true, false, true>>(p, ws, ws_bytes, stream);
        return launch<SwarPol<B, false, false, true>>(p, ws, ws_bytes, stream);
    }
    if constexpr (B <= 16) {
        // the plain compressstore takes the kernel that carries only its own path; with an input
        // mask in its 16-warp form: the 24-warp form's two stages and two survivor slots fill the
        // 227 KB, and the mask's stage would leave room for one slot (compute warps then wait for
        // the encoder every tile: 0.25 vs 0.11 ms on a one-cluster mask)
        if (p.has_out && p.compact && !p.has_agg && !p.mask_out && p.out.format == AMX_SLAB && p.out.bits == B &&
            p.vbits <= 16)
            return p.has_mask_in ? launch<SwarPol<B, true, false, false, true>>(p, ws, ws_bytes, stream)
                                 : launch<SwarPol<B, true>>(p, ws, ws_bytes, stream);
    }
    return launch<SwarPol<B>>(p, ws, ws_bytes, stream);
}

template amx_status launch_swar_w<1>(PipeParams&, void*, size_t, cudaStream_t);
template amx_status launch_swar_w<2>(PipeParams&, void*, size_t, cudaStream_t);
template amx_status launch_swar_w<3>(PipeParams&, void*, size_t, cudaStream_t);
template amx_status launch_swar_w<4>(PipeParams&, void*, size_t, cudaStream_t);
template amx_status launch_swar_w<5>(PipeParams&, void*, size_t, cudaStream_t);
template amx_status launch_swar_w<6>(PipeParams&, void*, size_t, cudaStream_t);
template amx_status launch_swar_w<7>(PipeParams&, void*, size_t, cudaStream_t);
template amx_status launch_swar_w<8>(PipeParams&, void*, size_t, cudaStream_t);

}  // namespace amx
