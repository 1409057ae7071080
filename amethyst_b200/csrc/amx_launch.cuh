// amx_launch.cuh -- host side of one tile-pipeline launch: shared-memory layout, ring depth,
// workspace checks and the persistent grid.  Included by every file that instantiates
// pipe_kernel for some decode policy.
#pragma once

#include "amx_dispatch.h"
#include "amx_pipeline.cuh"

namespace amx {

inline uint32_t round_up(uint32_t x, uint32_t a) { return (x + a - 1) / a * a; }

// shared-memory bytes to stage one tile of column c (tile_elems elements), with 16 bytes of
// alignment shift and 32 bytes of read-ahead slack
inline uint32_t stage_need(const ColDev& c, uint32_t tile_elems)
{
    uint64_t b = 0;
    switch (c.format) {
        case AMX_PLAIN32: b = 4ull * tile_elems; break;
        case AMX_PLAIN64: b = 8ull * tile_elems; break;
        case AMX_SLAB: b = 8ull * (tile_elems / c.eps + 2); break;
        case AMX_NOGAPS: b = 8ull * ((uint64_t)tile_elems * c.bits / 64 + 2); break;
        default: b = tile_elems / 8 + 8; break;
    }
    return round_up((uint32_t)b + 48, 128);
}

// bytes of column c per tile when every tile starts and ends on a storage-word boundary
inline uint64_t tile_stride(const ColDev& c, uint32_t tile_elems)
{
    switch (c.format) {
        case AMX_PLAIN32: return 4ull * tile_elems;
        case AMX_PLAIN64: return 8ull * tile_elems;
        case AMX_SLAB: return tile_elems % c.eps == 0 ? 8ull * (tile_elems / c.eps) : 0;
        case AMX_NOGAPS: return ((uint64_t)tile_elems * c.bits) % 64 == 0 ? (uint64_t)tile_elems * c.bits / 8 : 0;
        default: return tile_elems % 32 == 0 ? tile_elems / 8 : 0;  // bitmask words
    }
}

template <class Pol>
amx_status launch(PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream)
{
    constexpr uint32_t TILE = Pol::kCompute * Pol::R;
    constexpr uint32_t THREADS = Pol::kCompute + kCtlThreads;  // compute + loader, look-back, encoder warps
    p.tile_elems = TILE;
    p.num_tiles = (p.n + TILE - 1) / TILE;
    const uint64_t need = sizeof(WsHeader) + 8 * p.num_tiles;
    if (!ws) return fail(AMX_ERR_WORKSPACE, "workspace is null");
    if (ws_bytes < need)
        return fail(AMX_ERR_WORKSPACE, "workspace of %zu bytes, %llu needed", ws_bytes, (unsigned long long)need);
    if (((uintptr_t)ws) & 15) return fail(AMX_ERR_ALIGNMENT, "workspace not 16-byte aligned");
    p.ws = reinterpret_cast<WsHeader*>(ws);
    p.status = reinterpret_cast<uint64_t*>(reinterpret_cast<uint8_t*>(ws) + sizeof(WsHeader));

    p.a_stride = tile_stride(p.a, TILE);
    p.b_stride = p.has_b ? tile_stride(p.b, TILE) : 0;
    p.m_stride = p.has_mask_in ? tile_stride(p.m, TILE) : 0;
    p.a_off = 0;
    uint32_t off = stage_need(p.a, TILE);
    p.b_off = off;
    if (p.has_b) off += stage_need(p.b, TILE);
    p.m_off = off;
    if (p.has_mask_in) off += stage_need(p.m, TILE);
    p.stage_bytes = off;
    using V = typename Pol::V;
    // Gathered survivors: one slot for element-wise outputs; for compacting passes as many slots
    // (2..kMaxSlots) as fit, so the look-back and the encoder warps trail the compute warps by
    // several tiles.  16-bit slots when the values fit.
    p.cv16 = p.has_out && p.vbits <= 16 ? 1 : 0;
    p.slot_bytes = round_up(TILE * (p.cv16 ? 2u : (uint32_t)sizeof(V)), 128);
    // shared memory to plan with: the whole 227 KB for the 24-compute-warp kernels (their tiles
    // are 1.5 times larger), else 220 KB
    const uint32_t budget = Pol::kMinBlocks >= 2 ? 110 * 1024 : (Pol::kCompute > 512 ? 227 * 1024 : 220 * 1024);
    const bool compact = p.has_out && p.compact;
    p.slots = p.has_out ? 1 : 0;
    if (compact) {
        p.slots = kMaxSlots;
        while (p.slots > 1 && kCvOff + p.slots * p.slot_bytes + 2 * p.stage_bytes > budget) p.slots--;
    }
    p.smem_fixed = round_up(kCvOff + p.slots * p.slot_bytes, 128);
    // Enough stages to keep ~64 KiB of the CTA's input in flight (HBM latency x bandwidth per
    // SM); compacting passes keep two, since every held ticket delays the moment that tile's
    // count is published for the other CTAs' look-backs.
    uint32_t stages = (p.stage_target + p.stage_bytes - 1) / p.stage_bytes;
    if (stages < 2) stages = 2;
    if (stages > kMaxStages) stages = kMaxStages;
    if (compact) stages = p.stage_target_compact;
    while (stages > 2 && p.smem_fixed + stages * p.stage_bytes > budget) stages--;
    p.stages = stages;
    const uint32_t smem = p.smem_fixed + stages * p.stage_bytes;
    if (smem > 227 * 1024) return fail(AMX_ERR_UNSUPPORTED, "pipeline needs %u bytes of shared memory", smem);

    cudaError_t e = cudaMemsetAsync(ws, 0, need, stream);
    if (e != cudaSuccess) return cuda_fail(e, "workspace clear");
    auto kern = pipe_kernel<Pol>;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_fail(e, "shared memory attribute");
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, THREADS, smem);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy");
    if (per_sm < 1) return fail(AMX_ERR_UNSUPPORTED, "pipeline kernel does not fit on an SM");
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > p.num_tiles) grid = p.num_tiles;
    if (grid < 1) grid = 1;
    kern<<<(unsigned)grid, THREADS, smem, stream>>>(p);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "pipeline launch");
    return AMX_OK;
}

}  // namespace amx
