// amx_dispatch.h -- host-side request description and helpers shared by the C ABI files.
#pragma once

#include <cuda_runtime.h>

#include "amx_internal.h"

namespace amx {

constexpr uint64_t kMaxElements = 1ull << 40;
// smallest tile of any pipeline policy (bounds the look-back status array)
constexpr uint64_t kMinTile = 4096;

// One pass of the tile pipeline: v = op(a, b) & mask(vbits), keep pred(v) (and the input
// mask), then any of mask_out / out (compacted or element-wise) / count / aggregate.
struct ChainReq {
    const amx_column* a = nullptr;
    const amx_column* b = nullptr;
    const uint32_t* mask_in = nullptr;
    const amx_predicate* pred = nullptr;
    uint32_t op = AMX_OP_LHS;
    uint32_t vbits = 64;
    const amx_column* out = nullptr;
    uint32_t compact = 0;
    uint32_t* mask_out = nullptr;
    uint64_t* count_out = nullptr;
    uint32_t has_agg = 0;
    uint32_t agg = AMX_AGG_SUM;
    uint64_t* agg_out = nullptr;
    int force_policy = -1;  // -1 = automatic; otherwise a policy id (tests and the autotuner)
};

// launch tuning of this host thread (amx_set_tuning); zero fields mean "automatic"
amx_tuning& tuning();

amx_status fail(amx_status s, const char* fmt, ...);
amx_status cuda_fail(cudaError_t e, const char* what);
uint64_t mask_of(uint32_t bits);
uint64_t magic64(uint32_t d);
uint64_t storage_bytes(uint32_t format, uint32_t bits, uint64_t n);
amx_status check_column(const amx_column* c, const char* name);
ColDev col_dev(const amx_column* c);
ColDev mask_dev(const uint32_t* m, uint64_t n);
OutDev out_dev(const amx_column* c);
amx_status normalize_pred(const amx_predicate* p, uint64_t& lo, uint64_t& span, uint32_t& neg);
int sm_count();

amx_status run_chain(const ChainReq& r, void* ws, size_t ws_bytes, cudaStream_t stream);

// plain compacting two-column policy `id` (amx_pairs.cu): one kernel per pair and cheap op
amx_status launch_plain_pair(int id, PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream);

// field-parallel slab policy (amx_swar.cu): predicate constants, and the launch for width `bits`
void swar_setup(PipeParams& p);
amx_status launch_swar(uint32_t bits, PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream);

}  // namespace amx
