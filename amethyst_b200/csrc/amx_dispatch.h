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
    const uint64_t* n_dev = nullptr;  // device-resident length (<= a->n), read by the kernel
};

// launch tuning of this host thread (amx_set_tuning); zero fields mean "automatic"
amx_tuning& tuning();

// look-back fault injection of this host thread (amx_test_lookback_timeout)
struct LookbackFault {
    uint64_t withhold_plus1 = 0;  // tile + 1 whose count the kernel never publishes, 0: none
    uint32_t wait_polls = 0;      // 0: kWaitSpins
};
LookbackFault& lookback_fault();

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

// amx_groupby with an optional device-resident length of the key and value columns (<= keys->n)
amx_status groupby_run(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                       const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                       uint64_t* d_groups, void* ws, size_t ws_bytes, void* stream, const uint64_t* n_dev);
// offset of the tile-pipeline workspace inside a group-by workspace when the groups of keys of
// that width are extracted by the pipeline, else UINT64_MAX
uint64_t groupby_pipeline_offset(uint32_t key_bits);

// plain compacting two-column policy `id` (amx_pairs.cu): one kernel per pair and cheap op
amx_status launch_plain_pair(int id, PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream);

// field-parallel slab policy (amx_swar.cu): predicate constants, and the launch for width `bits`
void swar_setup(PipeParams& p);
amx_status launch_swar(uint32_t bits, PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream);

}  // namespace amx
