// amx_dispatch.cu -- builds the tile-pipeline parameters for a request, picks the decode
// policy, clears the workspace and launches the persistent grid.
#include "amx_dispatch.h"
#include "amx_launch.cuh"
#include "amx_policies.cuh"

namespace amx {

// input bytes the loader keeps staged ahead of the compute warps unless tuned otherwise
constexpr uint32_t kDefaultStagedBytes = 160 * 1024;

amx_tuning& tuning()
{
    static thread_local amx_tuning t{};
    return t;
}

LookbackFault& lookback_fault()
{
    static thread_local LookbackFault f{};
    return f;
}

amx_status run_chain(const ChainReq& r, void* ws, size_t ws_bytes, cudaStream_t stream)
{
    PipeParams p{};
    p.withhold_plus1 = lookback_fault().withhold_plus1;
    p.wait_polls = lookback_fault().wait_polls ? lookback_fault().wait_polls : kWaitSpins;
    p.a = col_dev(r.a);
    p.n = r.a->n;
    p.n_dev = r.n_dev;
    if (r.b) {
        p.b = col_dev(r.b);
        p.has_b = 1;
    }
    if (r.mask_in) {
        p.m = mask_dev(r.mask_in, p.n);
        p.has_mask_in = 1;
    }
    if (r.out) {
        p.out = out_dev(r.out);
        p.has_out = 1;
        p.compact = r.compact;
    }
    p.op = r.b ? r.op : AMX_OP_LHS;
    p.vbits = r.vbits;
    p.vmask = mask_of(r.vbits);
    {
        // op results that provably fit vbits need no masking
        uint32_t widest = p.a.bits;
        if (r.b) {
            const uint32_t mx = p.a.bits > p.b.bits ? p.a.bits : p.b.bits;
            switch (p.op) {
                case AMX_OP_ADD: widest = mx + 1; break;
                case AMX_OP_MUL: widest = p.a.bits + p.b.bits; break;
                case AMX_OP_MIN:
                case AMX_OP_MAX:
                case AMX_OP_AND:
                case AMX_OP_OR:
                case AMX_OP_XOR: widest = mx; break;
                case AMX_OP_DIV:
                case AMX_OP_MOD:
                case AMX_OP_LHS: widest = p.a.bits; break;
                case AMX_OP_BOOL_OR:
                case AMX_OP_BOOL_XOR: widest = 1; break;
                default: widest = 64; break;  // sub wraps, math can be all ones
            }
        }
        p.need_vmask = widest > r.vbits ? 1 : 0;
    }
    if (r.pred) {
        amx_status st = normalize_pred(r.pred, p.pred_lo, p.pred_span, p.pred_neg);
        if (st) return st;
        p.has_pred = 1;
        // for values below 2^32 the range test is exact in 32-bit arithmetic when the range
        // starts below 2^32 and does not wrap
        if (p.pred_lo < (1ull << 32) && p.pred_lo + p.pred_span >= p.pred_lo) {
            const uint64_t room = 0xffffffffull - p.pred_lo;
            p.pred_lo32 = (uint32_t)p.pred_lo;
            p.pred_span32 = (uint32_t)(p.pred_span < room ? p.pred_span : room);
            p.pred32_ok = 1;
        }
    }
    p.agg = r.agg;
    p.has_agg = r.has_agg;
    p.mask_out = r.mask_out;
    p.count_out = r.count_out;
    p.agg_out = r.agg_out;
    const amx_tuning& tu = tuning();
    p.stage_target = tu.staged_bytes ? tu.staged_bytes : kDefaultStagedBytes;
    p.stage_target_compact = tu.compact_stages ? (tu.compact_stages > kMaxStages ? kMaxStages : tu.compact_stages) : 2;
    if (p.stage_target_compact < 2) p.stage_target_compact = 2;
    const int force = r.force_policy >= 0 ? r.force_policy : tu.policy - 1;

    const int id = choose_policy(p, force);
    if (id > kSwarPolicyBase) {
        if (p.has_pred) {
            swar_setup(p);
        }
        else {  // an input mask or an aggregate alone: every field passes the (absent) predicate
            p.sw_mode = 0;
            p.sw_l1 = p.sw_l2 = 0;
        }
        return launch_swar((uint32_t)(id - kSwarPolicyBase), p, ws, ws_bytes, stream);
    }
    // element-wise output with nothing else (conversions, binary ops): the runtime-format map
    // variant, where its larger tiles still leave room for two stages and the output slot
    if (id == 0 && p.has_out && !p.compact && !p.has_mask_in && !p.mask_out && !p.has_agg) {
        constexpr uint32_t kT = 512 * 12;
        const uint64_t stage = stage_need(p.a, kT) + (p.has_b ? stage_need(p.b, kT) : 0);
        const uint64_t slot = round_up(kT * (p.vbits <= 16 ? 2u : 8u), 128);
        if (kCvOff + slot + 2 * stage <= 220 * 1024) return launch<GenericPolT<12, false, true>>(p, ws, ws_bytes, stream);
    }
    if (plain_compacting(p)) {  // the variants that carry only this path
        if (id == 0) return launch<GenericPolT<12, true>>(p, ws, ws_bytes, stream);
        switch (id) {
#define AMX_PLAIN_CASE(id, a, b) case id:
            AMX_SLAB2_PAIRS(AMX_PLAIN_CASE)
#undef AMX_PLAIN_CASE
            return launch_plain_pair(id, p, ws, ws_bytes, stream);
            default: break;
        }
    }
    switch (id) {
#define AMX_POLICY_CASE(id, Pol) \
    case id: return launch<Pol>(p, ws, ws_bytes, stream);
        AMX_POLICY_LIST(AMX_POLICY_CASE)
#undef AMX_POLICY_CASE
        default: return launch<GenericPol>(p, ws, ws_bytes, stream);
    }
}

}  // namespace amx
