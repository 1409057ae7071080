// amx_pairs.cu -- the plain compacting variants of the two-column policies (Slab2Pol<A, B, true,
// OP>): one kernel per slab-width pair and cheap element-wise op, so that a kernel carries only
// the path of its request -- the compute warps share the instruction cache with the other warp
// roles, and cold variants of the op and of the aggregate cost fetch bandwidth.
#include "amx_launch.cuh"
#include "amx_policies.cuh"

namespace amx {

template <int A, int B>
static amx_status launch_pair_op(PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream)
{
    switch (p.op) {
        case AMX_OP_ADD: return launch<Slab2Pol<A, B, true, AMX_OP_ADD>>(p, ws, ws_bytes, stream);
        case AMX_OP_SUB: return launch<Slab2Pol<A, B, true, AMX_OP_SUB>>(p, ws, ws_bytes, stream);
        case AMX_OP_MUL: return launch<Slab2Pol<A, B, true, AMX_OP_MUL>>(p, ws, ws_bytes, stream);
        case AMX_OP_MIN: return launch<Slab2Pol<A, B, true, AMX_OP_MIN>>(p, ws, ws_bytes, stream);
        case AMX_OP_MAX: return launch<Slab2Pol<A, B, true, AMX_OP_MAX>>(p, ws, ws_bytes, stream);
        case AMX_OP_AND: return launch<Slab2Pol<A, B, true, AMX_OP_AND>>(p, ws, ws_bytes, stream);
        case AMX_OP_OR: return launch<Slab2Pol<A, B, true, AMX_OP_OR>>(p, ws, ws_bytes, stream);
        case AMX_OP_XOR: return launch<Slab2Pol<A, B, true, AMX_OP_XOR>>(p, ws, ws_bytes, stream);
        default: return launch<Slab2Pol<A, B, true>>(p, ws, ws_bytes, stream);
    }
}

amx_status launch_plain_pair(int id, PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream)
{
    switch (id) {
#define AMX_PAIR_CASE(pid, a, b) \
    case pid: return launch_pair_op<a, b>(p, ws, ws_bytes, stream);
        AMX_SLAB2_PAIRS(AMX_PAIR_CASE)
#undef AMX_PAIR_CASE
        default: return fail(AMX_ERR_UNSUPPORTED, "no two-column policy %d", id);
    }
}

}  // namespace amx
