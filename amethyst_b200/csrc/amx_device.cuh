// amx_device.cuh -- device building blocks shared by the Amethyst B200 kernels:
// mbarrier + bulk-copy (TMA) staging, bounded waits, look-back status words, predicate and
// operator evaluation, and the per-format element readers.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "amx_internal.h"

namespace amx {

// ---------------------------------------------------------------------------------------------
// shared-memory addresses, mbarriers and 1-D bulk copies (cp.async.bulk, no multicast)
// ---------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// global -> shared bulk copy completing on an mbarrier; dst, src 16-byte aligned, bytes % 16 == 0
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// try_wait that suspends the thread until the phase completes or `ns` nanoseconds pass, so a
// waiting warp issues a handful of instructions per wait instead of a spin loop
__device__ __forceinline__ bool mbar_try_wait_hint(uint64_t* bar, uint32_t parity, uint32_t ns)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase: at most kWaitSuspends suspensions of kWaitSuspendNs each
// (about 1.3 s in all).  Returns false when the limit ran out; the caller records
// AMX_ERR_TIMEOUT and stops using the stage.
constexpr uint32_t kWaitSuspendNs = 20000;
constexpr uint32_t kWaitSuspends = 1u << 16;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity)
{
    for (uint32_t i = 0; i < kWaitSuspends; i++)
        if (mbar_try_wait_hint(bar, parity, kWaitSuspendNs)) return true;
    return false;
}

// Reads of a staged tile that the warp releases right after reading, before it is done with the
// values: volatile, so the compiler can neither read the stage again later (when the loader may
// already be refilling it) nor move the read past the release.  A packed-matrix kernel that read
// its stage with plain loads and released it early got rows with data of the next slice when the
// compiler re-read the stage after the release.
__device__ __forceinline__ uint64_t lds_u64_v(const void* p)
{
    uint64_t v;
    asm volatile("ld.volatile.shared.u64 %0, [%1];" : "=l"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t lds_u32_v(const void* p)
{
    uint32_t v;
    asm volatile("ld.volatile.shared.u32 %0, [%1];" : "=r"(v) : "r"(smem_u32(p)) : "memory");
    return v;
}

__device__ __forceinline__ uint4 lds_v4_v(const void* p)
{
    uint4 v;
    asm volatile("ld.volatile.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(smem_u32(p))
                 : "memory");
    return v;
}

// ---------------------------------------------------------------------------------------------
// look-back status words: [63:62] flag, [61:0] value
// ---------------------------------------------------------------------------------------------
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;

__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void record_error(uint32_t* err, uint32_t code) { atomicCAS(err, 0u, code); }

// ---------------------------------------------------------------------------------------------
// predicate and operator evaluation
// ---------------------------------------------------------------------------------------------
// A predicate normalised on the host to  keep(v) = ((v - lo) <= span) != neg.
struct PredN {
    uint64_t lo;
    uint64_t span;
    uint32_t neg;
    uint32_t pad;
};

template <typename V>
__device__ __forceinline__ bool pred_eval(const PredN& p, V v)
{
    return (((uint64_t)v - p.lo) <= p.span) != (p.neg != 0);
}

__device__ __forceinline__ uint64_t binop_eval(uint32_t op, uint64_t l, uint64_t r)
{
    switch (op) {
        case AMX_OP_ADD: return l + r;
        case AMX_OP_SUB: return l - r;
        case AMX_OP_MUL: return l * r;
        case AMX_OP_DIV: return r ? l / r : ~0ull;
        case AMX_OP_MOD: return r ? l % r : l;
        case AMX_OP_MIN: return l < r ? l : r;
        case AMX_OP_MAX: return l > r ? l : r;
        case AMX_OP_AND: return l & r;
        case AMX_OP_OR: return l | r;
        case AMX_OP_XOR: return l ^ r;
        case AMX_OP_BOOL_OR: return (l || r) ? 1ull : 0ull;
        case AMX_OP_BOOL_XOR: return ((l && !r) || (!l && r)) ? 1ull : 0ull;
        case AMX_OP_MATH: {
            const uint64_t den = l * l + r * r + 5 * l;
            return den ? (l * l + r * r + 4 * l) / den : ~0ull;
        }
        default: return l;
    }
}

// Aggregations are kept in an encoded form so that every one of them has identity 0 and a
// native 64-bit atomic: min(x) = ~max(~x), and(x) = ~or(~x).
__device__ __forceinline__ uint64_t agg_encode(uint32_t agg, uint64_t v)
{
    return (agg == AMX_AGG_MIN || agg == AMX_AGG_AND) ? ~v : v;
}
__device__ __forceinline__ uint64_t agg_combine(uint32_t agg, uint64_t a, uint64_t e)
{
    switch (agg) {
        case AMX_AGG_SUM: return a + e;
        case AMX_AGG_MIN:
        case AMX_AGG_MAX: return a > e ? a : e;
        case AMX_AGG_AND:
        case AMX_AGG_OR: return a | e;
        case AMX_AGG_XOR: return a ^ e;
    }
    return a;
}
__device__ __forceinline__ void agg_atomic(uint32_t agg, unsigned long long* p, uint64_t e)
{
    switch (agg) {
        case AMX_AGG_SUM: atomicAdd(p, (unsigned long long)e); break;
        case AMX_AGG_MIN:
        case AMX_AGG_MAX: atomicMax(p, (unsigned long long)e); break;
        case AMX_AGG_AND:
        case AMX_AGG_OR: atomicOr(p, (unsigned long long)e); break;
        case AMX_AGG_XOR: atomicXor(p, (unsigned long long)e); break;
    }
}
__device__ __forceinline__ uint64_t agg_decode(uint32_t agg, uint64_t a)
{
    return (agg == AMX_AGG_MIN || agg == AMX_AGG_AND) ? ~a : a;
}

__device__ __forceinline__ uint64_t mask_bits(uint32_t bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1); }

// n / d for n < 2^58 and d in 1..64 with a precomputed magic m = floor(2^64 / d) + 1 (d >= 2):
// a multiply-high instead of the long software 64-bit division
__device__ __forceinline__ uint64_t udiv64(uint64_t n, uint64_t m, uint32_t d) { return d == 1 ? n : __umul64hi(n, m); }

}  // namespace amx
