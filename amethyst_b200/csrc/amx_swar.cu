// amx_swar.cu -- host side of the field-parallel slab policy: the predicate as an interval of
// field values, and the dispatch to the pipe_kernel<SwarPol<B>> launches (B = 1..32).
#include "amx_dispatch.h"
#include "amx_internal.h"

namespace amx {

// The passing values of [0, 2^b) under the normalised predicate ((v - lo) mod 2^64 <= span) xor
// neg, as an interval [a, z] or its complement, turned into the words the kernel subtracts.
void swar_setup(PipeParams& p)
{
    const uint32_t b = p.a.bits;
    const uint64_t M = mask_of(b);
    const uint32_t eps = 64 / b;
    uint64_t H = 0, LM = 0;
    for (uint32_t k = 0; k < eps; k++) {
        H |= 1ull << (k * b + b - 1);
        LM |= mask_of(b - 1) << (k * b);
    }
    auto rep = [&](uint64_t c) {
        uint64_t r = 0;
        for (uint32_t k = 0; k < eps; k++) r |= c << (k * b);
        return r;
    };
    const uint64_t lo = p.pred_lo, span = p.pred_span;
    bool complement = p.pred_neg != 0, empty = false;
    uint64_t a = 0, z = M;
    if (span <= ~0ull - lo) {  // [lo, lo + span] without wrap-around
        if (lo > M)
            empty = true;
        else {
            a = lo;
            z = span > M - lo ? M : lo + span;
        }
    }
    else {  // [lo, 2^64) together with [0, lo + span - 2^64]
        const uint64_t hw = lo + span;  // wrapped end, below lo
        if (lo > M) {
            a = 0;
            z = hw > M ? M : hw;
        }
        else if (hw + 1 < lo) {  // [0, hw] and [lo, M]: the complement of [hw + 1, lo - 1]
            a = hw + 1;
            z = lo - 1;
            complement = !complement;
        }
        // else every value passes: a = 0, z = M
    }
    uint32_t mode = 0;
    p.sw_l1 = p.sw_l2 = 0;
    if (empty) {
        mode = complement ? 0 : kSwNone;
    }
    else {
        if (a > 0) {
            mode |= kSwLo;
            if ((a >> (b - 1)) & 1) mode |= kSwLoTop;
            p.sw_l1 = rep(a) & LM;
        }
        if (z < M) {
            const uint64_t z1 = z + 1;
            mode |= kSwHi;
            if ((z1 >> (b - 1)) & 1) mode |= kSwHiTop;
            p.sw_l2 = rep(z1) & LM;
        }
        if (complement) mode |= kSwNeg;
    }
    p.sw_mode = mode;
    p.sw_h = H;
}

// pipe_kernel<SwarPol<B>> launches, instantiated in amx_swar_w*.cu (split for build parallelism)
template <int B>
amx_status launch_swar_w(PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream);

amx_status launch_swar(uint32_t bits, PipeParams& p, void* ws, size_t ws_bytes, cudaStream_t stream)
{
    switch (bits) {
#define AMX_SWAR_CASE(b) \
    case b: return launch_swar_w<b>(p, ws, ws_bytes, stream);
        AMX_SWAR_CASE(1) AMX_SWAR_CASE(2) AMX_SWAR_CASE(3) AMX_SWAR_CASE(4) AMX_SWAR_CASE(5) AMX_SWAR_CASE(6)
        AMX_SWAR_CASE(7) AMX_SWAR_CASE(8) AMX_SWAR_CASE(9) AMX_SWAR_CASE(10) AMX_SWAR_CASE(11) AMX_SWAR_CASE(12)
        AMX_SWAR_CASE(13) AMX_SWAR_CASE(14) AMX_SWAR_CASE(15) AMX_SWAR_CASE(16) AMX_SWAR_CASE(17) AMX_SWAR_CASE(18)
        AMX_SWAR_CASE(19) AMX_SWAR_CASE(20) AMX_SWAR_CASE(21) AMX_SWAR_CASE(22) AMX_SWAR_CASE(23) AMX_SWAR_CASE(24)
        AMX_SWAR_CASE(25) AMX_SWAR_CASE(26) AMX_SWAR_CASE(27) AMX_SWAR_CASE(28) AMX_SWAR_CASE(29) AMX_SWAR_CASE(30)
        AMX_SWAR_CASE(31) AMX_SWAR_CASE(32)
#undef AMX_SWAR_CASE
        default: return fail(AMX_ERR_UNSUPPORTED, "field-parallel policy for %u-bit slabs", bits);
    }
}

}  // namespace amx
