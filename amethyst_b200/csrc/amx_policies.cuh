// amx_policies.cuh -- compile-time-width decode policies of the tile pipeline and the rule
// that picks one for a request.
//
// A policy fixes R (elements per thread per tile) and decodes a thread's run of R elements
// from the staged words.  GenericPol (amx_pipeline.cuh) handles any format and width with
// warp-major runtime readers.  The policies here fix the slab widths at compile time so every
// shift and mask is a constant and each thread's run starts on a slab boundary:
//   SlabPol<B>           one slab column of width B (filter, compressstore, reduce, convert)
//   Slab2Pol<BA, BB>     two slab columns (binary op, fused chains)
// Values are 32-bit, so these policies serve value widths up to 32.
#pragma once

#include "amx_pipeline.cuh"

namespace amx {

template <int A, int B>
struct ct_gcd {
    static constexpr int value = ct_gcd<B, A % B>::value;
};
template <int A>
struct ct_gcd<A, 0> {
    static constexpr int value = A;
};

template <int B, int K>
__device__ __forceinline__ uint32_t field(uint64_t slab)
{
    return (uint32_t)((slab >> (K * B)) & ((1ull << B) - 1));
}

template <int B, int EPS, int N, int R>
__device__ __forceinline__ void unpack_slabs(const uint64_t (&w)[N], uint32_t (&v)[R])
{
#pragma unroll
    for (int j = 0; j < N; j++)
#pragma unroll
        for (int k = 0; k < EPS; k++) v[j * EPS + k] = (uint32_t)((w[j] >> (k * B)) & ((1ull << B) - 1));
}

// mask to the value width and evaluate the predicate on 32-bit values
template <int R>
__device__ __forceinline__ void finish32(const PipeParams& p, uint32_t (&v)[R], uint64_t& fl)
{
    if (p.need_vmask) {
        const uint32_t vm = (uint32_t)p.vmask;
#pragma unroll
        for (int i = 0; i < R; i++) v[i] &= vm;
    }
    if (!p.has_pred) {
        fl = ~0ull;
        return;
    }
    fl = 0;
    if (p.pred32_ok) {
        const uint32_t lo = p.pred_lo32, span = p.pred_span32;
        if (lo == 0) {
#pragma unroll
            for (int i = 0; i < R; i++) fl |= (uint64_t)(v[i] <= span) << i;
        }
        else {
#pragma unroll
            for (int i = 0; i < R; i++) fl |= (uint64_t)((v[i] - lo) <= span) << i;
        }
        if (p.pred_neg) fl = ~fl;
    }
    else {
        const PredN pn{p.pred_lo, p.pred_span, p.pred_neg, 0};
#pragma unroll
        for (int i = 0; i < R; i++) fl |= (uint64_t)pred_eval(pn, (uint64_t)v[i]) << i;
    }
}

template <int B>
struct SlabPol {
    using V = uint32_t;
    static constexpr int EPS = 64 / B;
    static constexpr int SPT = EPS >= 32 ? 1 : 32 / EPS;
    static constexpr int R = EPS * SPT;
    static constexpr bool kWarpMajor = false;
    static constexpr bool kSwar = false;
    static constexpr bool kPlain = false;
    static constexpr bool kFilter = false;
    static constexpr bool kAggOnly = false;
    static constexpr bool kMap = false;
    static constexpr bool kWide = false;
    // one CTA per SM: 16 compute warps, or 8 for the register-heavy 64-element runs and for
    // widths >= 17 (10+ slabs per thread: a 16-warp tile would not fit twice in shared memory)
    static constexpr uint32_t kCompute = (R > 40 || B >= 17) ? 256 : 512;
    static constexpr int kMinBlocks = 1;

    __device__ __forceinline__ static void decode(const PipeParams& p, const uint8_t* st, const uint64_t* sb,
                                                  uint64_t e0, V (&v)[R], uint64_t& fl)
    {
        const uint64_t first = e0 + threadIdx.x * R;
        const uint64_t* w = reinterpret_cast<const uint64_t*>(st + p.a_off) + (first / EPS - sb[0] / 8);
        uint64_t s[SPT];
        lds_words<SPT>(w, s);
        unpack_slabs<B, EPS, SPT, R>(s, v);
        finish32<R>(p, v, fl);
    }

    // value of element i of this thread's run, re-read from the staged words (sparse gather)
    __device__ __forceinline__ static V value_at(const PipeParams& p, const uint8_t* st, const uint64_t* sb,
                                                 uint64_t e0, int i)
    {
        const uint64_t first = e0 + threadIdx.x * R;
        const uint64_t* w = reinterpret_cast<const uint64_t*>(st + p.a_off) + (first / EPS - sb[0] / 8);
        const uint32_t j = (uint32_t)i / EPS, k = (uint32_t)i - j * EPS;
        uint32_t x = (uint32_t)((w[j] >> (k * B)) & ((1ull << B) - 1));
        if (p.need_vmask) x &= (uint32_t)p.vmask;
        return x;
    }
};

// v[j*EPS + k] = op(v[j*EPS + k], field k of slab j), in place (no second value array)
template <int B, int EPS, int N, int R, typename F>
__device__ __forceinline__ void combine_slabs(const uint64_t (&w)[N], uint32_t (&v)[R], F f)
{
#pragma unroll
    for (int j = 0; j < N; j++)
#pragma unroll
        for (int k = 0; k < EPS; k++)
            v[j * EPS + k] = f(v[j * EPS + k], (uint32_t)((w[j] >> (k * B)) & ((1ull << B) - 1)));
}

// One of the cheap element-wise ops of the two-column policies, fixed at compile time.
template <int OP>
struct OpFn {
    __device__ __forceinline__ uint32_t operator()(uint32_t a, uint32_t b) const
    {
        if constexpr (OP == AMX_OP_ADD) return a + b;
        else if constexpr (OP == AMX_OP_SUB) return a - b;
        else if constexpr (OP == AMX_OP_MUL) return a * b;
        else if constexpr (OP == AMX_OP_MIN) return a < b ? a : b;
        else if constexpr (OP == AMX_OP_MAX) return a > b ? a : b;
        else if constexpr (OP == AMX_OP_AND) return a & b;
        else if constexpr (OP == AMX_OP_OR) return a | b;
        else return a ^ b;
    }
};

// Width of op(a, b) for a-bit and b-bit operands (amx_binary_out_bits for the cheap ops).
constexpr int op_out_bits(int op, int a, int b)
{
    return op == AMX_OP_ADD ? (a > b ? a : b) + 1
           : op == AMX_OP_MUL ? a + b
           : (op == AMX_OP_MIN || op == AMX_OP_AND) ? (a < b ? a : b)
                                                    : (a > b ? a : b);
}

// PLAIN: the request is known to be a compacting pass with 16-bit gathered values, no input
// mask, no bitmask out and at most a sum, so the kernel carries only that path.  OP >= 0: the
// element-wise op is fixed too (one of the eight cheap ops); -1: chosen at run time.
template <int BA, int BB, bool PLAIN = false, int OP = -1>
struct Slab2Pol {
    using V = uint32_t;
    static constexpr int EA = 64 / BA;
    static constexpr int EB = 64 / BB;
    static constexpr int L = EA / ct_gcd<EA, EB>::value * EB;
    static constexpr int R = L >= 32 ? L : L * (32 / L);
    static constexpr int SA = R / EA;
    static constexpr int SB = R / EB;
    static constexpr bool kWarpMajor = false;
    static constexpr bool kSwar = false;
    static constexpr bool kPlain = PLAIN;
    static constexpr bool kFilter = false;
    static constexpr bool kAggOnly = false;
    static constexpr bool kMap = false;
    static constexpr bool kWide = false;
    // output width the encoder warps pack at compile time (slabs of the op's natural width)
    static constexpr int kOutBits = OP >= 0 ? op_out_bits(OP, BA, BB) : 0;
    // the plain variants run 20 compute warps where two stages and two slots of 16-bit values
    // still fit in 227 KB of shared memory (5632 bytes of control data first)
    static constexpr uint32_t kT20 = 640 * R;
    static constexpr bool kFits20 =
        5632u + 2u * (2u * kT20) + 2u * (8u * (kT20 / EA + 2) + 8u * (kT20 / EB + 2) + 352u) <= 227u * 1024u;
    static constexpr uint32_t kCompute = R > 40 ? 256 : ((PLAIN && kFits20) ? 640 : 512);
    static constexpr int kMinBlocks = 1;
    static_assert(R <= 64, "run too long for the flag word");

    __device__ __forceinline__ static void decode(const PipeParams& p, const uint8_t* st, const uint64_t* sb,
                                                  uint64_t e0, V (&v)[R], uint64_t& fl)
    {
        const uint64_t first = e0 + threadIdx.x * R;
        {
            const uint64_t* w = reinterpret_cast<const uint64_t*>(st + p.a_off) + (first / EA - sb[0] / 8);
            uint64_t s[SA];
            lds_words<SA>(w, s);
            unpack_slabs<BA, EA, SA, R>(s, v);
        }
        {
            const uint64_t* w = reinterpret_cast<const uint64_t*>(st + p.b_off) + (first / EB - sb[1] / 8);
            uint64_t s[SB];
            lds_words<SB>(w, s);
            if constexpr (OP >= 0) {
                combine_slabs<BB, EB, SB, R>(s, v, OpFn<OP>{});
            }
            else switch (p.op) {
                case AMX_OP_ADD: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a + b; }); break;
                case AMX_OP_SUB: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a - b; }); break;
                case AMX_OP_MUL: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a * b; }); break;
                case AMX_OP_MIN: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a < b ? a : b; }); break;
                case AMX_OP_MAX: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a > b ? a : b; }); break;
                case AMX_OP_AND: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a & b; }); break;
                case AMX_OP_OR: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a | b; }); break;
                default: combine_slabs<BB, EB, SB, R>(s, v, [](uint32_t a, uint32_t b) { return a ^ b; }); break;
            }
        }
        finish32<R>(p, v, fl);
    }

    // value of element i of this thread's run, re-read from the staged words (sparse gather)
    __device__ __forceinline__ static V value_at(const PipeParams& p, const uint8_t* st, const uint64_t* sb,
                                                 uint64_t e0, int i)
    {
        const uint64_t first = e0 + threadIdx.x * R;
        const uint64_t* wa = reinterpret_cast<const uint64_t*>(st + p.a_off) + (first / EA - sb[0] / 8);
        const uint64_t* wb = reinterpret_cast<const uint64_t*>(st + p.b_off) + (first / EB - sb[1] / 8);
        const uint32_t ja = (uint32_t)i / EA, ka = (uint32_t)i - ja * EA;
        const uint32_t jb = (uint32_t)i / EB, kb = (uint32_t)i - jb * EB;
        const uint32_t a = (uint32_t)((wa[ja] >> (ka * BA)) & ((1ull << BA) - 1));
        const uint32_t b = (uint32_t)((wb[jb] >> (kb * BB)) & ((1ull << BB) - 1));
        uint32_t x;
        if constexpr (OP >= 0) x = OpFn<OP>{}(a, b);
        else switch (p.op) {
            case AMX_OP_ADD: x = a + b; break;
            case AMX_OP_SUB: x = a - b; break;
            case AMX_OP_MUL: x = a * b; break;
            case AMX_OP_MIN: x = a < b ? a : b; break;
            case AMX_OP_MAX: x = a > b ? a : b; break;
            case AMX_OP_AND: x = a & b; break;
            case AMX_OP_OR: x = a | b; break;
            default: x = a ^ b; break;
        }
        if (p.need_vmask) x &= (uint32_t)p.vmask;
        return x;
    }
};

// Policy ids: 0 generic, 1..32 SlabPol<B>, 100+ Slab2Pol pairs, 201..232 SwarPol<B>.
constexpr int kSwarPolicyBase = 200;
#define AMX_SLAB2_PAIRS(X) X(100, 7, 13) X(101, 13, 7) X(102, 11, 11) X(103, 13, 13)

#define AMX_POLICY_LIST(X)                                                                                             \
    X(1, SlabPol<1>) X(2, SlabPol<2>) X(3, SlabPol<3>) X(4, SlabPol<4>) X(5, SlabPol<5>) X(6, SlabPol<6>)             \
    X(7, SlabPol<7>) X(8, SlabPol<8>) X(9, SlabPol<9>) X(10, SlabPol<10>) X(11, SlabPol<11>) X(12, SlabPol<12>)       \
    X(13, SlabPol<13>) X(14, SlabPol<14>) X(15, SlabPol<15>) X(16, SlabPol<16>) X(17, SlabPol<17>)                    \
    X(18, SlabPol<18>) X(19, SlabPol<19>) X(20, SlabPol<20>) X(21, SlabPol<21>) X(22, SlabPol<22>)                    \
    X(23, SlabPol<23>) X(24, SlabPol<24>) X(25, SlabPol<25>) X(26, SlabPol<26>) X(27, SlabPol<27>)                    \
    X(28, SlabPol<28>) X(29, SlabPol<29>) X(30, SlabPol<30>) X(31, SlabPol<31>) X(32, SlabPol<32>)                    \
    X(100, AMX_PAIR(7, 13)) X(101, AMX_PAIR(13, 7)) X(102, AMX_PAIR(11, 11)) X(103, AMX_PAIR(13, 13))
#define AMX_PAIR(a, b) Slab2Pol<a, b>

// A request the field-parallel slab policy (SwarPol) serves: one slab column of width <= 32, a
// predicate on the field values themselves and/or an input mask, and a compacted output or none;
// or a sum alone (every field passes) at a width whose field-parallel or bit-plane sum applies, or
// at 7 bits (field visit).  671M-element column against the compile-time policy: 11 bits 0.234 vs
// 0.366 ms, 8 bits 0.178 vs 0.336, 32 bits 0.473 vs 0.763, 1 bit 0.035 vs 0.361, 3 bits 0.083 vs
// 0.481, 7 bits 0.263 vs 0.397.  At 9 and 21 bits the compile-time policy keeps the sum: bit planes
// measured 0.482 vs 0.375 ms at 9 bits (the b <= 32 test comes first: the rule divides by 64 / b).
inline bool swar_applicable(const PipeParams& p)
{
    const int b = (int)p.a.bits;
    const bool agg_alone = !p.has_out && !p.mask_out && p.has_agg && p.agg == AMX_AGG_SUM && b <= 32 &&
                           (swar_sum_fits_slab(b) || b <= kSwarPlaneMax || b == 7);
    return !p.has_b && p.a.format == AMX_SLAB && p.a.bits <= 32 && (p.has_pred || p.has_mask_in || agg_alone) &&
           (!p.has_out || p.compact) && p.op == AMX_OP_LHS && !p.need_vmask && p.vbits <= 32;
}

// A request the PLAIN variants serve: compacting, 16-bit values, no input mask, no bitmask out,
// no aggregate or a sum.
inline bool plain_compacting(const PipeParams& p)
{
    return p.has_out && p.compact && !p.has_mask_in && !p.mask_out && p.vbits <= 16 &&
           (!p.has_agg || p.agg == AMX_AGG_SUM);
}

// Policy for a request: the field-parallel policy when it applies, else compile-time widths
// when every input is a slab column of width <= 32 and values fit 32 bits, else the generic
// runtime-width policy.  `force` >= 0 selects a policy directly (the autotuner and the tests);
// an inapplicable force falls back to the automatic choice.
inline int choose_policy(const PipeParams& p, int force)
{
    const bool v32 = p.vbits <= 32;
    const bool a_slab = p.a.format == AMX_SLAB && p.a.bits <= 32;
    const bool swar = swar_applicable(p);
    int auto_id = 0;
    int slab_id = -1;
    if (v32 && a_slab && !p.has_b) slab_id = (int)p.a.bits;
    // two-column compile-time policies cover the 32-bit-exact ops; the rest take the generic path
    const bool cheap_op = p.op == AMX_OP_ADD || p.op == AMX_OP_SUB || p.op == AMX_OP_MUL || p.op == AMX_OP_MIN ||
                          p.op == AMX_OP_MAX || p.op == AMX_OP_AND || p.op == AMX_OP_OR || p.op == AMX_OP_XOR;
    if (v32 && a_slab && p.has_b && p.b.format == AMX_SLAB && cheap_op) {
#define AMX_PAIR_MATCH(id, x, y) \
    if (p.a.bits == x && p.b.bits == y) slab_id = id;
        AMX_SLAB2_PAIRS(AMX_PAIR_MATCH)
#undef AMX_PAIR_MATCH
    }
    if (slab_id > 0) auto_id = slab_id;
    if (swar) auto_id = kSwarPolicyBase + (int)p.a.bits;
    if (force == 0) return 0;
    if (force > 0 && (force == slab_id || (swar && force == kSwarPolicyBase + (int)p.a.bits))) return force;
    return auto_id;
}

}  // namespace amx
