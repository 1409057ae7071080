// amx_swar.cuh -- field-parallel ("SIMD within a register") predicates on slab words.
//
// A slab word holds eps = floor(64/B) fields of B bits.  Instead of extracting every field and
// comparing it, one 64-bit subtraction compares all fields of a word with a constant at once:
//
//   H  = the top bit of every field,  LM = the other B-1 bits of every field,
//   t  = (x | H) - (rep(c) & LM)       per field: (x_low + 2^(B-1)) - c_low, never borrows
//                                      across fields, and its top bit is [x_low >= c_low];
//   ge = (c_top ? x & t : x | t) & H   top bit of every field = [x >= c]
//
// so a predicate costs a handful of integer instructions per word instead of per element.
// The flags stay in place (bit k*B+B-1 of g = element k of the word passes); counting is a
// popcount, and survivors are read back from the word they came from.  The predicate is
// turned into an interval of passing values (or its complement) on the host.
//
// The reference evaluates the predicate element by element after unpacking each field
// (src/kernels/filter_slabs.cuh:31-55, get_element in src/common_code.cuh:43-50).
#pragma once

#include "amx_device.cuh"

namespace amx {

// load N consecutive 64-bit words from a stage released right after (volatile reads), 16 bytes
// at a time when aligned
template <int N>
__device__ __forceinline__ void lds_words(const uint64_t* src, uint64_t (&w)[N])
{
    if constexpr (N % 2 == 0) {
        const uint4* s = reinterpret_cast<const uint4*>(src);
#pragma unroll
        for (int i = 0; i < N / 2; i++) {
            const uint4 x = lds_v4_v(s + i);
            w[2 * i] = ((uint64_t)x.y << 32) | x.x;
            w[2 * i + 1] = ((uint64_t)x.w << 32) | x.z;
        }
    }
    else {
#pragma unroll
        for (int i = 0; i < N; i++) w[i] = lds_u64_v(src + i);
    }
}

// The 8 consecutive 64-bit words of this thread, for threads that own 64 contiguous bytes each
// (src 128-byte aligned for even lanes).  Read as four 16-byte chunks in the natural order, the
// 8 lanes of a quarter warp would hit only two 16-byte bank groups (a 4-way conflict); lane pair
// r = (lane / 2) mod 4 reads its chunks rotated by r instead, so the quarter warp covers all 8
// groups, and two register selects per chunk rotate them back.
__device__ __forceinline__ void lds_words8_rot(const uint64_t* src, uint64_t (&w)[8])
{
    const uint32_t r = (threadIdx.x >> 1) & 3;
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4 t[4], u[4];
#pragma unroll
    for (int k = 0; k < 4; k++) t[k] = lds_v4_v(s + ((k + r) & 3));  // t[k] = chunk (k + r) mod 4
#pragma unroll
    for (int c = 0; c < 4; c++) u[c] = (r & 1) ? t[(c + 3) & 3] : t[c];  // u[c] = t[c - (r & 1)]
#pragma unroll
    for (int c = 0; c < 4; c++) t[c] = (r & 2) ? u[(c + 2) & 3] : u[c];  // t[c] = chunk c
#pragma unroll
    for (int c = 0; c < 4; c++) {
        w[2 * c] = ((uint64_t)t[c].y << 32) | t[c].x;
        w[2 * c + 1] = ((uint64_t)t[c].w << 32) | t[c].z;
    }
}

// the top bit of each of the floor(64/b) fields of a slab word
__host__ __device__ constexpr uint64_t swar_top_bits(int b)
{
    uint64_t h = 0;
    for (int k = 0; k < 64 / b; k++) h |= 1ull << (k * b + b - 1);
    return h;
}

// One slab column of width B with a predicate, evaluated field-parallel.  Each compute thread
// owns SPT consecutive slabs of a tile (R = SPT * eps elements, R <= 64).  PLAIN: the request is
// known to be the plain compressstore (slabs of width B <= 16 out, 16-bit gathered values, no
// aggregate, no bitmask), so the kernel carries only that path: less code for the instruction
// cache to hold next to the other warp roles.  FILTER: likewise for a request that only writes
// the bitmask; AGGONLY: for one that only counts and aggregates.  WIDE (with AGGONLY, for a count
// and at most a sum, no input mask): 8 slabs per thread at every width, runs past 64 elements, as
// no flag or mask word of the run is kept (1-4-bit columns: tiles of 4-12 KB otherwise).
template <int B, bool PLAIN = false, bool FILTER = false, bool AGGONLY = false, bool NARROW = false,
          bool WIDE = false>
struct SwarPol {
    using V = uint32_t;
    static constexpr int kBits = B;
    static constexpr int EPS = 64 / B;
    static constexpr int SPT = WIDE ? 8 : (EPS >= 64 ? 1 : (64 / EPS < 8 ? 64 / EPS : 8));
    static constexpr int R = EPS * SPT;
    static constexpr bool kWarpMajor = false;
    static constexpr bool kSwar = true;
    static constexpr bool kPlain = PLAIN;
    static constexpr bool kFilter = FILTER;    // the request only writes the bitmask
    static constexpr bool kAggOnly = AGGONLY;  // the request only counts and aggregates
    static constexpr bool kWide = WIDE;        // ... and at most sums, with no input mask
    static constexpr bool kMap = false;
    // the plain compressstore at widths of at most 5 fields per slab runs 24 compute warps (its
    // registers allow 960 threads): more warps to hide the compute warps' latencies
    // (NARROW: 16 compute warps always -- the plain compressstore by an input mask, whose mask
    // stage would leave the 24-warp form one survivor slot)
    static constexpr uint32_t kCompute = ((PLAIN || FILTER || AGGONLY) && EPS * SPT <= 40 && !NARROW) ? 768 : 512;
    static constexpr int kMinBlocks = 1;
    static constexpr uint64_t kField = (1ull << B) - 1;  // one field
    static constexpr uint64_t kTop = swar_top_bits(B);    // the top bit of every field
    static_assert(R <= 64 || (WIDE && AGGONLY), "a thread's run must fit one 64-bit flag word");
    static_assert(!PLAIN || B <= 16, "the plain compressstore gathers 16-bit values");
};

// The E = floor(64/B) flags of a slab word (the top bit of each B-bit field of g, nothing else
// set) gathered into bits 0..E-1 by one multiplication, for B >= 8.  With
// M = sum_j 2^((E-1-j)(B-1)) the product term of field k and multiplier term j sits at bit
// E(B-1) + k + (k-j)(B-1): j = k lands field k's flag at bit E(B-1) + k; k > j lands at or above
// E(B-1) + E for B >= 9 (at B = 8 past bit 63); k < j lands below E(B-1), at distinct bits whose
// sum stays below 2^(E(B-1)), so nothing carries into the window.  Terms past bit 63 drop out of
// the 64-bit product without touching it.  tests/test_swar_cpu.py checks every pattern of every
// width 8..32 (and that B = 7 fails).
__host__ __device__ constexpr uint64_t swar_gather_mul(int b)
{
    uint64_t m = 0;
    for (int j = 0; j < 64 / b; j++) m |= 1ull << ((64 / b - 1 - j) * (b - 1));
    return m;
}

template <int B>
__device__ __forceinline__ uint32_t swar_gather_flags(uint64_t g)
{
    static_assert(B >= 8 && B <= 32, "the single-product gather is exact for 8..32-bit fields");
    constexpr int E = 64 / B;
    return (uint32_t)((g * swar_gather_mul(B)) >> (E * (B - 1))) & ((1u << E) - 1);
}

// The inverse of swar_gather_flags: bits 0..E-1 of m (E = floor(64/B)) placed on the top bits of
// the E fields of a slab word, for an input mask.  A chunk of C <= B-1 flags times
// D = sum_{j<C} 2^(j(B-1)) puts flag k at bit kB (term j = k); every other term (k != j, at bit
// k + j(B-1)) falls on a bit that is no multiple of B and that no other term takes, since
// |k - k'| < B - 1, so the product is a plain OR of shifted copies with no carries.  Chunks are
// ORed in at offsets k0*B, and one shift and mask move bit kB to the field's top bit.  Bits of m
// above E land past bit 63 or off the field tops.  One product per word for B >= 9, two for
// B = 6..8, up to 32 for B = 2.  tests/test_swar_cpu.py checks every width against bit-by-bit
// placement.
__host__ __device__ constexpr uint64_t swar_deposit_mul(int b, int c)
{
    uint64_t d = 0;
    for (int j = 0; j < c; j++) d |= 1ull << (j * (b - 1));
    return d;
}

template <int B>
__device__ __forceinline__ uint64_t swar_deposit_flags(uint64_t m)
{
    if constexpr (B == 1) {
        return m;
    }
    else {
        constexpr int E = 64 / B;
        constexpr int C = (B - 1) < E ? (B - 1) : E;
        constexpr uint64_t D = swar_deposit_mul(B, C);
        uint64_t r = 0;
#pragma unroll
        for (int k0 = 0; k0 < E; k0 += C) r |= (((m >> k0) & ((1ull << C) - 1)) * D) << (k0 * B);
        return (r << (B - 1)) & swar_top_bits(B);
    }
}

// g[i] = in-place flags of word x[i] for the interval test selected by the template flags
template <int B, int N, bool LO, bool HI, bool LOTOP, bool HITOP>
__device__ __forceinline__ void swar_flags_t(const uint64_t (&x)[N], uint64_t (&g)[N], uint64_t l1, uint64_t l2)
{
    constexpr uint64_t H = SwarPol<B>::kTop;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint64_t xh = x[i] | H;
        uint64_t f = H;
        if (LO) {
            const uint64_t t = xh - l1;
            f = LOTOP ? (x[i] & t & H) : ((x[i] | t) & H);
        }
        if (HI) {
            const uint64_t t = xh - l2;
            const uint64_t ge = HITOP ? (x[i] & t) : (x[i] | t);
            f &= ~ge;
        }
        g[i] = f;
    }
}

template <int B, int N>
__device__ __forceinline__ void swar_flags(uint32_t mode, const uint64_t (&x)[N], uint64_t (&g)[N], uint64_t l1,
                                           uint64_t l2)
{
    constexpr uint64_t H = SwarPol<B>::kTop;
    switch (mode & 15) {
#define AMX_SW_CASE(m) \
    case m: swar_flags_t<B, N, (m & 1) != 0, (m & 2) != 0, (m & 4) != 0, (m & 8) != 0>(x, g, l1, l2); break;
        AMX_SW_CASE(0) AMX_SW_CASE(1) AMX_SW_CASE(2) AMX_SW_CASE(3) AMX_SW_CASE(5) AMX_SW_CASE(7) AMX_SW_CASE(10)
        AMX_SW_CASE(11) AMX_SW_CASE(15)
#undef AMX_SW_CASE
        default:  // unreachable: a top flag is only set together with its test
#pragma unroll
            for (int i = 0; i < N; i++) g[i] = 0;
            break;
    }
    if (mode & kSwNone) {
#pragma unroll
        for (int i = 0; i < N; i++) g[i] = 0;
    }
    if (mode & kSwNeg) {
#pragma unroll
        for (int i = 0; i < N; i++) g[i] ^= H;
    }
}

// Sum of the passing fields of a thread's SPT words, field-parallel: the flags (top bits of the
// passing fields) times the field mask give whole-field masks (each product term fills exactly its
// own field: no carries), and the even and the odd fields accumulate in two words whose lanes are
// two fields wide.  swar_sum_fits<B, SPT>() says whether every lane holds the sum of SPT fields
// (tests/test_swar_cpu.py models it against field-by-field sums); the others sum field by field.
__host__ __device__ constexpr bool swar_sum_fits_w(int B, int SPT)
{
    int need = B;
    for (int s = SPT; s > 0; s >>= 1) need++;  // B + bit length of SPT
    for (int k = 0; k < 64 / B; k++) {
        // odd fields are shifted down by B: odd field k's lane starts at bit (k - 1) B, and the top
        // lane of either accumulator may grow to bit 63
        int room = (k % 2 == 0) ? 64 - k * B : 64 - (k - 1) * B;
        if (room > 2 * B) room = 2 * B;
        if (room < need) return false;
    }
    return true;
}

template <int B, int SPT>
__host__ __device__ constexpr bool swar_sum_fits()
{
    return swar_sum_fits_w(B, SPT);
}

// The same for SwarPol<B>'s own SPT (min(8, 64 / EPS), 1 at EPS = 64), at a width known at run time
__host__ __device__ constexpr bool swar_sum_fits_slab(int B)
{
    return swar_sum_fits_w(B, 64 / B >= 64 ? 1 : (64 / (64 / B) < 8 ? 64 / (64 / B) : 8));
}
static_assert(swar_sum_fits_slab(7) == swar_sum_fits<7, SwarPol<7>::SPT>() &&
                  swar_sum_fits_slab(11) == swar_sum_fits<11, SwarPol<11>::SPT>() &&
                  swar_sum_fits_slab(16) == swar_sum_fits<16, SwarPol<16>::SPT>() &&
                  swar_sum_fits_slab(1) == swar_sum_fits<1, SwarPol<1>::SPT>(),
              "host rule follows the policy's SPT");

template <int B, int SPT>
__device__ __forceinline__ uint64_t swar_masked_sum(const uint64_t (&x)[SPT], const uint64_t (&g)[SPT])
{
    constexpr int EPS = 64 / B;
    constexpr uint64_t FM = (1ull << B) - 1;
    constexpr uint64_t EVEN = [] {
        uint64_t e = 0;
        for (int k = 0; k < 64 / B; k += 2) e |= ((1ull << B) - 1) << (k * B);
        return e;
    }();
    uint64_t a = 0, b = 0;
#pragma unroll
    for (int i = 0; i < SPT; i++) {
        const uint64_t m = x[i] & ((g[i] >> (B - 1)) * FM);
        a += m & EVEN;
        b += (m >> B) & EVEN;
    }
    uint64_t t = 0;
#pragma unroll
    for (int k = 0; k < EPS; k += 2) {
        const int ra = 64 - k * B < 2 * B ? 64 - k * B : 2 * B;
        t += (a >> (k * B)) & (ra >= 64 ? ~0ull : ((1ull << ra) - 1));
        if (k + 1 < EPS) {
            const int rb = ra;  // odd field k + 1, shifted down to bit k B
            t += (b >> (k * B)) & (rb >= 64 ? ~0ull : ((1ull << rb) - 1));
        }
    }
    return t;
}

// Sum of the passing fields by bit planes, for the narrow widths whose lanes swar_masked_sum cannot
// hold at the policy's SPT (3 bits; 1-3 bits with the wide variant's 8 slabs per thread): the
// passing fields (whole-field masks as there) are counted per bit position b and each count weighted
// by 2^b.  B population counts per word, nothing to overflow.  671M-field column, no predicate:
// 1 bit 0.035 ms, 3 bits 0.083 against 0.361 and 0.481 with the compile-time policy (at 4 bits the
// lanes beat the planes, 0.100 vs 0.118 ms; at 7 bits the field visit, 0.263 vs 0.312 ms; at 9 the
// compile-time policy).  kSwarPlaneMax is also the widest width of the wide count-and-sum variant.
constexpr int kSwarPlaneMax = 4;

template <int B, int SPT>
__device__ __forceinline__ uint64_t swar_plane_sum(const uint64_t (&x)[SPT], const uint64_t (&g)[SPT])
{
    constexpr uint64_t FM = (1ull << B) - 1;
    constexpr uint64_t LOW = [] {
        uint64_t e = 0;
        for (int k = 0; k < 64 / B; k++) e |= 1ull << (k * B);
        return e;
    }();
    uint32_t cnt[B];
#pragma unroll
    for (int b = 0; b < B; b++) cnt[b] = 0;
#pragma unroll
    for (int i = 0; i < SPT; i++) {
        const uint64_t m = x[i] & ((g[i] >> (B - 1)) * FM);
#pragma unroll
        for (int b = 0; b < B; b++) cnt[b] += __popcll(m & (LOW << b));
    }
    uint64_t t = 0;
#pragma unroll
    for (int b = 0; b < B; b++) t += (uint64_t)cnt[b] << b;
    return t;
}

// Dense walk of the plain compressstore: for every field whose flag is set, the low 16 bits from
// the field's first bit on (the field, then bits of the next one, which the slab encoder masks off)
// stored at the running position.  Works on the 32-bit halves of each word: a field costs a flag
// test, one shift (none for field 0; a funnel shift for the field across the halves), and the
// predicated store and advance.
template <int B, int SPT>
__device__ __forceinline__ void swar_store_dense_raw(const uint64_t (&x)[SPT], const uint64_t (&g)[SPT],
                                                     uint16_t* d)
{
    constexpr int EPS = 64 / B;
#pragma unroll
    for (int i = 0; i < SPT; i++) {
        const uint32_t lo = (uint32_t)x[i], hi = (uint32_t)(x[i] >> 32);
        const uint32_t glo = (uint32_t)g[i], ghi = (uint32_t)(g[i] >> 32);
#pragma unroll
        for (int k = 0; k < EPS; k++) {
            const int sb = k * B, fb = sb + B - 1;
            const bool pass = fb < 32 ? ((glo >> fb) & 1u) != 0 : ((ghi >> (fb - 32)) & 1u) != 0;
            uint32_t v;
            if (sb >= 32)
                v = hi >> (sb - 32);
            else if (sb + B <= 32)
                v = lo >> sb;
            else
                v = __funnelshift_r(lo, hi, sb);
            if (pass) *d++ = (uint16_t)v;
        }
    }
}

// Visit the passing elements of a thread's run in element order: store each value to dst[pos++]
// (when DST) and fold it into the aggregate `a` (when AGG).  Dense warps walk every field with a
// predicated store (no branches, independent extractions); sparse warps walk the set flag bits
// only, a serial chain per survivor that only pays off when survivors are rare.
template <int B, int N, typename D, bool DST, bool AGG>
__device__ __forceinline__ void swar_visit(const uint64_t (&x)[N], const uint64_t (&g)[N], bool dense, D* dst,
                                           uint32_t pos, uint32_t agg, uint64_t& a)
{
    constexpr int EPS = SwarPol<B>::EPS;
    constexpr uint64_t FM = SwarPol<B>::kField;
    if (dense) {
#pragma unroll
        for (int i = 0; i < N; i++)
#pragma unroll
            for (int k = 0; k < EPS; k++)
                if ((g[i] >> (k * B + B - 1)) & 1) {
                    const uint32_t v = (uint32_t)((x[i] >> (k * B)) & FM);
                    if (DST) dst[pos++] = (D)v;
                    if (AGG) a = agg_combine(agg, a, agg_encode(agg, v));
                }
    }
    else {
#pragma unroll
        for (int i = 0; i < N; i++)
            for (uint64_t f = g[i]; f; f &= f - 1) {
                const int bp = __ffsll((long long)f) - 1;
                const uint32_t v = (uint32_t)((x[i] >> (bp - (B - 1))) & FM);
                if (DST) dst[pos++] = (D)v;
                if (AGG) a = agg_combine(agg, a, agg_encode(agg, v));
            }
    }
}

}  // namespace amx
