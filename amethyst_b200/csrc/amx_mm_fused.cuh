// amx_mm_fused.cuh -- the packed-matrix multiply with both operands unpacked in shared memory
// and the product packed straight out of the tensor memory (no u8 operand and no int32 product
// in HBM).  Instantiated for slab operands of one width W = 1..8 in amx_mm_fused_w*.cu; the
// host side (bound, edge clearing, finish) is in amx_mm_fused.cu.
//
// One persistent CTA per SM, 128 x 256 output tiles, K in 128-entry slices.  Two rings:
//   packed stages (2): the slice's packed words, staged by 2-D TMA loads of 64-bit elements --
//     A: 128 rows x 18 words (144-byte rows), B: 128 k-rows x 34 words (272-byte rows) -- from an
//     even word index at or below the slice's first word, so every copy starts 16-byte aligned;
//     rows and words past the matrix come in as zeros.  When a row pitch is not a multiple of 16
//     bytes (no tensor map possible) the unpackers read the words from global memory instead.
//   u8 stages (2), in the canonical tcgen05 layouts:
//     A slice (128 rows x 128 k, K-major, 128-byte swizzle): row r at r*128, its 16-byte chunk c
//       at ((c ^ (r & 7)) << 4) -- the layout a 2-D TMA load with SWIZZLE_128B writes;
//     B slice (128 k x 256 n, MN-major, 128-byte swizzle): 1024-byte atoms of 8 k-rows x 128 n;
//       atom (k-group g, n-half h) at g*2048 + h*1024, k-row r of the atom at r*128, 16-byte
//       chunk c of n at ((c ^ r) << 4).  The MMA's descriptor strides: 1024 bytes between
//       n-atoms, 2048 between k-groups (read either way round, a descriptor stays inside its
//       32 KB stage).
// Warp roles (18 warps):
//   warp 0       one lane issues the TMA loads of the packed stages;
//   warp 1       one lane issues tcgen05.mma kind::i8 (u8 x u8 -> s32, M 128, N 256, K 32; A
//                K-major, B MN-major) into one of two 256-column TMEM accumulators and releases
//                each u8 stage with tcgen05.commit;
//   warps 2..5   the epilogue: tcgen05.ld of the finished accumulator, the largest entry, and
//                the entries packed into the output format at the packing width;
//   warps 6..17  unpackers: per slice each takes 32 rows of A (4 warps) or 32 k-rows of one
//                128-column half of B (8 warps).  Lane = row, so all lanes of a warp start their
//                128-entry run at the same field o of a slab word: every warp extracts from
//                field 0 with compile-time word indices and shifts (two instructions per entry)
//                and drops the first o bytes with byte permutes (one code path for every
//                residue: small enough for the instruction cache).  A lane reads its words,
//                writes 8 swizzled 16-byte chunks and fences them for the tensor core's async
//                proxy; the warp then arrives on the u8 stage's full barrier and releases the
//                packed stage.
// Entries past M, N or K (and dirty padding fields of the slab rows) become zeros.
#pragma once

#include "amx_mm_common.cuh"

namespace amx {

constexpr uint32_t kMfUnpackWarps = 12;
constexpr uint32_t kMfThreads = 32 * (2 + 4 + kMfUnpackWarps);
constexpr uint32_t kMfStages = 2;                  // u8 stages
constexpr uint32_t kMfPStages = 2;                 // packed stages
constexpr uint32_t kMfPWordsA = 18, kMfPWordsB = 34;  // words per staged row (144 and 272 bytes)
constexpr uint32_t kMfPStageA = kMmBM * kMfPWordsA * 8;  // 18 KB
constexpr uint32_t kMfPStageB = kMmBK * kMfPWordsB * 8;  // 34 KB
constexpr uint32_t kMfSmem = 1024 + kMfStages * (kMmStageA + kMmStageB) + kMfPStages * (kMfPStageA + kMfPStageB) + 256;
// A K-major, B MN-major (instruction descriptor bit 16)
constexpr uint32_t kMfIdesc = kMmIdesc | (1u << 16);

struct MfParams {
    uint32_t M, N, K;
    uint32_t tiles_m, tiles_n, kblocks;
    const uint64_t* a;  // M rows of a_rs slab words
    const uint64_t* b;  // K rows of b_rs slab words
    uint32_t a_rs, b_rs;
    void* out;
    uint32_t out_format;
    uint32_t fixed_bits;  // packing width given by the caller, or 0: the width in hdr[2]
    uint32_t* hdr;        // [0] largest entry, [1] error word, [2] packing width
    uint32_t direct;      // 1: unpackers read the packed words from global memory (no tensor maps)
};

// shared-memory matrix descriptor: MN-major, 128-byte swizzle, n-atoms 1024 bytes apart, k-groups
// of 8 rows 2048 bytes apart
__device__ __forceinline__ uint64_t sdesc_mn_sw128(const void* p)
{
    const uint32_t a = smem_u32(p);
    return (uint64_t)((a & 0x3FFFFu) >> 4) | ((uint64_t)(1024 >> 4) << 16) | ((uint64_t)(2048 >> 4) << 32) |
           (1ull << 46) | (2ull << 61);
}

__host__ __device__ constexpr int mf_gcd(int a, int b) { return b == 0 ? a : mf_gcd(b, a % b); }

// A run of 128 entries of a W-bit slab row starting at a multiple of 128 starts at field
// O = e0 mod EPS of its first word, O a multiple of G = gcd(EPS, 128), so O <= EPS - G.  The
// extraction always starts at field 0 of that word and produces 128 + XB entries (XB = EPS - G
// rounded up to whole 32-bit words), then drops the first O bytes; NW words cover it.
template <int W>
struct MfRun {
    static constexpr int EPS = 64 / W;
    static constexpr int G = mf_gcd(EPS, 128);
    static constexpr int XB = (EPS - G + 3) / 4 * 4;
    static constexpr int NW = (127 + XB) / EPS + 1;
};

// bytes 0 .. 4N-1 of o[] (its first N little-endian words) = fields F0 .. F0 + 4N - 1 of the
// words w[] (w[0] holding field 0): compile-time word indices and shifts, two instructions per
// entry
template <int W, int F0, int N, int NO>
__device__ __forceinline__ void mf_extract(const uint64_t (&w)[MfRun<W>::NW], uint32_t (&o)[NO])
{
    static_assert(N <= NO, "output words");
    constexpr int EPS = 64 / W;
    constexpr uint32_t FM = (1u << W) - 1;
#pragma unroll
    for (int q = 0; q < N; q++) {
        const int f0 = F0 + 4 * q;
        uint32_t acc = 0;
        if (f0 % EPS + 3 < EPS) {
            // the 4 fields lie in one slab word: one shift brings them to bits 0, W, 2W, 3W, and
            // products by 2^(8b - bW) (the multiplier's pipe, not the shifter's) spread them
            const uint32_t t = (uint32_t)(w[f0 / EPS] >> ((f0 % EPS) * W));
            acc = t & FM;
#pragma unroll
            for (int b = 1; b < 4; b++) acc |= (t * (1u << (b * (8 - W)))) & (FM << (8 * b));
        }
        else {
#pragma unroll
            for (int b = 0; b < 4; b++) {
                const int f = f0 + b;
                const int i = f / EPS;
                const int s = (f % EPS) * W - 8 * b;  // field bit position minus its byte position
                const uint32_t x = s >= 0 ? (uint32_t)(w[i] >> s) : (uint32_t)(w[i] << (-s));
                acc |= x & (FM << (8 * b));
            }
        }
        o[q] = acc;
    }
}

// out[q] = bytes 4(q + D) + r .. +3 of x (r = the byte shift in `sel`), for D known here
template <int D, int N, int NX>
__device__ __forceinline__ void mf_shift_bytes(const uint32_t (&x)[NX], uint32_t sel, uint32_t (&out)[N])
{
#pragma unroll
    for (int q = 0; q < N; q++) out[q] = __byte_perm(x[q + D], x[q + D + 1], sel);
}

template <int DMAX, int N, int NX, int D = 0>
__device__ __forceinline__ void mf_shift_bytes_at(int d, const uint32_t (&x)[NX], uint32_t sel, uint32_t (&out)[N])
{
    if constexpr (D <= DMAX) {
        if (d == D) {
            mf_shift_bytes<D, N, NX>(x, sel, out);
            return;
        }
        mf_shift_bytes_at<DMAX, N, NX, D + 1>(d, x, sel, out);
    }
}

// half H of a run: bytes 64H .. 64H+63 = fields o + 64H .. o + 64H + 63 (o warp-uniform)
template <int W, int H>
__device__ __forceinline__ void mf_unpack_half(int o, const uint64_t (&w)[MfRun<W>::NW], uint32_t (&out)[16])
{
    constexpr int XB = MfRun<W>::XB;
    if constexpr (XB == 0) {
        mf_extract<W, 64 * H, 16>(w, out);
    }
    else {
        uint32_t x[16 + XB / 4 + 1];
        mf_extract<W, 64 * H, 16 + XB / 4>(w, x);
        x[16 + XB / 4] = 0;
        const uint32_t sel = 0x3210u + 0x1111u * (uint32_t)(o & 3);
        mf_shift_bytes_at<XB / 4>(o >> 2, x, sel, out);
    }
}

// The words of one unpacker task: lane = row `row` of a packed matrix (rows x rs words), the
// NW words from the one holding entry e0 -- read from the packed stage (`st`: this row's staged
// words, the first of them word x0 of the row) or, in direct mode, from global memory.
template <int W>
__device__ __forceinline__ void mf_words(const uint64_t* m, uint32_t rs, uint32_t rows, uint32_t row, uint32_t e0,
                                         uint32_t lim, const uint64_t* st, uint32_t x0, bool direct,
                                         uint64_t (&w)[MfRun<W>::NW])
{
    constexpr int EPS = MfRun<W>::EPS;
    constexpr int NW = MfRun<W>::NW;
    const uint32_t s0 = e0 / EPS;
    if (direct) {
        const bool live = row < rows && e0 < lim;
        const uint64_t* rp = m + (size_t)row * rs + s0;
#pragma unroll
        for (int i = 0; i < NW; i++)
            w[i] = (live && s0 + i < rs) ? __ldg(reinterpret_cast<const unsigned long long*>(rp + i)) : 0ull;
    }
    else {
        const uint64_t* sp = st + (s0 - x0);
#pragma unroll
        for (int i = 0; i < NW; i++) w[i] = sp[i];
    }
}

// entries e0 .. e0+127 from the words (entries >= lim are zero), written as 8 swizzled 16-byte
// chunks at dst + ((c ^ x) << 4); extracted and stored 64 entries at a time to keep the live
// registers down
template <int W>
__device__ __forceinline__ void mf_unpack_store(const uint64_t (&w)[MfRun<W>::NW], uint32_t e0, uint32_t lim, uint8_t* dst,
                                                uint32_t x)
{
    constexpr int EPS = MfRun<W>::EPS;
    const int o = (int)(e0 - (e0 / EPS) * EPS);
    const int keep = lim > e0 ? (int)(lim - e0) : 0;  // entries below lim
#pragma unroll
    for (int h = 0; h < 2; h++) {
        uint32_t out[16];
        if (h == 0)
            mf_unpack_half<W, 0>(o, w, out);
        else
            mf_unpack_half<W, 1>(o, w, out);
        if (keep < 64 * h + 64) {  // the ragged end of K or N (and dirty padding fields)
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int k = keep - 64 * h - 4 * q;
                out[q] = k <= 0 ? 0u : (k >= 4 ? out[q] : (out[q] & ((1u << (8 * k)) - 1)));
            }
        }
#pragma unroll
        for (int c = 0; c < 4; c++)
            *reinterpret_cast<uint4*>(dst + (((4 * h + c) ^ x) << 4)) =
                make_uint4(out[4 * c], out[4 * c + 1], out[4 * c + 2], out[4 * c + 3]);
    }
}

// ---------------------------------------------------------------------------------------------
// epilogue packers: one thread packs columns [c0, c1) of one row, in column order
// ---------------------------------------------------------------------------------------------
// A word the thread completed: stored, or or-ed in when it shares fields with a neighbouring
// tile (the word was cleared before the kernel).
__device__ __forceinline__ void mf_emit(uint64_t* out, uint64_t gw, uint64_t v, bool shared)
{
    if (shared)
        atomicOr(reinterpret_cast<unsigned long long*>(out + gw), (unsigned long long)v);
    else
        out[gw] = v;
}

struct MfSlabPacker {
    uint64_t* out;
    uint64_t gw, acc, fm;
    uint32_t f, eps, w;
    bool shared;
    __device__ __forceinline__ void start(void* o, uint32_t width, uint32_t N, uint32_t row, uint32_t c0)
    {
        out = reinterpret_cast<uint64_t*>(o);
        w = width;
        eps = 64 / width;
        fm = width >= 64 ? ~0ull : ((1ull << width) - 1);
        const uint32_t rw = (N + eps - 1) / eps;
        gw = (uint64_t)row * rw + c0 / eps;
        f = c0 % eps;
        shared = f != 0;
        acc = 0;
    }
    __device__ __forceinline__ void put(uint32_t v)
    {
        acc |= ((uint64_t)v & fm) << (f * w);
        if (++f == eps) {
            mf_emit(out, gw, acc, shared);
            gw++;
            f = 0;
            acc = 0;
            shared = false;
        }
    }
    __device__ __forceinline__ void finish()
    {
        if (f) mf_emit(out, gw, acc, true);
    }
};

struct MfBitsPacker {  // nogaps: entry (r, c) at bits [(r*N + c)*w, +w) of the stream
    uint64_t* out;
    uint64_t gw, acc, fm;
    uint32_t sh, w;
    bool shared;
    __device__ __forceinline__ void start(void* o, uint32_t width, uint32_t N, uint32_t row, uint32_t c0)
    {
        out = reinterpret_cast<uint64_t*>(o);
        w = width;
        fm = width >= 64 ? ~0ull : ((1ull << width) - 1);
        const uint64_t bit = ((uint64_t)row * N + c0) * width;
        gw = bit >> 6;
        sh = (uint32_t)(bit & 63);
        shared = sh != 0;
        acc = 0;
    }
    __device__ __forceinline__ void put(uint32_t v)
    {
        const uint64_t x = (uint64_t)v & fm;
        acc |= x << sh;
        if (sh + w >= 64) {
            mf_emit(out, gw, acc, shared);
            shared = false;
            gw++;
            acc = sh + w > 64 ? x >> (64 - sh) : 0;
            sh = sh + w - 64;
        }
        else {
            sh += w;
        }
    }
    __device__ __forceinline__ void finish()
    {
        if (sh) mf_emit(out, gw, acc, true);
    }
};

// ---------------------------------------------------------------------------------------------
// the kernel
// ---------------------------------------------------------------------------------------------
template <int W>
__global__ void __launch_bounds__(kMfThreads, 1)
    mf_gemm_kernel(const __grid_constant__ CUtensorMap tma, const __grid_constant__ CUtensorMap tmb,
                   const __grid_constant__ MfParams p)
{
    constexpr int EPS = MfRun<W>::EPS;
    extern __shared__ uint8_t mf_smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(mf_smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = sA + kMfStages * kMmStageA;
    uint8_t* pA = sB + kMfStages * kMmStageB;
    uint8_t* pB = pA + kMfPStages * kMfPStageA;
    uint64_t* full = reinterpret_cast<uint64_t*>(pB + kMfPStages * kMfPStageB);
    uint64_t* empty = full + kMfStages;
    uint64_t* pfull = empty + kMfStages;
    uint64_t* pempty = pfull + kMfPStages;
    uint64_t* tfull = pempty + kMfPStages;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* err = p.hdr + 1;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < kMfStages; s++) {
            mbar_init(&full[s], kMfUnpackWarps);  // one arrival per unpacker warp
            mbar_init(&empty[s], 1);              // tcgen05.commit
        }
        for (uint32_t s = 0; s < kMfPStages; s++) {
            mbar_init(&pfull[s], 1);                // the producer's arrival (+ the copies' bytes)
            mbar_init(&pempty[s], kMfUnpackWarps);  // every unpacker has consumed its words
        }
        for (uint32_t a = 0; a < 2; a++) {
            mbar_init(&tfull[a], 1);
            mbar_init(&tempty[a], 4);  // one arrival per epilogue warp
        }
        fence_mbar_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(kMmTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const uint32_t ntiles = p.tiles_m * p.tiles_n;

    if (warp == 0) {
        if (lane == 0) {  // packed-stage producer
            uint32_t st = 0, ph = 0;
            for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
                const uint32_t m0 = (t % p.tiles_m) * kMmBM, n0 = (t / p.tiles_m) * kMmBN;
                for (uint32_t kb = 0; kb < p.kblocks; kb++) {
                    wait_or_flag(&pempty[st], ph ^ 1, err);
                    if (p.direct) {
                        mbar_arrive(&pfull[st]);
                    }
                    else {
                        mbar_arrive_expect_tx(&pfull[st], kMfPStageA + kMfPStageB);
                        tma_load_2d(pA + st * kMfPStageA, &tma, (int32_t)((kb * kMmBK / EPS) & ~1u), (int32_t)m0, &pfull[st]);
                        tma_load_2d(pB + st * kMfPStageB, &tmb, (int32_t)((n0 / EPS) & ~1u), (int32_t)(kb * kMmBK), &pfull[st]);
                    }
                    if (++st == kMfPStages) {
                        st = 0;
                        ph ^= 1;
                    }
                }
            }
            // every issued copy has landed once the unpackers have released its stage
            for (uint32_t i = 0; i < kMfPStages; i++) {
                wait_or_flag(&pempty[st], ph ^ 1, err);
                if (++st == kMfPStages) {
                    st = 0;
                    ph ^= 1;
                }
            }
        }
        __syncwarp();
    }
    else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            uint32_t st = 0, ph = 0, i = 0;
            for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
                const uint32_t acc = i & 1, aph = (i >> 1) & 1;
                wait_or_flag(&tempty[acc], aph ^ 1, err);  // the epilogue has drained this accumulator
                tc_fence_after();
                const uint32_t d = tmem + acc * kMmBN;
                for (uint32_t kb = 0; kb < p.kblocks; kb++) {
                    wait_or_flag(&full[st], ph, err);
                    tc_fence_after();
                    const uint8_t* a_st = sA + st * kMmStageA;
                    const uint8_t* b_st = sB + st * kMmStageB;
#pragma unroll
                    for (uint32_t kk = 0; kk < kMmBK / 32; kk++)
                        umma_i8(d, sdesc_sw128(a_st) + 2 * kk, sdesc_mn_sw128(b_st + kk * 8192), kMfIdesc,
                                (kb | kk) != 0);
                    umma_commit(&empty[st]);  // the stage is free once these MMAs have read it
                    if (++st == kMfStages) {
                        st = 0;
                        ph ^= 1;
                    }
                }
                umma_commit(&tfull[acc]);  // accumulator complete
            }
        }
        __syncwarp();
    }
    else if (warp <= 5) {  // epilogue: TMEM lanes 32*(warp%4) .. +31
        const uint32_t q = warp & 3;
        const uint32_t width = p.fixed_bits ? p.fixed_bits : p.hdr[2];
        uint32_t mymax = 0, i = 0;
        for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
            const uint32_t acc = i & 1, aph = (i >> 1) & 1;
            wait_or_flag(&tfull[acc], aph, err);
            __syncwarp();  // tcgen05.ld is warp-collective
            tc_fence_after();
            const uint32_t row = (t % p.tiles_m) * kMmBM + q * 32 + lane;
            const uint32_t colt = (t / p.tiles_m) * kMmBN;
            const uint32_t cend = colt + kMmBN < p.N ? colt + kMmBN : p.N;
            const bool live = row < p.M;
            MfSlabPacker sp;
            MfBitsPacker bp;
            if (live && p.out_format == AMX_SLAB) sp.start(p.out, width, p.N, row, colt);
            if (live && p.out_format == AMX_NOGAPS) bp.start(p.out, width, p.N, row, colt);
            const uint64_t fm = (p.fixed_bits == 0 || p.fixed_bits >= 32) ? 0xffffffffull : ((1ull << p.fixed_bits) - 1);
#pragma unroll 1
            for (uint32_t cb = 0; cb < kMmBN / 32; cb++) {
                uint32_t r[32];
                tmem_ld32(tmem + acc * kMmBN + cb * 32 + ((q * 32) << 16), r);
                const uint32_t col0 = colt + cb * 32;
                if (!live || col0 >= cend) continue;
                const uint32_t cnt = cend - col0 < 32 ? cend - col0 : 32;
#pragma unroll
                for (int e = 0; e < 32; e++)
                    if ((uint32_t)e < cnt) mymax = r[e] > mymax ? r[e] : mymax;
                if (p.out_format == AMX_PLAIN32) {
                    uint32_t* dst = reinterpret_cast<uint32_t*>(p.out) + (size_t)row * p.N + col0;
                    if (cnt == 32 && (p.N & 3) == 0) {
#pragma unroll
                        for (int e = 0; e < 8; e++)
                            reinterpret_cast<uint4*>(dst)[e] =
                                make_uint4(r[4 * e] & (uint32_t)fm, r[4 * e + 1] & (uint32_t)fm, r[4 * e + 2] & (uint32_t)fm,
                                           r[4 * e + 3] & (uint32_t)fm);
                    }
                    else {
#pragma unroll
                        for (int e = 0; e < 32; e++)
                            if ((uint32_t)e < cnt) dst[e] = r[e] & (uint32_t)fm;
                    }
                }
                else if (p.out_format == AMX_PLAIN64) {
                    unsigned long long* dst = reinterpret_cast<unsigned long long*>(p.out) + (size_t)row * p.N + col0;
                    if (cnt == 32 && (p.N & 1) == 0) {
#pragma unroll
                        for (int e = 0; e < 16; e++)
                            reinterpret_cast<ulonglong2*>(dst)[e] = make_ulonglong2(r[2 * e] & fm, r[2 * e + 1] & fm);
                    }
                    else {
#pragma unroll
                        for (int e = 0; e < 32; e++)
                            if ((uint32_t)e < cnt) dst[e] = r[e] & fm;
                    }
                }
                else if (p.out_format == AMX_SLAB) {
#pragma unroll
                    for (int e = 0; e < 32; e++)
                        if ((uint32_t)e < cnt) sp.put(r[e]);
                }
                else {
#pragma unroll
                    for (int e = 0; e < 32; e++)
                        if ((uint32_t)e < cnt) bp.put(r[e]);
                }
            }
            if (live && p.out_format == AMX_SLAB) sp.finish();
            if (live && p.out_format == AMX_NOGAPS) bp.finish();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[acc]);
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) {
            const uint32_t y = __shfl_xor_sync(0xffffffffu, mymax, o);
            mymax = y > mymax ? y : mymax;
        }
        if (lane == 0 && mymax) atomicMax(p.hdr, mymax);
    }
    else {  // unpackers
        const uint32_t u = warp - 6;
        const bool is_a = u < 4;
        const uint32_t g = is_a ? u : (u - 4) & 3;  // row group of 32
        const uint32_t h = is_a ? 0 : (u - 4) >> 2;  // B: n-half of the slice
        const uint32_t x = lane & 7;                 // swizzle row of this lane's rows
        const uint32_t r = 32 * g + lane;            // row of the slice (A: tile row, B: k-row)
        uint32_t st = 0, ph = 0, pst = 0, pph = 0;
        for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const uint32_t m0 = (t % p.tiles_m) * kMmBM, n0 = (t / p.tiles_m) * kMmBN;
            for (uint32_t kb = 0; kb < p.kblocks; kb++) {
                uint64_t w[MfRun<W>::NW];
                const uint32_t e0 = is_a ? kb * kMmBK : n0 + 128 * h;
                wait_or_flag(&pfull[pst], pph, err);
                if (is_a)
                    mf_words<W>(p.a, p.a_rs, p.M, m0 + r, e0, p.K,
                                reinterpret_cast<const uint64_t*>(pA + pst * kMfPStageA) + r * kMfPWordsA,
                                (kb * kMmBK / EPS) & ~1u, p.direct != 0, w);
                else
                    mf_words<W>(p.b, p.b_rs, p.K, kb * kMmBK + r, e0, p.N,
                                reinterpret_cast<const uint64_t*>(pB + pst * kMfPStageB) + r * kMfPWordsB,
                                (n0 / EPS) & ~1u, p.direct != 0, w);
                // The packed stage is released only once its words have been consumed (after the
                // u8 chunks are written and fenced below): released right after the loads, the
                // compiler may read the words from shared memory again later, when the next TMA
                // load is already filling the stage (measured: wrong A entries in some rows).
                const uint32_t rel = pst;
                if (++pst == kMfPStages) {
                    pst = 0;
                    pph ^= 1;
                }
                wait_or_flag(&empty[st], ph ^ 1, err);
                if (is_a)
                    mf_unpack_store<W>(w, e0, p.K, sA + st * kMmStageA + r * 128, x);
                else
                    mf_unpack_store<W>(w, e0, p.N, sB + st * kMmStageB + (r >> 3) * 2048 + h * 1024 + (r & 7) * 128, x);
                // the tensor core reads the stage through the async proxy
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) mbar_arrive(&full[st]);
                if (lane == 0) mbar_arrive(&pempty[rel]);  // every word has been consumed
                if (++st == kMfStages) {
                    st = 0;
                    ph ^= 1;
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMmTmemCols) : "memory");
    }
}

template <int W>
amx_status mf_launch_w(const CUtensorMap& tma, const CUtensorMap& tmb, const MfParams& p, cudaStream_t s)
{
    cudaError_t e = cudaFuncSetAttribute(mf_gemm_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMfSmem);
    if (e != cudaSuccess) return cuda_fail(e, "matmul: shared memory attribute");
    const uint32_t tiles = p.tiles_m * p.tiles_n;
    const uint32_t grid = tiles < (uint32_t)sm_count() ? tiles : (uint32_t)sm_count();
    mf_gemm_kernel<W><<<grid, kMfThreads, kMfSmem, s>>>(tma, tmb, p);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: fused launch");
    return AMX_OK;
}

}  // namespace amx
