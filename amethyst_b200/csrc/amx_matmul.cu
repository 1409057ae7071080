// amx_matmul.cu -- dense packed-integer matrix multiply on the 5th-generation tensor cores.
//
// C (M x N) = A (M x K) * B (K x N) for unsigned entries of at most 8 bits, exact, with int32
// accumulation (the caller's widths must keep K * max(A) * max(B) below 2^31).  The reference
// has no matrix kernel; it defines the slab matrix layout (get_matrix_element,
// src/common_code.cuh:124-129: row-major, every row padded to whole slabs) that the packed
// operands and the packed result use here.
//
// Two paths.  The fused path (amx_mm_fused.cuh; slab operands of one width 1..8, selected with
// amx_tuning.policy = 2 or 3): unpacker warps of the GEMM kernel turn the packed operands into
// u8 tiles in its shared memory and the epilogue packs the product straight from the tensor
// memory, so no operand or product is ever decompressed to HBM.  It unpacks every A slice once
// per tile column and every B slice once per tile row (16x and 32x at 4096^3) on the ALU pipes,
// and measured 1.5-2.3x slower than the two-pass path for K = 128..4096 at 4 and 7 bits, so the
// automatic choice is the two-pass path here, three stream-ordered steps:
//   1. mm_unpack_rows / mm_unpack_cols: the packed operands become u8 matrices in the workspace,
//      A as M x K and B transposed to N x K (both K-major, rows padded to 128 bytes, padding 0).
//   2. mm_gemm_kernel: persistent CTAs, one per SM, 128 x 256 output tiles.  One lane of warp 0
//      streams 128-byte-deep K slices of A and B into a 4-stage shared-memory ring with 2-D TMA
//      loads (128-byte swizzle, no multicast); one lane of warp 1 issues tcgen05.mma kind::i8
//      (u8 x u8 -> s32, 128 x 256 x 32 per instruction) into one of two 256-column TMEM
//      accumulators and releases each stage with tcgen05.commit; warps 2..5 drain the other
//      accumulator with tcgen05.ld, store int32 C and track its largest entry.
//   3. mm_pack: C is written in the output format at the requested width, or at the narrowest
//      width that holds the largest entry (written to *d_out_bits).
// Every mbarrier wait is bounded; a wait that runs out records AMX_ERR_TIMEOUT in the workspace.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "amx_dispatch.h"
#include "amx_mm_common.cuh"

namespace amx {

struct MmParams {
    uint32_t M, N, K;
    uint32_t tiles_m, tiles_n, kblocks;
    int32_t* c;  // M x N, row pitch N
    uint32_t* hdr;  // [0] largest entry, [1] error word
};

// ---------------------------------------------------------------------------------------------
// GEMM
// ---------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kMmThreads, 1)
    mm_gemm_kernel(const __grid_constant__ CUtensorMap tma, const __grid_constant__ CUtensorMap tmb,
                   const __grid_constant__ MmParams p)
{
    extern __shared__ uint8_t mm_smem_raw[];
    uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(mm_smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t* sA = smem;
    uint8_t* sB = smem + kMmStages * kMmStageA;
    uint64_t* full = reinterpret_cast<uint64_t*>(sB + kMmStages * kMmStageB);
    uint64_t* empty = full + kMmStages;
    uint64_t* tfull = empty + kMmStages;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tempty + 2);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint32_t* err = p.hdr + 1;

    if (threadIdx.x == 0) {
        for (uint32_t s = 0; s < kMmStages; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
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
        if (lane == 0) {  // TMA producer
            uint32_t st = 0, ph = 0;
            for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x) {
                const int32_t ym = (int32_t)((t % p.tiles_m) * kMmBM), yn = (int32_t)((t / p.tiles_m) * kMmBN);
                for (uint32_t kb = 0; kb < p.kblocks; kb++) {
                    wait_or_flag(&empty[st], ph ^ 1, err);
                    mbar_arrive_expect_tx(&full[st], kMmStageA + kMmStageB);
                    tma_load_2d(sA + st * kMmStageA, &tma, (int32_t)(kb * kMmBK), ym, &full[st]);
                    tma_load_2d(sB + st * kMmStageB, &tmb, (int32_t)(kb * kMmBK), yn, &full[st]);
                    if (++st == kMmStages) {
                        st = 0;
                        ph ^= 1;
                    }
                }
            }
            // every issued copy has landed once the MMA warp has released its stage
            for (uint32_t i = 0; i < kMmStages; i++) {
                wait_or_flag(&empty[st], ph ^ 1, err);
                if (++st == kMmStages) {
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
                    const uint64_t ad = sdesc_sw128(sA + st * kMmStageA), bd = sdesc_sw128(sB + st * kMmStageB);
#pragma unroll
                    for (uint32_t kk = 0; kk < kMmBK / 32; kk++)
                        umma_i8(d, ad + 2 * kk, bd + 2 * kk, kMmIdesc, (kb | kk) != 0);
                    umma_commit(&empty[st]);  // the stage is free once these MMAs have read it
                    if (++st == kMmStages) {
                        st = 0;
                        ph ^= 1;
                    }
                }
                umma_commit(&tfull[acc]);  // accumulator complete
            }
        }
        __syncwarp();
    }
    else {  // epilogue warps 2..5: TMEM lanes 32*(warp%4) .. +31
        const uint32_t q = warp & 3;
        uint32_t mymax = 0, i = 0;
        for (uint32_t t = blockIdx.x; t < ntiles; t += gridDim.x, i++) {
            const uint32_t acc = i & 1, aph = (i >> 1) & 1;
            wait_or_flag(&tfull[acc], aph, err);
            __syncwarp();  // tcgen05.ld is warp-collective
            tc_fence_after();
            const uint32_t row = (t % p.tiles_m) * kMmBM + q * 32 + lane;
            const uint32_t colt = (t / p.tiles_m) * kMmBN;
            int32_t* crow = p.c + (size_t)row * p.N;
#pragma unroll 1
            for (uint32_t cb = 0; cb < kMmBN / 32; cb++) {
                uint32_t r[32];
                tmem_ld32(tmem + acc * kMmBN + cb * 32 + ((q * 32) << 16), r);
                const uint32_t col0 = colt + cb * 32;
                if (row < p.M && col0 < p.N) {
                    if (col0 + 32 <= p.N && (p.N & 3) == 0) {
#pragma unroll
                        for (int e = 0; e < 32; e++) mymax = r[e] > mymax ? r[e] : mymax;
                        uint4* dst = reinterpret_cast<uint4*>(crow + col0);
#pragma unroll
                        for (int e = 0; e < 8; e++) dst[e] = make_uint4(r[4 * e], r[4 * e + 1], r[4 * e + 2], r[4 * e + 3]);
                    }
                    else {
#pragma unroll
                        for (int e = 0; e < 32; e++)
                            if (col0 + e < p.N) {
                                crow[col0 + e] = (int32_t)r[e];
                                mymax = r[e] > mymax ? r[e] : mymax;
                            }
                    }
                }
            }
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
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kMmTmemCols) : "memory");
    }
}

// ---------------------------------------------------------------------------------------------
// unpack and pack
// ---------------------------------------------------------------------------------------------
// The 16 entries c0 .. c0 + cnt - 1 (cnt <= 16) of row r of a matrix in format F, as bytes
// (entries have at most 8 bits).  Every word the run touches is loaded up front: with at most 8
// bits per entry a slab run of 16 spans at most 3 slab words and a nogaps run at most 3 words.
template <uint32_t F>
__device__ __forceinline__ void read_run16(const ColDev& m, uint32_t cols, uint32_t row_slabs, uint32_t r, uint32_t c0,
                                           uint32_t cnt, uint32_t (&v)[4])
{
    v[0] = v[1] = v[2] = v[3] = 0;
    if (F == AMX_SLAB) {
        const unsigned long long* w = reinterpret_cast<const unsigned long long*>(m.data) + (size_t)r * row_slabs;
        const uint32_t s = c0 < (1u << 17) ? __umulhi(c0, m.magic) : c0 / m.eps;  // exact below 2^17
        const uint32_t last = (c0 + cnt - 1) < (1u << 17) ? __umulhi(c0 + cnt - 1, m.magic) : (c0 + cnt - 1) / m.eps;
        uint64_t w0 = __ldg(w + s);
        uint64_t w1 = last >= s + 1 ? __ldg(w + s + 1) : 0;
        uint64_t w2 = last >= s + 2 ? __ldg(w + s + 2) : 0;
        uint32_t k = c0 - s * m.eps;
#pragma unroll
        for (uint32_t e = 0; e < 16; e++) {
            if (e < cnt) v[e >> 2] |= (uint32_t)((w0 >> (k * m.bits)) & m.mask) << ((e & 3) * 8);
            if (++k == m.eps) {
                k = 0;
                w0 = w1;
                w1 = w2;
            }
        }
    }
    else if (F == AMX_NOGAPS) {
        const unsigned long long* w = reinterpret_cast<const unsigned long long*>(m.data);
        const uint64_t b0 = ((uint64_t)r * cols + c0) * m.bits;
        const uint64_t wi = b0 >> 6, wl = (b0 + (uint64_t)cnt * m.bits - 1) >> 6;
        const uint64_t x0 = __ldg(w + wi), x1 = wl >= wi + 1 ? __ldg(w + wi + 1) : 0, x2 = wl >= wi + 2 ? __ldg(w + wi + 2) : 0;
        uint32_t off = (uint32_t)(b0 & 63);
#pragma unroll
        for (uint32_t e = 0; e < 16; e++) {
            // bits [off, off + bits) of the 192-bit window x2:x1:x0
            uint64_t x = off < 64 ? (x0 >> off) | (off ? x1 << (64 - off) : 0)
                                  : (off < 128 ? (x1 >> (off - 64)) | (off > 64 ? x2 << (128 - off) : 0) : x2 >> (off - 128));
            if (e < cnt) v[e >> 2] |= (uint32_t)(x & m.mask) << ((e & 3) * 8);
            off += m.bits;
        }
    }
    else {
#pragma unroll
        for (uint32_t e = 0; e < 16; e++) {
            uint32_t x = 0;
            if (e < cnt) {
                const size_t i = (size_t)r * cols + c0 + e;
                x = F == AMX_PLAIN32 ? (uint32_t)(__ldg(reinterpret_cast<const uint32_t*>(m.data) + i) & m.mask)
                                     : (uint32_t)(__ldg(reinterpret_cast<const unsigned long long*>(m.data) + i) & m.mask);
            }
            v[e >> 2] |= x << ((e & 3) * 8);
        }
    }
}

// A (rows x cols) -> u8 [rows_pad][cols_pad]: rows over grid.y, 16-entry chunks of a row over the
// threads, zero padding
template <uint32_t F>
__global__ void __launch_bounds__(256) mm_unpack_rows(const __grid_constant__ ColDev a, uint32_t rows, uint32_t cols,
                                                      uint32_t row_slabs, uint32_t rows_pad, uint32_t cols_pad,
                                                      uint8_t* out)
{
    const uint32_t chunks = cols_pad / 16;
    for (uint32_t r = blockIdx.y; r < rows_pad; r += gridDim.y) {
        uint4* dst = reinterpret_cast<uint4*>(out + (size_t)r * cols_pad);
        for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < chunks; j += gridDim.x * blockDim.x) {
            const uint32_t c0 = j * 16;
            uint32_t v[4] = {0, 0, 0, 0};
            if (r < rows && c0 < cols) read_run16<F>(a, cols, row_slabs, r, c0, cols - c0 < 16 ? cols - c0 : 16, v);
            dst[j] = make_uint4(v[0], v[1], v[2], v[3]);
        }
    }
}

// B (rows = K x cols = N) -> u8 [cols_pad][rows_pad] (transposed), 64 x 64 blocks through shared memory
template <uint32_t F>
__global__ void __launch_bounds__(256) mm_unpack_cols(const __grid_constant__ ColDev b, uint32_t rows, uint32_t cols,
                                                      uint32_t row_slabs, uint32_t rows_pad, uint8_t* out)
{
    __shared__ uint8_t tile[64][68];
    const uint32_t k0 = blockIdx.x * 64, n0 = blockIdx.y * 64;
    {
        const uint32_t kk = threadIdx.x >> 2, part = threadIdx.x & 3;  // row k0 + kk, entries n0 + 16 part ..
        const uint32_t k = k0 + kk, c0 = n0 + part * 16;
        uint32_t cnt = 0;
        if (k < rows && c0 < cols) cnt = cols - c0 < 16 ? cols - c0 : 16;
        uint32_t v[4] = {0, 0, 0, 0};
        if (cnt) read_run16<F>(b, cols, row_slabs, k, c0, cnt, v);
#pragma unroll
        for (uint32_t e = 0; e < 16; e++) tile[part * 16 + e][kk] = (uint8_t)(v[e >> 2] >> ((e & 3) * 8));
    }
    __syncthreads();
    const uint32_t nn = threadIdx.x / 4, part = threadIdx.x % 4;
    uint32_t v[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const uint8_t* s = &tile[nn][part * 16 + 4 * e];
        v[e] = (uint32_t)s[0] | ((uint32_t)s[1] << 8) | ((uint32_t)s[2] << 16) | ((uint32_t)s[3] << 24);
    }
    *reinterpret_cast<uint4*>(out + (size_t)(n0 + nn) * rows_pad + k0 + part * 16) = make_uint4(v[0], v[1], v[2], v[3]);
}

// one row of slab words with EPS entries each (EPS > 0 at compile time, or eps at run time)
template <int EPS>
__device__ __forceinline__ void pack_slab_row(const uint32_t* src, uint64_t* dst, uint32_t N, uint32_t row_slabs,
                                              uint32_t eps_rt, uint32_t bits, uint64_t m, uint32_t tx, uint32_t sx)
{
    const uint32_t eps = EPS > 0 ? (uint32_t)EPS : eps_rt;
    const uint32_t full = N / eps;  // words whose entries all exist
    for (uint32_t s = tx; s < row_slabs; s += sx) {
        const uint32_t c0 = s * eps;
        uint64_t acc = 0;
        if (EPS > 0 && s < full) {
#pragma unroll
            for (int k = 0; k < (EPS > 0 ? EPS : 1); k++) acc |= ((uint64_t)__ldg(src + c0 + k) & m) << (k * bits);
        }
        else {
            const uint32_t cnt = N - c0 < eps ? N - c0 : eps;
            for (uint32_t k = 0; k < cnt; k++) acc |= ((uint64_t)__ldg(src + c0 + k) & m) << (k * bits);
        }
        dst[s] = acc;
    }
}

// C (int32, M x N) -> the output format at `fixed_bits`, or (fixed_bits == 0) at the narrowest
// width holding the largest entry; the width used goes to *d_out_bits.  Rows are spread over
// grid.y, the words of a row over grid.x and the threads.
__global__ void __launch_bounds__(256) mm_pack(const int32_t* c, uint32_t M, uint32_t N, void* out, uint32_t format,
                                               uint32_t fixed_bits, const uint32_t* hdr, uint32_t* d_out_bits)
{
    const uint32_t mx = hdr[0];
    const uint32_t bits = fixed_bits ? fixed_bits : (mx ? 32 - __clz(mx) : 1);
    const uint64_t m = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0 && d_out_bits) *d_out_bits = bits;
    const uint32_t* cu = reinterpret_cast<const uint32_t*>(c);
    const uint32_t tx = blockIdx.x * blockDim.x + threadIdx.x, sx = gridDim.x * blockDim.x;
    if (format == AMX_SLAB) {
        const uint32_t eps = 64 / bits;
        const uint32_t row_slabs = (N + eps - 1) / eps;
        for (uint32_t r = blockIdx.y; r < M; r += gridDim.y) {
            const uint32_t* src = cu + (size_t)r * N;
            uint64_t* dst = reinterpret_cast<uint64_t*>(out) + (size_t)r * row_slabs;
            switch (eps) {
                case 2: pack_slab_row<2>(src, dst, N, row_slabs, eps, bits, m, tx, sx); break;
                case 3: pack_slab_row<3>(src, dst, N, row_slabs, eps, bits, m, tx, sx); break;
                case 4: pack_slab_row<4>(src, dst, N, row_slabs, eps, bits, m, tx, sx); break;
                default: pack_slab_row<0>(src, dst, N, row_slabs, eps, bits, m, tx, sx); break;
            }
        }
        return;
    }
    if (format == AMX_PLAIN32 || format == AMX_PLAIN64) {
        for (uint32_t r = blockIdx.y; r < M; r += gridDim.y) {
            const uint32_t* src = cu + (size_t)r * N;
            for (uint32_t j = tx; j < N; j += sx) {
                const uint64_t v = __ldg(src + j) & m;
                if (format == AMX_PLAIN32)
                    reinterpret_cast<uint32_t*>(out)[(size_t)r * N + j] = (uint32_t)v;
                else
                    reinterpret_cast<uint64_t*>(out)[(size_t)r * N + j] = v;
            }
        }
        return;
    }
    // nogaps: word w holds bits [64w, 64w + 64) of the row-major stream
    const uint64_t n = (uint64_t)M * N;
    const uint64_t words = (n * bits + 63) / 64;
    const uint64_t t0 = (uint64_t)blockIdx.y * sx + tx, stride = (uint64_t)sx * gridDim.y;
    for (uint64_t w = t0; w < words; w += stride) {
        const uint64_t lo = w * 64;
        uint64_t e = lo / bits;
        uint64_t acc = 0;
        for (; e < n && e * bits < lo + 64; e++) {
            const int64_t sh = (int64_t)(e * bits) - (int64_t)lo;
            const uint64_t v = __ldg(cu + e) & m;
            acc |= sh >= 0 ? (v << sh) : (v >> (-sh));
        }
        reinterpret_cast<uint64_t*>(out)[w] = acc;
    }
}

// ---------------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------------
static uint64_t up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

// Workspace: header, the fused path's column norms, u8 A and B^T of the two-pass path, and the
// int32 product of the two-pass path (the fused path's repack scratch, up to 8 ceil(N/2) bytes a
// row at widths of at most 31 bits).
struct MmLayout {
    uint64_t hdr, colsq, a8, b8, c32, total;
    uint32_t kpad, mpad, npad;
};

static MmLayout mm_layout(uint32_t M, uint32_t N, uint32_t K)
{
    MmLayout l{};
    l.kpad = (uint32_t)up(K ? K : 1, kMmBK);
    l.mpad = (uint32_t)up(M ? M : 1, kMmBM);
    l.npad = (uint32_t)up(N ? N : 1, kMmBN);
    l.hdr = 0;
    l.colsq = 1024;
    l.a8 = up(l.colsq + 8ull * l.npad, 1024);
    l.b8 = up(l.a8 + (uint64_t)l.mpad * l.kpad, 1024);
    l.c32 = up(l.b8 + (uint64_t)l.npad * l.kpad, 1024);
    l.total = up(l.c32 + 4ull * M * N + 8ull * M + 16, 1024);
    return l;
}

static uint32_t bit_length(uint64_t x)
{
    uint32_t b = 0;
    while (x) {
        b++;
        x >>= 1;
    }
    return b;
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }
    return fn;
}

// 2-D u8 tensor map over a [outer][inner] matrix with a box of box_outer rows x 128 bytes
static amx_status make_map(CUtensorMap* m, void* base, uint64_t inner, uint64_t outer, uint32_t box_outer)
{
    auto enc = tensor_map_encoder();
    if (!enc) return fail(AMX_ERR_CUDA, "matmul: cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {inner};
    cuuint32_t box[2] = {kMmBK, box_outer};
    cuuint32_t es[2] = {1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(AMX_ERR_CUDA, "matmul: tensor map encoding failed (%d)", (int)r);
    return AMX_OK;
}

static uint32_t row_slabs_of(const amx_column* c, uint32_t cols)
{
    return c->format == AMX_SLAB ? (cols + 64 / c->bits - 1) / (64 / c->bits) : 0;
}

static uint64_t matrix_bytes(uint32_t format, uint32_t bits, uint64_t rows, uint64_t cols)
{
    if (format == AMX_SLAB) {
        const uint64_t eps = 64 / bits;
        return 8 * rows * ((cols + eps - 1) / eps);
    }
    return storage_bytes(format, bits, rows * cols);
}

}  // namespace amx

using namespace amx;

extern "C" {

uint64_t amx_matmul_workspace_bytes(uint32_t M, uint32_t N, uint32_t K) { return mm_layout(M, N, K).total; }

uint64_t amx_matmul_out_bytes(uint32_t format, uint32_t out_bits, uint32_t M, uint32_t N, uint32_t K, uint32_t a_bits,
                              uint32_t b_bits)
{
    if (format > AMX_NOGAPS || a_bits < 1 || a_bits > kMmMaxBits || b_bits < 1 || b_bits > kMmMaxBits) return 0;
    uint32_t w = out_bits;
    if (!w) {
        w = bit_length((uint64_t)K * mask_of(a_bits) * mask_of(b_bits));
        if (w < 1) w = 1;
    }
    if (w > (format == AMX_PLAIN32 ? 32u : 64u)) return 0;
    return matrix_bytes(format, w, M, N);
}

amx_status amx_matmul(const amx_column* a, const amx_column* b, uint32_t M, uint32_t N, uint32_t K,
                      const amx_column* out, uint32_t* d_out_bits, void* ws, size_t ws_bytes, void* stream)
{
    amx_status st = check_column(a, "matmul: a");
    if (st) return st;
    if ((st = check_column(b, "matmul: b"))) return st;
    if (!out || !out->data) return fail(AMX_ERR_INVALID_ARG, "matmul: null output");
    if (out->format > AMX_NOGAPS) return fail(AMX_ERR_INVALID_ARG, "matmul: unknown output format %u", out->format);
    if (out->bits > (out->format == AMX_PLAIN32 ? 32u : 64u))
        return fail(AMX_ERR_INVALID_ARG, "matmul: output width %u", out->bits);
    if (((uintptr_t)out->data) & 15) return fail(AMX_ERR_ALIGNMENT, "matmul: output not 16-byte aligned");
    if (a->n != (uint64_t)M * K || b->n != (uint64_t)K * N)
        return fail(AMX_ERR_INVALID_ARG, "matmul: a holds %llu entries (M*K = %llu), b %llu (K*N = %llu)",
                    (unsigned long long)a->n, (unsigned long long)M * K, (unsigned long long)b->n,
                    (unsigned long long)K * N);
    if (out->n < (uint64_t)M * N) return fail(AMX_ERR_INVALID_ARG, "matmul: output capacity below M*N");
    if (a->bits > kMmMaxBits || b->bits > kMmMaxBits)
        return fail(AMX_ERR_UNSUPPORTED, "matmul: entries of %u and %u bits (at most %u on the u8 tensor path)",
                    a->bits, b->bits, kMmMaxBits);
    if ((uint64_t)K * mask_of(a->bits) * mask_of(b->bits) > 0x7fffffffull)
        return fail(AMX_ERR_UNSUPPORTED, "matmul: K * max(a) * max(b) may exceed the int32 accumulator");
    if (out->bits && out->bits > 64) return fail(AMX_ERR_INVALID_ARG, "matmul: output width");
    const MmLayout L = mm_layout(M, N, K);
    if (!ws || ws_bytes < L.total)
        return fail(AMX_ERR_WORKSPACE, "matmul: workspace of %zu bytes, %llu needed", ws_bytes,
                    (unsigned long long)L.total);
    if (((uintptr_t)ws) & 1023) return fail(AMX_ERR_ALIGNMENT, "matmul: workspace not 1024-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* w = static_cast<uint8_t*>(ws);
    uint32_t* hdr = reinterpret_cast<uint32_t*>(w + L.hdr);
    cudaError_t e = cudaMemsetAsync(hdr, 0, 256, s);
    if (e != cudaSuccess) return cuda_fail(e, "matmul: header clear");
    int32_t* c32 = reinterpret_cast<int32_t*>(w + L.c32);
    const uint64_t mn = (uint64_t)M * N;
    if (mn && K && mf_applicable(a, b))  // unpacked in shared memory, packed from the accumulators
        return mf_run(a, b, M, N, K, out, d_out_bits, hdr, reinterpret_cast<unsigned long long*>(w + L.colsq), c32, s);
    if (mn && K) {
        const ColDev ad = col_dev(a), bd = col_dev(b);
        const uint32_t chunks = L.kpad / 16;
        const dim3 ga((chunks + 255) / 256, L.mpad < 65535 ? L.mpad : 65535);
        const dim3 gb(L.kpad / 64, L.npad / 64);
        const uint32_t ars = row_slabs_of(a, K), brs = row_slabs_of(b, N);
        switch (a->format) {
            case AMX_PLAIN32: mm_unpack_rows<AMX_PLAIN32><<<ga, 256, 0, s>>>(ad, M, K, ars, L.mpad, L.kpad, w + L.a8); break;
            case AMX_PLAIN64: mm_unpack_rows<AMX_PLAIN64><<<ga, 256, 0, s>>>(ad, M, K, ars, L.mpad, L.kpad, w + L.a8); break;
            case AMX_SLAB: mm_unpack_rows<AMX_SLAB><<<ga, 256, 0, s>>>(ad, M, K, ars, L.mpad, L.kpad, w + L.a8); break;
            default: mm_unpack_rows<AMX_NOGAPS><<<ga, 256, 0, s>>>(ad, M, K, ars, L.mpad, L.kpad, w + L.a8); break;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: unpack a");
        switch (b->format) {
            case AMX_PLAIN32: mm_unpack_cols<AMX_PLAIN32><<<gb, 256, 0, s>>>(bd, K, N, brs, L.kpad, w + L.b8); break;
            case AMX_PLAIN64: mm_unpack_cols<AMX_PLAIN64><<<gb, 256, 0, s>>>(bd, K, N, brs, L.kpad, w + L.b8); break;
            case AMX_SLAB: mm_unpack_cols<AMX_SLAB><<<gb, 256, 0, s>>>(bd, K, N, brs, L.kpad, w + L.b8); break;
            default: mm_unpack_cols<AMX_NOGAPS><<<gb, 256, 0, s>>>(bd, K, N, brs, L.kpad, w + L.b8); break;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: unpack b");

        CUtensorMap tma, tmb;
        if ((st = make_map(&tma, w + L.a8, L.kpad, L.mpad, kMmBM))) return st;
        if ((st = make_map(&tmb, w + L.b8, L.kpad, L.npad, kMmBN))) return st;
        MmParams p{};
        p.M = M;
        p.N = N;
        p.K = K;
        p.tiles_m = L.mpad / kMmBM;
        p.tiles_n = L.npad / kMmBN;
        p.kblocks = L.kpad / kMmBK;
        p.c = c32;
        p.hdr = hdr;
        e = cudaFuncSetAttribute(mm_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMmSmem);
        if (e != cudaSuccess) return cuda_fail(e, "matmul: shared memory attribute");
        const uint32_t tiles = p.tiles_m * p.tiles_n;
        const uint32_t grid = tiles < (uint32_t)sm_count() ? tiles : (uint32_t)sm_count();
        mm_gemm_kernel<<<grid, kMmThreads, kMmSmem, s>>>(tma, tmb, p);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: gemm launch");
    }
    else if (mn) {
        e = cudaMemsetAsync(c32, 0, 4 * mn, s);  // K == 0: the product is all zeros
        if (e != cudaSuccess) return cuda_fail(e, "matmul: zero product");
    }
    // rows over grid.y (at most 65535), the words of a row over grid.x
    const uint32_t gy = M ? (M < 4096 ? M : 4096) : 1;
    const uint32_t gx = 1;
    mm_pack<<<dim3(gx, gy), 256, 0, s>>>(c32, M, N, out->data, out->format, out->bits, hdr, d_out_bits);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: pack launch");
    return AMX_OK;
}

// device-side failure recorded by the last amx_matmul on this workspace (synchronises the stream)
amx_status amx_matmul_status(const void* ws, void* stream)
{
    if (!ws) return fail(AMX_ERR_INVALID_ARG, "matmul_status: null workspace");
    uint32_t h[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, ws, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "matmul_status");
    if (h[1]) return fail((amx_status)h[1], "matmul: a device-side wait timed out");
    return AMX_OK;
}

}  // extern "C"
