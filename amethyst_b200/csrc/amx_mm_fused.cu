// amx_mm_fused.cu -- host side of the fused packed-matrix multiply (amx_mm_fused.cuh) and its
// small helper kernels.
//
// The output is packed inside the GEMM's epilogue, so its width must be known before the first
// tile is done.  With a caller-given width that is the width.  For "the narrowest width that
// holds the largest entry" the epilogue packs at a width bounded in advance by Cauchy-Schwarz:
// every entry is a_i . b_j <= |a_i| |b_j| <= sqrt(max_i |a_i|^2 * max_j |b_j|^2), so
// mf_bound computes the largest squared row norm of A and column norm of B (one read of each
// packed operand, which also leaves them in L2 for the GEMM), and the width of
// min(isqrt(that product), K * max(a) * max(b)).  For uniform 7-bit operands at K = 4096 this is
// the exact minimal width (25 bits: entries reach about 1.77e7, the bound about 2.3e7 < 2^25).
// When the largest entry turns out narrower, mf_finish repacks the output through the workspace.
//
// Tiles share the slab or nogaps words that straddle their column boundaries; mf_zero_edges
// clears exactly those words first and the epilogue or-s its fields into them.
#include "amx_dispatch.h"
#include "amx_mm_fused.cuh"

namespace amx {

template <int W>
amx_status mf_launch_w(const CUtensorMap& tma, const CUtensorMap& tmb, const MfParams& p, cudaStream_t s);

static amx_status mf_launch(uint32_t w, const CUtensorMap& ta, const CUtensorMap& tb, const MfParams& p, cudaStream_t s)
{
    switch (w) {
        case 1: return mf_launch_w<1>(ta, tb, p, s);
        case 2: return mf_launch_w<2>(ta, tb, p, s);
        case 3: return mf_launch_w<3>(ta, tb, p, s);
        case 4: return mf_launch_w<4>(ta, tb, p, s);
        case 5: return mf_launch_w<5>(ta, tb, p, s);
        case 6: return mf_launch_w<6>(ta, tb, p, s);
        case 7: return mf_launch_w<7>(ta, tb, p, s);
        case 8: return mf_launch_w<8>(ta, tb, p, s);
        default: return fail(AMX_ERR_UNSUPPORTED, "matmul: fused path for %u-bit slabs", w);
    }
}

// 2-D tensor map of 64-bit words over a packed matrix (rows x rs words), box of box_words words x
// 128 rows, no swizzle; words and rows past the matrix read as zeros
static amx_status mf_make_map(CUtensorMap* m, const void* base, uint32_t rs, uint32_t rows, uint32_t box_words)
{
    auto enc = tensor_map_encoder();
    if (!enc) return fail(AMX_ERR_CUDA, "matmul: cuTensorMapEncodeTiled unavailable");
    cuuint64_t dims[2] = {rs, rows};
    cuuint64_t strides[1] = {8ull * rs};
    cuuint32_t box[2] = {box_words, 128};
    cuuint32_t es[2] = {1, 1};
    const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT64, 2, const_cast<void*>(base), dims, strides, box, es,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(AMX_ERR_CUDA, "matmul: tensor map encoding failed (%d)", (int)r);
    return AMX_OK;
}

// header words (uint32 units) beyond [0] largest entry, [1] error word, [2] packing width
constexpr uint32_t kMfRowNorm = 4;  // uint64 at words 4..5: largest squared row norm of A
constexpr uint32_t kMfDone = 6;     // blocks of mf_bound finished

__device__ __forceinline__ uint64_t mf_isqrt(uint64_t v)
{
    uint64_t s = (uint64_t)sqrt((double)v);
    while (s * s > v) s--;
    while ((s + 1) * (s + 1) <= v) s++;
    return s;
}

// Blocks [0, ablocks): one warp per row of A, the largest sum of squares over the rows.  The other
// blocks: 64 columns of B over 256 rows of K each, sums of squares added into colsq.
// The last block to finish turns both into the packing width (hdr[2]).
__global__ void __launch_bounds__(256) mf_bound(const uint64_t* a, uint32_t a_rs, const uint64_t* b, uint32_t b_rs,
                                                uint32_t w, uint32_t M, uint32_t N, uint32_t K, uint32_t ablocks,
                                                uint32_t cblocks, unsigned long long* colsq, uint32_t* hdr,
                                                uint64_t static_bound)
{
    const uint32_t eps = 64 / w;
    const uint64_t fm = (1ull << w) - 1;
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned long long* rowmax = reinterpret_cast<unsigned long long*>(hdr + kMfRowNorm);
    if (blockIdx.x < ablocks) {
        for (uint32_t r = blockIdx.x * 8 + warp; r < M; r += ablocks * 8) {
            const uint64_t* row = a + (size_t)r * a_rs;
            uint64_t acc = 0;
            for (uint32_t s = lane; s < a_rs; s += 32) {
                const uint64_t x = __ldg(reinterpret_cast<const unsigned long long*>(row + s));
                for (uint32_t f = 0; f < eps; f++)
                    if ((uint64_t)s * eps + f < K) {
                        const uint64_t v = (x >> (f * w)) & fm;
                        acc += v * v;
                    }
            }
#pragma unroll
            for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (lane == 0) atomicMax(rowmax, (unsigned long long)acc);
        }
    }
    else {  // 64 columns x 4 row lanes; each thread sums 64 rows, 8 loads in flight
        const uint32_t bi = blockIdx.x - ablocks;
        const uint32_t j = (bi % cblocks) * 64 + (threadIdx.x & 63), rl = threadIdx.x >> 6;
        const uint32_t k0 = (bi / cblocks) * 256;
        uint64_t acc = 0;
        if (j < N) {
            const uint32_t s = j / eps, sh = (j % eps) * w;
            const unsigned long long* col = reinterpret_cast<const unsigned long long*>(b) + s;
#pragma unroll 8
            for (uint32_t i = 0; i < 64; i++) {
                const uint32_t k = k0 + rl + 4 * i;
                const uint64_t v = k < K ? (__ldg(col + (size_t)k * b_rs) >> sh) & fm : 0;
                acc += v * v;
            }
        }
        __shared__ uint64_t part[256];
        part[threadIdx.x] = acc;
        __syncthreads();
        if (threadIdx.x < 64 && j < N) {
            const uint64_t t = part[threadIdx.x] + part[threadIdx.x + 64] + part[threadIdx.x + 128] + part[threadIdx.x + 192];
            if (t) atomicAdd(colsq + j, (unsigned long long)t);
        }
    }
    __threadfence();
    __syncthreads();
    __shared__ uint32_t last;
    if (threadIdx.x == 0) last = atomicAdd(hdr + kMfDone, 1u) == gridDim.x - 1 ? 1u : 0u;
    __syncthreads();
    if (!last) return;
    __threadfence();
    uint64_t cm = 0;
    for (uint32_t i = threadIdx.x; i < N; i += 256) {
        const uint64_t v = __ldcg(colsq + i);
        cm = v > cm ? v : cm;
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        const uint64_t y = __shfl_xor_sync(0xffffffffu, cm, o);
        cm = y > cm ? y : cm;
    }
    __shared__ uint64_t wm[8];
    if (lane == 0) wm[warp] = cm;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 0; i < 8; i++) cm = wm[i] > cm ? wm[i] : cm;
        const uint64_t rm = __ldcg(rowmax);
        // rm <= K max(a)^2 and cm <= K max(b)^2: the product is at most (K max(a) max(b))^2 < 2^62
        uint64_t bound = mf_isqrt(rm * cm);
        if (bound > static_bound) bound = static_bound;
        uint32_t bits = 1;
        while (bits < 64 && (bound >> bits)) bits++;
        hdr[2] = bits;
    }
}

// clear the output words that two tiles share: the first and the last word of every tile row
// segment whose boundary falls inside a word
__global__ void __launch_bounds__(256) mf_zero_edges(void* out, uint32_t format, uint32_t fixed, const uint32_t* hdr,
                                                     uint32_t M, uint32_t N, uint32_t tiles_n)
{
    const uint32_t w = fixed ? fixed : hdr[2];
    uint64_t* o = reinterpret_cast<uint64_t*>(out);
    const uint64_t total = (uint64_t)M * tiles_n;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t r = (uint32_t)(i / tiles_n), t = (uint32_t)(i % tiles_n);
        const uint32_t c0 = t * kMmBN, c1 = c0 + kMmBN < N ? c0 + kMmBN : N;
        if (format == AMX_SLAB) {
            const uint32_t eps = 64 / w;
            const uint64_t rw = (N + eps - 1) / eps;
            if (c0 % eps) o[r * rw + c0 / eps] = 0;
            if (c1 % eps) o[r * rw + (c1 - 1) / eps] = 0;
        }
        else {
            const uint64_t b0 = ((uint64_t)r * N + c0) * w, b1 = ((uint64_t)r * N + c1) * w;
            if (b0 & 63) o[b0 >> 6] = 0;
            if (b1 & 63) o[b1 >> 6] = 0;
        }
    }
}

// bits [pos, pos + w) of a word stream (w <= 32)
__device__ __forceinline__ uint64_t mf_bits_at(const uint64_t* src, uint64_t pos, uint32_t w)
{
    const uint64_t wi = pos >> 6;
    const uint32_t sh = (uint32_t)(pos & 63);
    uint64_t v = src[wi] >> sh;
    if (sh + w > 64) v |= src[wi + 1] << (64 - sh);
    return v & ((1ull << w) - 1);
}

// The final width (the caller's, or the narrowest holding the largest entry) to *d_out_bits;
// when it is below the packing width, the output repacked at the final width into `scratch`.
__global__ void __launch_bounds__(256) mf_finish(const void* out, void* scratch, uint32_t format, uint32_t fixed,
                                                 const uint32_t* hdr, uint32_t* d_out_bits, uint32_t M, uint32_t N)
{
    const uint32_t mx = hdr[0];
    const uint32_t wf = fixed ? fixed : (mx ? 32 - __clz(mx) : 1);
    if (blockIdx.x == 0 && threadIdx.x == 0 && d_out_bits) *d_out_bits = wf;
    if (fixed || (format != AMX_SLAB && format != AMX_NOGAPS)) return;
    const uint32_t wb = hdr[2];
    if (wf >= wb) return;
    const uint64_t* src = reinterpret_cast<const uint64_t*>(out);
    uint64_t* dst = reinterpret_cast<uint64_t*>(scratch);
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    if (format == AMX_SLAB) {
        const uint32_t ef = 64 / wf, eb = 64 / wb;
        const uint64_t rwf = (N + ef - 1) / ef, rwb = (N + eb - 1) / eb;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (uint64_t)M * rwf; i += stride) {
            const uint64_t r = i / rwf, s = i % rwf;
            uint64_t acc = 0;
            for (uint32_t f = 0; f < ef; f++) {
                const uint64_t c = s * ef + f;
                if (c >= N) break;
                const uint64_t v = (src[r * rwb + c / eb] >> ((c % eb) * wb)) & ((1ull << wb) - 1);
                acc |= v << (f * wf);
            }
            dst[i] = acc;
        }
    }
    else {
        const uint64_t n = (uint64_t)M * N, words = (n * wf + 63) / 64;
        for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += stride) {
            const uint64_t lo = i * 64;
            uint64_t acc = 0;
            for (uint64_t e = lo / wf; e < n && e * wf < lo + 64; e++) {
                const uint64_t v = mf_bits_at(src, e * wb, wb);
                const int64_t sh = (int64_t)(e * wf) - (int64_t)lo;
                acc |= sh >= 0 ? (v << sh) : (v >> (-sh));
            }
            dst[i] = acc;
        }
    }
}

__global__ void __launch_bounds__(256) mf_copy_back(void* out, const void* scratch, uint32_t format, const uint32_t* hdr,
                                                    uint32_t M, uint32_t N)
{
    const uint32_t mx = hdr[0];
    const uint32_t wf = mx ? 32 - __clz(mx) : 1;
    if (wf >= hdr[2]) return;
    uint64_t words;
    if (format == AMX_SLAB) {
        const uint32_t ef = 64 / wf;
        words = (uint64_t)M * ((N + ef - 1) / ef);
    }
    else {
        words = ((uint64_t)M * N * wf + 63) / 64;
    }
    const uint64_t* s = reinterpret_cast<const uint64_t*>(scratch);
    uint64_t* d = reinterpret_cast<uint64_t*>(out);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (uint64_t)gridDim.x * blockDim.x)
        d[i] = s[i];
}

bool mf_applicable(const amx_column* a, const amx_column* b)
{
    const int32_t pol = tuning().policy;
    return (pol == 2 || pol == 3) && a->format == AMX_SLAB && b->format == AMX_SLAB && a->bits == b->bits &&
           a->bits >= 1 && a->bits <= 8;
}

amx_status mf_run(const amx_column* a, const amx_column* b, uint32_t M, uint32_t N, uint32_t K, const amx_column* out,
                  uint32_t* d_out_bits, uint32_t* hdr, unsigned long long* colsq, void* scratch, cudaStream_t s)
{
    const uint32_t w = a->bits;
    const uint32_t eps = 64 / w;
    const uint32_t a_rs = (K + eps - 1) / eps, b_rs = (N + eps - 1) / eps;
    const uint32_t fixed = out->bits;
    const bool packed = out->format == AMX_SLAB || out->format == AMX_NOGAPS;
    const uint32_t tiles_m = (M + kMmBM - 1) / kMmBM, tiles_n = (N + kMmBN - 1) / kMmBN;
    const uint32_t sms = (uint32_t)sm_count();
    cudaError_t e;
    if (packed && !fixed) {
        if ((e = cudaMemsetAsync(colsq, 0, 8ull * N, s)) != cudaSuccess) return cuda_fail(e, "matmul: norm clear");
        const uint32_t ablocks = (M + 7) / 8 < 4 * sms ? (M + 7) / 8 : 4 * sms;
        const uint32_t cblocks = (N + 63) / 64, kchunks = (K + 255) / 256;
        const uint64_t static_bound = (uint64_t)K * mask_of(a->bits) * mask_of(b->bits);
        mf_bound<<<ablocks + cblocks * kchunks, 256, 0, s>>>(reinterpret_cast<const uint64_t*>(a->data), a_rs,
                                                             reinterpret_cast<const uint64_t*>(b->data), b_rs, w, M, N,
                                                             K, ablocks, cblocks, colsq, hdr, static_bound);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: bound launch");
    }
    if (packed) {
        const uint64_t edges = (uint64_t)M * tiles_n;
        const uint32_t g = (uint32_t)((edges + 255) / 256 < 8ull * sms ? (edges + 255) / 256 : 8ull * sms);
        mf_zero_edges<<<g ? g : 1, 256, 0, s>>>(out->data, out->format, fixed, hdr, M, N, tiles_n);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: edge clear launch");
    }
    MfParams p{};
    p.M = M;
    p.N = N;
    p.K = K;
    p.tiles_m = tiles_m;
    p.tiles_n = tiles_n;
    p.kblocks = (K + kMmBK - 1) / kMmBK;
    p.a = reinterpret_cast<const uint64_t*>(a->data);
    p.b = reinterpret_cast<const uint64_t*>(b->data);
    p.a_rs = a_rs;
    p.b_rs = b_rs;
    p.out = out->data;
    p.out_format = out->format;
    p.fixed_bits = fixed;
    p.hdr = hdr;
    // packed stages by TMA when both row pitches are whole 16-byte units and the boxes fit the
    // matrices; otherwise the unpackers read global memory directly
    CUtensorMap ta{}, tb{};
    p.direct = (a_rs % 2 || b_rs % 2 || a_rs < kMfPWordsA || b_rs < kMfPWordsB || M < kMmBM || K < kMmBK ||
                tuning().policy == 3) ? 1u : 0u;
    amx_status st;
    if (!p.direct) {
        if ((st = mf_make_map(&ta, a->data, a_rs, M, kMfPWordsA))) return st;
        if ((st = mf_make_map(&tb, b->data, b_rs, K, kMfPWordsB))) return st;
    }
    if ((st = mf_launch(w, ta, tb, p, s))) return st;
    mf_finish<<<8 * sms, 256, 0, s>>>(out->data, scratch, out->format, fixed, hdr, d_out_bits, M, N);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: finish launch");
    if (packed && !fixed) {
        mf_copy_back<<<8 * sms, 256, 0, s>>>(out->data, scratch, out->format, hdr, M, N);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "matmul: copy launch");
    }
    return AMX_OK;
}

}  // namespace amx
