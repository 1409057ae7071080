// amx_stats.cu -- column statistics for the format selector: the histogram of the bit widths
// the values of a column need.  One read of the column; a shared-memory histogram per CTA
// (one copy per warp, so lanes of different warps never contend), folded into the caller's
// 65 uint64 counters with one atomic per nonzero bin and CTA.  No reference counterpart.
#include "amx_dispatch.h"
#include "amx_device.cuh"

namespace amx {

constexpr uint32_t kHistBins = 65;
constexpr uint32_t kHistThreads = 256;
constexpr uint32_t kHistWarps = kHistThreads / 32;

__device__ __forceinline__ uint32_t bit_len(uint64_t v) { return 64u - (uint32_t)__clzll((long long)v); }

__global__ void __launch_bounds__(kHistThreads) bit_hist_kernel(ColDev c, unsigned long long* hist)
{
    __shared__ uint32_t h[kHistWarps][kHistBins];
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    for (uint32_t i = tid; i < kHistWarps * kHistBins; i += blockDim.x) (&h[0][0])[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t first = (uint64_t)blockIdx.x * blockDim.x + tid;
    if (c.format == AMX_SLAB) {
        // one slab word per thread and step: eps fields, the tail word's missing fields skipped
        const uint64_t words = udiv64(c.n + c.eps - 1, c.magic64, c.eps);
        const unsigned long long* w = reinterpret_cast<const unsigned long long*>(c.data);
        for (uint64_t i = first; i < words; i += stride) {
            uint64_t x = __ldg(w + i);
            const uint64_t e0 = i * c.eps;
            const uint32_t k = c.n - e0 < c.eps ? (uint32_t)(c.n - e0) : c.eps;
            for (uint32_t f = 0; f < k; f++) {
                atomicAdd(&h[warp][bit_len(x & c.mask)], 1u);
                x >>= c.bits;
            }
        }
    }
    else {
        for (uint64_t e = first; e < c.n; e += stride) {
            uint64_t v;
            if (c.format == AMX_PLAIN32)
                v = __ldg(reinterpret_cast<const uint32_t*>(c.data) + e) & c.mask;
            else if (c.format == AMX_PLAIN64)
                v = __ldg(reinterpret_cast<const unsigned long long*>(c.data) + e) & c.mask;
            else {
                const uint64_t bp = e * c.bits, wi = bp >> 6;
                const uint32_t off = (uint32_t)(bp & 63);
                const unsigned long long* w = reinterpret_cast<const unsigned long long*>(c.data);
                v = __ldg(w + wi) >> off;
                if (off + c.bits > 64) v |= (uint64_t)__ldg(w + wi + 1) << (64 - off);
                v &= c.mask;
            }
            atomicAdd(&h[warp][bit_len(v)], 1u);
        }
    }
    __syncthreads();
    for (uint32_t b = tid; b < kHistBins; b += blockDim.x) {
        uint64_t s = 0;
        for (uint32_t k = 0; k < kHistWarps; k++) s += h[k][b];
        if (s) atomicAdd(hist + b, (unsigned long long)s);
    }
}

}  // namespace amx

using namespace amx;

extern "C" amx_status amx_bit_histogram(const amx_column* in, uint64_t* d_hist, void* stream)
{
    amx_status st = check_column(in, "bit_histogram: in");
    if (st) return st;
    if (!d_hist) return fail(AMX_ERR_INVALID_ARG, "bit_histogram: null histogram");
    if (!in->n) return AMX_OK;
    const ColDev c = col_dev(in);
    // a warp's 32-bit shared counters see at most 2^20 units per thread x 32 lanes x 64 fields
    uint64_t grid = (uint64_t)sm_count() * 8;
    const uint64_t units = c.format == AMX_SLAB ? (c.n + c.eps - 1) / c.eps : c.n;
    const uint64_t need = (units + kHistThreads - 1) / kHistThreads;
    if (grid > need) grid = need ? need : 1;
    while ((units + grid * kHistThreads - 1) / (grid * kHistThreads) >= (1ull << 20)) grid *= 2;
    bit_hist_kernel<<<(unsigned)grid, kHistThreads, 0, (cudaStream_t)stream>>>(c, reinterpret_cast<unsigned long long*>(d_hist));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "bit_histogram: launch");
    return AMX_OK;
}
