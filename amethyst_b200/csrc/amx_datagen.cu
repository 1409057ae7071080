// amx_datagen.cu -- seeded synthetic column generators for benchmarks and tests.
//
// Element i is a pure function of (seed, i): state = splitmix64(seed + i * golden) followed by
// one xorshift64 (13, 7, 17) step; the value is the top `bits` bits.  The generators have no
// reference counterpart (the reference fills host arrays with PCG32, src/main.cu:242-251,
// which the oracle restates for the parity fixtures).
#include "amx_dispatch.h"

namespace amx {

__host__ __device__ inline uint64_t gen_draw(uint64_t seed, uint64_t i)
{
    uint64_t z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    z ^= z << 13;
    z ^= z >> 7;
    z ^= z << 17;
    return z;
}

__global__ void fill_uniform_kernel(void* out, uint64_t n, uint32_t elem_bytes, uint32_t bits, uint64_t seed)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t r = gen_draw(seed, i);
        const uint64_t v = bits >= 64 ? r : (r >> (64 - bits));
        if (elem_bytes == 4)
            reinterpret_cast<uint32_t*>(out)[i] = (uint32_t)v;
        else
            reinterpret_cast<uint64_t*>(out)[i] = v;
    }
}

// Zipf keys by inverse CDF: u uniform in [0, 1) from the draw, key = first k with cdf[k] > u.
__global__ void fill_cdf_kernel(uint32_t* out, uint64_t n, const double* cdf, uint32_t groups, uint64_t seed)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double u = (double)(gen_draw(seed, i) >> 11) * (1.0 / 9007199254740992.0);
        uint32_t lo = 0, hi = groups - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi) >> 1;
            if (cdf[mid] > u)
                hi = mid;
            else
                lo = mid + 1;
        }
        out[i] = lo;
    }
}

}  // namespace amx

using namespace amx;

extern "C" {

amx_status amx_fill_uniform(void* d_out, uint64_t n, uint32_t elem_bytes, uint32_t bits, uint64_t seed, void* stream)
{
    if (!d_out && n) return fail(AMX_ERR_INVALID_ARG, "fill_uniform: null output");
    if (elem_bytes != 4 && elem_bytes != 8) return fail(AMX_ERR_INVALID_ARG, "fill_uniform: elem_bytes must be 4 or 8");
    if (bits < 1 || bits > elem_bytes * 8) return fail(AMX_ERR_INVALID_ARG, "fill_uniform: bad width %u", bits);
    if (!n) return AMX_OK;
    const uint64_t blocks = (n + 255) / 256;
    fill_uniform_kernel<<<(unsigned)(blocks < 8192 ? blocks : 8192), 256, 0, (cudaStream_t)stream>>>(d_out, n, elem_bytes,
                                                                                                     bits, seed);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AMX_OK : cuda_fail(e, "fill_uniform launch");
}

amx_status amx_fill_from_cdf(uint32_t* d_out, uint64_t n, const double* d_cdf, uint32_t groups, uint64_t seed,
                             void* stream)
{
    if ((!d_out && n) || !d_cdf || groups < 1) return fail(AMX_ERR_INVALID_ARG, "fill_from_cdf: bad arguments");
    if (!n) return AMX_OK;
    const uint64_t blocks = (n + 255) / 256;
    fill_cdf_kernel<<<(unsigned)(blocks < 8192 ? blocks : 8192), 256, 0, (cudaStream_t)stream>>>(d_out, n, d_cdf, groups,
                                                                                                 seed);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? AMX_OK : cuda_fail(e, "fill_from_cdf launch");
}

}  // extern "C"
