// amx_noalloc.cu -- fused filter + compressstore for callers that cannot allocate device memory.
//
// The regular entry points never allocate either, but they need a caller-provided workspace, so
// the caller must own device memory to lend.  Some callers own none at call time: a query engine
// whose memory manager has already handed out every byte of its pool, a plugin invoked on an
// execution thread where cudaMalloc is forbidden because it can synchronise the device and stall
// other streams, or code recorded into a CUDA graph whose capture mode rejects allocation calls.
// For them this entry point brings its own scratch: a fixed array in the library's device memory.
//
// Limits and sharing rules (also stated in include/amethyst.h):
//   * the scratch is a file-scope __device__ array of kNoAllocScratchBytes (1 MiB + 256 bytes);
//     every GPU that loads the library holds one copy of it until the process exits;
//   * it holds the look-back state of at most 2^29 input elements; longer columns are rejected
//     with AMX_ERR_CAPACITY before anything is launched;
//   * every call shares the one array and leaves its contents behind; each call clears the part it
//     uses (cudaMemsetAsync) before its kernel runs, so calls that follow one another on a stream
//     are safe, but calls that may overlap on the GPU (other streams, other host threads) race;
//   * the first call on a device looks up the array's device address there (cudaGetSymbolAddress)
//     and caches it; make that first call before any stream capture begins.  The cached address
//     belongs to the device's primary context: after cudaDeviceReset it is stale, so a process
//     that resets a device must not call this entry point on that device again;
//   * a device-side failure (a bounded wait that ran out) is recorded in the array's header;
//     amx_filter_compressstore_noalloc_status() reads it back.  The next call clears it, so check
//     it before the next call.
// No cudaMalloc, cudaFree or allocating library routine is called on this path.
#include <mutex>

#include "amx_dispatch.h"

namespace amx {

constexpr uint64_t kNoAllocMaxElements = 1ull << 29;
// header + one look-back status word per tile of the smallest tile size, rounded up
constexpr size_t kNoAllocScratchBytes = (1u << 20) + 256;
static_assert(sizeof(WsHeader) + 8 * (kNoAllocMaxElements / kMinTile) <= kNoAllocScratchBytes, "scratch too small");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Host code must not use g_noalloc_scratch directly: on the host that name is a stand-in object,
// not a device address.  The device address is looked up once per device.
static void* g_scratch_ptr[64];
static std::mutex g_scratch_mu;

static amx_status scratch_for_current_device(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "filter_compressstore_noalloc: current device");
    if (dev < 0 || dev >= 64) return fail(AMX_ERR_UNSUPPORTED, "filter_compressstore_noalloc: device %d", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "filter_compressstore_noalloc: scratch address");
        g_scratch_ptr[dev] = ptr;
    }
    *out = g_scratch_ptr[dev];
    return AMX_OK;
}

}  // namespace amx

using namespace amx;

extern "C" amx_status amx_filter_compressstore_noalloc(const amx_column* in, const amx_predicate* pred,
                                                       const amx_column* out, uint64_t* d_count, void* stream)
{
    amx_status st = check_column(in, "filter_compressstore_noalloc: in");
    if (st) return st;
    if ((st = check_column(out, "filter_compressstore_noalloc: out"))) return st;
    if (!pred) return fail(AMX_ERR_INVALID_ARG, "filter_compressstore_noalloc: null predicate");
    if (out->n < in->n)
        return fail(AMX_ERR_INVALID_ARG, "filter_compressstore_noalloc: output capacity below input length");
    if (in->n > kNoAllocMaxElements)
        return fail(AMX_ERR_CAPACITY,
                    "filter_compressstore_noalloc: %llu elements exceed the built-in scratch limit of 2^29 "
                    "(536870912); use amx_filter_compressstore with a caller workspace",
                    (unsigned long long)in->n);
    void* scratch = nullptr;
    if ((st = scratch_for_current_device(&scratch))) return st;
    ChainReq r{};
    r.a = in;
    r.pred = pred;
    r.vbits = in->bits;
    r.out = out;
    r.compact = 1;
    r.count_out = d_count;
    return run_chain(r, scratch, kNoAllocScratchBytes, (cudaStream_t)stream);
}

extern "C" amx_status amx_filter_compressstore_noalloc_status(void* stream)
{
    void* scratch = nullptr;
    amx_status st = scratch_for_current_device(&scratch);
    if (st) return st;
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "filter_compressstore_noalloc_status: stream");
    uint32_t err = 0;
    e = cudaMemcpy(&err, &static_cast<const WsHeader*>(scratch)->err, sizeof(err), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "filter_compressstore_noalloc_status: read");
    if (err) return fail((amx_status)err, "device-side failure recorded by the last no-alloc call (%u)", err);
    return AMX_OK;
}
