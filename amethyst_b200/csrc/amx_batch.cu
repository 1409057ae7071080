// amx_batch.cu -- filter + compressstore + sum over many slab columns of uneven length and width
// in ONE persistent launch.
//
// The reference runs one launch per operator and column (src/main.cu:300-340 drives the benches
// column by column; src/op_chaining_demo.cu:137-152 chains launches).  Here the columns of a batch
// are cut into tiles (threads x words-per-thread slab words), the tiles of all columns form one
// work list in column-major order, and persistent CTAs take work items from an atomic ticket.
// Per item:
//   1. the item's column comes from a host-built item -> column map, its tile from the column's
//      first item; each thread issues the loads of its slab words straight from global memory;
//   2. while those loads are in flight, the CTA encodes the PREVIOUS item's survivors (its
//      offset is already known, so no other CTA waits on that work);
//   3. the column's predicate is evaluated field-parallel (the runtime-mask form of the
//      single-column policy: whole-word subtractions against the column's repeated bounds);
//   4. a block scan gives every thread its survivors' places inside the tile, and the tile's
//      count is published for the look-back at once;
//   5. warp 0 runs a decoupled look-back over the column's earlier items (aggregate / inclusive
//      prefix flags in one status word per item; bounded spins) while every warp gathers its
//      survivors into shared memory; the item is encoded in the next iteration (step 2).
// A ticket is taken only when its item is about to be worked on: a ticket held ahead of time would
// delay the publication of that item's count, and every later item of its column waits for it.
// Work items are handed out in column-major order, so every item's predecessors are already held
// by running CTAs and the look-back cannot wait on an item that has not started.
#include <type_traits>
#include <vector>

#include "amx_dispatch.h"
#include "amx_pipeline.cuh"

namespace amx {

struct BatchCol {
    const unsigned long long* data;
    unsigned long long* out;
    uint64_t n;
    uint64_t nwords;  // slab words of the column
    uint64_t item0;   // first work item of the column
    uint64_t items;   // work items of the column
    uint64_t sw_h, sw_l1, sw_l2;
    uint32_t bits, eps, spt, te;  // te = elements per tile = threads * spt * eps
    uint32_t sw_mode, cv16;
    uint64_t eps_m64;  // magic divisor of eps (udiv64)
};

struct BatchHdr {
    unsigned long long ticket;
    uint32_t err;
    uint32_t pad;
    uint64_t pad1[2];
};

constexpr uint64_t kBatchP = 1ull << 63;  // inclusive prefix published
constexpr uint64_t kBatchA = 1ull << 62;  // tile aggregate published
constexpr uint64_t kBatchVal = kBatchA - 1;
constexpr uint32_t kBatchMaxSpt = 8;
// survivors of one tile: u16 for widths <= 16 (at most 64 per thread), else u32 (at most 24 per thread)
template <uint32_t THREADS>
__host__ __device__ constexpr uint32_t batch_cv_bytes() { return THREADS * 128; }

// slab words per thread for a width: R = spt * eps <= 64 elements, at most `wpt` (<= 8) words
inline uint32_t batch_spt(uint32_t bits, uint32_t wpt)
{
    const uint32_t eps = 64 / bits;
    const uint32_t s = 64 / eps;
    const uint32_t cap = wpt < 1 ? 1 : (wpt > kBatchMaxSpt ? kBatchMaxSpt : wpt);
    return s < 1 ? 1 : (s > cap ? cap : s);
}

__device__ __forceinline__ uint64_t batch_flags(const BatchCol& c, uint64_t x)
{
    const uint64_t H = c.sw_h;
    const uint32_t mode = c.sw_mode;
    uint64_t f = H;
    const uint64_t xh = x | H;
    if (mode & kSwLo) {
        const uint64_t t = xh - c.sw_l1;
        f = (mode & kSwLoTop) ? (x & t & H) : ((x | t) & H);
    }
    if (mode & kSwHi) {
        const uint64_t t = xh - c.sw_l2;
        const uint64_t ge = (mode & kSwHiTop) ? (x & t) : (x | t);
        f &= ~ge;
    }
    if (mode & kSwNone) f = 0;
    if (mode & kSwNeg) f ^= H;
    return f;
}

// The survivors of a thread's words in element order into the survivor buffer, and their sum, at
// the compile-time width B: fully unrolled field tests for dense warps of widths with at most 12
// fields per slab, a walk over the set flag bits otherwise.
template <int B>
__device__ __forceinline__ void batch_gather_ct(const uint64_t (&x)[kBatchMaxSpt], const uint64_t (&g)[kBatchMaxSpt],
                                                uint32_t spt, bool dense, uint8_t* cvbuf, uint32_t pos,
                                                unsigned long long& sum)
{
    constexpr int EPS = 64 / B;
    constexpr uint64_t FM = (1ull << B) - 1;
    using D = typename std::conditional<(B <= 16), uint16_t, uint32_t>::type;
    D* dst = reinterpret_cast<D*>(cvbuf);
#pragma unroll
    for (uint32_t i = 0; i < kBatchMaxSpt; i++) {
        if (i >= spt) break;
        if (EPS <= 12 && dense) {
#pragma unroll
            for (int k = 0; k < (EPS <= 12 ? EPS : 1); k++)
                if ((g[i] >> (k * B + B - 1)) & 1) {
                    const uint32_t v = (uint32_t)((x[i] >> (k * B)) & FM);
                    dst[pos++] = (D)v;
                    sum += v;
                }
        }
        else {
            for (uint64_t f = g[i]; f; f &= f - 1) {
                const int bp = __ffsll((long long)f) - 1;
                const uint32_t v = (uint32_t)((x[i] >> (bp - (B - 1))) & FM);
                dst[pos++] = (D)v;
                sum += v;
            }
        }
    }
}

#define AMX_BATCH_WIDTHS(X) \
    X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14) X(15) X(16) X(17) X(18) X(19) \
    X(20) X(21) X(22) X(23) X(24) X(25) X(26) X(27) X(28) X(29) X(30) X(31) X(32)

// Encodes the gathered survivors of one finished item at its looked-back offset and accounts its
// sum and, for a column's last item, its count.
struct BatchPending {
    unsigned long long* out;
    uint64_t g0;
    uint64_t eps_m64;
    uint32_t total, bits, eps, cv16, last, ci;
    unsigned long long sum;
    uint64_t item, first;  // the item and its column's first item (for the deferred look-back)
};

// Decoupled look-back of item `item` (warp 0): the survivors of the column's items before it.
// Every item publishes its own count (kBatchA) right after its block scan and its inclusive
// prefix (kBatchP) once this look-back is done.
__device__ __forceinline__ uint64_t batch_lookback(uint64_t* status, uint64_t item, uint64_t first, uint32_t total,
                                                   BatchHdr* hdr, uint32_t lane)
{
    uint64_t excl = 0;
    uint64_t jj = item;  // items [first, jj) remain to be visited
    bool done = item == first;
    while (!done) {
        const bool in = jj > first + lane;
        const uint64_t idx = jj - 1 - lane;
        uint64_t st = in ? ld_relaxed_u64(&status[idx]) : kBatchP;
        uint32_t spins = 0;
        while (in && (st & (kBatchP | kBatchA)) == 0) {
            if (++spins > kWaitSpins) {
                record_error(&hdr->err, AMX_ERR_TIMEOUT);
                st = kBatchP;
                break;
            }
            if (spins > 8) __nanosleep(32);
            st = ld_relaxed_u64(&status[idx]);
        }
        const uint32_t pmask = __ballot_sync(0xffffffffu, (st & kBatchP) != 0);
        const uint32_t stop = pmask ? (uint32_t)(__ffs(pmask) - 1) : 31;
        uint64_t v = (in && lane <= stop) ? (st & kBatchVal) : 0;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        done = pmask != 0;
        jj = jj > 32 ? jj - 32 : 0;
    }
    if (item != first && lane == 0) st_relaxed_u64(&status[item], kBatchP | (excl + total));
    return excl;
}

template <uint32_t THREADS>
__device__ __forceinline__ void batch_encode(const BatchPending& q, const uint8_t* cvbuf, uint32_t tid,
                                             unsigned long long* counts, unsigned long long* sums)
{
    OutDev o{};
    o.data = q.out;
    o.mask = (1ull << q.bits) - 1;
    o.format = AMX_SLAB;
    o.bits = q.bits;
    o.eps = q.eps;
    o.eps_m64 = q.eps_m64;
    switch (q.bits) {  // block-uniform: the compile-time-width encoder of the column's width
#define AMX_BATCH_ENC(b)                                                                                            \
    case b:                                                                                                          \
        encode_slab_ct<b, typename std::conditional<(b <= 16), uint16_t, uint32_t>::type>(                           \
            o, reinterpret_cast<const typename std::conditional<(b <= 16), uint16_t, uint32_t>::type*>(cvbuf), q.total, \
            q.g0, q.last, tid, THREADS);                                                                             \
        break;
        AMX_BATCH_WIDTHS(AMX_BATCH_ENC)
#undef AMX_BATCH_ENC
        default: break;
    }
    if (tid == 0) {
        if (q.sum) atomicAdd(&sums[q.ci], q.sum);
        if (q.last) counts[q.ci] = q.g0 + q.total;
    }
}

template <uint32_t THREADS>
__global__ void __launch_bounds__(THREADS, THREADS == 512 ? 2 : 4) batch_fc_kernel(const BatchCol* __restrict__ cols,
                                                           const uint32_t* __restrict__ colmap, uint64_t total_items,
                                                           uint64_t* status, BatchHdr* hdr,
                                                           unsigned long long* counts, unsigned long long* sums)
{
    constexpr uint32_t NW = THREADS / 32;
    extern __shared__ __align__(16) uint8_t cvbuf[];
    __shared__ uint64_t s_item;
    __shared__ uint32_t s_wtot[NW];
    __shared__ unsigned long long s_wsum[NW];
    __shared__ uint64_t s_excl;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    BatchPending pend{};
    bool pending = false;

    for (;;) {
        // the previous item's look-back, deferred to here: its prefix is only needed by its
        // encode below, and by now its predecessors have mostly published theirs
        if (pending && warp == 0) {
            const uint64_t excl = batch_lookback(status, pend.item, pend.first, pend.total, hdr, lane);
            if (lane == 0) s_excl = excl;
        }
        if (tid == 0) s_item = atomicAdd(&hdr->ticket, 1ull);
        __syncthreads();  // the ticket and the previous item's prefix; every read of its shared values is done
        if (pending) pend.g0 = s_excl;
        const uint64_t item = s_item;
        if (item >= total_items) break;
        const uint32_t ci = __ldg(colmap + item);
        const BatchCol c = cols[ci];
        const uint64_t t = item - c.item0;
        const uint64_t e0 = t * c.te;
        const uint64_t rem = c.n - e0;
        const uint32_t valid = rem < c.te ? (uint32_t)rem : c.te;
        const uint32_t R = c.spt * c.eps;
        const uint32_t B = c.bits;

        // 1. this item's slab words, loads in flight ...
        uint64_t x[kBatchMaxSpt], g[kBatchMaxSpt];
        const uint64_t s0 = t * (uint64_t)(THREADS * c.spt) + (uint64_t)tid * c.spt;
#pragma unroll
        for (uint32_t i = 0; i < kBatchMaxSpt; i++) x[i] = (i < c.spt && s0 + i < c.nwords) ? __ldg(c.data + s0 + i) : 0;
        // 2. ... while the previous item is encoded (it frees the survivor buffer for this one)
        if (pending) batch_encode<THREADS>(pend, cvbuf, tid, counts, sums);
        // 3. field-parallel flags
        {
            const uint32_t le0 = tid * R;
#pragma unroll
            for (uint32_t i = 0; i < kBatchMaxSpt; i++) {
                uint64_t f = i < c.spt ? batch_flags(c, x[i]) : 0;
                const int left = (int)valid - (int)(le0 + i * c.eps);
                f &= left <= 0 ? 0ull : (left >= (int)c.eps ? ~0ull : ((1ull << (left * B)) - 1));
                g[i] = f;
            }
        }
        uint32_t cnt = 0;
#pragma unroll
        for (uint32_t i = 0; i < kBatchMaxSpt; i++) cnt += __popcll(g[i]);

        // 4. block scan
        uint32_t incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        if (lane == 31) s_wtot[warp] = incl;
        __syncthreads();  // warp totals; the previous item's encode is done everywhere
        uint32_t before = 0, total = 0;
#pragma unroll
        for (uint32_t w = 0; w < NW; w++) {
            const uint32_t v = s_wtot[w];
            before += w < warp ? v : 0;
            total += v;
        }
        const uint32_t pos0 = before + incl - cnt;

        // 5. this item's count for the look-backs of the column's later items (the first item's
        // count is already its inclusive prefix); its own look-back waits for the next iteration
        if (tid == 0) st_relaxed_u64(&status[item], (t == 0 ? kBatchP : kBatchA) | total);

        // every warp gathers its survivors and sums them
        unsigned long long mysum = 0;
        {
            const bool dense = 25 * __reduce_add_sync(0xffffffffu, cnt) > 32 * R;  // above ~4% survivors
            switch (B) {  // block-uniform
#define AMX_BATCH_GATHER(b) \
    case b: batch_gather_ct<b>(x, g, c.spt, dense, cvbuf, pos0, mysum); break;
                AMX_BATCH_WIDTHS(AMX_BATCH_GATHER)
#undef AMX_BATCH_GATHER
                default: break;
            }
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) mysum += __shfl_xor_sync(0xffffffffu, mysum, o);
        if (lane == 0) s_wsum[warp] = mysum;
        __syncthreads();  // survivors gathered, the warp sums visible

        // the encode waits for the next item's loads to be in flight (step 2)
        pend.out = c.out;
        pend.g0 = 0;  // set after the next look-back
        pend.item = item;
        pend.first = c.item0;
        pend.eps_m64 = c.eps_m64;
        pend.total = total;
        pend.bits = B;
        pend.eps = c.eps;
        pend.cv16 = c.cv16;
        pend.last = t + 1 == c.items;
        pend.ci = ci;
        pend.sum = 0;
        if (tid == 0)
            for (uint32_t w = 0; w < NW; w++) pend.sum += s_wsum[w];
        pending = true;
    }
    if (pending) batch_encode<THREADS>(pend, cvbuf, tid, counts, sums);  // its prefix came with the last ticket
}

}  // namespace amx

using namespace amx;

namespace {

constexpr uint64_t kBatchHdrBytes = 256;

uint64_t up256(uint64_t x) { return (x + 255) & ~255ull; }

struct BatchLayout {
    uint64_t hdr, cols, colmap, status, total;
};

BatchLayout batch_layout(uint32_t ncols, uint64_t items)
{
    BatchLayout l{};
    l.hdr = 0;
    l.cols = kBatchHdrBytes;
    l.colmap = up256(l.cols + sizeof(BatchCol) * (uint64_t)ncols);
    l.status = up256(l.colmap + 4 * items);
    l.total = up256(l.status + 8 * items);
    return l;
}

uint32_t tuned_threads(const amx_batch_tuning* t) { return (t && t->threads == 512) ? 512 : 256; }
uint32_t tuned_wpt(const amx_batch_tuning* t)
{
    return (t && t->words_per_thread) ? (t->words_per_thread > kBatchMaxSpt ? kBatchMaxSpt : t->words_per_thread)
                                      : kBatchMaxSpt;
}

uint64_t column_items(const amx_column& c, uint32_t threads, uint32_t wpt)
{
    const uint32_t eps = 64 / c.bits;
    const uint64_t te = (uint64_t)threads * batch_spt(c.bits, wpt) * eps;
    return (c.n + te - 1) / te;
}

template <uint32_t T>
cudaError_t batch_attr(uint32_t smem, int* per_sm)
{
    cudaError_t e = cudaFuncSetAttribute(batch_fc_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, batch_fc_kernel<T>, T, smem);
    return e;
}

}  // namespace

extern "C" {

uint64_t amx_batch_workspace_bytes(const amx_column* ins, uint32_t ncols, const amx_batch_tuning* tuning)
{
    if (!ins) return 0;
    const uint32_t T = tuned_threads(tuning), W = tuned_wpt(tuning);
    uint64_t items = 0;
    for (uint32_t i = 0; i < ncols; i++) {
        if (ins[i].format != AMX_SLAB || ins[i].bits < 1 || ins[i].bits > 32) return 0;
        items += column_items(ins[i], T, W);
    }
    return batch_layout(ncols, items).total;
}

amx_status amx_batch_prepare(const amx_column* ins, const amx_predicate* preds, const amx_column* outs, uint32_t ncols,
                             const amx_batch_tuning* tuning, amx_batch_plan* plan, void* ws, size_t ws_bytes,
                             void* stream)
{
    if (!plan) return fail(AMX_ERR_INVALID_ARG, "batch_prepare: null plan");
    if (ncols && (!ins || !preds || !outs)) return fail(AMX_ERR_INVALID_ARG, "batch_prepare: null column arrays");
    const uint32_t T = tuned_threads(tuning), W = tuned_wpt(tuning);
    std::vector<BatchCol> cols(ncols);
    uint64_t items = 0;
    for (uint32_t i = 0; i < ncols; i++) {
        const amx_column& a = ins[i];
        const amx_column& o = outs[i];
        amx_status st = check_column(&a, "batch: input column");
        if (st) return st;
        if ((st = check_column(&o, "batch: output column"))) return st;
        if (a.format != AMX_SLAB || a.bits > 32)
            return fail(AMX_ERR_UNSUPPORTED, "batch: column %u is not a slab column of at most 32 bits", i);
        if (o.format != AMX_SLAB || o.bits != a.bits)
            return fail(AMX_ERR_UNSUPPORTED, "batch: output %u must be slabs of the input width", i);
        if (o.n < a.n) return fail(AMX_ERR_INVALID_ARG, "batch: output %u capacity below input length", i);
        PipeParams p{};
        p.a = col_dev(&a);
        if ((st = normalize_pred(&preds[i], p.pred_lo, p.pred_span, p.pred_neg))) return st;
        swar_setup(p);
        BatchCol& c = cols[i];
        c.data = reinterpret_cast<const unsigned long long*>(a.data);
        c.out = reinterpret_cast<unsigned long long*>(o.data);
        c.n = a.n;
        c.bits = a.bits;
        c.eps = 64 / a.bits;
        c.nwords = (a.n + c.eps - 1) / c.eps;
        c.spt = batch_spt(a.bits, W);
        c.te = T * c.spt * c.eps;
        c.item0 = items;
        c.items = (a.n + c.te - 1) / c.te;
        c.sw_h = p.sw_h;
        c.sw_l1 = p.sw_l1;
        c.sw_l2 = p.sw_l2;
        c.sw_mode = p.sw_mode;
        c.cv16 = a.bits <= 16 ? 1 : 0;
        c.eps_m64 = magic64(c.eps);
        items += c.items;
    }
    const BatchLayout L = batch_layout(ncols, items);
    if (!ws || ws_bytes < L.total)
        return fail(AMX_ERR_WORKSPACE, "batch: workspace of %zu bytes, %llu needed", ws_bytes,
                    (unsigned long long)L.total);
    if (((uintptr_t)ws) & 255) return fail(AMX_ERR_ALIGNMENT, "batch: workspace not 256-byte aligned");
    std::vector<uint32_t> colmap(items);
    for (uint32_t i = 0; i < ncols; i++)
        for (uint64_t k = 0; k < cols[i].items; k++) colmap[cols[i].item0 + k] = i;
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* w = static_cast<uint8_t*>(ws);
    cudaError_t e = cudaSuccess;
    if (ncols) e = cudaMemcpyAsync(w + L.cols, cols.data(), sizeof(BatchCol) * ncols, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && items)
        e = cudaMemcpyAsync(w + L.colmap, colmap.data(), 4 * items, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);  // the host tables die with this call
    if (e != cudaSuccess) return cuda_fail(e, "batch_prepare: table upload");

    int per_sm = 0;
    const int want = (tuning && tuning->ctas_per_sm) ? (int)tuning->ctas_per_sm : 0;
    const uint32_t smem = T * 128;
    e = T == 512 ? batch_attr<512>(smem, &per_sm) : batch_attr<256>(smem, &per_sm);
    if (e != cudaSuccess) return cuda_fail(e, "batch_prepare: occupancy");
    if (per_sm < 1) return fail(AMX_ERR_UNSUPPORTED, "batch: kernel does not fit on an SM");
    if (want > 0 && want < per_sm) per_sm = want;
    uint64_t grid = (uint64_t)per_sm * sm_count();
    if (grid > items) grid = items ? items : 1;
    plan->ncols = ncols;
    plan->threads = T;
    plan->grid = (uint32_t)grid;
    plan->items = items;
    plan->workspace_bytes = L.total;
    return AMX_OK;
}

amx_status amx_batch_run(const amx_batch_plan* plan, uint64_t* d_counts, uint64_t* d_sums, void* ws, size_t ws_bytes,
                         void* stream)
{
    if (!plan) return fail(AMX_ERR_INVALID_ARG, "batch_run: null plan");
    if (plan->ncols && (!d_counts || !d_sums)) return fail(AMX_ERR_INVALID_ARG, "batch_run: null counts or sums");
    if (!ws || ws_bytes < plan->workspace_bytes) return fail(AMX_ERR_WORKSPACE, "batch_run: workspace too small");
    const BatchLayout L = batch_layout(plan->ncols, plan->items);
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* w = static_cast<uint8_t*>(ws);
    cudaError_t e = cudaMemsetAsync(w, 0, kBatchHdrBytes, s);
    if (e == cudaSuccess && plan->items) e = cudaMemsetAsync(w + L.status, 0, 8 * plan->items, s);
    if (e == cudaSuccess && plan->ncols) e = cudaMemsetAsync(d_sums, 0, 8 * (uint64_t)plan->ncols, s);
    if (e == cudaSuccess && plan->ncols) e = cudaMemsetAsync(d_counts, 0, 8 * (uint64_t)plan->ncols, s);
    if (e != cudaSuccess) return cuda_fail(e, "batch_run: clear");
    if (!plan->items) return AMX_OK;
    const BatchCol* cols = reinterpret_cast<const BatchCol*>(w + L.cols);
    const uint32_t* colmap = reinterpret_cast<const uint32_t*>(w + L.colmap);
    uint64_t* status = reinterpret_cast<uint64_t*>(w + L.status);
    BatchHdr* hdr = reinterpret_cast<BatchHdr*>(w);
    auto* cnt = reinterpret_cast<unsigned long long*>(d_counts);
    auto* sum = reinterpret_cast<unsigned long long*>(d_sums);
    if (plan->threads == 512)
        batch_fc_kernel<512><<<plan->grid, 512, batch_cv_bytes<512>(), s>>>(cols, colmap, plan->items, status, hdr,
                                                                          cnt, sum);
    else
        batch_fc_kernel<256><<<plan->grid, 256, batch_cv_bytes<256>(), s>>>(cols, colmap, plan->items, status, hdr,
                                                                          cnt, sum);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "batch_run: launch");
    return AMX_OK;
}

amx_status amx_batch_status(const void* ws, void* stream)
{
    if (!ws) return fail(AMX_ERR_INVALID_ARG, "batch_status: null workspace");
    BatchHdr h{};
    cudaError_t e = cudaMemcpyAsync(&h, ws, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "batch_status");
    if (h.err) return fail((amx_status)h.err, "batch: a device-side wait timed out");
    return AMX_OK;
}

}  // extern "C"
