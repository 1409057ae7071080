// amx_groupby_sort.cu -- sort-based group-by: sum and count per key, groups in ascending key
// order, for keys of 1..32 bits and values of 1..64 bits in any format.
//
// The reference's sort-based group-by (src/benchs/bench_groupby_sort_cub.cu:48-66) sorts the
// key/value pairs with cub::DeviceRadixSort::SortPairs and reduces them with
// cub::DeviceReduce::ReduceByKey.  This is the same algorithm in kernels of this library:
//   1. the keys and values become plain 32-bit keys and 32- or 64-bit values in the workspace (the
//      tile pipeline's conversion, or its compressstore when a mask selects the rows; the count
//      then stays on the device and every later kernel reads it);
//   2. an LSD radix sort in 8-bit digits, ceil(key_bits / 8) passes of
//        gs_hist_kernel     per tile of 4096 pairs, the digit histogram (one per warp in shared
//                           memory), digit-major so that
//        gs_scan_kernel     one CTA per digit turns the column of tile counts into offsets, and
//        gs_scatter_kernel  ranks every pair stably inside its tile (a warp multisplit of 8 ballots
//                           per 32 pairs, in element order), reorders the tile by digit in
//                           shared memory and
//                           writes each digit's run to its place: consecutive threads, consecutive
//                           addresses;
//   3. reduce-by-key over the sorted pairs: gs_heads_kernel counts the first pair of every key
//      run per tile, gs_scan_heads_kernel turns the counts into group numbers (and writes the
//      group count), and gs_reduce_kernel sums each run as the difference of two running sums of
//      a block scan; runs that cross a tile boundary are added with global atomics, all others
//      stored;
//   4. the tile pipeline encodes keys, sums and counts into the caller's columns, reading the
//      group count on the device.
// The cost is independent of the number of groups: about 20 bytes per pair and pass moved
// through HBM.  The hash-table group-by (amx_groupby) is faster with few groups, this one with
// many (tens of thousands and up), where the hash tables' flushes and global probes dominate.
#include "amx_dispatch.h"
#include "amx_pipeline.cuh"

namespace amx {

constexpr uint32_t kGsThreads = 256;
constexpr uint32_t kGsPer = 16;                      // pairs per thread
constexpr uint32_t kGsTile = kGsThreads * kGsPer;    // 4096 pairs per tile
constexpr uint32_t kGsWarps = kGsThreads / 32;

struct GsHeader {
    uint32_t err;
    uint32_t pad;
    uint64_t n;       // pairs after the mask (compressstore count)
    uint64_t groups;  // when the caller passes no d_groups
};

__device__ __forceinline__ uint64_t gs_len(uint64_t n_max, const uint64_t* n_dev)
{
    if (!n_dev) return n_max;
    const uint64_t d = *n_dev;
    return d < n_max ? d : n_max;
}

// element of thread (warp w, lane) in round i: tile order (round-major, then lane)
__device__ __forceinline__ uint32_t gs_slot(uint32_t w, uint32_t i, uint32_t lane)
{
    return w * (32 * kGsPer) + i * 32 + lane;
}

// Lanes of the warp whose 8-bit digit equals this lane's (valid lanes only): one ballot per digit
// bit (the warp multisplit), cheaper than match_any.
__device__ __forceinline__ uint32_t gs_peers(uint32_t d, bool ok)
{
    uint32_t m = __ballot_sync(0xffffffffu, ok);
#pragma unroll
    for (int b = 0; b < 8; b++) {
        const uint32_t bb = __ballot_sync(0xffffffffu, (d >> b) & 1u);
        m &= ((d >> b) & 1u) ? bb : ~bb;
    }
    return m;
}

// Per tile, the count of every digit, digit-major: counts[d * tiles + tile].
__global__ void __launch_bounds__(kGsThreads) gs_hist_kernel(const uint32_t* keys, uint64_t n_max,
                                                             const uint64_t* n_dev, uint32_t shift, uint32_t* counts,
                                                             uint64_t tiles)
{
    __shared__ uint32_t h[kGsWarps][256];  // one histogram per warp
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint64_t tile = blockIdx.x;
    const uint64_t n = gs_len(n_max, n_dev);
    const uint64_t e0 = tile * kGsTile;
#pragma unroll
    for (uint32_t k = 0; k < kGsWarps; k++) h[k][tid] = 0;
    __syncthreads();
    uint32_t key[kGsPer];
#pragma unroll
    for (uint32_t i = 0; i < kGsPer; i++) {
        const uint64_t e = e0 + gs_slot(w, i, lane);
        key[i] = e < n ? keys[e] : 0u;
    }
#pragma unroll
    for (uint32_t i = 0; i < kGsPer; i++)
        if (e0 + gs_slot(w, i, lane) < n) atomicAdd(&h[w][(key[i] >> shift) & 255u], 1u);
    __syncthreads();
    uint32_t c = 0;
#pragma unroll
    for (uint32_t k = 0; k < kGsWarps; k++) c += h[k][tid];
    counts[(uint64_t)tid * tiles + tile] = c;
}

// Digit d = blockIdx.x: exclusive prefix of its tile counts (in place), its total to tot[d].
__global__ void __launch_bounds__(1024) gs_scan_kernel(uint32_t* counts, uint64_t tiles, uint32_t* tot)
{
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    uint32_t* c = counts + (uint64_t)blockIdx.x * tiles;
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (uint64_t b = 0; b < tiles; b += 1024) {
        const uint64_t i = b + tid;
        const uint32_t v = i < tiles ? c[i] : 0;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= (uint32_t)o) s += y;
            }
            wsum[lane] = s;  // inclusive over warps
        }
        __syncthreads();
        const uint32_t before = carry + (w ? wsum[w - 1] : 0) + x - v;
        if (i < tiles) c[i] = before;
        __syncthreads();
        if (tid == 1023) carry += wsum[31];
        __syncthreads();
    }
    if (tid == 0) tot[blockIdx.x] = carry;
}

// exclusive prefix of 256 values held one per thread of a 256-thread block
__device__ __forceinline__ uint32_t gs_block_excl256(uint32_t v, uint32_t* wsum)
{
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t k = 0; k < w; k++) before += wsum[k];
    __syncthreads();
    return before + x - v;
}

// One LSD pass: every pair of the tile to its place in the output, stable.
template <typename V>
__global__ void __launch_bounds__(kGsThreads, 4) gs_scatter_kernel(const uint32_t* kin, const V* vin, uint32_t* kout,
                                                                V* vout, uint64_t n_max, const uint64_t* n_dev,
                                                                uint32_t shift, const uint32_t* counts, uint64_t tiles,
                                                                const uint32_t* tot)
{
    __shared__ uint32_t wcnt[kGsWarps][256];
    __shared__ uint32_t dstart[256];
    __shared__ uint64_t gbase[256];
    __shared__ uint32_t wsum[kGsWarps];
    extern __shared__ uint4 gs_dyn[];  // the tile sorted by digit: kGsTile keys, then kGsTile values
    uint32_t* sk = reinterpret_cast<uint32_t*>(gs_dyn);
    V* sv = reinterpret_cast<V*>(sk + kGsTile);
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint64_t tile = blockIdx.x;
    const uint64_t n = gs_len(n_max, n_dev);
    const uint64_t e0 = tile * kGsTile;
    if (e0 >= n) return;
    const uint32_t valid = n - e0 < kGsTile ? (uint32_t)(n - e0) : kGsTile;
#pragma unroll
    for (uint32_t k = 0; k < kGsWarps; k++) wcnt[k][tid] = 0;
    // the digit's first output position: the tiles before this one plus every smaller digit
    const uint32_t dbase = gs_block_excl256(tot[tid], wsum);
    gbase[tid] = (uint64_t)dbase + counts[(uint64_t)tid * tiles + tile];
    __syncthreads();

    // only the ranks stay in registers between the phases (keys and values are read again below:
    // cache hits), so more CTAs fit per SM
    uint32_t key[kGsPer], rank[kGsPer];
#pragma unroll
    for (uint32_t i = 0; i < kGsPer; i++) {
        const uint32_t s = gs_slot(w, i, lane);
        key[i] = s < valid ? kin[e0 + s] : 0u;
    }
#pragma unroll
    for (uint32_t i = 0; i < kGsPer; i++) {
        const uint32_t s = gs_slot(w, i, lane);
        const bool ok = s < valid;
        const uint32_t d = (key[i] >> shift) & 255u;
        const uint32_t peers = gs_peers(d, ok);
        const uint32_t below = (uint32_t)__popc(peers & ((1u << lane) - 1));
        const uint32_t have = ok ? wcnt[w][d] : 0u;
        rank[i] = have + below;
        __syncwarp();
        if (ok && below == 0) wcnt[w][d] = have + (uint32_t)__popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // per digit: the warps' exclusive prefix, and the digit's start inside the sorted tile
    uint32_t tcount = 0;
#pragma unroll
    for (uint32_t k = 0; k < kGsWarps; k++) {
        const uint32_t c = wcnt[k][tid];
        wcnt[k][tid] = tcount;
        tcount += c;
    }
    dstart[tid] = gs_block_excl256(tcount, wsum);
    __syncthreads();
#pragma unroll 4
    for (uint32_t i = 0; i < kGsPer; i++) {
        const uint32_t s = gs_slot(w, i, lane);
        if (s < valid) {
            const uint32_t k = kin[e0 + s];
            const uint32_t d = (k >> shift) & 255u;
            const uint32_t pos = dstart[d] + wcnt[w][d] + rank[i];
            sk[pos] = k;
            sv[pos] = vin[e0 + s];
        }
    }
    __syncthreads();
    for (uint32_t j = tid; j < valid; j += kGsThreads) {
        const uint32_t k = sk[j];
        const uint32_t d = (k >> shift) & 255u;
        const uint64_t dst = gbase[d] + (j - dstart[d]);
        kout[dst] = k;
        vout[dst] = sv[j];
    }
}

// first pair of a key run: the first pair, or a key different from its predecessor's
__device__ __forceinline__ bool gs_head(const uint32_t* keys, uint64_t e)
{
    return e == 0 || keys[e] != keys[e - 1];
}

__global__ void __launch_bounds__(kGsThreads) gs_heads_kernel(const uint32_t* keys, uint64_t n_max,
                                                              const uint64_t* n_dev, uint32_t* tile_heads)
{
    __shared__ uint32_t wsum[kGsWarps];
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint64_t tile = blockIdx.x;
    const uint64_t n = gs_len(n_max, n_dev);
    const uint64_t e0 = tile * kGsTile;
    uint32_t c = 0;
    for (uint32_t i = 0; i < kGsPer; i++) {
        const uint64_t e = e0 + gs_slot(w, i, lane);
        c += (e < n && gs_head(keys, e)) ? 1u : 0u;
    }
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) wsum[w] = c;
    __syncthreads();
    if (tid == 0) {
        uint32_t t = 0;
        for (uint32_t k = 0; k < kGsWarps; k++) t += wsum[k];
        tile_heads[tile] = t;
    }
}

// exclusive prefix of the tiles' head counts (group number of each tile's first head), and the
// group count
__global__ void __launch_bounds__(1024) gs_scan_heads_kernel(const uint32_t* tile_heads, uint64_t tiles,
                                                             uint64_t* seg_base, uint64_t* d_groups)
{
    __shared__ uint64_t wsum[32];
    __shared__ uint64_t carry;
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (uint64_t b = 0; b < tiles; b += 1024) {
        const uint64_t i = b + tid;
        const uint64_t v = i < tiles ? tile_heads[i] : 0;
        uint64_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint64_t s = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint64_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= (uint32_t)o) s += y;
            }
            wsum[lane] = s;
        }
        __syncthreads();
        if (i < tiles) seg_base[i] = carry + (w ? wsum[w - 1] : 0) + x - v;
        __syncthreads();
        if (tid == 1023) carry += wsum[31];
        __syncthreads();
    }
    if (tid == 0) *d_groups = carry;
}

// Sums and counts of the key runs.  Thread t takes pairs 16t .. 16t+15 of the tile; a block scan
// of the head counts numbers the runs (group g = the tile's first group number + the heads up to
// the pair - 1; run 0 is the one continuing from the tile before) and a block scan of the values
// gives every pair's running sum.  The thread holding a run's first pair records the running sum
// before it and its position; the thread holding its last pair turns them into the run's sum and
// length.  Runs that start and end inside the tile are stored, the first (continuing from the tile
// before) and the last (continuing into the next) are added with atomics into the zeroed outputs.
template <typename V>
__global__ void __launch_bounds__(kGsThreads) gs_reduce_kernel(const uint32_t* keys, const V* vals, uint64_t n_max,
                                                               const uint64_t* n_dev, const uint64_t* seg_base,
                                                               uint32_t* okey, unsigned long long* osum,
                                                               unsigned long long* ocnt, uint64_t cap, uint32_t* err)
{
    extern __shared__ uint4 gs_dyn[];  // per run: running sum before its first pair, then that position
    unsigned long long* rstart = reinterpret_cast<unsigned long long*>(gs_dyn);
    uint32_t* pstart = reinterpret_cast<uint32_t*>(rstart + kGsTile + 1);
    __shared__ uint32_t wh[kGsWarps];
    __shared__ unsigned long long wv[kGsWarps];
    const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint64_t tile = blockIdx.x;
    const uint64_t n = gs_len(n_max, n_dev);
    const uint64_t e0 = tile * kGsTile;
    if (e0 >= n) return;
    const uint32_t valid = n - e0 < kGsTile ? (uint32_t)(n - e0) : kGsTile;
    const uint32_t b = tid * kGsPer;
    uint32_t k[kGsPer];
    unsigned long long v[kGsPer];
    if (b + kGsPer <= valid) {  // 16-byte loads: the buffers and the caller's columns are 16-byte aligned
        const uint4* kq = reinterpret_cast<const uint4*>(keys + e0 + b);
#pragma unroll
        for (uint32_t q = 0; q < kGsPer / 4; q++) {
            const uint4 x = kq[q];
            k[4 * q] = x.x;
            k[4 * q + 1] = x.y;
            k[4 * q + 2] = x.z;
            k[4 * q + 3] = x.w;
        }
        const uint4* vq = reinterpret_cast<const uint4*>(vals + e0 + b);
        if constexpr (sizeof(V) == 4) {
#pragma unroll
            for (uint32_t q = 0; q < kGsPer / 4; q++) {
                const uint4 x = vq[q];
                v[4 * q] = x.x;
                v[4 * q + 1] = x.y;
                v[4 * q + 2] = x.z;
                v[4 * q + 3] = x.w;
            }
        }
        else {
#pragma unroll
            for (uint32_t q = 0; q < kGsPer / 2; q++) {
                const uint4 x = vq[q];
                v[2 * q] = ((unsigned long long)x.y << 32) | x.x;
                v[2 * q + 1] = ((unsigned long long)x.w << 32) | x.z;
            }
        }
    }
    else {
#pragma unroll
        for (uint32_t j = 0; j < kGsPer; j++) {
            const bool ok = b + j < valid;
            k[j] = ok ? keys[e0 + b + j] : 0u;
            v[j] = ok ? (unsigned long long)vals[e0 + b + j] : 0ull;
        }
    }
    const bool has_prev = e0 + b > 0 && b < valid;
    const uint32_t kprev = has_prev ? keys[e0 + b - 1] : 0u;
    const bool has_next = b + kGsPer < valid || (b + kGsPer == kGsTile && e0 + kGsTile < n);
    const uint32_t knext = has_next ? keys[e0 + b + kGsPer] : 0u;
    uint32_t hf = 0;  // bit j: pair j starts a run
    unsigned long long vs = 0;
#pragma unroll
    for (uint32_t j = 0; j < kGsPer; j++) {
        const bool ok = b + j < valid;
        const bool head = ok && (j ? k[j] != k[j - 1] : (!has_prev || k[0] != kprev));
        hf |= (head ? 1u : 0u) << j;
        vs += v[j];
    }
    // block scans: heads and values before this thread
    uint32_t hx = (uint32_t)__popc(hf);
    unsigned long long vx = vs;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t yh = __shfl_up_sync(0xffffffffu, hx, o);
        const unsigned long long yv = __shfl_up_sync(0xffffffffu, vx, o);
        if (lane >= (uint32_t)o) {
            hx += yh;
            vx += yv;
        }
    }
    if (lane == 31) {
        wh[w] = hx;
        wv[w] = vx;
    }
    __syncthreads();
    uint32_t hbefore = hx - (uint32_t)__popc(hf), total_heads = 0;
    unsigned long long vbefore = vx - vs;
    for (uint32_t q = 0; q < kGsWarps; q++) {
        if (q < w) {
            hbefore += wh[q];
            vbefore += wv[q];
        }
        total_heads += wh[q];
    }
    if (tid == 0 && !(hf & 1u)) {  // the run continuing from the tile before
        rstart[0] = 0;
        pstart[0] = 0;
    }
    // run starts
    {
        uint32_t loc = hbefore;
        unsigned long long run = vbefore;
#pragma unroll
        for (uint32_t j = 0; j < kGsPer; j++) {
            if ((hf >> j) & 1u) {
                loc++;
                rstart[loc] = run;
                pstart[loc] = b + j;
            }
            run += v[j];
        }
    }
    __syncthreads();
    // run ends: the last valid pair of the tile, or a pair followed by a head
    const bool open_end = valid == kGsTile && e0 + kGsTile < n && keys[e0 + kGsTile] == keys[e0 + kGsTile - 1];
    const uint64_t g0 = seg_base[tile];  // group number of the tile's first head
    uint32_t loc = hbefore;
    unsigned long long run = vbefore;
#pragma unroll
    for (uint32_t j = 0; j < kGsPer; j++) {
        const bool ok = b + j < valid;
        if ((hf >> j) & 1u) {
            loc++;
            const uint64_t g = g0 + loc - 1;
            if (g < cap) okey[g] = k[j];
        }
        run += v[j];
        const bool last = b + j + 1 == valid;
        const bool next_head = j + 1 < kGsPer ? ((hf >> (j + 1)) & 1u) != 0 : (has_next && knext != k[j]);
        if (ok && (last || next_head)) {
            const unsigned long long sum = run - rstart[loc];
            const unsigned long long cnt = (unsigned long long)(b + j + 1 - pstart[loc]);
            const uint64_t g = g0 + loc - 1;  // loc 0: the run that began before this tile
            if (g >= cap) {
                record_error(err, AMX_ERR_CAPACITY);
            }
            else if (loc == 0 || (loc == total_heads && last && open_end)) {
                atomicAdd(&osum[g], sum);
                atomicAdd(&ocnt[g], cnt);
            }
            else {
                osum[g] = sum;
                ocnt[g] = cnt;
            }
        }
    }
}

static uint64_t gs_align(uint64_t x) { return (x + 255) & ~255ull; }

// Workspace of a sort-based group-by over n pairs with values carried in `vbytes` bytes:
//   header | keys A | keys B | values A | values B | digit counts | digit totals | tile heads |
//   group bases | group keys | group sums | group counts | pipeline workspace
struct GsLayout {
    uint64_t hdr, ka, kb, va, vb, counts, tot, heads, base, okey, osum, ocnt, ws, total, tiles;
};

static GsLayout gs_layout(uint64_t n, uint32_t vbytes)
{
    GsLayout l{};
    const uint64_t m = n ? n : 1;
    l.tiles = (m + kGsTile - 1) / kGsTile;
    l.hdr = 0;
    l.ka = 256;
    l.kb = gs_align(l.ka + 4 * m + 16);
    l.va = gs_align(l.kb + 4 * m + 16);
    l.vb = gs_align(l.va + (uint64_t)vbytes * m + 16);
    l.counts = gs_align(l.vb + (uint64_t)vbytes * m + 16);
    l.tot = gs_align(l.counts + 4ull * 256 * l.tiles);
    l.heads = gs_align(l.tot + 4 * 256);
    l.base = gs_align(l.heads + 4 * l.tiles);
    l.okey = gs_align(l.base + 8 * l.tiles);
    l.osum = gs_align(l.okey + 4 * m + 16);
    l.ocnt = gs_align(l.osum + 8 * m);
    l.ws = gs_align(l.ocnt + 8 * m);
    l.total = gs_align(l.ws + amx_workspace_bytes(m));
    return l;
}

amx_status groupby_sort_run(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                            const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                            uint64_t* d_groups, void* ws, size_t ws_bytes, void* stream, const uint64_t* n_dev)
{
    amx_status st = check_column(keys, "groupby_sort: keys");
    if (st) return st;
    if ((st = check_column(vals, "groupby_sort: values"))) return st;
    if (keys->n != vals->n) return fail(AMX_ERR_INVALID_ARG, "groupby_sort: keys and values lengths differ");
    if (keys->bits > 32) return fail(AMX_ERR_UNSUPPORTED, "groupby_sort: keys of %u bits (at most 32)", keys->bits);
    if (((uintptr_t)d_mask) & 15) return fail(AMX_ERR_ALIGNMENT, "groupby_sort: mask not 16-byte aligned");
    const uint64_t n = keys->n;
    const uint32_t vbytes = vals->bits <= 32 ? 4 : 8;
    const GsLayout L = gs_layout(n, vbytes);
    if (!ws || ws_bytes < L.total)
        return fail(AMX_ERR_WORKSPACE, "groupby_sort: workspace of %zu bytes, %llu needed", ws_bytes,
                    (unsigned long long)L.total);
    if (((uintptr_t)ws) & 255) return fail(AMX_ERR_ALIGNMENT, "groupby_sort: workspace not 256-byte aligned");
    const amx_column* outs[3] = {out_keys, out_sums, out_counts};
    const char* names[3] = {"groupby_sort: out_keys", "groupby_sort: out_sums", "groupby_sort: out_counts"};
    uint64_t cap = n ? n : 1;
    for (int i = 0; i < 3; i++) {
        if (!outs[i]) continue;
        if ((st = check_column(outs[i], names[i]))) return st;
        if (outs[i]->n < cap) cap = outs[i]->n;
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* w = static_cast<uint8_t*>(ws);
    GsHeader* hdr = reinterpret_cast<GsHeader*>(w + L.hdr);
    uint64_t* groups = d_groups ? d_groups : &hdr->groups;
    cudaError_t e = cudaMemsetAsync(w, 0, 256, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w + L.osum, 0, L.ws - L.osum, s);  // sums and counts
    if (e == cudaSuccess && d_groups) e = cudaMemsetAsync(d_groups, 0, 8, s);
    if (e != cudaSuccess) return cuda_fail(e, "groupby_sort: clear");
    void* pws = w + L.ws;
    const size_t pws_bytes = L.total - L.ws;

    // 1. plain keys and values (compacted by the mask, the count on the device)
    uint32_t* ka = reinterpret_cast<uint32_t*>(w + L.ka);
    uint32_t* kb = reinterpret_cast<uint32_t*>(w + L.kb);
    void* va = w + L.va;
    void* vb = w + L.vb;
    const uint64_t* len = n_dev;
    // 32-bit slabs hold two fields per word, low first: the layout of a plain uint32 array, so
    // such keys (and such values, or 64-bit plain ones) are read in place when no mask selects
    const bool keys_plain = keys->bits == 32 && (keys->format == AMX_PLAIN32 || keys->format == AMX_SLAB);
    const bool vals_plain = (vbytes == 4 && vals->bits == 32 && (vals->format == AMX_PLAIN32 || vals->format == AMX_SLAB)) ||
                            (vbytes == 8 && vals->bits == 64 && (vals->format == AMX_PLAIN64 || vals->format == AMX_SLAB));
    const uint32_t* k_in = ka;
    const void* v_in = va;
    if (n) {
        const amx_column pk{ka, n, AMX_PLAIN32, 32};
        const amx_column pv{va, n, (uint32_t)(vbytes == 4 ? AMX_PLAIN32 : AMX_PLAIN64), vbytes == 4 ? 32u : 64u};
        ChainReq r{};
        r.a = keys;
        r.vbits = keys->bits;
        r.out = &pk;
        r.n_dev = n_dev;
        if (d_mask) {
            r.mask_in = d_mask;
            r.compact = 1;
            r.count_out = &hdr->n;
        }
        if (d_mask || !keys_plain) {
            if ((st = run_chain(r, pws, pws_bytes, s))) return st;
        }
        else {
            k_in = static_cast<const uint32_t*>(keys->data);
        }
        if (d_mask || !vals_plain) {
            r.a = vals;
            r.vbits = vals->bits;
            r.out = &pv;
            r.count_out = nullptr;
            if ((st = run_chain(r, pws, pws_bytes, s))) return st;
        }
        else {
            v_in = vals->data;
        }
        if (d_mask) len = &hdr->n;
    }

    // 2. LSD radix sort in 8-bit digits
    const uint64_t tiles = L.tiles;
    uint32_t* counts = reinterpret_cast<uint32_t*>(w + L.counts);
    uint32_t* tot = reinterpret_cast<uint32_t*>(w + L.tot);
    const uint32_t passes = n ? (keys->bits + 7) / 8 : 0;
    const size_t scat_smem = (size_t)kGsTile * (4 + vbytes);
    const size_t red_smem = (size_t)(kGsTile + 1) * (8 + 4);  // run starts: running sum and position
    if (vbytes == 4) {
        e = cudaFuncSetAttribute(gs_scatter_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scat_smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(gs_reduce_kernel<uint32_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)red_smem);
    }
    else {
        e = cudaFuncSetAttribute(gs_scatter_kernel<unsigned long long>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)scat_smem);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(gs_reduce_kernel<unsigned long long>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)red_smem);
    }
    if (e != cudaSuccess) return cuda_fail(e, "groupby_sort: shared memory attribute");
    // pass 0 reads k_in / v_in (the caller's columns or buffers A) and writes buffers B; later
    // passes alternate between A and B
    for (uint32_t pass = 0; pass < passes; pass++) {
        const uint32_t shift = 8 * pass;
        const uint32_t* src_k = pass ? ka : k_in;
        const void* src_v = pass ? va : v_in;
        gs_hist_kernel<<<(unsigned)tiles, kGsThreads, 0, s>>>(src_k, n, len, shift, counts, tiles);
        gs_scan_kernel<<<256, 1024, 0, s>>>(counts, tiles, tot);
        if (vbytes == 4)
            gs_scatter_kernel<uint32_t><<<(unsigned)tiles, kGsThreads, scat_smem, s>>>(
                src_k, reinterpret_cast<const uint32_t*>(src_v), kb, reinterpret_cast<uint32_t*>(vb), n, len, shift,
                counts, tiles, tot);
        else
            gs_scatter_kernel<unsigned long long><<<(unsigned)tiles, kGsThreads, scat_smem, s>>>(
                src_k, reinterpret_cast<const unsigned long long*>(src_v), kb, reinterpret_cast<unsigned long long*>(vb),
                n, len, shift, counts, tiles, tot);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "groupby_sort: radix pass launch");
        uint32_t* tk = ka;
        ka = kb;
        kb = tk;
        void* tv = va;
        va = vb;
        vb = tv;
    }

    // 3. reduce by key
    uint32_t* heads = reinterpret_cast<uint32_t*>(w + L.heads);
    uint64_t* base = reinterpret_cast<uint64_t*>(w + L.base);
    uint32_t* okey = reinterpret_cast<uint32_t*>(w + L.okey);
    unsigned long long* osum = reinterpret_cast<unsigned long long*>(w + L.osum);
    unsigned long long* ocnt = reinterpret_cast<unsigned long long*>(w + L.ocnt);
    if (n) {
        gs_heads_kernel<<<(unsigned)tiles, kGsThreads, 0, s>>>(ka, n, len, heads);
        gs_scan_heads_kernel<<<1, 1024, 0, s>>>(heads, tiles, base, groups);
        if (vbytes == 4)
            gs_reduce_kernel<uint32_t><<<(unsigned)tiles, kGsThreads, red_smem, s>>>(
                ka, reinterpret_cast<const uint32_t*>(va), n, len, base, okey, osum, ocnt, cap, &hdr->err);
        else
            gs_reduce_kernel<unsigned long long><<<(unsigned)tiles, kGsThreads, red_smem, s>>>(
                ka, reinterpret_cast<const unsigned long long*>(va), n, len, base, okey, osum, ocnt, cap, &hdr->err);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "groupby_sort: reduce launch");
    }

    // 4. the groups into the caller's columns, as many as the device count says
    const amx_column tk{okey, cap, AMX_PLAIN32, 32}, ts{osum, cap, AMX_PLAIN64, 64}, tc{ocnt, cap, AMX_PLAIN64, 64};
    const amx_column* srcs[3] = {&tk, &ts, &tc};
    for (int i = 0; i < 3; i++) {
        if (!outs[i] || !n) continue;
        ChainReq r{};
        r.a = srcs[i];
        r.vbits = outs[i]->bits;
        r.out = outs[i];
        r.n_dev = groups;
        if ((st = run_chain(r, pws, pws_bytes, s))) return st;
    }
    return AMX_OK;
}

}  // namespace amx

using namespace amx;

extern "C" {

uint64_t amx_groupby_sort_workspace_bytes(uint64_t n, uint32_t key_bits, uint32_t value_bits)
{
    if (key_bits < 1 || key_bits > 32 || value_bits < 1 || value_bits > 64 || n > kMaxElements) return 0;
    return gs_layout(n, value_bits <= 32 ? 4 : 8).total;
}

amx_status amx_groupby_sort(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                            const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                            uint64_t* d_groups, void* ws, size_t ws_bytes, void* stream)
{
    return groupby_sort_run(keys, vals, d_mask, out_keys, out_sums, out_counts, d_groups, ws, ws_bytes, stream, nullptr);
}

amx_status amx_groupby_sort_status(const void* workspace, void* stream)
{
    if (!workspace) return fail(AMX_ERR_INVALID_ARG, "groupby_sort_status: null workspace");
    GsHeader h{};
    cudaError_t e = cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "groupby_sort_status");
    if (h.err) return fail((amx_status)h.err, "groupby_sort: device-side failure (%u)", h.err);
    return AMX_OK;
}

}  // extern "C"
