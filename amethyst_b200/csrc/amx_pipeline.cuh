// amx_pipeline.cuh -- the tile pipeline kernel behind filter, compressstore, binary ops,
// conversion, aggregation and fused chains.
//
// One persistent CTA per SM slot pulls tiles from an atomic ticket counter.  For each tile:
//   1. one thread stages the tile's bytes of every input into shared memory with 1-D bulk
//      copies (cp.async.bulk, completion on an mbarrier), two tiles ahead;
//   2. every thread decodes R elements straight from the staged packed words (a policy:
//      warp-major runtime-width readers, or thread-contiguous compile-time-width readers),
//      applies the binary op and the predicate, and keeps a flag word;
//   3. flags feed (a) the bitmask (warp ballots or a shared-memory bitmap), (b) the aggregate,
//      (c) a block scan that publishes the tile's survivor count for the decoupled look-back
//      and gathers the survivors into shared memory.
//   4. the PREVIOUS tile's look-back (now short: its predecessors have had a whole tile of
//      time to publish) gives its output offset, and its gathered survivors are re-encoded in
//      the output format; boundary words shared with neighbouring tiles merge by atomics.
// Replaces the reference's separate filter / popcount / CUB scan / write kernels
// (src/kernels/filter_slabs.cuh:4-57, src/kernels/compressstore_slabs.cuh:4-206,
// src/benchs/bench_compressstore_slabs.cu:38-56) with one pass and no mask round trip.
#pragma once

#include "amx_device.cuh"

namespace amx {

// byte range [b0, b1) of column c that holds elements [e0, e1)
__device__ __forceinline__ void col_range(const ColDev& c, uint64_t e0, uint64_t e1, uint64_t& b0, uint64_t& b1)
{
    switch (c.format) {
        case AMX_PLAIN32: b0 = 4 * e0; b1 = 4 * e1; break;
        case AMX_PLAIN64: b0 = 8 * e0; b1 = 8 * e1; break;
        case AMX_SLAB: b0 = 8 * (e0 / c.eps); b1 = 8 * ((e1 + c.eps - 1) / c.eps); break;
        case AMX_NOGAPS: b0 = 8 * ((e0 * c.bits) >> 6); b1 = 8 * ((e1 * c.bits + 63) >> 6); break;
        default: b0 = 4 * (e0 >> 5); b1 = 4 * ((e1 + 31) >> 5); break;  // bitmask words
    }
    if (b1 > c.bytes) b1 = c.bytes;
    if (b0 > b1) b0 = b1;
}

struct Copy {
    const uint8_t* src;
    uint8_t* dst;
    uint32_t bytes;
};

// Plan the staging of one column: the 16-byte-aligned body goes through the bulk-copy unit;
// a ragged tail at the very end of the column (< 16 bytes) is copied here with plain loads.
__device__ __forceinline__ void stage_plan(const ColDev& c, uint64_t e0, uint64_t e1, uint8_t* dst, uint64_t* sbase,
                                           Copy* cp, int& ncp, uint32_t& tx)
{
    uint64_t b0, b1;
    col_range(c, e0, e1, b0, b1);
    const uint64_t s16 = b0 & ~15ull;
    *sbase = s16;
    uint64_t tend = (b1 + 15) & ~15ull;
    const uint64_t total16 = c.bytes & ~15ull;
    if (tend > total16) tend = total16;
    const uint8_t* src = reinterpret_cast<const uint8_t*>(c.data);
    if (tend > s16) {
        cp[ncp++] = Copy{src + s16, dst, (uint32_t)(tend - s16)};
        tx += (uint32_t)(tend - s16);
    }
    for (uint64_t x = tend > s16 ? tend : s16; x < b1; x++) dst[x - s16] = src[x];
}

// Issue the staging of one tile into stage buffer `st` (called by a single thread).
__device__ __forceinline__ void stage_issue(const PipeParams& p, uint8_t* st, uint64_t* sbase, uint64_t* bar,
                                            uint64_t tile, uint32_t tile_elems)
{
    const uint64_t e0 = tile * tile_elems;
    uint64_t e1 = e0 + tile_elems;
    if (e1 > p.n) e1 = p.n;
    Copy cp[3];
    int ncp = 0;
    uint32_t tx = 0;
    stage_plan(p.a, e0, e1, st + p.a_off, &sbase[0], cp, ncp, tx);
    if (p.has_b) stage_plan(p.b, e0, e1, st + p.b_off, &sbase[1], cp, ncp, tx);
    if (p.has_mask_in) stage_plan(p.m, e0, e1, st + p.m_off, &sbase[2], cp, ncp, tx);
    mbar_arrive_expect_tx(bar, tx);
    for (int i = 0; i < ncp; i++) bulk_g2s(cp[i].dst, cp[i].src, cp[i].bytes, bar);
}

// bits [bit, bit+R) of a little-endian uint32 word array (R <= 64)
template <int R>
__device__ __forceinline__ uint64_t bits_at(const uint32_t* w, uint32_t bit)
{
    const uint32_t wi = bit >> 5, sh = bit & 31;
    uint64_t x = ((uint64_t)w[wi] | ((uint64_t)w[wi + 1] << 32)) >> sh;
    if (R + sh > 64) x |= (uint64_t)w[wi + 2] << (64 - sh);
    return R == 64 ? x : (x & ((1ull << R) - 1));
}

template <typename V>
__device__ __forceinline__ V warp_incl_scan(V x)
{
    const uint32_t lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const V y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    return x;
}

// Bank-skewed index of the gathered-values buffer: one pad entry per 32 (4-byte values) or
// per 16 (8-byte values), so that strided per-thread access patterns spread over banks.
template <typename V>
__device__ __forceinline__ uint32_t sk(uint32_t p)
{
    return sizeof(V) == 4 ? p + (p >> 5) : p + (p >> 4);
}

// Re-encode cnt gathered values cv[0..cnt) as output elements [g, g+cnt).  Words wholly
// owned by this tile are stored; words shared with neighbouring tiles are merged with
// atomicAnd (clear own bits) + atomicOr (set own bits), which commute across tiles because
// owners are disjoint.  Dead slab bits belong to the owner of the slab's last field; the
// bits past the column's last element are cleared by the last tile (`last`).
template <typename V>
__device__ __forceinline__ void encode_tile(const OutDev& o, const V* cv, uint32_t cnt, uint64_t g, bool last)
{
    const uint32_t tid = threadIdx.x;
    const uint32_t T = blockDim.x;
    const uint64_t m = o.mask;
    switch (o.format) {
        case AMX_PLAIN32: {
            uint32_t* out = reinterpret_cast<uint32_t*>(o.data) + g;
            for (uint32_t r = tid; r < cnt; r += T) out[r] = (uint32_t)((uint64_t)cv[sk<V>(r)] & m);
            return;
        }
        case AMX_PLAIN64: {
            uint64_t* out = reinterpret_cast<uint64_t*>(o.data) + g;
            for (uint32_t r = tid; r < cnt; r += T) out[r] = (uint64_t)cv[sk<V>(r)] & m;
            return;
        }
        case AMX_SLAB: {
            unsigned long long* out = reinterpret_cast<unsigned long long*>(o.data);
            const uint32_t eps = o.eps, b = o.bits;
            const uint64_t live = eps * b >= 64 ? ~0ull : ((1ull << (eps * b)) - 1);
            if (cnt) {
                const uint64_t w0 = g / eps, w1 = (g + cnt - 1) / eps;
                for (uint64_t w = w0 + tid; w <= w1; w += T) {
                    const int64_t r0 = (int64_t)(w * eps) - (int64_t)g;
                    uint64_t acc = 0;
                    if (r0 >= 0 && r0 + eps <= cnt) {
                        for (uint32_t k = 0; k < eps; k++) acc |= ((uint64_t)cv[sk<V>((uint32_t)r0 + k)] & m) << (k * b);
                        out[w] = acc;
                    }
                    else {
                        uint64_t own = 0;
                        for (uint32_t k = 0; k < eps; k++) {
                            const int64_t r = r0 + k;
                            if (r >= 0 && r < (int64_t)cnt) {
                                acc |= ((uint64_t)cv[sk<V>((uint32_t)r)] & m) << (k * b);
                                own |= m << (k * b);
                            }
                        }
                        if (r0 + (int64_t)eps - 1 < (int64_t)cnt && r0 + (int64_t)eps - 1 >= 0) own |= ~live;
                        atomicAnd(&out[w], ~own);
                        atomicOr(&out[w], acc);
                    }
                }
            }
            if (last && tid == 0) {
                const uint64_t total = g + cnt;
                const uint32_t k = (uint32_t)(total % eps);
                if (k) atomicAnd(&out[total / eps], (1ull << (k * b)) - 1);
            }
            return;
        }
        default: {  // nogaps
            unsigned long long* out = reinterpret_cast<unsigned long long*>(o.data);
            const uint32_t b = o.bits;
            const uint64_t bit0 = g * b, bit1 = (g + cnt) * b;
            if (cnt) {
                const uint64_t w0 = bit0 >> 6, w1 = (bit1 - 1) >> 6;
                for (uint64_t w = w0 + tid; w <= w1; w += T) {
                    const uint64_t lo = w << 6, hi = lo + 64;
                    const uint64_t ob0 = lo > bit0 ? lo : bit0, ob1 = hi < bit1 ? hi : bit1;
                    const uint64_t own = (ob1 - ob0 >= 64) ? ~0ull : (((1ull << (ob1 - ob0)) - 1) << (ob0 - lo));
                    uint64_t p0 = lo / b;
                    if (p0 < g) p0 = g;
                    uint64_t p1 = (hi - 1) / b;
                    if (p1 > g + cnt - 1) p1 = g + cnt - 1;
                    uint64_t acc = 0;
                    for (uint64_t q = p0; q <= p1; q++) {
                        const uint64_t v = (uint64_t)cv[sk<V>((uint32_t)(q - g))] & m;
                        const int64_t s = (int64_t)(q * b) - (int64_t)lo;
                        acc |= s >= 0 ? (v << s) : (v >> (-s));
                    }
                    if (own == ~0ull)
                        out[w] = acc;
                    else {
                        atomicAnd(&out[w], ~own);
                        atomicOr(&out[w], acc & own);
                    }
                }
            }
            if (last && tid == 0) {
                const uint32_t k = (uint32_t)(bit1 & 63);
                if (k) atomicAnd(&out[bit1 >> 6], (1ull << k) - 1);
            }
            return;
        }
    }
}

// Look-back for a tile whose survivor count (AGG) is already published: returns the number
// of survivors in all earlier tiles and publishes the tile's inclusive prefix (INC).  All 32
// lanes of one warp call it.  Each round reads kLookWindow predecessor status words at once
// (8 per lane, independent loads), so one round usually reaches a published prefix.  Every
// wait is bounded: on timeout the error word is set and the missing value is taken as 0.
constexpr int kLookPerLane = 8;

__device__ __forceinline__ uint64_t lookback_prev(uint64_t* status, uint64_t tile, uint64_t agg, uint32_t* err)
{
    const uint32_t lane = threadIdx.x & 31;
    if (tile == 0) return 0;  // tile 0 published its inclusive prefix directly
    uint64_t excl = 0;
    int64_t j = (int64_t)tile - 1;
    while (true) {
        uint64_t st[kLookPerLane];
#pragma unroll
        for (int m = 0; m < kLookPerLane; m++) {
            const int64_t idx = j - (int64_t)(lane + 32 * m);
            st[m] = idx >= 0 ? ld_relaxed_u64(&status[idx]) : kFlagInc;
        }
        // wait for unpublished predecessors (they are decoding now)
#pragma unroll
        for (int m = 0; m < kLookPerLane; m++) {
            const int64_t idx = j - (int64_t)(lane + 32 * m);
            uint32_t spins = 0;
            while ((st[m] >> 62) == 0) {
                if (++spins > kWaitSpins) {
                    record_error(err, AMX_ERR_TIMEOUT);
                    st[m] = kFlagInc;
                    break;
                }
                if (spins > 8) __nanosleep(20);
                st[m] = ld_relaxed_u64(&status[idx]);
            }
        }
        // nearest inclusive prefix: smallest window position p = lane + 32 m
        int mine = 1 << 30;
#pragma unroll
        for (int m = kLookPerLane - 1; m >= 0; m--)
            if ((st[m] >> 62) == 2) mine = (int)lane + 32 * m;
        int pmin = mine;
#pragma unroll
        for (int o = 16; o; o >>= 1) pmin = min(pmin, __shfl_xor_sync(0xffffffffu, pmin, o));
        uint64_t v = 0;
#pragma unroll
        for (int m = 0; m < kLookPerLane; m++)
            if ((int)lane + 32 * m <= pmin) v += st[m] & kValMask;
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (pmin < (1 << 30)) break;
        j -= 32 * kLookPerLane;
    }
    if (lane == 0) st_relaxed_u64(&status[tile], kFlagInc | (excl + agg));
    return excl;
}

// Shared-memory map of the pipeline kernel (dynamic shared memory):
//   [0,64)     mbarriers            [64,128)  tickets        [128,256) stage base offsets
//   [256,320)  warp totals          [320,384) broadcast      [384,448) warp aggregates
//   [512,2560) tile bitmap (thread-contiguous policies, <= 16384 elements)
//   [kCvOff, smem_fixed)  gathered values (bank-skewed);  [smem_fixed, ...) 2 stage buffers
constexpr uint32_t kBitmapOff = 512;
constexpr uint32_t kCvOff = 2560;

template <class Pol>
__global__ void __launch_bounds__(kPipeThreads) pipe_kernel(const __grid_constant__ PipeParams p)
{
    using V = typename Pol::V;
    constexpr int R = Pol::R;
    constexpr bool WM = Pol::kWarpMajor;
    constexpr uint32_t T = kPipeThreads;
    constexpr uint32_t NW = T / 32;
    constexpr uint32_t TILE = T * R;
    static_assert(TILE / 32 * 4 <= kCvOff - kBitmapOff, "bitmap region");
    static_assert(!WM || R <= 32, "warp-major runs keep one ballot per lane");

    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);
    volatile uint64_t* tickets = reinterpret_cast<volatile uint64_t*>(smem + 64);
    uint64_t* sbase = reinterpret_cast<uint64_t*>(smem + 128);
    volatile uint64_t* warp_tot = reinterpret_cast<volatile uint64_t*>(smem + 256);
    volatile uint64_t* bcast = reinterpret_cast<volatile uint64_t*>(smem + 320);
    uint64_t* warp_agg = reinterpret_cast<uint64_t*>(smem + 384);
    uint32_t* bitmap = reinterpret_cast<uint32_t*>(smem + kBitmapOff);
    V* cv = reinterpret_cast<V*>(smem + kCvOff);
    uint8_t* stage0 = smem + p.smem_fixed;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        for (uint32_t s = 0; s < kStages; s++) mbar_init(&mbar[s], 1);
        fence_mbar_init();
    }
    if (!WM)
        for (uint32_t i = tid; i < TILE / 32; i += T) bitmap[i] = 0;
    __syncthreads();
    uint64_t next_tk = 0;  // thread 0: the ticket for the stage freed next
    if (tid == 0) {
        for (uint32_t s = 0; s < kStages; s++) {
            const uint64_t tk = atomicAdd(&p.ws->ticket, 1u);
            tickets[s] = tk;
            if (tk < p.num_tiles) stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &mbar[s], tk, TILE);
        }
        next_tk = atomicAdd(&p.ws->ticket, 1u);
    }
    __syncthreads();

    uint64_t my_count = 0, my_agg = 0;
    bool have_prev = false;
    uint64_t prev_tile = 0;
    uint32_t prev_total = 0;

    // look-back (compacting) + encode of the previous tile's gathered survivors
    auto finish_prev = [&]() {
        uint64_t g;
        if (p.compact) {
            if (warp == 0) {
                const uint64_t x = lookback_prev(p.status, prev_tile, prev_total, &p.ws->err);
                if (lane == 0) bcast[0] = x;
            }
            __syncthreads();
            g = bcast[0];
        }
        else {
            g = prev_tile * TILE;
        }
        encode_tile<V>(p.out, cv, prev_total, g, prev_tile == p.num_tiles - 1);
        __syncthreads();
    };

    for (uint32_t it = 0;; it++) {
        const uint32_t s = it % kStages;
        const uint64_t tile = tickets[s];
        if (tile >= p.num_tiles) break;
        if (!mbar_wait_bounded(&mbar[s], (it / kStages) & 1)) record_error(&p.ws->err, AMX_ERR_TIMEOUT);

        const uint64_t e0 = tile * TILE;
        const uint64_t rem = p.n - e0;
        const uint32_t valid = rem < TILE ? (uint32_t)rem : TILE;
        const uint8_t* st = stage0 + s * p.stage_bytes;

        V v[R];
        uint64_t fl;
        Pol::decode(p, st, sbase + 3 * s, e0, v, fl);
        // element of flag bit i: thread-contiguous tid*R + i, warp-major warp*32R + 32i + lane
        if (p.has_mask_in) {
            const uint32_t* mw = reinterpret_cast<const uint32_t*>(st + p.m_off);
            if (WM) {
                uint64_t mfl = 0;
#pragma unroll
                for (int i = 0; i < R; i++) mfl |= (uint64_t)((mw[warp * R + i] >> lane) & 1u) << i;
                fl &= mfl;
            }
            else {
                fl &= bits_at<R>(mw, tid * R);
            }
        }
        if (WM) {
            const uint32_t base = warp * 32 * R + lane;
            if (base + 32 * (R - 1) >= valid) {
#pragma unroll
                for (int i = 0; i < R; i++)
                    if (base + 32 * i >= valid) fl &= ~(1ull << i);
            }
        }
        else {
            const uint32_t le0 = tid * R;
            if (le0 >= valid)
                fl = 0;
            else if (valid - le0 < (uint32_t)R)
                fl &= (1ull << (valid - le0)) - 1;
        }
        if (R < 64) fl &= (1ull << R) - 1;

        __syncthreads();  // every thread is done with stage s
        if (tid == 0) {
            tickets[s] = next_tk;
            if (next_tk < p.num_tiles)
                stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &mbar[s], next_tk, TILE);
            next_tk = atomicAdd(&p.ws->ticket, 1u);
        }

        if (p.has_agg) {
#pragma unroll
            for (int i = 0; i < R; i++)
                if ((fl >> i) & 1) my_agg = agg_combine(p.agg, my_agg, agg_encode(p.agg, (uint64_t)v[i]));
        }

        // ballots (warp-major) give mask words and in-warp ranks directly
        uint32_t bal[WM ? R : 1];
        uint32_t c = 0;
        if (WM) {
#pragma unroll
            for (int i = 0; i < R; i++) {
                bal[i] = __ballot_sync(0xffffffffu, (fl >> i) & 1);
                c += __popc(bal[i]);
            }
            if (p.mask_out) {
                uint32_t word = 0;
#pragma unroll
                for (int i = 0; i < R; i++)
                    if ((int)lane == i) word = bal[i];
                const uint32_t local = warp * 32 * R + 32 * lane;
                if ((int)lane < R && local < valid) p.mask_out[(e0 + local) / 32] = word;
            }
        }
        else {
            c = __popcll(fl);
            if (p.mask_out && fl) {
                const uint32_t le0 = tid * R;
                const uint32_t wi = le0 >> 5, sh = le0 & 31;
                atomicOr(&bitmap[wi], (uint32_t)(fl << sh));
                if (sh + R > 32) atomicOr(&bitmap[wi + 1], (uint32_t)(fl >> (32 - sh)));
                if (sh + R > 64) atomicOr(&bitmap[wi + 2], (uint32_t)(fl >> (64 - sh)));
            }
        }
        // warp-major: c is the warp's count (same in every lane); thread-contiguous: own count
        my_count += WM ? (lane == 0 ? c : 0) : c;

        if (p.has_out) {
            // block scan: survivors before this thread (or warp) inside the tile
            uint32_t pos, total;
            if (WM) {
                if (lane == 0) warp_tot[warp] = c;
                __syncthreads();
                uint32_t before = 0;
                total = 0;
#pragma unroll
                for (uint32_t w = 0; w < NW; w++) {
                    const uint32_t x = (uint32_t)warp_tot[w];
                    before += w < warp ? x : 0;
                    total += x;
                }
                pos = before;
            }
            else {
                const uint32_t incl = warp_incl_scan<uint32_t>(c);
                if (lane == 31) warp_tot[warp] = incl;
                __syncthreads();
                uint32_t before = 0;
                total = 0;
#pragma unroll
                for (uint32_t w = 0; w < NW; w++) {
                    const uint32_t x = (uint32_t)warp_tot[w];
                    before += w < warp ? x : 0;
                    total += x;
                }
                pos = before + incl - c;
            }
            if (p.compact && tid == 0) st_relaxed_u64(&p.status[tile], (tile == 0 ? kFlagInc : kFlagAgg) | total);

            if (have_prev) finish_prev();  // ends with __syncthreads: cv is free

            if (WM) {
                const uint32_t lt = (1u << lane) - 1;
#pragma unroll
                for (int i = 0; i < R; i++) {
                    if ((fl >> i) & 1) cv[sk<V>(pos + __popc(bal[i] & lt))] = v[i];
                    pos += __popc(bal[i]);
                }
            }
            else {
#pragma unroll
                for (int i = 0; i < R; i++)
                    if ((fl >> i) & 1) cv[sk<V>(pos++)] = v[i];
            }
            have_prev = true;
            prev_tile = tile;
            prev_total = total;
        }
        if (!WM && p.mask_out) {
            __syncthreads();
            const uint32_t words = (valid + 31) / 32;
            for (uint32_t i = tid; i < words; i += T) {
                p.mask_out[e0 / 32 + i] = bitmap[i];
                bitmap[i] = 0;
            }
        }
        __syncthreads();
    }
    if (have_prev) finish_prev();

    // CTA totals -> workspace; the last CTA to finish publishes the scalar results
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        my_count += __shfl_xor_sync(0xffffffffu, my_count, o);
        my_agg = agg_combine(p.agg, my_agg, __shfl_xor_sync(0xffffffffu, my_agg, o));
    }
    __syncthreads();
    if (lane == 0) {
        warp_tot[warp] = my_count;
        warp_agg[warp] = my_agg;
    }
    __syncthreads();
    if (tid == 0) {
        uint64_t cnt = 0, ag = 0;
        for (uint32_t w = 0; w < NW; w++) {
            cnt += warp_tot[w];
            ag = agg_combine(p.agg, ag, warp_agg[w]);
        }
        atomicAdd(&p.ws->count, (unsigned long long)cnt);
        if (p.has_agg) agg_atomic(p.agg, &p.ws->agg, ag);
        __threadfence();
        const uint32_t prev = atomicAdd(&p.ws->done, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            const uint64_t tot = atomicAdd(&p.ws->count, 0ull);
            const uint64_t a = atomicAdd(&p.ws->agg, 0ull);
            if (p.count_out) *p.count_out = tot;
            if (p.agg_out) *p.agg_out = agg_decode(p.agg, a);
        }
    }
}

// ---------------------------------------------------------------------------------------------
// decode policies
// ---------------------------------------------------------------------------------------------
template <int R_, typename V>
__device__ __forceinline__ void finish_values(const PipeParams& p, V (&v)[R_], uint64_t& fl)
{
#pragma unroll
    for (int i = 0; i < R_; i++) v[i] = (V)((uint64_t)v[i] & p.vmask);
    if (p.has_pred) {
        const PredN pn{p.pred_lo, p.pred_span, p.pred_neg, 0};
        fl = 0;
#pragma unroll
        for (int i = 0; i < R_; i++) fl |= (uint64_t)pred_eval(pn, v[i]) << i;
    }
    else {
        fl = ~0ull;
    }
}

// Warp-major reader with runtime format and width: lane `lane` of warp `warp` reads tile
// elements warp*32R + 32i + lane, i = 0..R-1 (consecutive lanes hit consecutive or shared
// words: no bank conflicts).
template <int R>
__device__ __forceinline__ void read_warp_major(const ColDev& c, const uint8_t* st, uint64_t sb, uint64_t e0,
                                                uint64_t (&out)[R])
{
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t base = warp * 32 * R + lane;
    const uint64_t m = c.mask;
    switch (c.format) {
        case AMX_PLAIN32: {
            const uint32_t* w = reinterpret_cast<const uint32_t*>(st) + (e0 - sb / 4) + base;
#pragma unroll
            for (int i = 0; i < R; i++) out[i] = w[32 * i] & m;
            break;
        }
        case AMX_PLAIN64: {
            const uint64_t* w = reinterpret_cast<const uint64_t*>(st) + (e0 - sb / 8) + base;
#pragma unroll
            for (int i = 0; i < R; i++) out[i] = w[32 * i] & m;
            break;
        }
        case AMX_SLAB: {
            const uint64_t s0 = e0 / c.eps;
            const uint32_t r0 = (uint32_t)(e0 - s0 * c.eps);
            const uint64_t* w = reinterpret_cast<const uint64_t*>(st) + (s0 - sb / 8);
            const uint32_t eps = c.eps, b = c.bits, mg = c.magic;
#pragma unroll
            for (int i = 0; i < R; i++) {
                const uint32_t x = r0 + base + 32 * i;
                const uint32_t s = eps == 1 ? x : __umulhi(x, mg);
                const uint32_t k = x - s * eps;
                out[i] = (w[s] >> (k * b)) & m;
            }
            break;
        }
        default: {  // nogaps
            const uint64_t b = c.bits;
            const uint64_t bit0 = e0 * b - sb * 8 + (uint64_t)base * b;
            const uint64_t* w = reinterpret_cast<const uint64_t*>(st);
#pragma unroll
            for (int i = 0; i < R; i++) {
                const uint64_t bp = bit0 + (uint64_t)(32 * i) * b;
                const uint32_t wi = (uint32_t)(bp >> 6), off = (uint32_t)(bp & 63);
                const uint64_t lo = w[wi], hi = w[wi + 1];
                out[i] = (off ? ((lo >> off) | (hi << (64 - off))) : lo) & m;
            }
            break;
        }
    }
}

// Any formats and widths: warp-major runtime readers, 64-bit values, 16 elements per thread.
struct GenericPol {
    using V = uint64_t;
    static constexpr int R = 16;
    static constexpr bool kWarpMajor = true;

    __device__ __forceinline__ static void decode(const PipeParams& p, const uint8_t* st, const uint64_t* sb,
                                                  uint64_t e0, V (&v)[R], uint64_t& fl)
    {
        read_warp_major<R>(p.a, st + p.a_off, sb[0], e0, v);
        if (p.has_b) {
            uint64_t r[R];
            read_warp_major<R>(p.b, st + p.b_off, sb[1], e0, r);
            switch (p.op) {
                case AMX_OP_ADD:
#pragma unroll
                    for (int i = 0; i < R; i++) v[i] += r[i];
                    break;
                case AMX_OP_SUB:
#pragma unroll
                    for (int i = 0; i < R; i++) v[i] -= r[i];
                    break;
                case AMX_OP_MUL:
#pragma unroll
                    for (int i = 0; i < R; i++) v[i] *= r[i];
                    break;
                default:
#pragma unroll
                    for (int i = 0; i < R; i++) v[i] = binop_eval(p.op, v[i], r[i]);
                    break;
            }
        }
        finish_values<R, V>(p, v, fl);
    }
};

}  // namespace amx
