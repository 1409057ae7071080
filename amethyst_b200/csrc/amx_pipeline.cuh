// amx_pipeline.cuh -- the tile pipeline kernel behind filter, compressstore, binary ops,
// conversion, aggregation and fused chains.
//
// Persistent CTAs (two per SM) of ten warps with three roles, handing work over through
// shared-memory mbarriers so that no compute warp ever waits on global-memory latency:
//   * the loader warp (one lane) takes tiles from an atomic ticket counter and stages each
//     tile's bytes of every input into a two-deep ring of shared-memory stages with 1-D bulk
//     copies (cp.async.bulk, completion on the stage's `full` mbarrier);
//   * eight compute warps decode R elements per thread straight from the staged packed words
//     (a policy: warp-major runtime-width readers or thread-contiguous compile-time-width
//     readers), apply the op and the predicate, build the bitmask / aggregate / count, scan the
//     tile's survivors, publish the count for the decoupled look-back, gather the survivors in
//     shared memory, and re-encode the PREVIOUS tile's survivors in the output format;
//   * the look-back warp turns each tile's published count into its output offset (the tile's
//     predecessors have had a whole tile of time to publish) and hands it to the compute warps.
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
        case AMX_SLAB:
            b0 = 8 * udiv64(e0, c.magic64, c.eps);
            b1 = 8 * udiv64(e1 + c.eps - 1, c.magic64, c.eps);
            break;
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

// Issue the staging of one tile into stage buffer `st` (one thread).
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

// Re-encode cnt gathered values cv[0..cnt) as output elements [g, g+cnt), using the compute
// threads (tid < nthreads).  Words wholly owned by this tile are stored; words shared with
// neighbouring tiles are merged with atomicAnd (clear own bits) + atomicOr (set own bits), which
// commute across tiles because owners are disjoint.  Dead slab bits belong to the owner of the
// slab's last field; bits past the column's last element are cleared by the last tile (`last`).
template <typename V>
__device__ __forceinline__ void encode_tile(const OutDev& o, const V* cv, uint32_t cnt, uint64_t g, bool last,
                                            uint32_t tid, uint32_t T)
{
    const uint64_t m = o.mask;
    switch (o.format) {
        case AMX_PLAIN32: {
            uint32_t* out = reinterpret_cast<uint32_t*>(o.data) + g;
            for (uint32_t r = tid; r < cnt; r += T) out[r] = (uint32_t)((uint64_t)cv[r] & m);
            return;
        }
        case AMX_PLAIN64: {
            uint64_t* out = reinterpret_cast<uint64_t*>(o.data) + g;
            for (uint32_t r = tid; r < cnt; r += T) out[r] = (uint64_t)cv[r] & m;
            return;
        }
        case AMX_SLAB: {
            unsigned long long* out = reinterpret_cast<unsigned long long*>(o.data);
            const uint32_t eps = o.eps, b = o.bits;
            const uint64_t live = eps * b >= 64 ? ~0ull : ((1ull << (eps * b)) - 1);
            if (cnt) {
                const uint64_t w0 = udiv64(g, o.eps_m64, eps), w1 = udiv64(g + cnt - 1, o.eps_m64, eps);
                for (uint64_t w = w0 + tid; w <= w1; w += T) {
                    const int64_t r0 = (int64_t)(w * eps) - (int64_t)g;
                    uint64_t acc = 0;
                    if (r0 >= 0 && r0 + eps <= cnt) {
                        const V* c = cv + r0;
                        for (uint32_t k = 0; k < eps; k++) acc |= ((uint64_t)c[k] & m) << (k * b);
                        out[w] = acc;
                    }
                    else {
                        uint64_t own = 0;
                        for (uint32_t k = 0; k < eps; k++) {
                            const int64_t r = r0 + k;
                            if (r >= 0 && r < (int64_t)cnt) {
                                acc |= ((uint64_t)cv[r] & m) << (k * b);
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
                const uint64_t tw = udiv64(total, o.eps_m64, eps);
                const uint32_t k = (uint32_t)(total - tw * eps);
                if (k) atomicAnd(&out[tw], (1ull << (k * b)) - 1);
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
                    uint64_t p0 = udiv64(lo, o.bits_m64, b);
                    if (p0 < g) p0 = g;
                    uint64_t p1 = udiv64(hi - 1, o.bits_m64, b);
                    if (p1 > g + cnt - 1) p1 = g + cnt - 1;
                    uint64_t acc = 0;
                    for (uint64_t q = p0; q <= p1; q++) {
                        const uint64_t v = (uint64_t)cv[q - g] & m;
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
// lanes of one warp call it.  Each round reads 256 predecessor status words at once (8 per
// lane, independent loads), so one round usually reaches a published prefix.  Every wait is
// bounded: on timeout the error word is set and the missing value is taken as 0.
constexpr int kLookPerLane = 8;

__device__ __forceinline__ uint64_t lookback_prev(uint64_t* status, uint64_t tile, uint64_t agg, uint32_t* err)
{
    const uint32_t lane = threadIdx.x & 31;
    if (tile == 0) return 0;  // tile 0 published its inclusive prefix directly
    uint64_t excl = 0;
    int64_t j = (int64_t)tile - 1;
    bool done = false;
    while (!done) {
        uint64_t st[kLookPerLane];
#pragma unroll
        for (int m = 0; m < kLookPerLane; m++) {  // all loads of the round in flight together
            const int64_t idx = j - (int64_t)(lane + 32 * m);
            st[m] = idx >= 0 ? ld_relaxed_u64(&status[idx]) : kFlagInc;
        }
        // consume the window nearest-first, 32 predecessors at a time, and stop at the first
        // group holding an inclusive prefix: never wait on tiles beyond it
#pragma unroll
        for (int m = 0; m < kLookPerLane; m++) {
            if (done) break;
            const int64_t idx = j - (int64_t)(lane + 32 * m);
            uint32_t spins = 0;
            while ((st[m] >> 62) == 0) {  // an earlier tile still decoding
                if (++spins > kWaitSpins) {
                    record_error(err, AMX_ERR_TIMEOUT);
                    st[m] = kFlagInc;
                    break;
                }
                if (spins > 8) __nanosleep(20);
                st[m] = ld_relaxed_u64(&status[idx]);
            }
            const uint32_t inc = __ballot_sync(0xffffffffu, (st[m] >> 62) == 2);
            const int first = __ffs(inc) - 1;
            uint64_t v = (first < 0 || (int)lane <= first) ? (st[m] & kValMask) : 0;
#pragma unroll
            for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            excl += v;
            done = first >= 0;
        }
        j -= 32 * kLookPerLane;
    }
    if (lane == 0) st_relaxed_u64(&status[tile], kFlagInc | (excl + agg));
    return excl;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void compute_bar()
{
    asm volatile("bar.sync 1, %0;" ::"n"(kPipeCompute) : "memory");
}

__device__ __forceinline__ void wait_or_flag(uint64_t* bar, uint32_t parity, uint32_t* err)
{
    if (!mbar_wait_bounded(bar, parity)) record_error(err, AMX_ERR_TIMEOUT);
}

// Shared-memory map (dynamic shared memory), for up to kMaxStages stages:
//   [0,64) full[8]  [64,128) empty[8]  [128,144) agg[2]  [144,160) gready[2]   (mbarriers)
//   [160,224)  tickets[8]              [224,416) stage base offsets [8][3]
//   [416,480)  warp totals [2][8]      [480,544) warp counts      [544,592) per-slot tile / total / offset
//   [608,672)  warp aggregates         [1024,3072) tile bitmap (thread-contiguous policies)
//   [kCvOff, smem_fixed)  gathered values;  [smem_fixed, ...) p.stages stage buffers
constexpr uint32_t kBitmapOff = 1024;
constexpr uint32_t kCvOff = 3072;
constexpr uint64_t kNoTile = ~0ull;

template <class Pol>
__global__ void __launch_bounds__(kPipeThreads, Pol::kMinBlocks) pipe_kernel(const __grid_constant__ PipeParams p)
{
    using V = typename Pol::V;
    constexpr int R = Pol::R;
    constexpr bool WM = Pol::kWarpMajor;
    constexpr uint32_t T = kPipeCompute;
    constexpr uint32_t NW = T / 32;
    constexpr uint32_t TILE = T * R;
    static_assert(TILE / 32 * 4 <= kCvOff - kBitmapOff, "bitmap region");
    static_assert(!WM || R <= 32, "warp-major runs keep one ballot per lane");

    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kMaxStages;
    uint64_t* aggb = full + 2 * kMaxStages;
    uint64_t* gready = aggb + 2;
    volatile uint64_t* tickets = reinterpret_cast<volatile uint64_t*>(smem + 160);
    uint64_t* sbase = reinterpret_cast<uint64_t*>(smem + 224);
    volatile uint32_t* warp_tot = reinterpret_cast<volatile uint32_t*>(smem + 416);
    uint64_t* warp_cnt = reinterpret_cast<uint64_t*>(smem + 480);
    volatile uint64_t* slot_tile = reinterpret_cast<volatile uint64_t*>(smem + 544);
    volatile uint32_t* slot_total = reinterpret_cast<volatile uint32_t*>(smem + 560);
    volatile uint64_t* slot_g = reinterpret_cast<volatile uint64_t*>(smem + 576);
    uint64_t* warp_agg = reinterpret_cast<uint64_t*>(smem + 608);
    const uint32_t S = p.stages;
    uint32_t* bitmap = reinterpret_cast<uint32_t*>(smem + kBitmapOff);
    V* cv = reinterpret_cast<V*>(smem + kCvOff);
    uint8_t* stage0 = smem + p.smem_fixed;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        for (uint32_t s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NW);
        }
        for (int q = 0; q < 2; q++) {
            mbar_init(&aggb[q], 1);
            mbar_init(&gready[q], 1);
        }
        fence_mbar_init();
    }
    if (!WM)
        for (uint32_t i = tid; i < TILE / 32; i += blockDim.x) bitmap[i] = 0;
    __syncthreads();  // the last CTA-wide barrier: roles split below

    // ---------------------------------------------------------------- loader warp
    if (warp == NW) {
        if (lane == 0) {
            // iteration j of the compute warps consumes stage j % S.  `stop_at` is the first
            // iteration whose stage holds an invalid ticket: the compute warps leave the loop
            // there, so they release no stage from that iteration on.
            uint64_t stop_at = kNoTile;
            for (uint32_t s = 0; s < S; s++) {
                const uint64_t tk = stop_at == kNoTile ? atomicAdd(&p.ws->ticket, 1u) : p.num_tiles;
                tickets[s] = tk;
                if (tk < p.num_tiles)
                    stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &full[s], tk, TILE);
                else {
                    mbar_arrive(&full[s]);
                    if (stop_at == kNoTile) stop_at = s;
                }
            }
            // the next ticket is taken one refill ahead, so its atomic latency overlaps the wait
            uint64_t next = stop_at == kNoTile ? atomicAdd(&p.ws->ticket, 1u) : p.num_tiles;
            uint32_t s = 0, phase = 0;
            for (uint64_t j = 0; j < stop_at; j++) {
                wait_or_flag(&empty[s], phase, &p.ws->err);  // iteration j released stage s
                const uint64_t tk = stop_at == kNoTile ? next : p.num_tiles;
                if (tk < p.num_tiles) next = atomicAdd(&p.ws->ticket, 1u);
                tickets[s] = tk;  // for iteration j + S
                if (tk < p.num_tiles)
                    stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &full[s], tk, TILE);
                else {
                    mbar_arrive(&full[s]);
                    if (stop_at == kNoTile) stop_at = j + S;
                }
                if (++s == S) {
                    s = 0;
                    phase ^= 1;
                }
            }
        }
        return;
    }
    // ---------------------------------------------------------------- look-back warp
    if (warp == NW + 1) {
        if (p.has_out && p.compact) {
            for (uint32_t j = 0;; j++) {
                const uint32_t q = j & 1;
                wait_or_flag(&aggb[q], (j >> 1) & 1, &p.ws->err);
                const uint64_t tile = slot_tile[q];
                if (tile == kNoTile) break;
                const uint64_t g = lookback_prev(p.status, tile, slot_total[q], &p.ws->err);
                if (lane == 0) {
                    slot_g[q] = g;
                    mbar_arrive(&gready[q]);
                }
                __syncwarp();
            }
        }
        return;
    }

    // ---------------------------------------------------------------- compute warps
    uint64_t my_count = 0, my_agg = 0;
    bool have_prev = false;
    uint64_t prev_tile = 0;
    uint32_t prev_total = 0, prev_j = 0;

    auto finish_prev = [&]() {
        uint64_t g;
        if (p.compact) {
            wait_or_flag(&gready[prev_j & 1], (prev_j >> 1) & 1, &p.ws->err);
            g = slot_g[prev_j & 1];
        }
        else {
            g = prev_tile * TILE;
        }
        encode_tile<V>(p.out, cv, prev_total, g, prev_tile == p.num_tiles - 1, tid, T);
        compute_bar();  // cv is free
    };

    uint32_t j = 0, s = 0, sphase = 0;
    for (;; j++) {
        if (j) {
            if (++s == S) {
                s = 0;
                sphase ^= 1;
            }
        }
        wait_or_flag(&full[s], sphase, &p.ws->err);
        const uint64_t tile = tickets[s];
        if (tile >= p.num_tiles) break;

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
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s

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

        if (p.has_agg) {
            uint64_t a = 0;
            switch (p.agg) {
                case AMX_AGG_SUM:
#pragma unroll
                    for (int i = 0; i < R; i++) a += ((fl >> i) & 1) ? (uint64_t)v[i] : 0;
                    break;
                case AMX_AGG_MIN:
                case AMX_AGG_AND:
#pragma unroll
                    for (int i = 0; i < R; i++) {
                        const uint64_t e = ((fl >> i) & 1) ? ~(uint64_t)v[i] : 0;
                        a = p.agg == AMX_AGG_MIN ? (a > e ? a : e) : (a | e);
                    }
                    break;
                case AMX_AGG_MAX:
#pragma unroll
                    for (int i = 0; i < R; i++) {
                        const uint64_t e = ((fl >> i) & 1) ? (uint64_t)v[i] : 0;
                        a = a > e ? a : e;
                    }
                    break;
                case AMX_AGG_OR:
#pragma unroll
                    for (int i = 0; i < R; i++) a |= ((fl >> i) & 1) ? (uint64_t)v[i] : 0;
                    break;
                default:
#pragma unroll
                    for (int i = 0; i < R; i++) a ^= ((fl >> i) & 1) ? (uint64_t)v[i] : 0;
                    break;
            }
            my_agg = agg_combine(p.agg, my_agg, a);
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
        my_count += WM ? (lane == 0 ? c : 0) : c;

        if (p.has_out) {
            // block scan: survivors before this thread (or warp) inside the tile
            volatile uint32_t* wt = warp_tot + 8 * (j & 1);
            uint32_t pos, total = 0, before = 0;
            if (WM) {
                if (lane == 0) wt[warp] = c;
                compute_bar();
#pragma unroll
                for (uint32_t w = 0; w < NW; w++) {
                    const uint32_t x = wt[w];
                    before += w < warp ? x : 0;
                    total += x;
                }
                pos = before;
            }
            else {
                const uint32_t incl = warp_incl_scan<uint32_t>(c);
                if (lane == 31) wt[warp] = incl;
                compute_bar();
#pragma unroll
                for (uint32_t w = 0; w < NW; w++) {
                    const uint32_t x = wt[w];
                    before += w < warp ? x : 0;
                    total += x;
                }
                pos = before + incl - c;
            }
            if (p.compact && tid == 0) {
                st_relaxed_u64(&p.status[tile], (tile == 0 ? kFlagInc : kFlagAgg) | total);
                slot_tile[j & 1] = tile;
                slot_total[j & 1] = total;
                mbar_arrive(&aggb[j & 1]);  // hand the tile to the look-back warp
            }

            if (have_prev) finish_prev();  // ends with a compute barrier: cv is free

            if (WM) {
                const uint32_t lt = (1u << lane) - 1;
#pragma unroll
                for (int i = 0; i < R; i++) {
                    if ((fl >> i) & 1) cv[pos + __popc(bal[i] & lt)] = v[i];
                    pos += __popc(bal[i]);
                }
            }
            else {
                V* dst = cv + pos;
#pragma unroll
                for (int i = 0; i < R; i++)
                    if ((fl >> i) & 1) *dst++ = v[i];
            }
            have_prev = true;
            prev_tile = tile;
            prev_total = total;
            prev_j = j;
        }
        if (!WM && p.mask_out) {
            compute_bar();
            const uint32_t words = (valid + 31) / 32;
            for (uint32_t i = tid; i < words; i += T) {
                p.mask_out[e0 / 32 + i] = bitmap[i];
                bitmap[i] = 0;
            }
            compute_bar();
        }
    }
    if (p.has_out && p.compact && tid == 0) {  // release the look-back warp
        slot_tile[j & 1] = kNoTile;
        mbar_arrive(&aggb[j & 1]);
    }
    if (have_prev) finish_prev();

    // CTA totals -> workspace; the last CTA to finish publishes the scalar results
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        my_count += __shfl_xor_sync(0xffffffffu, my_count, o);
        my_agg = agg_combine(p.agg, my_agg, __shfl_xor_sync(0xffffffffu, my_agg, o));
    }
    compute_bar();
    if (lane == 0) {
        warp_cnt[warp] = my_count;
        warp_agg[warp] = my_agg;
    }
    compute_bar();
    if (tid == 0) {
        uint64_t cnt = 0, ag = 0;
        for (uint32_t w = 0; w < NW; w++) {
            cnt += warp_cnt[w];
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
    if (p.need_vmask) {
#pragma unroll
        for (int i = 0; i < R_; i++) v[i] = (V)((uint64_t)v[i] & p.vmask);
    }
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
            const uint64_t s0 = udiv64(e0, c.magic64, c.eps);
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
    static constexpr int kMinBlocks = 1;

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
