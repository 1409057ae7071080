// amx_pipeline.cuh -- the tile pipeline kernel behind filter, compressstore, binary ops,
// conversion, aggregation and fused chains.
//
// Persistent CTAs (one per SM) with four warp roles, handing work over through shared-memory
// mbarriers so that no compute warp waits on global-memory latency:
//   * the loader warp (one lane) takes tiles from an atomic ticket counter and stages each
//     tile's bytes of every input into a ring of 2..8 shared-memory stages with 1-D bulk
//     copies (cp.async.bulk, completion on the stage's `full` mbarrier);
//   * 8 to 24 compute warps (Pol::kCompute) decode R elements per thread straight from the
//     staged packed words (a policy: field-parallel slab words, thread-contiguous
//     compile-time-width readers, or warp-major runtime-width readers), apply the op and the
//     predicate, build the bitmask / aggregate / count, scan the tile's survivors, publish the
//     count for the look-back, and gather the survivors into one of up to four shared-memory
//     slots.  The request-specific policy variants (Pol::kPlain, kFilter, kAggOnly) compile only
//     their request's path, which keeps the hot loop small in the instruction cache the compute
//     warps share with the other roles, and frees the registers for more compute warps;
//   * the look-back warp turns each tile's published count into its output offset: the CTA's
//     tiles arrive in ticket order, so the offset is the end of the CTA's previous tile plus the
//     counts of the tiles other CTAs took in between;
//   * four encoder warps re-encode each slot's survivors in the output format at that offset and
//     hand the slot back to the compute warps.
// Replaces the reference's separate filter / popcount / CUB scan / write kernels
// (src/kernels/filter_slabs.cuh:4-57, src/kernels/compressstore_slabs.cuh:4-206,
// src/benchs/bench_compressstore_slabs.cu:38-56) with one pass and no mask round trip.
#pragma once

#include "amx_device.cuh"
#include "amx_swar.cuh"

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

// Byte range of one column for a tile: tile * stride when every tile of the column covers
// exactly `stride` bytes (precomputed on the host; 0 when tiles do not fall on word
// boundaries), else col_range.
__device__ __forceinline__ void tile_bytes(const ColDev& c, uint64_t stride, uint64_t tile, uint64_t e0, uint64_t e1,
                                           uint64_t& b0, uint64_t& b1)
{
    if (stride) {
        b0 = tile * stride;
        b1 = b0 + stride;
        if (b1 > c.bytes) b1 = c.bytes;
        if (b0 > b1) b0 = b1;
    }
    else {
        col_range(c, e0, e1, b0, b1);
    }
}

// Issue the staging of one tile into stage buffer `st` (one thread): plain scalar code, no
// arrays, so the loader spends as little time as possible per tile.
__device__ __forceinline__ void stage_issue(const PipeParams& p, uint8_t* st, uint64_t* sbase, uint64_t* bar,
                                            uint64_t tile, uint32_t tile_elems, uint64_t n)
{
    const uint64_t e0 = tile * tile_elems;
    uint64_t e1 = e0 + tile_elems;
    if (e1 > n) e1 = n;
    uint64_t a0, a1, b0 = 0, b1 = 0, m0 = 0, m1 = 0;
    tile_bytes(p.a, p.a_stride, tile, e0, e1, a0, a1);
    if (p.has_b) tile_bytes(p.b, p.b_stride, tile, e0, e1, b0, b1);
    if (p.has_mask_in) tile_bytes(p.m, p.m_stride, tile, e0, e1, m0, m1);
    // body of each range through the bulk-copy unit (16-byte aligned), ragged tail by hand
    const uint64_t as = a0 & ~15ull, bs = b0 & ~15ull, ms = m0 & ~15ull;
    uint64_t ae = (a1 + 15) & ~15ull, be = (b1 + 15) & ~15ull, me = (m1 + 15) & ~15ull;
    if (ae > (p.a.bytes & ~15ull)) ae = p.a.bytes & ~15ull;
    if (be > (p.b.bytes & ~15ull)) be = p.b.bytes & ~15ull;
    if (me > (p.m.bytes & ~15ull)) me = p.m.bytes & ~15ull;
    const uint32_t at = ae > as ? (uint32_t)(ae - as) : 0;
    const uint32_t bt = (p.has_b && be > bs) ? (uint32_t)(be - bs) : 0;
    const uint32_t mt = (p.has_mask_in && me > ms) ? (uint32_t)(me - ms) : 0;
    sbase[0] = as;
    sbase[1] = bs;
    sbase[2] = ms;
    if (a1 > (ae > as ? ae : as)) {  // ragged tail at the very end of the column (< 16 bytes)
        const uint8_t* src = reinterpret_cast<const uint8_t*>(p.a.data);
        for (uint64_t x = ae > as ? ae : as; x < a1; x++) st[p.a_off + (x - as)] = src[x];
    }
    if (p.has_b && b1 > (be > bs ? be : bs)) {
        const uint8_t* src = reinterpret_cast<const uint8_t*>(p.b.data);
        for (uint64_t x = be > bs ? be : bs; x < b1; x++) st[p.b_off + (x - bs)] = src[x];
    }
    if (p.has_mask_in && m1 > (me > ms ? me : ms)) {
        const uint8_t* src = reinterpret_cast<const uint8_t*>(p.m.data);
        for (uint64_t x = me > ms ? me : ms; x < m1; x++) st[p.m_off + (x - ms)] = src[x];
    }
    mbar_arrive_expect_tx(bar, at + bt + mt);
    if (at) bulk_g2s(st + p.a_off, reinterpret_cast<const uint8_t*>(p.a.data) + as, at, bar);
    if (bt) bulk_g2s(st + p.b_off, reinterpret_cast<const uint8_t*>(p.b.data) + bs, bt, bar);
    if (mt) bulk_g2s(st + p.m_off, reinterpret_cast<const uint8_t*>(p.m.data) + ms, mt, bar);
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

// bits_at for a stage released right after the read (volatile reads)
template <int R>
__device__ __forceinline__ uint64_t bits_at_v(const uint32_t* w, uint32_t bit)
{
    const uint32_t wi = bit >> 5, sh = bit & 31;
    uint64_t x = ((uint64_t)lds_u32_v(w + wi) | ((uint64_t)lds_u32_v(w + wi + 1) << 32)) >> sh;
    if (R + sh > 64) x |= (uint64_t)lds_u32_v(w + wi + 2) << (64 - sh);
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

// encode_tile for a slab output whose width OB is known at compile time: 32-bit tile-local
// indices, unrolled field loads, and a division by a constant.  Same ownership rules.
template <int OB, typename V>
__device__ __forceinline__ void encode_slab_ct(const OutDev& o, const V* cv, uint32_t cnt, uint64_t g, bool last,
                                               uint32_t tid, uint32_t T)
{
    constexpr int EPS = 64 / OB;
    constexpr uint64_t M = (1ull << OB) - 1;
    constexpr uint64_t LIVE = EPS * OB >= 64 ? ~0ull : ((1ull << (EPS * OB)) - 1);
    unsigned long long* out = reinterpret_cast<unsigned long long*>(o.data);
    if (cnt) {
        const uint64_t w0 = g / EPS;
        const uint32_t nw = (uint32_t)((g + cnt - 1) / EPS - w0 + 1);
        const int32_t r00 = (int32_t)(int64_t)(w0 * EPS - g);  // in (-EPS, 0]
        for (uint32_t i = tid; i < nw; i += T) {
            const int32_t r0 = r00 + (int32_t)(i * EPS);
            uint64_t acc = 0;
            if (r0 >= 0 && r0 + EPS <= (int32_t)cnt) {
                const V* c = cv + r0;
#pragma unroll
                for (int k = 0; k < EPS; k++) acc |= ((uint64_t)c[k] & M) << (k * OB);
                out[w0 + i] = acc;
            }
            else {
                uint64_t own = 0;
#pragma unroll
                for (int k = 0; k < EPS; k++) {
                    const int32_t r = r0 + k;
                    if (r >= 0 && r < (int32_t)cnt) {
                        acc |= ((uint64_t)cv[r] & M) << (k * OB);
                        own |= M << (k * OB);
                    }
                }
                if (r0 + EPS - 1 < (int32_t)cnt && r0 + EPS - 1 >= 0) own |= ~LIVE;
                atomicAnd(&out[w0 + i], ~own);
                atomicOr(&out[w0 + i], acc);
            }
        }
    }
    if (last && tid == 0) {
        const uint64_t total = g + cnt;
        const uint64_t tw = total / EPS;
        const uint32_t k = (uint32_t)(total - tw * EPS);
        if (k) atomicAnd(&out[tw], (1ull << (k * OB)) - 1);
    }
}

// Sum of the published survivor counts of tiles [lo, hi).  All 32 lanes of one warp call it;
// each round has 256 status loads in flight (8 per lane).  Waits for counts not yet published
// are bounded: on timeout the error word is set and the count is taken as 0.
constexpr int kLookPerLane = 8;

__device__ __forceinline__ uint64_t sum_counts(const uint64_t* status, uint64_t lo, uint64_t hi, uint32_t* err,
                                               uint32_t limit)
{
    const uint32_t lane = threadIdx.x & 31;
    uint64_t acc = 0;
    for (uint64_t base = lo; base < hi; base += 32 * kLookPerLane) {
        uint64_t st[kLookPerLane];
#pragma unroll
        for (int m = 0; m < kLookPerLane; m++) {
            const uint64_t idx = base + lane + 32 * m;
            st[m] = idx < hi ? ld_relaxed_u64(&status[idx]) : kFlagAgg;
        }
#pragma unroll
        for (int m = 0; m < kLookPerLane; m++) {
            const uint64_t idx = base + lane + 32 * m;
            uint32_t spins = 0;
            while ((st[m] >> 62) == 0) {  // that tile is still being decoded
                if (++spins > limit) {
                    record_error(err, AMX_ERR_TIMEOUT);
                    st[m] = kFlagAgg;
                    break;
                }
                if (spins > 8) __nanosleep(20);
                st[m] = ld_relaxed_u64(&status[idx]);
            }
            acc += st[m] & kValMask;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Exclusive prefix of this warp and the tile total from the NW warp totals in wt: one shared load
// per lane and a 4-step shuffle scan instead of every lane summing all NW entries.
template <uint32_t NW>
__device__ __forceinline__ void tile_prefix(volatile const uint32_t* wt, uint32_t warp, uint32_t lane,
                                            uint32_t& before, uint32_t& total)
{
    static_assert(NW <= 32, "one warp total per lane");
    uint32_t pre = lane < NW ? wt[lane] : 0;
#pragma unroll
    for (uint32_t o = 1; o < NW; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, pre, o);
        if (lane >= o) pre += y;
    }
    total = __shfl_sync(0xffffffffu, pre, NW - 1);
    const uint32_t b = __shfl_sync(0xffffffffu, pre, warp ? warp - 1 : 0);
    before = warp ? b : 0;
}

// named barrier 1 over the compute warps only (the loader and look-back warps never join it)
template <uint32_t N>
__device__ __forceinline__ void compute_bar_n()
{
    asm volatile("bar.sync 1, %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ void wait_or_flag(uint64_t* bar, uint32_t parity, uint32_t* err)
{
    if (!mbar_wait_bounded(bar, parity)) record_error(err, AMX_ERR_TIMEOUT);
}

// Shared-memory map (dynamic shared memory), for up to kMaxStages stages and kMaxSlots slots:
//   [0,64) full[8]  [64,128) empty[8]  [128,160) agg[4]  [160,192) gready[4]  [192,224) scat[4]
//   [224,256) cvfree[4]                                                        (mbarriers)
//   [256,320)  tickets[8]              [320,512) stage base offsets [8][3]
//   [512,768)  warp totals [2][32]     [768,1024) warp counts [32]  [1024,1280) warp aggregates [32]
//   [1280,1360) per-slot tile / total / offset  [1360,1376) run length, tiles                    [1536,5632) tile bitmap (thread-contiguous policies)
//   [kCvOff, smem_fixed)  gathered-value slots;  [smem_fixed, ...) p.stages stage buffers
constexpr uint32_t kBitmapOff = 1536;
constexpr uint32_t kCvOff = 5632;
constexpr uint64_t kNoTile = ~0ull;
constexpr uint32_t kEncoderWarps = 4;
constexpr int kSparseMax = 3;  // survivors per thread up to which a warp gathers sparsely
constexpr uint32_t kCtlThreads = 32 * (2 + kEncoderWarps);  // loader + look-back + encoders

// gathered values are kept as 16-bit words when the value width allows it
template <typename V>
__device__ __forceinline__ void cv_put(uint8_t* cv, bool cv16, uint32_t i, V x)
{
    if (cv16)
        reinterpret_cast<uint16_t*>(cv)[i] = (uint16_t)x;
    else
        reinterpret_cast<V*>(cv)[i] = x;
}

template <typename V>
__device__ __forceinline__ void encode_any(const OutDev& o, const uint8_t* cv, bool cv16, uint32_t cnt, uint64_t g,
                                           bool last, uint32_t tid, uint32_t T)
{
    if (cv16)
        encode_tile<uint16_t>(o, reinterpret_cast<const uint16_t*>(cv), cnt, g, last, tid, T);
    else
        encode_tile<V>(o, reinterpret_cast<const V*>(cv), cnt, g, last, tid, T);
}

template <class Pol>
__global__ void __launch_bounds__(Pol::kCompute + kCtlThreads, Pol::kMinBlocks)
    pipe_kernel(const __grid_constant__ PipeParams p)
{
    using V = typename Pol::V;
    constexpr int R = Pol::R;
    constexpr bool WM = Pol::kWarpMajor;
    constexpr uint32_t T = Pol::kCompute;
    constexpr uint32_t NW = T / 32;
    constexpr uint32_t TILE = T * R;
    static_assert(Pol::kWide || TILE / 32 * 4 <= kCvOff - kBitmapOff, "bitmap region");  // wide: no bitmap
    static_assert(NW <= 32, "warp arrays hold 32 compute warps");
    static_assert(!WM || R <= 32, "warp-major runs keep one ballot per lane");
    auto compute_bar = []() { compute_bar_n<T>(); };

    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* empty = full + kMaxStages;
    uint64_t* aggb = reinterpret_cast<uint64_t*>(smem + 128);
    uint64_t* gready = reinterpret_cast<uint64_t*>(smem + 160);
    uint64_t* scat = reinterpret_cast<uint64_t*>(smem + 192);
    uint64_t* cvfree = reinterpret_cast<uint64_t*>(smem + 224);
    volatile uint64_t* tickets = reinterpret_cast<volatile uint64_t*>(smem + 256);
    uint64_t* sbase = reinterpret_cast<uint64_t*>(smem + 320);
    volatile uint32_t* warp_tot = reinterpret_cast<volatile uint32_t*>(smem + 512);
    uint64_t* warp_cnt = reinterpret_cast<uint64_t*>(smem + 768);
    uint64_t* warp_agg = reinterpret_cast<uint64_t*>(smem + 1024);
    volatile uint64_t* slot_tile = reinterpret_cast<volatile uint64_t*>(smem + 1280);
    volatile uint32_t* slot_total = reinterpret_cast<volatile uint32_t*>(smem + 1312);
    volatile uint64_t* slot_g = reinterpret_cast<volatile uint64_t*>(smem + 1328);
    uint64_t* run_len = reinterpret_cast<uint64_t*>(smem + 1360);
    uint32_t* bitmap = reinterpret_cast<uint32_t*>(smem + kBitmapOff);
    uint8_t* cv = smem + kCvOff;
    uint8_t* stage0 = smem + p.smem_fixed;
    const uint32_t S = p.stages;
    const uint32_t NB = p.slots;
    const bool cv16 = p.cv16 != 0;
    const bool compact = p.has_out && p.compact;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        for (uint32_t s = 0; s < S; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NW);
        }
        for (uint32_t q = 0; q < NB; q++) {
            mbar_init(&aggb[q], 1);
            mbar_init(&gready[q], 1);
            mbar_init(&scat[q], NW);
            mbar_init(&cvfree[q], kEncoderWarps);
        }
        fence_mbar_init();
        // elements of this run: the capacity, or the device-resident length a previous kernel
        // on the stream wrote (a count that never reached the host)
        uint64_t len = p.n;
        if (p.n_dev) {
            const uint64_t d = *p.n_dev;
            if (d < len) len = d;
        }
        run_len[0] = len;
        run_len[1] = (len + TILE - 1) / TILE;
    }
    if (!WM && !Pol::kWide)
        for (uint32_t i = tid; i < TILE / 32; i += blockDim.x) bitmap[i] = 0;
    __syncthreads();  // the last CTA-wide barrier: roles split below
    const uint64_t n = run_len[0], num_tiles = run_len[1];

    // ---------------------------------------------------------------- loader warp
    if (warp == NW) {
        if (lane == 0) {
            // iteration j of the compute warps consumes stage j % S.  `stop_at` is the first
            // iteration whose stage holds an invalid ticket: the compute warps leave the loop
            // there, so they release no stage from that iteration on.
            uint64_t stop_at = kNoTile;
            for (uint32_t s = 0; s < S; s++) {
                const uint64_t tk = stop_at == kNoTile ? atomicAdd(&p.ws->ticket, 1u) : num_tiles;
                tickets[s] = tk;
                if (tk < num_tiles)
                    stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &full[s], tk, TILE, n);
                else {
                    mbar_arrive(&full[s]);
                    if (stop_at == kNoTile) stop_at = s;
                }
            }
            // the next ticket is taken one refill ahead, so its atomic latency overlaps the wait
            uint64_t next = stop_at == kNoTile ? atomicAdd(&p.ws->ticket, 1u) : num_tiles;
            uint32_t s = 0, phase = 0;
            for (uint64_t j = 0; j < stop_at; j++) {
                wait_or_flag(&empty[s], phase, &p.ws->err);  // iteration j released stage s
                const uint64_t tk = stop_at == kNoTile ? next : num_tiles;
                if (tk < num_tiles) next = atomicAdd(&p.ws->ticket, 1u);
                tickets[s] = tk;  // for iteration j + S
                if (tk < num_tiles)
                    stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &full[s], tk, TILE, n);
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
    // The CTA's tiles arrive in increasing ticket order, so the output offset of a tile is the
    // end of this CTA's previous tile plus the survivor counts of the tiles in between (other
    // CTAs publish each count right after the tile's scan).  No tile waits on another tile's
    // look-back: there is no chain of inclusive prefixes across CTAs.
    if (warp == NW + 1) {
        if (!Pol::kFilter && !Pol::kAggOnly && compact) {
            uint64_t prev_tile = 0, prev_end = 0;
            bool first = true;
            for (uint32_t j = 0, q = 0, ph = 0;; j++) {
                wait_or_flag(&aggb[q], ph, &p.ws->err);
                const uint64_t tile = slot_tile[q];
                if (tile != kNoTile) {
                    const uint64_t lo = first ? 0 : prev_tile + 1;
                    const uint64_t g = (first ? 0 : prev_end) + sum_counts(p.status, lo, tile, &p.ws->err, p.wait_polls);
                    first = false;
                    prev_tile = tile;
                    prev_end = g + slot_total[q];
                    if (lane == 0) slot_g[q] = g;
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&gready[q]);  // hands the slot to the encoder warps
                if (tile == kNoTile) break;
                if (++q == NB) {
                    q = 0;
                    ph ^= 1;
                }
            }
        }
        return;
    }
    // ---------------------------------------------------------------- encoder warps
    // Re-encode each slot's gathered survivors at the offset the look-back warp found, then
    // give the slot back to the compute warps.
    if (warp >= NW + 2) {
        if (!Pol::kFilter && !Pol::kAggOnly && compact) {
            const uint32_t etid = tid - (NW + 2) * 32;
            for (uint32_t j = 0, q = 0, ph = 0;; j++) {
                wait_or_flag(&gready[q], ph, &p.ws->err);
                const uint64_t tile = slot_tile[q];
                if (tile == kNoTile) break;
                wait_or_flag(&scat[q], ph, &p.ws->err);  // every compute warp has gathered
                const uint8_t* sv = cv + (size_t)q * p.slot_bytes;
                bool done = false;
                if constexpr (Pol::kSwar) {
                    // the usual compressstore: slabs of the input width in, slabs of it out
                    if (Pol::kPlain || (p.out.format == AMX_SLAB && p.out.bits == (uint32_t)Pol::kBits)) {
                        if (Pol::kPlain || cv16)
                            encode_slab_ct<Pol::kBits, uint16_t>(p.out, reinterpret_cast<const uint16_t*>(sv),
                                                                slot_total[q], slot_g[q], tile == num_tiles - 1,
                                                                etid, 32 * kEncoderWarps);
                        else if constexpr (!Pol::kPlain)
                            encode_slab_ct<Pol::kBits, uint32_t>(p.out, reinterpret_cast<const uint32_t*>(sv),
                                                                slot_total[q], slot_g[q], tile == num_tiles - 1,
                                                                etid, 32 * kEncoderWarps);
                        done = true;
                    }
                }
                if constexpr (!Pol::kPlain) {
                    if (!done)
                        encode_any<V>(p.out, sv, cv16, slot_total[q], slot_g[q], tile == num_tiles - 1, etid,
                                      32 * kEncoderWarps);
                }
                else if constexpr (!Pol::kSwar) {
                    const uint16_t* sv16 = reinterpret_cast<const uint16_t*>(sv);
                    const bool last = tile == num_tiles - 1;
                    if constexpr (Pol::kOutBits >= 1 && Pol::kOutBits <= 16) {
                        if (p.out.format == AMX_SLAB && p.out.bits == (uint32_t)Pol::kOutBits)
                            encode_slab_ct<Pol::kOutBits, uint16_t>(p.out, sv16, slot_total[q], slot_g[q], last, etid,
                                                                   32 * kEncoderWarps);
                        else
                            encode_tile<uint16_t>(p.out, sv16, slot_total[q], slot_g[q], last, etid, 32 * kEncoderWarps);
                    }
                    else {
                        encode_tile<uint16_t>(p.out, sv16, slot_total[q], slot_g[q], last, etid, 32 * kEncoderWarps);
                    }
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&cvfree[q]);
                if (++q == NB) {
                    q = 0;
                    ph ^= 1;
                }
            }
        }
        return;
    }

    // ---------------------------------------------------------------- compute warps
    uint64_t my_count = 0, my_agg = 0;
    uint32_t j = 0, s = 0, sphase = 0, q = 0, qphase = 0;
    if constexpr (Pol::kSwar) {
        // Field-parallel path (one slab column, a predicate and/or an input mask): the flags are
        // computed on whole slab words, the stage is released as soon as the thread's words (and
        // mask bits) are in registers, and only the passing fields are ever extracted.
        constexpr int B = Pol::kBits;
        constexpr int EPS = Pol::EPS;
        constexpr int SPT = Pol::SPT;
        for (;; j++) {
            if (j) {
                if (++s == S) {
                    s = 0;
                    sphase ^= 1;
                }
            }
            wait_or_flag(&full[s], sphase, &p.ws->err);
            const uint64_t tile = tickets[s];
            if (tile >= num_tiles) break;
            const uint64_t e0 = tile * TILE;
            const uint64_t rem = n - e0;
            const uint32_t valid = rem < TILE ? (uint32_t)rem : TILE;
            uint64_t x[SPT];
            uint64_t mb = 0;  // the thread's R input-mask bits
            {
                const uint8_t* st = stage0 + s * p.stage_bytes;
                const uint64_t first = tile * (uint64_t)(T * SPT) + tid * SPT;  // first slab of this thread
                const uint64_t* src = reinterpret_cast<const uint64_t*>(st + p.a_off) + (first - sbase[3 * s] / 8);
                if constexpr ((Pol::kPlain || Pol::kFilter || Pol::kAggOnly) && SPT == 8)
                    lds_words8_rot(src, x);  // tiles fall on 32 KB boundaries: 64-byte-aligned runs
                else
                    lds_words<SPT>(src, x);
                // tiles of T*R elements, T a multiple of 256: a tile's mask starts on a 32-byte
                // boundary, the first staged byte
                if constexpr (!Pol::kWide)
                    if (p.has_mask_in) mb = bits_at_v<R>(reinterpret_cast<const uint32_t*>(st + p.m_off), tid * R);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);  // the words are in registers: stage s is free

            uint64_t g[SPT];
            swar_flags<B, SPT>(p.sw_mode, x, g, p.sw_l1, p.sw_l2);
            if constexpr (!Pol::kWide) {
                if (p.has_mask_in) {
#pragma unroll
                    for (int i = 0; i < SPT; i++) g[i] &= swar_deposit_flags<B>(mb >> (i * EPS));
                }
            }
            const uint32_t le0 = tid * R;
            if (le0 + R > valid) {  // elements past the column's end do not pass
#pragma unroll
                for (int i = 0; i < SPT; i++) {
                    const int left = (int)valid - (int)(le0 + i * EPS);
                    g[i] &= left <= 0 ? 0ull : (left >= EPS ? ~0ull : ((1ull << (left * B)) - 1));
                }
            }
            uint32_t c = 0;
#pragma unroll
            for (int i = 0; i < SPT; i++) c += __popcll(g[i]);
            my_count += c;

            if constexpr (!Pol::kWide) if (Pol::kFilter || (!Pol::kPlain && !Pol::kAggOnly && p.mask_out)) {
                uint64_t fl = 0;
                if constexpr (B >= 8) {  // one multiplication per word (swar_gather_flags)
#pragma unroll
                    for (int i = 0; i < SPT; i++) fl |= (uint64_t)swar_gather_flags<B>(g[i]) << (i * EPS);
                }
                else {
#pragma unroll
                    for (int i = 0; i < SPT; i++)
#pragma unroll
                        for (int k = 0; k < EPS; k++) fl |= ((g[i] >> (k * B + B - 1)) & 1ull) << (i * EPS + k);
                }
                if (fl) {
                    const uint32_t wi = le0 >> 5, sh = le0 & 31;
                    atomicOr(&bitmap[wi], (uint32_t)(fl << sh));
                    if (sh + R > 32) atomicOr(&bitmap[wi + 1], (uint32_t)(fl >> (32 - sh)));
                    if (sh + R > 64) atomicOr(&bitmap[wi + 2], (uint32_t)(fl >> (64 - sh)));
                }
            }

            uint32_t pos = 0;
            uint8_t* slot = cv;
            if (!Pol::kFilter && !Pol::kAggOnly && (Pol::kPlain || p.has_out)) {  // compacting: block scan, publish, hand the tile to the look-back
                volatile uint32_t* wt = warp_tot + 32 * (j & 1);
                const uint32_t incl = warp_incl_scan<uint32_t>(c);
                if (lane == 31) wt[warp] = incl;
                compute_bar();
                uint32_t total, before;
                tile_prefix<NW>(wt, warp, lane, before, total);
                pos = before + incl - c;
                if (tid == 0 && tile + 1 != p.withhold_plus1) st_relaxed_u64(&p.status[tile], kFlagAgg | total);
                if (j >= NB) wait_or_flag(&cvfree[q], qphase ^ 1, &p.ws->err);
                if (tid == 0) {
                    slot_tile[q] = tile;
                    slot_total[q] = total;
                    mbar_arrive(&aggb[q]);
                }
                slot = cv + (size_t)q * p.slot_bytes;
            }
            if constexpr (Pol::kFilter) {
            }
            else if constexpr (Pol::kAggOnly) {
                if (p.has_agg) {
                    bool done = false;
                    if constexpr (swar_sum_fits<B, SPT>()) {
                        if (p.agg == AMX_AGG_SUM) {  // field-parallel: no field extracted
                            my_agg += swar_masked_sum<B, SPT>(x, g);
                            done = true;
                        }
                    }
                    else if constexpr (B <= kSwarPlaneMax) {
                        if (p.agg == AMX_AGG_SUM) {
                            my_agg += swar_plane_sum<B, SPT>(x, g);
                            done = true;
                        }
                    }
                    if constexpr (!Pol::kWide) {
                        if (!done) {
                            const uint32_t wc = __reduce_add_sync(0xffffffffu, c);
                            uint64_t a = 0;
                            swar_visit<B, SPT, uint32_t, false, true>(x, g, 25 * wc > 32 * (uint32_t)R, nullptr, 0,
                                                                      p.agg, a);
                            my_agg = agg_combine(p.agg, my_agg, a);
                        }
                    }
                }
            }
            else if constexpr (Pol::kPlain) {
                const uint32_t wc = __reduce_add_sync(0xffffffffu, c);
                if (25 * wc > 32 * (uint32_t)R) {
                    swar_store_dense_raw<B, SPT>(x, g, reinterpret_cast<uint16_t*>(slot) + pos);
                }
                else {
                    uint64_t a = 0;
                    swar_visit<B, SPT, uint16_t, true, false>(x, g, false, reinterpret_cast<uint16_t*>(slot), pos, 0, a);
                }
            }
            else if (p.has_out || p.has_agg) {
                // the walk over set bits wins only below ~4% survivors in the warp
                const uint32_t wc = __reduce_add_sync(0xffffffffu, c);
                const bool dense = 25 * wc > 32 * (uint32_t)R;
                uint64_t a = 0;
                if (p.has_out) {
                    if (cv16) {
                        if (p.has_agg)
                            swar_visit<B, SPT, uint16_t, true, true>(x, g, dense, reinterpret_cast<uint16_t*>(slot), pos, p.agg, a);
                        else
                            swar_visit<B, SPT, uint16_t, true, false>(x, g, dense, reinterpret_cast<uint16_t*>(slot), pos, p.agg, a);
                    }
                    else {
                        if (p.has_agg)
                            swar_visit<B, SPT, uint32_t, true, true>(x, g, dense, reinterpret_cast<uint32_t*>(slot), pos, p.agg, a);
                        else
                            swar_visit<B, SPT, uint32_t, true, false>(x, g, dense, reinterpret_cast<uint32_t*>(slot), pos, p.agg, a);
                    }
                }
                else {
                    swar_visit<B, SPT, uint32_t, false, true>(x, g, dense, nullptr, 0, p.agg, a);
                }
                if (p.has_agg) my_agg = agg_combine(p.agg, my_agg, a);
            }
            if (!Pol::kFilter && !Pol::kAggOnly && (Pol::kPlain || p.has_out)) {
                __syncwarp();
                if (lane == 0) mbar_arrive(&scat[q]);  // this warp's survivors are in slot q
                if (++q == NB) {
                    q = 0;
                    qphase ^= 1;
                }
            }
            if (!Pol::kWide && (Pol::kFilter || (!Pol::kPlain && !Pol::kAggOnly && p.mask_out))) {
                compute_bar();
                const uint32_t words = (valid + 31) / 32;
                for (uint32_t i = tid; i < words; i += T) {
                    p.mask_out[e0 / 32 + i] = bitmap[i];
                    bitmap[i] = 0;
                }
                compute_bar();
            }
        }
    }
    else {
    for (;; j++) {
        if (j) {
            if (++s == S) {
                s = 0;
                sphase ^= 1;
            }
        }
        wait_or_flag(&full[s], sphase, &p.ws->err);
        const uint64_t tile = tickets[s];
        if (tile >= num_tiles) break;

        const uint64_t e0 = tile * TILE;
        const uint64_t rem = n - e0;
        const uint32_t valid = rem < TILE ? (uint32_t)rem : TILE;
        const uint8_t* st = stage0 + s * p.stage_bytes;

        V v[R];
        uint64_t fl;
        Pol::decode(p, st, sbase + 3 * s, e0, v, fl);
        // element of flag bit i: thread-contiguous tid*R + i, warp-major warp*32R + 32i + lane
        if (!Pol::kPlain && !Pol::kMap && p.has_mask_in) {
            const uint32_t* mw = reinterpret_cast<const uint32_t*>(st + p.m_off);
            if (WM) {
                uint64_t mfl = 0;
#pragma unroll
                for (int i = 0; i < R; i++) mfl |= (uint64_t)((lds_u32_v(mw + warp * R + i) >> lane) & 1u) << i;
                fl &= mfl;
            }
            else {
                fl &= bits_at<R>(mw, tid * R);
            }
        }
        // Warp-major runs keep every value in registers and release the stage at once.  The
        // thread-contiguous (compile-time) policies keep the stage until their survivors are
        // gathered: a sparse warp re-reads only its few survivors from it.
        if (WM) {
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s
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

        // sparse warp: every thread has at most kSparseMax survivors; the aggregate and the
        // gather then visit the survivors only (set bits of fl) instead of all R elements
        const bool sparse = !WM && __all_sync(0xffffffffu, __popcll(fl) <= kSparseMax);

        if (Pol::kPlain && p.has_agg && !sparse) {  // a sum
            uint64_t a = 0;
#pragma unroll
            for (int i = 0; i < R; i++) a += ((fl >> i) & 1) ? (uint64_t)v[i] : 0;
            my_agg += a;
        }
        else if (!Pol::kPlain && !Pol::kMap && p.has_agg && !sparse) {
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
            if (!Pol::kPlain && !Pol::kMap && p.mask_out) {
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
            if (!Pol::kPlain && !Pol::kMap && p.mask_out && fl) {
                const uint32_t le0 = tid * R;
                const uint32_t wi = le0 >> 5, sh = le0 & 31;
                atomicOr(&bitmap[wi], (uint32_t)(fl << sh));
                if (sh + R > 32) atomicOr(&bitmap[wi + 1], (uint32_t)(fl >> (32 - sh)));
                if (sh + R > 64) atomicOr(&bitmap[wi + 2], (uint32_t)(fl >> (64 - sh)));
            }
        }
        my_count += WM ? (lane == 0 ? c : 0) : c;

        if (Pol::kPlain || Pol::kMap || p.has_out) {
            // block scan: survivors before this thread (or warp) inside the tile
            volatile uint32_t* wt = warp_tot + 32 * (j & 1);
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
                tile_prefix<NW>(wt, warp, lane, before, total);
                pos = before + incl - c;
            }
            uint8_t* slot = cv;
            if (Pol::kPlain || (!Pol::kMap && compact)) {
                // publish this tile's survivor count for the other CTAs' look-backs at once ...
                if (tid == 0 && tile + 1 != p.withhold_plus1) st_relaxed_u64(&p.status[tile], kFlagAgg | total);
                // ... but reuse slot q only after the encoder warps are done with its last tile
                if (j >= NB) wait_or_flag(&cvfree[q], qphase ^ 1, &p.ws->err);
                if (tid == 0) {
                    slot_tile[q] = tile;
                    slot_total[q] = total;
                    mbar_arrive(&aggb[q]);  // hand the tile to the look-back warp
                }
                slot = cv + (size_t)q * p.slot_bytes;
            }
            if (WM) {
                const uint32_t lt = (1u << lane) - 1;
#pragma unroll
                for (int i = 0; i < R; i++) {
                    if ((fl >> i) & 1) cv_put<V>(slot, cv16, pos + __popc(bal[i] & lt), v[i]);
                    pos += __popc(bal[i]);
                }
            }
            else if (sparse) {
                uint64_t a = 0;
                for (uint64_t f = fl; f; f &= f - 1) {
                    const V x = Pol::value_at(p, st, sbase + 3 * s, e0, __ffsll((long long)f) - 1);
                    if constexpr (Pol::kPlain) {
                        reinterpret_cast<uint16_t*>(slot)[pos++] = (uint16_t)x;
                        a += x;
                    }
                    else {
                        cv_put<V>(slot, cv16, pos++, x);
                        a = agg_combine(p.agg, a, agg_encode(p.agg, (uint64_t)x));
                    }
                }
                if (Pol::kPlain) {
                    if (p.has_agg) my_agg += a;
                }
                else if (p.has_agg)
                    my_agg = agg_combine(p.agg, my_agg, a);
            }
            else if (Pol::kPlain || cv16) {
                uint16_t* dst = reinterpret_cast<uint16_t*>(slot) + pos;
#pragma unroll
                for (int i = 0; i < R; i++)
                    if ((fl >> i) & 1) *dst++ = (uint16_t)v[i];
            }
            else if constexpr (!Pol::kPlain) {
                V* dst = reinterpret_cast<V*>(slot) + pos;
#pragma unroll
                for (int i = 0; i < R; i++)
                    if ((fl >> i) & 1) *dst++ = v[i];
            }
            if (Pol::kPlain || (!Pol::kMap && compact)) {
                __syncwarp();
                if (lane == 0) mbar_arrive(&scat[q]);  // this warp's survivors are in slot q
                if (++q == NB) {
                    q = 0;
                    qphase ^= 1;
                }
            }
            else if constexpr (!Pol::kPlain) {  // element-wise output: the offset is known, encode right away
                compute_bar();
                encode_any<V>(p.out, cv, cv16, total, e0, tile == num_tiles - 1, tid, T);
                compute_bar();
            }
        }
        if (!WM) {
            if (!Pol::kPlain && !Pol::kMap && !p.has_out && p.has_agg && sparse) {
                uint64_t a = 0;
                for (uint64_t f = fl; f; f &= f - 1) {
                    const V x = Pol::value_at(p, st, sbase + 3 * s, e0, __ffsll((long long)f) - 1);
                    a = agg_combine(p.agg, a, agg_encode(p.agg, (uint64_t)x));
                }
                my_agg = agg_combine(p.agg, my_agg, a);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);  // this warp is done with stage s
        }
        if (!Pol::kPlain && !Pol::kMap && !WM && p.mask_out) {
            compute_bar();
            const uint32_t words = (valid + 31) / 32;
            for (uint32_t i = tid; i < words; i += T) {
                p.mask_out[e0 / 32 + i] = bitmap[i];
                bitmap[i] = 0;
            }
            compute_bar();
        }
    }
    }
    if (compact) {  // release the look-back and encoder warps through the next free slot
        if (j >= NB) wait_or_flag(&cvfree[q], qphase ^ 1, &p.ws->err);
        if (tid == 0) {
            slot_tile[q] = kNoTile;
            mbar_arrive(&aggb[q]);
        }
    }

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
// words: no bank conflicts).  Volatile reads: the warp-major policies release the stage right
// after this.
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
            for (int i = 0; i < R; i++) out[i] = lds_u32_v(w + 32 * i) & m;
            break;
        }
        case AMX_PLAIN64: {
            const uint64_t* w = reinterpret_cast<const uint64_t*>(st) + (e0 - sb / 8) + base;
#pragma unroll
            for (int i = 0; i < R; i++) out[i] = lds_u64_v(w + 32 * i) & m;
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
                out[i] = (lds_u64_v(w + s) >> (k * b)) & m;
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
                const uint64_t lo = lds_u64_v(w + wi), hi = lds_u64_v(w + wi + 1);
                out[i] = (off ? ((lo >> off) | (hi << (64 - off))) : lo) & m;
            }
            break;
        }
    }
}

// Any formats and widths: warp-major runtime readers, 64-bit values, RR elements per thread.
// PLAIN: the variant for compacting requests with 16-bit values, no masks and at most a sum;
// MAP: for element-wise outputs (conversions, binary ops) with no masks and no aggregate.  Both
// carry their request's path only, with more elements per thread to cut the tiles.
template <int RR = 8, bool PLAIN = false, bool MAP = false>
struct GenericPolT {
    using V = uint64_t;
    static constexpr int R = RR;
    static constexpr bool kWarpMajor = true;
    static constexpr bool kSwar = false;
    static constexpr bool kPlain = PLAIN;
    static constexpr bool kFilter = false;
    static constexpr bool kAggOnly = false;
    static constexpr bool kMap = MAP;
    static constexpr bool kWide = false;
    static constexpr int kOutBits = 0;         // the encoder warps use the runtime encoder
    static constexpr uint32_t kCompute = 512;  // one CTA of 16 compute warps per SM
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

    // warp-major runs never take the sparse path (their values stay in registers)
    __device__ __forceinline__ static V value_at(const PipeParams&, const uint8_t*, const uint64_t*, uint64_t, int)
    {
        return 0;
    }
};
using GenericPol = GenericPolT<>;

}  // namespace amx
