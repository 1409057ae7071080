// amx_pipeline.cuh -- the tile pipeline kernel behind filter, compressstore, binary ops,
// conversion, aggregation and fused chains.
//
// One persistent CTA per SM slot pulls tiles from an atomic ticket counter.  For each tile:
//   1. one thread stages the tile's bytes of every input into shared memory with 1-D bulk
//      copies (cp.async.bulk, completion on an mbarrier), kStages tiles ahead;
//   2. every thread decodes a run of R consecutive elements straight from the staged packed
//      words (a policy: runtime-width streaming readers, or compile-time-width readers),
//      applies the binary op and the predicate, and keeps a flag word;
//   3. flags feed (a) a bitmask assembled in shared memory, (b) the aggregate, (c) a block
//      scan + decoupled look-back that places the survivors, which are gathered in shared
//      memory and re-encoded in the output format with boundary words merged by atomics.
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

// Re-encode cnt compacted values cv[0..cnt) as output elements [g, g+cnt).  Words wholly
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
                const uint64_t w0 = g / eps, w1 = (g + cnt - 1) / eps;
                for (uint64_t w = w0 + tid; w <= w1; w += T) {
                    const int64_t r0 = (int64_t)(w * eps) - (int64_t)g;
                    uint64_t acc = 0;
                    if (r0 >= 0 && r0 + eps <= cnt) {
                        for (uint32_t k = 0; k < eps; k++) acc |= ((uint64_t)cv[r0 + k] & m) << (k * b);
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
                    const uint64_t own =
                        (ob1 - ob0 >= 64) ? ~0ull : (((1ull << (ob1 - ob0)) - 1) << (ob0 - lo));
                    uint64_t p0 = lo / b;
                    if (p0 < g) p0 = g;
                    uint64_t p1 = (hi - 1) / b;
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

// Shared-memory map of the pipeline kernel (dynamic shared memory):
//   [0,64)     mbarriers            [64,128)  tickets        [128,256) stage base offsets
//   [256,320)  warp totals          [320,384) broadcast      [512,1024) tile bitmap (R*T/32 words, <= 2 KiB)
//   [kCvOff, smem_fixed)  compacted values;  [smem_fixed, ...) kStages stage buffers
constexpr uint32_t kBitmapOff = 512;
constexpr uint32_t kCvOff = 2560;

template <class Pol>
__global__ void __launch_bounds__(kPipeThreads) pipe_kernel(const __grid_constant__ PipeParams p)
{
    using V = typename Pol::V;
    constexpr int R = Pol::R;
    constexpr uint32_t T = kPipeThreads;
    constexpr uint32_t NW = T / 32;
    constexpr uint32_t TILE = T * R;
    static_assert(TILE / 32 * 4 <= kCvOff - kBitmapOff, "bitmap region");

    extern __shared__ __align__(128) uint8_t smem[];
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem);
    volatile uint64_t* tickets = reinterpret_cast<volatile uint64_t*>(smem + 64);
    uint64_t* sbase = reinterpret_cast<uint64_t*>(smem + 128);
    uint64_t* warp_tot = reinterpret_cast<uint64_t*>(smem + 256);
    volatile uint64_t* bcast = reinterpret_cast<volatile uint64_t*>(smem + 320);
    uint32_t* bitmap = reinterpret_cast<uint32_t*>(smem + kBitmapOff);
    V* cv = reinterpret_cast<V*>(smem + kCvOff);
    uint8_t* stage0 = smem + p.smem_fixed;

    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (tid == 0) {
        for (uint32_t s = 0; s < kStages; s++) mbar_init(&mbar[s], 1);
        fence_mbar_init();
    }
    for (uint32_t i = tid; i < TILE / 32; i += T) bitmap[i] = 0;
    __syncthreads();
    if (tid == 0) {
        for (uint32_t s = 0; s < kStages; s++) {
            const uint64_t tk = atomicAdd(&p.ws->ticket, 1u);
            tickets[s] = tk;
            if (tk < p.num_tiles) stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &mbar[s], tk, TILE);
        }
    }
    __syncthreads();

    uint64_t my_count = 0;
    uint64_t my_agg = 0;
    for (uint32_t it = 0;; it++) {
        const uint32_t s = it % kStages;
        const uint64_t tile = tickets[s];
        if (tile >= p.num_tiles) break;
        if (!mbar_wait_bounded(&mbar[s], (it / kStages) & 1)) record_error(&p.ws->err, AMX_ERR_TIMEOUT);

        const uint64_t e0 = tile * TILE;
        const uint64_t rem = p.n - e0;
        const uint32_t valid = rem < TILE ? (uint32_t)rem : TILE;
        const uint32_t le0 = tid * R;
        const uint8_t* st = stage0 + s * p.stage_bytes;

        V v[R];
        uint64_t fl;
        Pol::decode(p, st, sbase + 3 * s, e0 + le0, v, fl);
        if (p.has_mask_in) {
            const uint64_t mbit = e0 + le0 - sbase[3 * s + 2] * 8;
            fl &= bits_at<R>(reinterpret_cast<const uint32_t*>(st + p.m_off), (uint32_t)mbit);
        }
        if (le0 >= valid)
            fl = 0;
        else if (valid - le0 < (uint32_t)R)
            fl &= (1ull << (valid - le0)) - 1;
        if (R < 64) fl &= (1ull << R) - 1;

        __syncthreads();  // every thread is done with stage s
        if (tid == 0) {
            const uint64_t tk = atomicAdd(&p.ws->ticket, 1u);
            tickets[s] = tk;
            if (tk < p.num_tiles) stage_issue(p, stage0 + s * p.stage_bytes, sbase + 3 * s, &mbar[s], tk, TILE);
        }

        const uint32_t c = __popcll(fl);
        my_count += c;
        if (p.has_agg) {
#pragma unroll
            for (int i = 0; i < R; i++)
                if ((fl >> i) & 1) my_agg = agg_combine(p.agg, my_agg, agg_encode(p.agg, (uint64_t)v[i]));
        }
        if (p.mask_out && fl) {
            const uint32_t wi = le0 >> 5, sh = le0 & 31;
            atomicOr(&bitmap[wi], (uint32_t)(fl << sh));
            if (sh + R > 32) atomicOr(&bitmap[wi + 1], (uint32_t)(fl >> (32 - sh)));
            if (sh + R > 64) atomicOr(&bitmap[wi + 2], (uint32_t)(fl >> (64 - sh)));
        }

        if (p.has_out) {
            const uint64_t incl = warp_incl_scan<uint64_t>(c);
            if (lane == 31) warp_tot[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                uint64_t x = lane < NW ? warp_tot[lane] : 0;
                x = warp_incl_scan<uint64_t>(x);
                if (lane < NW) warp_tot[lane] = x;
            }
            __syncthreads();
            const uint32_t total = (uint32_t)warp_tot[NW - 1];
            uint32_t pos = (uint32_t)(incl - c + (warp ? warp_tot[warp - 1] : 0));
            if (p.compact && warp == 0) {
                const uint64_t g = lookback(p.status, tile, total, &p.ws->err);
                if (lane == 0) bcast[0] = g;
            }
#pragma unroll
            for (int i = 0; i < R; i++)
                if ((fl >> i) & 1) cv[pos++] = v[i];
            __syncthreads();
            const uint64_t g = p.compact ? bcast[0] : e0;
            encode_tile<V>(p.out, cv, total, g, tile == p.num_tiles - 1);
        }
        if (p.mask_out) {
            __syncthreads();
            const uint32_t words = (valid + 31) / 32;
            for (uint32_t i = tid; i < words; i += T) {
                p.mask_out[e0 / 32 + i] = bitmap[i];
                bitmap[i] = 0;
            }
        }
        __syncthreads();
    }

    // CTA totals -> workspace; the last CTA to finish publishes the scalar results
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        my_count += __shfl_xor_sync(0xffffffffu, my_count, o);
        my_agg = agg_combine(p.agg, my_agg, __shfl_xor_sync(0xffffffffu, my_agg, o));
    }
    __syncthreads();
    if (lane == 0) {
        warp_tot[warp] = my_count;
        reinterpret_cast<uint64_t*>(smem + 384)[warp] = my_agg;
    }
    __syncthreads();
    if (tid == 0) {
        uint64_t cnt = 0, ag = 0;
        for (uint32_t w = 0; w < NW; w++) {
            cnt += warp_tot[w];
            ag = agg_combine(p.agg, ag, reinterpret_cast<uint64_t*>(smem + 384)[w]);
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

// Any formats and widths: runtime streaming readers, 64-bit values, 16 elements per thread.
struct GenericPol {
    using V = uint64_t;
    static constexpr int R = 16;

    __device__ __forceinline__ static void decode(const PipeParams& p, const uint8_t* st, const uint64_t* sb,
                                                  uint64_t first, V (&v)[R], uint64_t& fl)
    {
        Stream sa;
        sa.init(p.a, st + p.a_off, sb[0], first);
#pragma unroll
        for (int i = 0; i < R; i++) v[i] = sa.next();
        if (p.has_b) {
            Stream sr;
            sr.init(p.b, st + p.b_off, sb[1], first);
#pragma unroll
            for (int c = 0; c < R; c += 8) {
                uint64_t r[8];
#pragma unroll
                for (int j = 0; j < 8; j++) r[j] = sr.next();
                switch (p.op) {
                    case AMX_OP_ADD:
#pragma unroll
                        for (int j = 0; j < 8; j++) v[c + j] += r[j];
                        break;
                    case AMX_OP_SUB:
#pragma unroll
                        for (int j = 0; j < 8; j++) v[c + j] -= r[j];
                        break;
                    case AMX_OP_MUL:
#pragma unroll
                        for (int j = 0; j < 8; j++) v[c + j] *= r[j];
                        break;
                    default:
#pragma unroll
                        for (int j = 0; j < 8; j++) v[c + j] = binop_eval(p.op, v[c + j], r[j]);
                        break;
                }
            }
        }
        finish_values<R, V>(p, v, fl);
    }
};

}  // namespace amx
