// amx_groupby.cu -- group-by sum + count over packed key and value columns.
//
// Replaces kernel_groupby_sm_array_gather / _writeout (src/kernels/groupby_sm_array.cuh:4-81) and
// the sort-based CUB path (src/benchs/bench_groupby_sort_cub.cu:50-63).  Differences by design:
// keys and values may have different formats and widths; sums are full uint64 (write them into a
// narrower output column to get the reference's sums masked to the key width); counts are
// emitted; groups come out in ascending key order (the reference's order is nondeterministic).
//
// 1. groupby_kernel: persistent CTAs of 512 threads (grid = CTAs that fit x SMs) walk chunks of
//    2^14 elements.  Each thread reads a run of 32 consecutive elements of the chunk straight from
//    the packed columns, one storage word at a time, and aggregates into a per-CTA shared table:
//      - keys up to 12 bits: a dense table (sum as 32-bit low word + carry word, 32-bit count);
//        values of at most 18 bits need no carry word (the table is flushed before a sum wraps);
//      - wider keys: an open-addressing hash table of 4096 slots (claimed by atomicCAS, linear
//        probing, 8 probes); a key that finds no slot goes straight to the global table.
//    A CTA flushes its shared table into the dense global table of uint64 sums and counts
//    (2^key_bits entries, 64-bit atomics) once, after its last chunk, or every 2^(32 - value
//    bits) elements (carry-free sums, at most 2^30) before a 32-bit field could overflow.
//    groupby_phase_kernel does the same for slab keys and slab values without a mask, with runs
//    whose length is a multiple of both columns' field counts: the lanes of a warp then change
//    words at the same element, and the next word is loaded a word ahead.
// 2. the groups are extracted: for at most 4096 groups by one CTA (gb_extract_kernel), else with
//    the tile pipeline itself: mask = filter(count != 0), then compressstore of the key indices,
//    the sums and the counts into the caller's output columns.
#include <cstddef>

#include "amx_dispatch.h"
#include "amx_pipeline.cuh"

namespace amx {

constexpr uint32_t kGbThreads = 512;
constexpr uint64_t kGbChunk = 1ull << 14;
constexpr uint32_t kGbRun = 32;  // consecutive elements per thread
static_assert(kGbThreads * kGbRun == kGbChunk, "a chunk is one run per thread");
constexpr uint64_t kGbFlushEvery = 1ull << 30;  // elements per CTA between flushes (32-bit counts)
constexpr uint32_t kGbDenseBits = 12;
constexpr uint32_t kGbHashSlots = 4096;
constexpr uint32_t kGbMaxKeyBits = 24;
constexpr uint32_t kGbCopies = 2;  // copies of a phase kernel's sums and counts
constexpr uint32_t kEmptyKey = 0xffffffffu;

struct GbParams {
    ColDev k, v;
    const uint32_t* mask;
    uint64_t n;
    uint32_t kbits;
    uint32_t dense;
    uint64_t flush_every;  // elements per CTA between flushes of its shared table
    uint32_t run;          // groupby_phase_kernel: elements per thread and chunk
    uint32_t copies;       // groupby_phase_kernel: copies of the table's sums and counts (1, 2 or 4)
    unsigned long long* gsum;
    unsigned long long* gcnt;
    const uint64_t* n_dev;  // optional device-resident length (<= n), read by the kernels
    // keys wider than kGbMaxKeyBits: gsum / gcnt are indexed by the slot of a global open-addressing
    // hash table (gkey[slot] = key, kGEmpty when free) of gcap_mask + 1 slots instead of by key
    unsigned long long* gkey;
    uint64_t gcap_mask;
    uint32_t gshift;  // 64 - log2(slots)
    uint32_t* err;    // AMX_ERR_CAPACITY when the table is full
};

constexpr unsigned long long kGEmpty = ~0ull;

// The global table slot of `key`: its index in the dense table, or -- for wide keys -- the hash
// slot holding it, claimed with atomicCAS on first sight (linear probing, at most one lap;
// UINT64_MAX when the table is full).
__device__ __forceinline__ uint64_t gb_gslot(const GbParams& p, uint32_t key)
{
    if (!p.gkey) return key;
    const uint64_t h = ((uint64_t)key * 0x9E3779B97F4A7C15ull) >> p.gshift;
    for (uint64_t probe = 0; probe <= p.gcap_mask; probe++) {
        const uint64_t s = (h + probe) & p.gcap_mask;
        const uint64_t cur = ld_relaxed_u64(reinterpret_cast<const uint64_t*>(p.gkey + s));
        if (cur == key) return s;
        if (cur == kGEmpty) {
            const unsigned long long prev = atomicCAS(p.gkey + s, kGEmpty, (unsigned long long)key);
            if (prev == kGEmpty || prev == key) return s;
        }
    }
    return ~0ull;
}

__device__ __forceinline__ void gb_global_add(const GbParams& p, uint32_t key, uint64_t sum, uint64_t cnt)
{
    const uint64_t s = gb_gslot(p, key);
    if (s == ~0ull) {
        record_error(p.err, AMX_ERR_CAPACITY);
        return;
    }
    atomicAdd(&p.gsum[s], (unsigned long long)sum);
    atomicAdd(&p.gcnt[s], (unsigned long long)cnt);
}

// elements of this run: n, or the device-resident length a previous kernel wrote
__device__ __forceinline__ uint64_t gb_len(const GbParams& p)
{
    if (!p.n_dev) return p.n;
    const uint64_t d = *p.n_dev;
    return d < p.n ? d : p.n;
}

// element e of column c read straight from global memory (consecutive lanes share words)
__device__ __forceinline__ uint64_t load_elem(const ColDev& c, uint64_t e)
{
    switch (c.format) {
        case AMX_PLAIN32: return __ldg(reinterpret_cast<const uint32_t*>(c.data) + e) & c.mask;
        case AMX_PLAIN64: return __ldg(reinterpret_cast<const unsigned long long*>(c.data) + e) & c.mask;
        case AMX_SLAB: {
            const uint64_t s = udiv64(e, c.magic64, c.eps);
            const uint32_t k = (uint32_t)(e - s * c.eps);
            return (__ldg(reinterpret_cast<const unsigned long long*>(c.data) + s) >> (k * c.bits)) & c.mask;
        }
        default: {
            const uint64_t bp = e * c.bits;
            const uint64_t wi = bp >> 6;
            const uint32_t off = (uint32_t)(bp & 63);
            const unsigned long long* w = reinterpret_cast<const unsigned long long*>(c.data);
            uint64_t x = __ldg(w + wi) >> off;
            if (off + c.bits > 64) x |= (uint64_t)__ldg(w + wi + 1) << (64 - off);
            return x & c.mask;
        }
    }
}

// Consecutive elements e, e + 1, ... of a column: one load per storage word instead of one per
// element, and one division by the slab's field count per run instead of one per element.
struct SeqReader {
    const unsigned long long* w;
    uint64_t cur;     // slab / nogaps: current word
    uint64_t wi;      // index of the current word
    uint64_t bitpos;  // nogaps: bit of the next element
    uint32_t k;       // slab: field of the next element in `cur`
};

__device__ __forceinline__ SeqReader seq_open(const ColDev& c, uint64_t e)
{
    SeqReader r{};
    r.w = reinterpret_cast<const unsigned long long*>(c.data);
    switch (c.format) {
        case AMX_PLAIN32:
        case AMX_PLAIN64: r.wi = e; break;
        case AMX_SLAB: {
            r.wi = udiv64(e, c.magic64, c.eps);
            r.k = (uint32_t)(e - r.wi * c.eps);
            r.cur = __ldg(r.w + r.wi);
            break;
        }
        default: r.bitpos = e * c.bits; break;
    }
    return r;
}

// the next element; `more` says whether another element of this run follows
__device__ __forceinline__ uint64_t seq_next(const ColDev& c, SeqReader& r, bool more)
{
    switch (c.format) {
        case AMX_PLAIN32: return __ldg(reinterpret_cast<const uint32_t*>(c.data) + r.wi++) & c.mask;
        case AMX_PLAIN64: return __ldg(r.w + r.wi++) & c.mask;
        case AMX_SLAB: {
            const uint64_t v = (r.cur >> (r.k * c.bits)) & c.mask;
            if (++r.k == c.eps) {
                r.k = 0;
                ++r.wi;
                if (more) r.cur = __ldg(r.w + r.wi);
            }
            return v;
        }
        default: {
            const uint64_t wi = r.bitpos >> 6;
            const uint32_t off = (uint32_t)(r.bitpos & 63);
            uint64_t x = __ldg(r.w + wi) >> off;
            if (off + c.bits > 64) x |= (uint64_t)__ldg(r.w + wi + 1) << (64 - off);
            r.bitpos += c.bits;
            return x & c.mask;
        }
    }
}

// Slab column read as a run of consecutive elements: the current word is shifted down by one
// field per element, so an element costs a mask, a shift and a field-count test.
struct SlabRun {
    const unsigned long long* w;
    uint64_t cur;  // current word, shifted so that the next element sits in the low bits
    uint64_t wi;
    uint32_t k;    // field of the next element
};

__device__ __forceinline__ SlabRun slab_open(const ColDev& c, uint64_t e)
{
    SlabRun r;
    r.w = reinterpret_cast<const unsigned long long*>(c.data);
    r.wi = udiv64(e, c.magic64, c.eps);
    r.k = (uint32_t)(e - r.wi * c.eps);
    r.cur = __ldg(r.w + r.wi) >> (r.k * c.bits);
    return r;
}

__device__ __forceinline__ uint32_t slab_next(const ColDev& c, SlabRun& r, bool more)
{
    const uint32_t v = (uint32_t)r.cur & (uint32_t)c.mask;
    r.cur >>= c.bits;
    if (++r.k == c.eps) {
        r.k = 0;
        ++r.wi;
        if (more) r.cur = __ldg(r.w + r.wi);
    }
    return v;
}

// A run reader: the slab form above when the column's format is known to be AMX_SLAB at
// compile time, else the general SeqReader (any format, chosen at run time).
template <bool SLAB>
struct RunReader {
    SeqReader r;
    __device__ __forceinline__ void open(const ColDev& c, uint64_t e) { r = seq_open(c, e); }
    __device__ __forceinline__ uint32_t next(const ColDev& c, bool more) { return (uint32_t)seq_next(c, r, more); }
};
template <>
struct RunReader<true> {
    SlabRun r;
    __device__ __forceinline__ void open(const ColDev& c, uint64_t e) { r = slab_open(c, e); }
    __device__ __forceinline__ uint32_t next(const ColDev& c, bool more) { return slab_next(c, r, more); }
};

// Narrow values (at most kGbNoCarryBits bits) need no carry word: the CTA flushes its table
// every gb_flush_every(value bits) elements, few enough that a 32-bit sum cannot wrap, so an
// element is two 32-bit shared-memory adds whose results are not read back.
constexpr uint32_t kGbNoCarryBits = 18;

__host__ __device__ constexpr uint64_t gb_flush_every(uint32_t vbits)
{
    // sums <= flush * (2^vbits - 1) < 2^32; counts <= flush <= 2^30; whole chunks
    return vbits > kGbNoCarryBits || 32 - vbits >= 30 ? kGbFlushEvery : (1ull << (32 - vbits));
}
static_assert(gb_flush_every(kGbNoCarryBits) % kGbChunk == 0, "flushes fall on chunk boundaries");

// Hash table probe: the slot holding `key`, claiming an empty one if needed; kEmptyKey when
// 8 probes find neither.
__device__ __forceinline__ uint32_t gb_probe(uint32_t* tkey, uint32_t key)
{
    const uint32_t h = (key * 2654435761u) >> 20;  // 12 bits: 4096 slots
    for (int probe = 0; probe < 8; probe++) {
        const uint32_t sl = (h + probe) & (kGbHashSlots - 1);
        const uint32_t cur = tkey[sl];
        if (cur == key) return sl;
        if (cur == kEmptyKey) {
            const uint32_t prev = atomicCAS(&tkey[sl], kEmptyKey, key);
            if (prev == kEmptyKey || prev == key) return sl;
        }
    }
    return kEmptyKey;
}

template <bool KSLAB, bool VSLAB, bool DENSE, bool NOCARRY>
__global__ void __launch_bounds__(kGbThreads) groupby_kernel(const __grid_constant__ GbParams p)
{
    extern __shared__ __align__(16) uint32_t tab[];
    const uint32_t slots = DENSE ? (1u << p.kbits) : kGbHashSlots;
    uint32_t* tkey = tab;              // hash: key per slot
    uint32_t* tlo = tab + slots;       // sum (low 32 bits)
    uint32_t* thi = tab + 2 * slots;   // carries out of the low word (unused when NOCARRY)
    uint32_t* tcnt = tab + 3 * slots;  // count
    const uint32_t tid = threadIdx.x;
    const uint64_t n = gb_len(p);
    const uint64_t nchunks = (n + kGbChunk - 1) / kGbChunk;
    const uint64_t flush_every = p.flush_every;

    auto clear = [&]() {
        for (uint32_t i = tid; i < slots; i += blockDim.x) {
            if (!DENSE) tkey[i] = kEmptyKey;
            tlo[i] = thi[i] = tcnt[i] = 0;
        }
    };
    clear();
    __syncthreads();
    uint64_t seen = 0;
    for (uint64_t chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
        const uint64_t e0 = chunk * kGbChunk;
        const uint64_t e1 = e0 + kGbChunk < n ? e0 + kGbChunk : n;
        // each thread walks a run of kGbRun consecutive elements of the chunk; a run starts on
        // a multiple of 32, so its mask bits are one mask word
        const uint64_t r0 = e0 + (uint64_t)tid * kGbRun;
        const uint32_t rn = r0 >= e1 ? 0 : (uint32_t)(e1 - r0 < kGbRun ? e1 - r0 : kGbRun);
        if (rn) {
            RunReader<KSLAB> kr;
            RunReader<VSLAB> vr;
            kr.open(p.k, r0);
            vr.open(p.v, r0);
            const uint32_t mw = p.mask ? __ldg(p.mask + (r0 >> 5)) : 0xffffffffu;
#pragma unroll 4
            for (uint32_t i = 0; i < rn; i++) {
                const bool more = i + 1 < rn;
                const uint32_t key = kr.next(p.k, more);
                const uint32_t val = vr.next(p.v, more);
                if (!((mw >> i) & 1u)) continue;
                uint32_t slot = key;
                if (!DENSE) {
                    // a crowded table, or the one key that marks free slots: straight to the global table
                    slot = key == kEmptyKey ? kEmptyKey : gb_probe(tkey, key);
                    if (slot == kEmptyKey) {
                        gb_global_add(p, key, val, 1);
                        continue;
                    }
                }
                if (NOCARRY) {
                    atomicAdd(&tlo[slot], val);
                    atomicAdd(&tcnt[slot], 1u);
                }
                else {
                    const uint32_t old = atomicAdd(&tlo[slot], val);
                    if (old + val < old) atomicAdd(&thi[slot], 1u);
                    atomicAdd(&tcnt[slot], 1u);
                }
            }
        }
        // the shared table only goes to the global table when this CTA is done, or before its
        // fields could overflow
        seen += e1 - e0;
        const bool last = chunk + gridDim.x >= nchunks;
        if (last || seen >= flush_every) {
            __syncthreads();
            for (uint32_t i = tid; i < slots; i += blockDim.x) {
                const uint32_t c = tcnt[i];
                const uint64_t sum = NOCARRY ? tlo[i] : ((uint64_t)thi[i] << 32) | tlo[i];
                if (c) gb_global_add(p, DENSE ? i : tkey[i], sum, c);
                if (!DENSE) tkey[i] = kEmptyKey;  // each thread clears the slots it flushed
                tlo[i] = thi[i] = tcnt[i] = 0;
            }
            __syncthreads();
            seen = 0;
        }
    }
}

// Slab keys and slab values, no mask: every thread's run starts on a slab boundary of BOTH
// columns (run length a multiple of the two field counts' lcm), so all lanes of a warp reach
// the end of a word at the same element.  The word after the current one is loaded as soon as
// the current one is taken, a whole word of elements ahead of its use.
struct PhaseRun {
    const unsigned long long* w;
    uint64_t cur;   // current word, shifted so that the next element sits in the low bits
    uint64_t nxt;   // the word after it (0 past the column's end)
    uint64_t wi;    // index of the current word
    uint64_t nw;    // words in the column
    uint32_t k;     // field of the next element
};

__device__ __forceinline__ PhaseRun phase_open(const ColDev& c, uint64_t e)
{
    PhaseRun r;
    r.w = reinterpret_cast<const unsigned long long*>(c.data);
    r.nw = c.bytes / 8;
    r.wi = udiv64(e, c.magic64, c.eps);  // e is a multiple of eps
    r.k = 0;
    r.cur = r.wi < r.nw ? __ldg(r.w + r.wi) : 0;
    r.nxt = r.wi + 1 < r.nw ? __ldg(r.w + r.wi + 1) : 0;
    return r;
}

__device__ __forceinline__ uint32_t phase_next(const ColDev& c, PhaseRun& r)
{
    const uint32_t v = (uint32_t)r.cur & (uint32_t)c.mask;
    r.cur >>= c.bits;
    if (++r.k == c.eps) {  // the same element for every lane of the warp
        r.k = 0;
        r.cur = r.nxt;
        ++r.wi;
        r.nxt = r.wi + 1 < r.nw ? __ldg(r.w + r.wi + 1) : 0;
    }
    return v;
}

// The sums and counts are kept in p.copies interleaved copies (entry slot * copies + c), lane
// group c = lane * copies / 32 updating copy c: a key that several lanes of a warp hit at once
// (a Zipf-hot key) serialises over fewer shared atomics.  The flushes fold the copies.
template <bool DENSE, bool NOCARRY>
__global__ void __launch_bounds__(kGbThreads) groupby_phase_kernel(const __grid_constant__ GbParams p)
{
    extern __shared__ __align__(16) uint32_t tab[];
    const uint32_t slots = DENSE ? (1u << p.kbits) : kGbHashSlots;
    const uint32_t cp = p.copies;
    uint32_t* tkey = tab;
    uint32_t* tlo = tab + slots;
    uint32_t* thi = tlo + slots * cp;
    uint32_t* tcnt = thi + slots * cp;
    const uint32_t tid = threadIdx.x;
    const uint32_t sub = ((tid & 31) * cp) >> 5;
    const uint32_t run = p.run;
    const uint64_t chunk_elems = (uint64_t)kGbThreads * run;
    const uint64_t n = gb_len(p);
    const uint64_t nchunks = (n + chunk_elems - 1) / chunk_elems;

    for (uint32_t i = tid; i < slots; i += blockDim.x)
        if (!DENSE) tkey[i] = kEmptyKey;
    for (uint32_t i = tid; i < slots * cp; i += blockDim.x) tlo[i] = thi[i] = tcnt[i] = 0;
    __syncthreads();
    uint64_t seen = 0;
    for (uint64_t chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
        const uint64_t e0 = chunk * chunk_elems;
        const uint64_t e1 = e0 + chunk_elems < n ? e0 + chunk_elems : n;
        const uint64_t r0 = e0 + (uint64_t)tid * run;
        const uint32_t rn = r0 >= e1 ? 0 : (uint32_t)(e1 - r0 < run ? e1 - r0 : run);
        if (rn) {
            PhaseRun kr = phase_open(p.k, r0);
            PhaseRun vr = phase_open(p.v, r0);
#pragma unroll 4
            for (uint32_t i = 0; i < rn; i++) {
                const uint32_t key = phase_next(p.k, kr);
                const uint32_t val = phase_next(p.v, vr);
                uint32_t slot = key;
                if (!DENSE) {
                    // a crowded table, or the one key that marks free slots: straight to the global table
                    slot = key == kEmptyKey ? kEmptyKey : gb_probe(tkey, key);
                    if (slot == kEmptyKey) {
                        gb_global_add(p, key, val, 1);
                        continue;
                    }
                }
                const uint32_t at = slot * cp + sub;
                if (NOCARRY) {
                    atomicAdd(&tlo[at], val);
                    atomicAdd(&tcnt[at], 1u);
                }
                else {
                    const uint32_t old = atomicAdd(&tlo[at], val);
                    if (old + val < old) atomicAdd(&thi[at], 1u);
                    atomicAdd(&tcnt[at], 1u);
                }
            }
        }
        // flush before the next chunk could take a field past its bound
        seen += e1 - e0;
        const bool last = chunk + gridDim.x >= nchunks;
        if (last || seen + chunk_elems > p.flush_every) {
            __syncthreads();
            for (uint32_t i = tid; i < slots; i += blockDim.x) {
                uint64_t c = 0, sum = 0;
                for (uint32_t j = 0; j < cp; j++) {
                    const uint32_t at = i * cp + j;
                    c += tcnt[at];
                    sum += NOCARRY ? (uint64_t)tlo[at] : (((uint64_t)thi[at] << 32) | tlo[at]);
                    tlo[at] = thi[at] = tcnt[at] = 0;
                }
                if (c) gb_global_add(p, DENSE ? i : tkey[i], sum, c);
                if (!DENSE) tkey[i] = kEmptyKey;
            }
            __syncthreads();
            seen = 0;
        }
    }
}

static uint32_t gcd_u32(uint32_t a, uint32_t b) { return b ? gcd_u32(b, a % b) : a; }

// Values wider than 32 bits: every element goes to the global table directly.
__global__ void groupby_wide_kernel(const __grid_constant__ GbParams p)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t n = gb_len(p);
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += stride) {
        if (p.mask && !((__ldg(p.mask + (e >> 5)) >> (e & 31)) & 1u)) continue;
        gb_global_add(p, (uint32_t)load_elem(p.k, e), load_elem(p.v, e), 1);
    }
}

// Groups of a table of at most kGbExtractMax entries, extracted by one CTA: the present keys
// (count != 0) in ascending order are compacted into shared memory with their sums and counts,
// then encoded into the caller's output columns (any format), and their number is written to
// d_groups.  One launch instead of the filter + three compressstores of the general path.
constexpr uint32_t kGbExtractMax = 4096;
constexpr uint32_t kGbExtractThreads = 1024;
constexpr uint32_t kGbExtractSmem = kGbExtractMax * (4 + 8 + 8);

__global__ void __launch_bounds__(kGbExtractThreads) gb_extract_kernel(const unsigned long long* gsum,
                                                                       const unsigned long long* gcnt, uint32_t g,
                                                                       OutDev ok, OutDev os, OutDev oc, uint32_t has,
                                                                       uint64_t* d_groups)
{
    extern __shared__ __align__(16) uint8_t xs[];
    uint64_t* sums = reinterpret_cast<uint64_t*>(xs);
    uint64_t* cnts = sums + kGbExtractMax;
    uint32_t* keys = reinterpret_cast<uint32_t*>(cnts + kGbExtractMax);
    __shared__ uint32_t wtot[32];
    constexpr uint32_t PER = kGbExtractMax / kGbExtractThreads;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint64_t c[PER];
    uint32_t n = 0;
#pragma unroll
    for (uint32_t j = 0; j < PER; j++) {
        const uint32_t i = tid * PER + j;
        c[j] = i < g ? gcnt[i] : 0;
        n += c[j] != 0;
    }
    uint32_t incl = n;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) wtot[warp] = incl;
    __syncthreads();
    uint32_t wpre = lane < 32 ? wtot[lane] : 0;  // every warp scans the 32 warp totals itself
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, wpre, o);
        if (lane >= (uint32_t)o) wpre += y;
    }
    const uint32_t total = __shfl_sync(0xffffffffu, wpre, 31);
    const uint32_t before = warp ? __shfl_sync(0xffffffffu, wpre, warp - 1) : 0;
    uint32_t pos = before + incl - n;
#pragma unroll
    for (uint32_t j = 0; j < PER; j++) {
        if (c[j]) {
            const uint32_t i = tid * PER + j;
            keys[pos] = i;
            sums[pos] = gsum[i];
            cnts[pos] = c[j];
            pos++;
        }
    }
    __syncthreads();
    if (has & 1) encode_tile<uint32_t>(ok, keys, total, 0, true, tid, kGbExtractThreads);
    if (has & 2) encode_tile<uint64_t>(os, sums, total, 0, true, tid, kGbExtractThreads);
    if (has & 4) encode_tile<uint64_t>(oc, cnts, total, 0, true, tid, kGbExtractThreads);
    if (tid == 0 && d_groups) *d_groups = total;
}

__global__ void iota_kernel(uint32_t* out, uint64_t n)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) out[i] = (uint32_t)i;
}

// ---- extraction for wide keys: hash slots -> ascending keys ----------------------------------
// The keys of the occupied slots are distinct, so the position of a key in ascending order is the
// number of present keys below it: mark every present key in a bitmap of the key space, count
// the bits of every 256-bit group, scan those counts (per 2048-group block, then the block
// totals), and a key's position is its block's offset + its group's offset inside the block +
// the set bits before it in its group.
constexpr uint32_t kGwGroupWords = 8;     // 32-bit bitmap words per group (256 keys)
constexpr uint32_t kGwBlockGroups = 2048; // groups per scan block

__global__ void gw_mark_kernel(const unsigned long long* gkey, const unsigned long long* gcnt, uint64_t slots,
                               uint32_t* bitmap)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += stride)
        if (gcnt[s]) {
            const uint32_t key = (uint32_t)gkey[s];
            atomicOr(bitmap + (key >> 5), 1u << (key & 31));
        }
}

// one CTA of 1024 threads per block of 2048 groups: exclusive in-block prefix of the groups'
// set bits, and the block's total
__global__ void __launch_bounds__(1024) gw_scan_blocks_kernel(const uint32_t* bitmap, uint64_t groups, uint32_t* gpre,
                                                              uint64_t* btot)
{
    __shared__ uint32_t wt[32];
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t g0 = (uint64_t)blockIdx.x * kGwBlockGroups + 2 * tid;
    uint32_t c[2] = {0, 0};
    for (int q = 0; q < 2; q++)
        if (g0 + q < groups) {
            const uint4* w = reinterpret_cast<const uint4*>(bitmap + (g0 + q) * kGwGroupWords);
            const uint4 a = w[0], b = w[1];
            c[q] = __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w) + __popc(b.x) + __popc(b.y) + __popc(b.z) +
                   __popc(b.w);
        }
    const uint32_t mine = c[0] + c[1];
    uint32_t incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= (uint32_t)o) incl += y;
    }
    if (lane == 31) wt[warp] = incl;
    __syncthreads();
    uint32_t wp = wt[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, wp, o);
        if (lane >= (uint32_t)o) wp += y;
    }
    const uint32_t before = (warp ? __shfl_sync(0xffffffffu, wp, warp - 1) : 0) + incl - mine;
    if (g0 < groups) gpre[g0] = before;
    if (g0 + 1 < groups) gpre[g0 + 1] = before + c[0];
    if (tid == 1023) btot[blockIdx.x] = wp;  // lane 31's inclusive scan of the warp totals: the block's total
}

// one CTA: exclusive scan of the block totals in place; the grand total is the number of groups
__global__ void __launch_bounds__(1024) gw_scan_top_kernel(uint64_t* btot, uint64_t blocks, uint64_t* d_groups)
{
    __shared__ unsigned long long wt[32];
    __shared__ unsigned long long carry;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) carry = 0;
    __syncthreads();
    for (uint64_t base = 0; base < blocks; base += 1024) {
        const uint64_t i = base + tid;
        const unsigned long long v = i < blocks ? btot[i] : 0;
        unsigned long long incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (uint32_t)o) incl += y;
        }
        if (lane == 31) wt[warp] = incl;
        __syncthreads();
        unsigned long long wp = wt[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, wp, o);
            if (lane >= (uint32_t)o) wp += y;
        }
        const unsigned long long before = (warp ? __shfl_sync(0xffffffffu, wp, warp - 1) : 0) + incl - v;
        const unsigned long long c0 = carry;
        if (i < blocks) btot[i] = c0 + before;
        __syncthreads();
        if (tid == 1023) carry = c0 + wp;  // lane 31's inclusive scan: this round's total
        __syncthreads();
    }
    if (tid == 0) *d_groups = carry;
}

// every occupied slot writes its key, sum and count at the key's ascending position (plain
// arrays of `cap` entries; positions at or past cap are counted as a capacity error)
__global__ void gw_place_kernel(const unsigned long long* gkey, const unsigned long long* gsum,
                                const unsigned long long* gcnt, uint64_t slots, const uint32_t* bitmap,
                                const uint32_t* gpre, const uint64_t* boff, uint32_t* okey, uint64_t* osum,
                                uint64_t* ocnt, uint64_t cap, uint32_t* err)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < slots; s += stride) {
        const uint64_t c = gcnt[s];
        if (!c) continue;
        const uint32_t key = (uint32_t)gkey[s];
        const uint64_t w = key >> 5, g = w / kGwGroupWords;
        uint64_t pos = boff[g / kGwBlockGroups] + gpre[g];
        for (uint64_t k = g * kGwGroupWords; k < w; k++) pos += __popc(bitmap[k]);
        pos += __popc(bitmap[w] & ((1u << (key & 31)) - 1u));
        if (pos >= cap) {
            record_error(err, AMX_ERR_CAPACITY);
            continue;
        }
        okey[pos] = key;
        osum[pos] = gsum[s];
        ocnt[pos] = c;
    }
}

// the aggregation kernel for a key / value format pair, table kind and carry handling
static const void* gb_kernel(bool kslab, bool vslab, bool dense, bool nocarry)
{
#define AMX_GB(K, V, D, P) reinterpret_cast<const void*>(&groupby_kernel<K, V, D, P>)
#define AMX_GB_PACK(K, V, D) (nocarry ? AMX_GB(K, V, D, true) : AMX_GB(K, V, D, false))
#define AMX_GB_DENSE(K, V) (dense ? AMX_GB_PACK(K, V, true) : AMX_GB_PACK(K, V, false))
    if (kslab) return vslab ? AMX_GB_DENSE(true, true) : AMX_GB_DENSE(true, false);
    return vslab ? AMX_GB_DENSE(false, true) : AMX_GB_DENSE(false, false);
#undef AMX_GB_DENSE
#undef AMX_GB_PACK
#undef AMX_GB
}

static uint64_t align256(uint64_t x) { return (x + 255) & ~255ull; }

struct GbLayout {
    uint64_t sums, counts, iota, mask, ws, total;
};

static GbLayout gb_layout(uint32_t kbits)
{
    const uint64_t g = 1ull << kbits;
    GbLayout l;
    l.sums = 0;
    l.counts = align256(l.sums + 8 * g);
    l.iota = align256(l.counts + 8 * g);
    l.mask = align256(l.iota + 4 * g);
    l.ws = align256(l.mask + 4 * ((g + 31) / 32) + 16);
    l.total = align256(l.ws + amx_workspace_bytes(g));
    return l;
}

uint64_t groupby_pipeline_offset(uint32_t key_bits)
{
    if (key_bits < 1 || key_bits > kGbMaxKeyBits || (1ull << key_bits) <= kGbExtractMax) return ~0ull;
    return gb_layout(key_bits).ws;
}

// Workspace of a wide-key group-by with a `slots`-entry hash table (a power of two):
//   header (error word, group count) | keys | sums | counts | key bitmap | group prefixes |
//   block offsets | placed keys | placed sums | placed counts | pipeline workspace
struct GwLayout {
    uint64_t hdr, keys, sums, counts, bitmap, gpre, boff, okey, osum, ocnt, ws, total;
    uint64_t bitmap_words, groups, blocks;
};

static GwLayout gw_layout(uint32_t kbits, uint64_t slots)
{
    GwLayout l{};
    l.bitmap_words = (1ull << kbits) / 32;
    l.groups = l.bitmap_words / kGwGroupWords;
    l.blocks = (l.groups + kGwBlockGroups - 1) / kGwBlockGroups;
    l.hdr = 0;
    l.keys = 256;
    l.sums = align256(l.keys + 8 * slots);
    l.counts = align256(l.sums + 8 * slots);
    l.bitmap = align256(l.counts + 8 * slots);
    l.gpre = align256(l.bitmap + 4 * l.bitmap_words);
    l.boff = align256(l.gpre + 4 * l.groups);
    l.okey = align256(l.boff + 8 * l.blocks);
    l.osum = align256(l.okey + 4 * slots + 16);
    l.ocnt = align256(l.osum + 8 * slots);
    l.ws = align256(l.ocnt + 8 * slots);
    l.total = align256(l.ws + amx_workspace_bytes(slots));
    return l;
}

// slots of the largest table that a workspace of `bytes` holds (0 if none of at least 1024)
static uint64_t gw_slots_for(uint32_t kbits, uint64_t bytes)
{
    uint64_t best = 0;
    for (uint64_t s = 1024; s <= (1ull << 33) && gw_layout(kbits, s).total <= bytes; s <<= 1) best = s;
    return best;
}

struct GwHeader {
    uint32_t err;
    uint32_t pad;
    uint64_t groups;
};

}  // namespace amx

using namespace amx;

extern "C" {

uint64_t amx_groupby_wide_workspace_bytes(uint32_t key_bits, uint64_t max_groups)
{
    if (key_bits <= kGbMaxKeyBits || key_bits > 32 || max_groups > (1ull << 32)) return 0;
    uint64_t slots = 1024;
    while (slots < 2 * max_groups) slots <<= 1;  // at most half full
    return gw_layout(key_bits, slots).total;
}

amx_status amx_groupby_status(const void* workspace, uint32_t key_bits, void* stream)
{
    if (!workspace) return fail(AMX_ERR_INVALID_ARG, "groupby_status: null workspace");
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "groupby_status: stream");
    uint64_t off = ~0ull;
    if (key_bits > kGbMaxKeyBits)
        off = 0;  // GwHeader::err
    else {
        const uint64_t g = groupby_pipeline_offset(key_bits);
        if (g != ~0ull) off = g + offsetof(WsHeader, err);
    }
    if (off == ~0ull) return AMX_OK;  // groups extracted by one CTA: nothing can fail on the device
    uint32_t err = 0;
    e = cudaMemcpy(&err, static_cast<const uint8_t*>(workspace) + off, sizeof(err), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "groupby_status: read");
    if (err) return fail((amx_status)err, "groupby: device-side failure (%u)", err);
    return AMX_OK;
}

uint64_t amx_groupby_workspace_bytes(uint32_t key_bits)
{
    if (key_bits < 1 || key_bits > kGbMaxKeyBits) return 0;
    return gb_layout(key_bits).total;
}

amx_status amx_groupby(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                       const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                       uint64_t* d_groups, void* ws, size_t ws_bytes, void* stream)
{
    return groupby_run(keys, vals, d_mask, out_keys, out_sums, out_counts, d_groups, ws, ws_bytes, stream, nullptr);
}

}  // extern "C"

namespace amx {

// Launches the aggregation of keys / values into the global table described by p (dense, or the
// wide-key hash table when p.gkey is set).
static amx_status gb_aggregate(GbParams& p, const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                               cudaStream_t s)
{
    cudaError_t e = cudaSuccess;
    if (p.n) {
        if (vals->bits <= 32) {
            // (wide keys with carry words and one flush per CTA measured 4.53 ms against 2.64 ms on
            // 2^26 keys over 100,000 groups: the returning shared atomics of the carry path cost
            // more than the flushes into the hash table)
            const bool nocarry = vals->bits <= kGbNoCarryBits;
            p.flush_every = nocarry ? gb_flush_every(vals->bits) : kGbFlushEvery;
            const uint32_t slots = p.dense ? (1u << p.kbits) : kGbHashSlots;
            size_t smem = 16ull * slots;
            p.copies = 1;
            const void* fn = gb_kernel(keys->format == AMX_SLAB, vals->format == AMX_SLAB, p.dense, nocarry);
            // slab keys and values without a mask: runs aligned to both columns' slabs, when
            // their length (a multiple of the field counts' lcm) stays short and a chunk of them
            // fits between two flushes
            if (keys->format == AMX_SLAB && vals->format == AMX_SLAB && !d_mask) {
                const uint32_t ek = p.k.eps, ev = p.v.eps;
                const uint32_t l = ek / gcd_u32(ek, ev) * ev;
                const uint32_t run = l <= 64 ? l * ((32 + l - 1) / l) : 0;
                if (run && run <= 64 && (uint64_t)kGbThreads * run <= p.flush_every) {
                    p.run = run;
                    // two copies of the sums and counts while the table stays within 54 KB (four
                    // 512-thread CTAs per SM still fit); 2^26 Zipf keys over 1000 groups at 10
                    // bits: 0.131 ms with one copy, 0.124 with two, 0.133 with four
                    while (p.copies < kGbCopies && 4ull * slots + 12ull * slots * (2 * p.copies) <= 54 * 1024) p.copies *= 2;
                    smem = 4ull * slots + 12ull * slots * p.copies;
                    fn = p.dense ? (nocarry ? reinterpret_cast<const void*>(&groupby_phase_kernel<true, true>)
                                            : reinterpret_cast<const void*>(&groupby_phase_kernel<true, false>))
                                 : (nocarry ? reinterpret_cast<const void*>(&groupby_phase_kernel<false, true>)
                                            : reinterpret_cast<const void*>(&groupby_phase_kernel<false, false>));
                }
            }
            e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return cuda_fail(e, "groupby: shared memory attribute");
            int per_sm = 0;
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kGbThreads, smem);
            uint64_t grid = (uint64_t)(per_sm > 0 ? per_sm : 1) * sm_count();
            const uint64_t chunk_elems = p.run ? (uint64_t)kGbThreads * p.run : kGbChunk;
            const uint64_t chunks = (p.n + chunk_elems - 1) / chunk_elems;
            if (grid > chunks) grid = chunks;
            if (tuning().max_ctas && grid > tuning().max_ctas) grid = tuning().max_ctas;
            void* args[] = {&p};
            e = cudaLaunchKernel(fn, dim3((unsigned)grid), dim3(kGbThreads), args, smem, s);
            if (e != cudaSuccess) return cuda_fail(e, "groupby: aggregation launch");
        }
        else {
            groupby_wide_kernel<<<sm_count() * 8, 256, 0, s>>>(p);
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "groupby: aggregation launch");
    }
    return AMX_OK;
}

// Keys of 25..32 bits: a global hash table sized by the workspace replaces the dense table; the
// groups come out in ascending key order through the bitmap ranks (gw_*_kernel) and are encoded
// into the caller's columns by the tile pipeline, reading the group count on the device.
static amx_status groupby_wide(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                               const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                               uint64_t* d_groups, void* ws, size_t ws_bytes, void* stream, const uint64_t* n_dev)
{
    amx_status st = AMX_OK;
    if (!ws || ((uintptr_t)ws) & 255) return fail(AMX_ERR_ALIGNMENT, "groupby: workspace null or not 256-byte aligned");
    const uint32_t kbits = keys->bits;
    const uint64_t slots = gw_slots_for(kbits, ws_bytes);
    if (!slots)
        return fail(AMX_ERR_WORKSPACE, "groupby: workspace of %zu bytes holds no hash table (%llu needed at least)",
                    ws_bytes, (unsigned long long)gw_layout(kbits, 1024).total);
    const GwLayout L = gw_layout(kbits, slots);
    const amx_column* outs[3] = {out_keys, out_sums, out_counts};
    const char* names[3] = {"groupby: out_keys", "groupby: out_sums", "groupby: out_counts"};
    uint64_t cap = slots;
    for (int i = 0; i < 3; i++) {
        if (!outs[i]) continue;
        if ((st = check_column(outs[i], names[i]))) return st;
        if (outs[i]->n < cap) cap = outs[i]->n;
    }
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* w = static_cast<uint8_t*>(ws);
    GwHeader* hdr = reinterpret_cast<GwHeader*>(w + L.hdr);
    cudaError_t e = cudaMemsetAsync(w, 0, 256, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(w + L.keys, 0xff, 8 * slots, s);  // every slot free
    if (e == cudaSuccess) e = cudaMemsetAsync(w + L.sums, 0, L.bitmap + 4 * L.bitmap_words - L.sums, s);
    if (e != cudaSuccess) return cuda_fail(e, "groupby: table clear");

    GbParams p{};
    p.k = col_dev(keys);
    p.v = col_dev(vals);
    p.mask = d_mask;
    p.n = keys->n;
    p.kbits = kbits;
    p.dense = 0;
    p.gsum = reinterpret_cast<unsigned long long*>(w + L.sums);
    p.gcnt = reinterpret_cast<unsigned long long*>(w + L.counts);
    p.gkey = reinterpret_cast<unsigned long long*>(w + L.keys);
    p.gcap_mask = slots - 1;
    p.gshift = 64 - (uint32_t)__builtin_ctzll(slots);
    p.err = &hdr->err;
    p.n_dev = n_dev;
    if ((st = gb_aggregate(p, keys, vals, d_mask, s))) return st;

    uint32_t* bitmap = reinterpret_cast<uint32_t*>(w + L.bitmap);
    uint32_t* gpre = reinterpret_cast<uint32_t*>(w + L.gpre);
    uint64_t* boff = reinterpret_cast<uint64_t*>(w + L.boff);
    uint64_t* groups = d_groups ? d_groups : &hdr->groups;
    const unsigned grid = (unsigned)(sm_count() * 8);
    gw_mark_kernel<<<grid, 256, 0, s>>>(p.gkey, p.gcnt, slots, bitmap);
    gw_scan_blocks_kernel<<<(unsigned)L.blocks, 1024, 0, s>>>(bitmap, L.groups, gpre, boff);
    gw_scan_top_kernel<<<1, 1024, 0, s>>>(boff, L.blocks, groups);
    uint32_t* okey = reinterpret_cast<uint32_t*>(w + L.okey);
    uint64_t* osum = reinterpret_cast<uint64_t*>(w + L.osum);
    uint64_t* ocnt = reinterpret_cast<uint64_t*>(w + L.ocnt);
    gw_place_kernel<<<grid, 256, 0, s>>>(p.gkey, p.gsum, p.gcnt, slots, bitmap, gpre, boff, okey, osum, ocnt, cap,
                                         &hdr->err);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "groupby: extraction launch");
    // the placed groups into the caller's columns (any format), as many as the device count says
    const amx_column tk{okey, cap, AMX_PLAIN32, 32}, ts{osum, cap, AMX_PLAIN64, 64}, tc{ocnt, cap, AMX_PLAIN64, 64};
    const amx_column* srcs[3] = {&tk, &ts, &tc};
    for (int i = 0; i < 3; i++) {
        if (!outs[i]) continue;
        ChainReq r{};
        r.a = srcs[i];
        r.vbits = outs[i]->bits;
        r.out = outs[i];
        r.n_dev = groups;
        if ((st = run_chain(r, w + L.ws, L.total - L.ws, s))) return st;
    }
    return AMX_OK;
}

amx_status groupby_run(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                       const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                       uint64_t* d_groups, void* ws, size_t ws_bytes, void* stream, const uint64_t* n_dev)
{
    amx_status st = check_column(keys, "groupby: keys");
    if (st) return st;
    if ((st = check_column(vals, "groupby: values"))) return st;
    if (keys->n != vals->n) return fail(AMX_ERR_INVALID_ARG, "groupby: keys and values lengths differ");
    if (keys->bits > 32) return fail(AMX_ERR_UNSUPPORTED, "groupby: keys of %u bits (at most 32)", keys->bits);
    if (((uintptr_t)d_mask) & 15) return fail(AMX_ERR_ALIGNMENT, "groupby: mask not 16-byte aligned");
    if (keys->bits > kGbMaxKeyBits)
        return groupby_wide(keys, vals, d_mask, out_keys, out_sums, out_counts, d_groups, ws, ws_bytes, stream, n_dev);
    const uint64_t g = 1ull << keys->bits;
    const amx_column* outs[3] = {out_keys, out_sums, out_counts};
    const char* names[3] = {"groupby: out_keys", "groupby: out_sums", "groupby: out_counts"};
    for (int i = 0; i < 3; i++) {
        if (!outs[i]) continue;
        if ((st = check_column(outs[i], names[i]))) return st;
        if (outs[i]->n < g) return fail(AMX_ERR_INVALID_ARG, "%s: capacity below 2^key_bits", names[i]);
    }
    const GbLayout L = gb_layout(keys->bits);
    if (!ws || ws_bytes < L.total)
        return fail(AMX_ERR_WORKSPACE, "groupby: workspace of %zu bytes, %llu needed", ws_bytes,
                    (unsigned long long)L.total);
    if (((uintptr_t)ws) & 255) return fail(AMX_ERR_ALIGNMENT, "groupby: workspace not 256-byte aligned");
    cudaStream_t s = (cudaStream_t)stream;
    uint8_t* w = static_cast<uint8_t*>(ws);
    cudaError_t e = cudaMemsetAsync(w, 0, L.iota, s);  // sums and counts
    if (e != cudaSuccess) return cuda_fail(e, "groupby: table clear");

    GbParams p{};
    p.k = col_dev(keys);
    p.v = col_dev(vals);
    p.mask = d_mask;
    p.n = keys->n;
    p.kbits = keys->bits;
    p.dense = keys->bits <= kGbDenseBits;
    p.gsum = reinterpret_cast<unsigned long long*>(w + L.sums);
    p.gcnt = reinterpret_cast<unsigned long long*>(w + L.counts);
    p.n_dev = n_dev;
    if ((st = gb_aggregate(p, keys, vals, d_mask, s))) return st;
    // groups: keys with a nonzero count, ascending
    if (g <= kGbExtractMax) {
        OutDev od[3] = {};
        uint32_t has = 0;
        for (int i = 0; i < 3; i++)
            if (outs[i]) {
                od[i] = out_dev(outs[i]);
                has |= 1u << i;
            }
        e = cudaFuncSetAttribute(gb_extract_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGbExtractSmem);
        if (e != cudaSuccess) return cuda_fail(e, "groupby: extraction shared memory attribute");
        gb_extract_kernel<<<1, kGbExtractThreads, kGbExtractSmem, s>>>(
            reinterpret_cast<const unsigned long long*>(w + L.sums), reinterpret_cast<const unsigned long long*>(w + L.counts),
            (uint32_t)g, od[0], od[1], od[2], has, d_groups);
        if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "groupby: extraction launch");
        return AMX_OK;
    }
    iota_kernel<<<(unsigned)((g + 255) / 256 < 4096 ? (g + 255) / 256 : 4096), 256, 0, s>>>(
        reinterpret_cast<uint32_t*>(w + L.iota), g);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "groupby: iota launch");
    amx_column counts{w + L.counts, g, AMX_PLAIN64, 64};
    amx_column sums{w + L.sums, g, AMX_PLAIN64, 64};
    amx_column iota{w + L.iota, g, AMX_PLAIN32, 32};
    uint32_t* mask = reinterpret_cast<uint32_t*>(w + L.mask);
    void* pws = w + L.ws;
    const size_t pws_bytes = L.total - L.ws;
    const amx_predicate nonzero{AMX_PRED_NE, 64, 0, 0};
    if ((st = amx_filter(&counts, &nonzero, mask, pws, pws_bytes, stream))) return st;
    const amx_column* srcs[3] = {&iota, &sums, &counts};
    bool counted = false;
    for (int i = 0; i < 3; i++) {
        if (!outs[i]) continue;
        if ((st = amx_compressstore(srcs[i], mask, outs[i], counted ? nullptr : d_groups, pws, pws_bytes, stream)))
            return st;
        counted = true;
    }
    if (!counted && d_groups) {  // no output column: count the groups only
        amx_chain_desc d{AMX_OP_LHS, 64, nonzero, AMX_AGG_SUM, 0};
        if ((st = amx_chain(&d, &counts, nullptr, nullptr, nullptr, d_groups, nullptr, pws, pws_bytes, stream)))
            return st;
    }
    return AMX_OK;
}

}  // namespace amx
