// amx_internal.h -- definitions shared by the host launchers and the kernels.
#pragma once

#include <cstddef>
#include <cstdint>

#include "../../include/amethyst.h"

namespace amx {

// Upper bound of the polls of one look-back status word (each poll after the eighth backs off
// with __nanosleep): well above a second of waiting.  mbarrier waits have their own bound
// (amx_device.cuh: kWaitSuspends suspensions of kWaitSuspendNs).
constexpr uint32_t kWaitSpins = 1u << 20;

// A column as the kernels see it.
struct ColDev {
    const void* data;
    uint64_t n;
    uint64_t bytes;  // storage bytes
    uint64_t mask;   // mask(bits)
    uint32_t format;
    uint32_t bits;
    uint32_t eps;    // elements per slab (slab format), else 0
    uint32_t magic;    // floor(2^32 / eps) + 1 for eps >= 2: x / eps == umulhi(x, magic) for x < 2^17
    uint64_t magic64;  // floor(2^64 / eps) + 1 for eps >= 2: n / eps == umul64hi(n, magic64) for n < 2^58
};

// Output column as the kernels see it.
struct OutDev {
    void* data;
    uint64_t mask;
    uint32_t format;
    uint32_t bits;
    uint32_t eps;
    uint32_t pad;
    uint64_t eps_m64;   // 64-bit magic divisors (see ColDev::magic64) for eps and for bits
    uint64_t bits_m64;
};

// Workspace header, followed by one uint64 look-back status word per tile.
struct WsHeader {
    uint32_t ticket;  // next tile to hand out
    uint32_t done;    // CTAs finished
    uint32_t err;     // first device-side error (amx_status), 0 if none
    uint32_t pad0;
    unsigned long long count;  // survivors over all tiles
    unsigned long long agg;    // encoded aggregate (identity 0)
    uint64_t pad1[4];
};
static_assert(sizeof(WsHeader) == 64, "workspace header layout");

constexpr uint32_t kFmtMask = 7;  // internal format tag of an input bitmask column
constexpr uint32_t kMaxStages = 8;  // depth of the shared-memory staging ring (runtime: PipeParams::stages)
constexpr uint32_t kMaxSlots = 4;   // gathered-value slots of a compacting pass (runtime: PipeParams::slots)

// Parameters of the tile pipeline kernel (passed by value as a __grid_constant__).
struct PipeParams {
    ColDev a;
    ColDev b;
    ColDev m;  // optional input bitmask (format = AMX_PLAIN32, bits = 32), data NULL if none
    OutDev out;
    uint32_t has_b;
    uint32_t has_mask_in;
    uint32_t has_out;
    uint32_t compact;  // 1: survivors are compacted (look-back); 0: element-wise map
    uint32_t op;
    uint32_t vbits;
    uint64_t vmask;
    uint64_t pred_lo;
    uint64_t pred_span;
    uint32_t pred_neg;
    uint32_t has_pred;
    uint32_t pred_lo32;   // 32-bit form of the predicate for values < 2^32 (pred32_ok)
    uint32_t pred_span32;
    uint32_t pred32_ok;
    uint32_t need_vmask;  // 0 when op results provably fit vbits (masking is a no-op)
    uint32_t agg;
    uint32_t has_agg;
    uint32_t* mask_out;
    uint64_t* count_out;
    uint64_t* agg_out;
    WsHeader* ws;
    uint64_t* status;
    uint64_t n;            // elements (the capacity when n_dev is set)
    uint64_t num_tiles;    // tiles of n elements
    const uint64_t* n_dev; // optional device-resident length: the kernel runs min(n, *n_dev) elements
    uint32_t tile_elems;
    uint32_t stage_bytes;  // bytes of one pipeline stage (a | b | m buffers)
    uint32_t stages;       // stages in the ring, 2..kMaxStages
    uint32_t slots;        // gathered-value slots between compute and encoder warps, 1..kMaxSlots
    uint32_t slot_bytes;   // bytes of one slot
    uint32_t cv16;         // gathered values stored as 16-bit words (value width <= 16)
    uint32_t stage_target;          // bytes of input to keep staged ahead (sets the ring depth)
    uint32_t stage_target_compact;  // ring depth of compacting passes
    uint32_t a_off, b_off, m_off;  // offsets of the buffers inside a stage
    uint64_t a_stride, b_stride, m_stride;  // bytes per tile when tiles fall on word boundaries, else 0
    uint32_t smem_fixed;           // bytes before the first stage
    // field-parallel predicate of the slab-word policies (SwarPol): the passing field values
    // form the interval [lo, hi1) or its complement; sw_l1 / sw_l2 are lo and hi1 repeated in
    // every field with the field's top bit cleared, sw_h has the top bit of every field set
    uint32_t sw_mode;  // kSw* bits
    uint32_t wait_polls;      // polls of a look-back status word before giving up (kWaitSpins)
    uint64_t withhold_plus1;  // test hook: tile + 1 whose count is never published (0: none)
    uint64_t sw_h;
    uint64_t sw_l1;
    uint64_t sw_l2;
};

// SwarPol predicate modes
constexpr uint32_t kSwLo = 1;      // test v >= lo
constexpr uint32_t kSwHi = 2;      // test v < hi1
constexpr uint32_t kSwLoTop = 4;   // top bit of lo's field
constexpr uint32_t kSwHiTop = 8;   // top bit of hi1's field
constexpr uint32_t kSwNeg = 16;    // complement the result
constexpr uint32_t kSwNone = 32;   // no value passes (before the complement)

}  // namespace amx
