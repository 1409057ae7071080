// amethyst.hpp -- C++ host mirror of the reference's operator launchers on top of the C ABI.
//
// The reference sketches its host-facing API as templates in src/lib.cuh:4-46 (dead code there:
// it includes files that do not exist).  This header keeps those names, template parameters and
// argument meanings, and routes every call through libamethyst_b200.so:
//
//   reference (src/lib.cuh)                                     here
//   binary_op_baseline<bits, op>(d_lhs, d_rhs, d_out, n)        same, op = amx_binop
//   binary_op_nogaps<bits, outbits, op, block>(.., n, grid)     same; grid/block accepted and ignored
//   binary_op_slabs<bits, outbits, op, block>(.., n, grid)      same; grid/block accepted and ignored
//   compressstore_baseline_cub<bits>(d_mask, d_elem, d_out, n)  same, returns the survivor count
//   filter_baseline<bits, predicate, block>(d_elem, d_mask, n, grid)  predicate = amx_predicate value
//
// and adds the slab and nogaps forms of filter / compressstore / hop (aggregation) that the
// reference only has as kernels (src/kernels/*.cuh).  The persistent grid is sized by the library,
// so the reference's grid and block parameters have no effect.
//
// Errors: the reference prints and exits (src/cuda_try.cuh:8-21); this mirror throws
// amethyst::error carrying the amx_status instead.  Workspaces: the C ABI never allocates; this
// convenience layer keeps one growing device workspace per host thread (cudaMalloc on first use).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "amethyst.h"

namespace amethyst {

struct error : std::runtime_error {
    amx_status status;
    error(amx_status s, const std::string& what) : std::runtime_error(what), status(s) {}
};

inline void check(amx_status s)
{
    if (s != AMX_OK) throw error(s, std::string(amx_status_string(s)) + ": " + amx_last_error());
}

struct ws_state {
    void* ws = nullptr;
    size_t cap = 0;
    uint64_t* scalars = nullptr;  // 8 device words for counts read back by the host
};

inline ws_state& ws_local()
{
    thread_local ws_state st;
    return st;
}

inline void* workspace(uint64_t n, size_t* bytes)
{
    ws_state& st = ws_local();
    const size_t need = (size_t)amx_workspace_bytes(n);
    if (need > st.cap) {
        if (st.ws) cudaFree(st.ws);
        st.ws = nullptr;
        if (cudaMalloc(&st.ws, need + 64) != cudaSuccess) throw error(AMX_ERR_CUDA, "workspace allocation failed");
        st.cap = need;
        st.scalars = reinterpret_cast<uint64_t*>(static_cast<uint8_t*>(st.ws) + need);
    }
    *bytes = st.cap;
    return st.ws;
}

inline amx_column column(void* d, uint64_t n, amx_format f, uint32_t bits) { return amx_column{d, n, (uint32_t)f, bits}; }

// FILTER_PREDICATE_OP<bits> of src/config.cuh:107-113
template <size_t bits>
inline amx_predicate pred_half()
{
    return amx_predicate{AMX_PRED_HALF, (uint32_t)bits, 0, 0};
}
inline amx_predicate pred(amx_pred_kind k, uint64_t k0 = 0, uint64_t k1 = 0, uint32_t bits = 0)
{
    return amx_predicate{(uint32_t)k, bits, k0, k1};
}

// ---- the launchers of src/lib.cuh ------------------------------------------------------------
template <size_t bits, amx_binop op>
void binary_op_baseline(uint64_t* d_lhs, uint64_t* d_rhs, uint64_t* d_out, size_t n, cudaStream_t s = 0)
{
    const uint32_t ob = amx_binary_out_bits(op, bits, bits);
    amx_column l = column(d_lhs, n, AMX_PLAIN64, bits), r = column(d_rhs, n, AMX_PLAIN64, bits);
    amx_column o = column(d_out, n, AMX_PLAIN64, ob);
    size_t wb;
    void* ws = workspace(n, &wb);
    check(amx_binary(op, &l, &r, &o, ws, wb, s));
}

template <size_t bits, size_t outbits, amx_binop op, size_t block_size = 256>
void binary_op_nogaps(uint64_t* d_lhs, uint64_t* d_rhs, uint64_t* d_out, size_t n, size_t /*grid_size*/ = 0,
                      cudaStream_t s = 0)
{
    amx_column l = column(d_lhs, n, AMX_NOGAPS, bits), r = column(d_rhs, n, AMX_NOGAPS, bits);
    amx_column o = column(d_out, n, AMX_NOGAPS, outbits);
    size_t wb;
    void* ws = workspace(n, &wb);
    check(amx_binary(op, &l, &r, &o, ws, wb, s));
}

template <size_t bits, size_t outbits, amx_binop op, size_t block_size = 256>
void binary_op_slabs(uint64_t* d_lhs, uint64_t* d_rhs, uint64_t* d_out, size_t n, size_t /*grid_size*/ = 0,
                     cudaStream_t s = 0)
{
    amx_column l = column(d_lhs, n, AMX_SLAB, bits), r = column(d_rhs, n, AMX_SLAB, bits);
    amx_column o = column(d_out, n, AMX_SLAB, outbits);
    size_t wb;
    void* ws = workspace(n, &wb);
    check(amx_binary(op, &l, &r, &o, ws, wb, s));
}

// the mask is the reference's LSB-first bit array (src/bit_iterator.cuh:18-21); it must be
// readable as uint32 words, i.e. 16-byte aligned like any cudaMalloc pointer
template <size_t bits>
size_t compressstore_baseline_cub(uint8_t* d_mask, uint64_t* d_elements, uint64_t* d_out, size_t n, cudaStream_t s = 0)
{
    amx_column in = column(d_elements, n, AMX_PLAIN64, bits), out = column(d_out, n, AMX_PLAIN64, bits);
    size_t wb;
    void* ws = workspace(n, &wb);
    uint64_t* d_count = ws_local().scalars;
    check(amx_compressstore(&in, reinterpret_cast<const uint32_t*>(d_mask), &out, d_count, ws, wb, s));
    uint64_t count = 0;
    if (cudaMemcpyAsync(&count, d_count, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        throw error(AMX_ERR_CUDA, "reading the survivor count failed");
    return (size_t)count;
}

template <size_t bits, size_t block_size = 256>
void filter_baseline(uint64_t* d_elements, uint64_t* d_output_bitmask, size_t n, const amx_predicate& p,
                     size_t /*grid_size*/ = 0, cudaStream_t s = 0)
{
    amx_column in = column(d_elements, n, AMX_PLAIN64, bits);
    size_t wb;
    void* ws = workspace(n, &wb);
    check(amx_filter(&in, &p, reinterpret_cast<uint32_t*>(d_output_bitmask), ws, wb, s));
}

// ---- slab / nogaps forms of the reference's kernels ------------------------------------------
// kernel_filter_slabs / kernel_filter_nogaps (src/kernels/filter_slabs.cuh:4-57, filter_nogaps.cuh:4-65)
template <size_t bits>
void filter(amx_format fmt, uint64_t* d_data, size_t n, uint64_t* d_bitmask, const amx_predicate& p, cudaStream_t s = 0)
{
    amx_column in = column(d_data, n, fmt, bits);
    size_t wb;
    void* ws = workspace(n, &wb);
    check(amx_filter(&in, &p, reinterpret_cast<uint32_t*>(d_bitmask), ws, wb, s));
}

// popcount -> scan -> kernel_compresstore_slabs_write (src/benchs/bench_compressstore_slabs.cu:38-56);
// the count stays on the device
template <size_t bits>
void compressstore_slabs(const uint8_t* d_mask, uint64_t* d_elements, uint64_t* d_out, size_t n, uint64_t* d_count,
                         cudaStream_t s = 0)
{
    amx_column in = column(d_elements, n, AMX_SLAB, bits), out = column(d_out, n, AMX_SLAB, bits);
    size_t wb;
    void* ws = workspace(n, &wb);
    check(amx_compressstore(&in, reinterpret_cast<const uint32_t*>(d_mask), &out, d_count, ws, wb, s));
}

// kernel_hop_slabs / kernel_hop_nogaps (src/kernels/hop.cuh:7-76): HOP_OP = sum into d_out
template <size_t bits>
void hop(amx_format fmt, uint64_t* d_data, size_t n, uint64_t* d_out, amx_agg agg = AMX_AGG_SUM, cudaStream_t s = 0)
{
    amx_column in = column(d_data, n, fmt, bits);
    size_t wb;
    void* ws = workspace(n, &wb);
    check(amx_reduce(agg, &in, nullptr, d_out, ws, wb, s));
}

// ---- operator-chain programs and graphs (amx_program_*, amx_graph_*) -------------------------
// RAII owners: a program plans its steps and holds its device workspace (cudaMalloc once, at
// construction); a graph captures programs once and replays them.  The reference has no
// counterpart: it runs operators one at a time (src/op_chaining_demo.cu:137-152).
class program {
  public:
    program(const amx_column& x, const std::vector<amx_step>& steps)
    {
        check(amx_program_create(&x, steps.data(), (uint32_t)steps.size(), &p_));
        bytes_ = (size_t)amx_program_workspace_bytes(p_);
        if (cudaMalloc(&ws_, bytes_) != cudaSuccess) {
            amx_program_destroy(p_);
            throw error(AMX_ERR_CUDA, "program workspace allocation failed");
        }
    }
    program(const program&) = delete;
    program& operator=(const program&) = delete;
    ~program()
    {
        cudaFree(ws_);
        amx_program_destroy(p_);
    }
    void run(cudaStream_t s = 0) { check(amx_program_run(p_, ws_, bytes_, s)); }
    // the final column of the last run and a device pointer to its length (nullptr: x.n)
    amx_column output(const uint64_t** d_len) const
    {
        amx_column c{};
        check(amx_program_output(p_, ws_, &c, d_len));
        return c;
    }
    void status(cudaStream_t s = 0) const { check(amx_program_status(p_, ws_, s)); }
    const amx_program* get() const { return p_; }
    void* workspace() const { return ws_; }
    uint64_t workspace_bytes() const { return bytes_; }

  private:
    amx_program* p_ = nullptr;
    void* ws_ = nullptr;
    size_t bytes_ = 0;
};

class graph {
  public:
    graph(const std::vector<const program*>& progs, uint32_t lanes)
    {
        std::vector<const amx_program*> h;
        std::vector<void*> ws;
        std::vector<uint64_t> wb;
        for (const program* p : progs) {
            h.push_back(p->get());
            ws.push_back(p->workspace());
            wb.push_back(p->workspace_bytes());
        }
        check(amx_graph_capture(h.data(), ws.data(), wb.data(), (uint32_t)h.size(), lanes, &g_));
    }
    graph(const graph&) = delete;
    graph& operator=(const graph&) = delete;
    ~graph() { amx_graph_destroy(g_); }
    void launch(cudaStream_t s = 0) const { check(amx_graph_launch(g_, s)); }

  private:
    amx_graph* g_ = nullptr;
};

}  // namespace amethyst
