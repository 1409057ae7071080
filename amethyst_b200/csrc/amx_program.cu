// amx_program.cu -- operator-chain programs and the CUDA graphs that batch them.
//
// A program is a chain of steps over one column (filter, compressstore, binary op, reduce,
// group-by).  Lengths that a step produces stay in device memory: the compressstore's last CTA
// writes its survivor count into a length slot of the program's workspace, and every later
// kernel reads its element count from there (PipeParams::n_dev, GbParams::n_dev).  A run is
// therefore a fixed sequence of stream-ordered launches with no host round trip, which a CUDA
// graph can capture once and replay.  The reference runs its operators one by one with the
// count copied to the host in between (src/op_chaining_demo.cu:137-152,
// src/benchs/bench_compressstore_slabs.cu:60-62).
//
// Workspace layout (every part 256-byte aligned):
//   length slots       one uint64 per step
//   pipeline headers   one amx_workspace_bytes(n) area per step (each keeps its own error word)
//   mask               the live filter mask, amx_mask_bytes(n) + 16
//   buffers 0 and 1    ping-pong storage of the produced columns (the widest one at capacity n)
//   group-by           one group-by workspace per group-by step (its own error word when the
//                      groups are extracted by the tile pipeline)
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "amx_dispatch.h"

namespace amx {

static uint64_t al256(uint64_t x) { return (x + 255) & ~255ull; }

}  // namespace amx

using namespace amx;

struct amx_program {
    amx_column x;
    std::vector<amx_step> steps;
    uint64_t len_off, pipe_off, pipe_bytes, mask_off, buf_off[2], buf_bytes, total;
    std::vector<uint64_t> gb_off;  // per step: offset of its group-by workspace (group-by steps)
    // how each step runs: merged steps launch nothing of their own
    std::vector<uint8_t> merged;   // runs inside another step's pass
    std::vector<int> pred_from;    // COMPRESSSTORE: the FILTER whose predicate it applies, else -1
    std::vector<int> fused_from;   // COMPRESSSTORE: the fused BINARY it evaluates first, else -1
    std::vector<int> agg_from;     // the REDUCE whose aggregate this step's pass also computes, else -1
    // final x after a run: -1 the input, else the buffer index; whether its length is on the device
    int final_buf;
    uint32_t final_format, final_bits;
    int final_len_slot;
};

struct amx_graph {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

namespace amx {

static bool fmt_ok(uint32_t f, uint32_t bits)
{
    if (bits < 1) return false;
    if (f == AMX_PLAIN32) return bits <= 32;
    return f <= AMX_NOGAPS && bits <= 64;
}

static amx_status check_step(const amx_column* x, const amx_step& s, uint32_t i, uint32_t nsteps, const amx_step* all)
{
    char name[64];
    snprintf(name, sizeof(name), "program: step %u aux", i);
    switch (s.kind) {
        case AMX_STEP_FILTER: return AMX_OK;
        case AMX_STEP_COMPRESSSTORE:
            if (!fmt_ok(s.out_format, s.out_bits))
                return fail(AMX_ERR_INVALID_ARG, "program: step %u: output format %u / width %u", i, s.out_format,
                            s.out_bits);
            return AMX_OK;
        case AMX_STEP_BINARY: {
            amx_status st = check_column(&s.aux, name);
            if (st) return st;
            if (s.aux.n < x->n) return fail(AMX_ERR_INVALID_ARG, "program: step %u: aux shorter than x", i);
            if (s.op > AMX_OP_LHS) return fail(AMX_ERR_INVALID_ARG, "program: step %u: unknown op %u", i, s.op);
            if (s.value_bits < 1 || s.value_bits > 64)
                return fail(AMX_ERR_INVALID_ARG, "program: step %u: value_bits must be 1..64", i);
            if (s.out_format == AMX_FORMAT_FUSED) {
                const bool next_cs = i + 1 < nsteps && all[i + 1].kind == AMX_STEP_COMPRESSSTORE;
                const bool filter_cs = i + 2 < nsteps && all[i + 1].kind == AMX_STEP_FILTER &&
                                       all[i + 2].kind == AMX_STEP_COMPRESSSTORE;
                if (!next_cs && !filter_cs)
                    return fail(AMX_ERR_INVALID_ARG, "program: step %u: a fused binary op must precede a compressstore", i);
                return AMX_OK;
            }
            if (!fmt_ok(s.out_format, s.out_bits))
                return fail(AMX_ERR_INVALID_ARG, "program: step %u: output format %u / width %u", i, s.out_format,
                            s.out_bits);
            return AMX_OK;
        }
        case AMX_STEP_REDUCE:
            if (s.op > AMX_AGG_XOR) return fail(AMX_ERR_INVALID_ARG, "program: step %u: unknown aggregation %u", i, s.op);
            if (!s.d_result) return fail(AMX_ERR_INVALID_ARG, "program: step %u: null result", i);
            return AMX_OK;
        case AMX_STEP_GROUPBY: {
            amx_status st = check_column(&s.aux, name);
            if (st) return st;
            if (s.aux.n < x->n) return fail(AMX_ERR_INVALID_ARG, "program: step %u: keys shorter than x", i);
            if (amx_groupby_workspace_bytes(s.aux.bits) == 0)
                return fail(AMX_ERR_UNSUPPORTED, "program: step %u: keys of %u bits", i, s.aux.bits);
            const amx_column* outs[3] = {&s.group_keys, &s.group_sums, &s.group_counts};
            for (int k = 0; k < 3; k++) {
                if (!outs[k]->data) continue;
                if ((st = check_column(outs[k], "program: group output"))) return st;
                if (outs[k]->n < (1ull << s.aux.bits))
                    return fail(AMX_ERR_INVALID_ARG, "program: step %u: group output capacity below 2^key_bits", i);
            }
            return AMX_OK;
        }
    }
    return fail(AMX_ERR_INVALID_ARG, "program: step %u: unknown kind %u", i, s.kind);
}

}  // namespace amx

extern "C" {

amx_status amx_program_create(const amx_column* x, const amx_step* steps, uint32_t nsteps, amx_program** prog)
{
    if (!prog) return fail(AMX_ERR_INVALID_ARG, "program: null output");
    *prog = nullptr;
    amx_status st = check_column(x, "program: x");
    if (st) return st;
    if (nsteps > AMX_PROGRAM_MAX_STEPS) return fail(AMX_ERR_CAPACITY, "program: %u steps (at most %u)", nsteps, AMX_PROGRAM_MAX_STEPS);
    if (nsteps && !steps) return fail(AMX_ERR_INVALID_ARG, "program: null steps");
    for (uint32_t i = 0; i < nsteps; i++)
        if ((st = check_step(x, steps[i], i, nsteps, steps))) return st;

    amx_program* p = new (std::nothrow) amx_program();
    if (!p) return fail(AMX_ERR_CAPACITY, "program: out of host memory");
    p->x = *x;
    p->steps.assign(steps, steps + nsteps);
    const uint64_t n = x->n;
    uint64_t buf = 16;
    p->final_buf = -1;
    p->final_format = x->format;
    p->final_bits = x->bits;
    p->final_len_slot = -1;
    int produced = 0;
    for (uint32_t i = 0; i < nsteps; i++) {
        const amx_step& s = steps[i];
        const bool makes = s.kind == AMX_STEP_COMPRESSSTORE || (s.kind == AMX_STEP_BINARY && s.out_format != AMX_FORMAT_FUSED);
        if (makes) {
            buf = std::max(buf, storage_bytes(s.out_format, s.out_bits, n) + 16);
            p->final_buf = produced++ & 1;
            p->final_format = s.out_format;
            p->final_bits = s.out_bits;
        }
        if (s.kind == AMX_STEP_COMPRESSSTORE) p->final_len_slot = (int)i;
    }
    // Merge the steps one pass can serve: a FILTER whose mask only a COMPRESSSTORE reads becomes
    // that compressstore's predicate; a REDUCE right after a COMPRESSSTORE, a FILTER, or a
    // BINARY op while no mask is live is computed in that step's pass (the aggregate of the
    // survivors, of the passing elements, of all elements).
    p->merged.assign(nsteps, 0);
    p->pred_from.assign(nsteps, -1);
    p->fused_from.assign(nsteps, -1);
    p->agg_from.assign(nsteps, -1);
    bool live = false;
    for (uint32_t i = 0; i < nsteps; i++) {
        if (p->merged[i]) continue;
        const amx_step& s = steps[i];
        const bool next_reduce = i + 1 < nsteps && steps[i + 1].kind == AMX_STEP_REDUCE;
        bool takes_reduce = false;
        switch (s.kind) {
            case AMX_STEP_FILTER:
                if (i + 1 < nsteps && steps[i + 1].kind == AMX_STEP_COMPRESSSTORE) {
                    p->merged[i] = 1;
                    p->pred_from[i + 1] = (int)i;
                }
                else {
                    live = true;
                    takes_reduce = next_reduce;
                }
                break;
            case AMX_STEP_BINARY:
                if (s.out_format == AMX_FORMAT_FUSED)
                    p->merged[i] = 1;
                else
                    takes_reduce = next_reduce && !live;
                break;
            case AMX_STEP_COMPRESSSTORE: {
                int k = (int)i - 1;
                if (p->pred_from[i] >= 0) k = p->pred_from[i] - 1;
                if (k >= 0 && steps[k].kind == AMX_STEP_BINARY && steps[k].out_format == AMX_FORMAT_FUSED)
                    p->fused_from[i] = k;
                live = false;
                takes_reduce = next_reduce;
                break;
            }
            default: break;
        }
        if (takes_reduce) {
            p->agg_from[i] = (int)i + 1;
            p->merged[i + 1] = 1;
        }
    }
    p->pipe_bytes = al256(amx_workspace_bytes(n));
    p->len_off = 0;
    p->pipe_off = al256(8ull * (nsteps ? nsteps : 1));
    p->mask_off = p->pipe_off + p->pipe_bytes * (nsteps ? nsteps : 1);
    p->buf_bytes = al256(buf);
    p->buf_off[0] = al256(p->mask_off + amx_mask_bytes(n) + 16);
    p->buf_off[1] = p->buf_off[0] + p->buf_bytes;
    uint64_t off = p->buf_off[1] + p->buf_bytes;
    p->gb_off.assign(nsteps, 0);
    for (uint32_t i = 0; i < nsteps; i++)
        if (steps[i].kind == AMX_STEP_GROUPBY) {
            p->gb_off[i] = off;
            off += al256(amx_groupby_workspace_bytes(steps[i].aux.bits));
        }
    p->total = off;
    *prog = p;
    return AMX_OK;
}

uint64_t amx_program_workspace_bytes(const amx_program* prog) { return prog ? prog->total : 0; }

amx_status amx_program_run(const amx_program* prog, void* ws, size_t ws_bytes, void* stream)
{
    if (!prog) return fail(AMX_ERR_INVALID_ARG, "program: null program");
    if (!ws || ws_bytes < prog->total)
        return fail(AMX_ERR_WORKSPACE, "program: workspace of %zu bytes, %llu needed", ws_bytes,
                    (unsigned long long)prog->total);
    if (((uintptr_t)ws) & 255) return fail(AMX_ERR_ALIGNMENT, "program: workspace not 256-byte aligned");
    uint8_t* w = static_cast<uint8_t*>(ws);
    uint64_t* lens = reinterpret_cast<uint64_t*>(w + prog->len_off);
    uint32_t* mask = reinterpret_cast<uint32_t*>(w + prog->mask_off);
    const uint64_t n = prog->x.n;
    cudaStream_t s = (cudaStream_t)stream;

    amx_column x = prog->x;          // current column (n = capacity)
    const uint64_t* len = nullptr;   // device-resident length, NULL while it is x.n
    bool mask_live = false;
    int produced = 0;
    const uint32_t ns = (uint32_t)prog->steps.size();
    for (uint32_t i = 0; i < ns; i++) {
        if (prog->merged[i]) continue;  // served by another step's pass
        const amx_step& st = prog->steps[i];
        void* pws = w + prog->pipe_off + (uint64_t)i * prog->pipe_bytes;
        const size_t pwb = prog->pipe_bytes;
        amx_status rc = AMX_OK;
        amx_column aux = st.aux;
        aux.n = n;  // the prefix that pairs with x
        const amx_step* red = prog->agg_from[i] >= 0 ? &prog->steps[prog->agg_from[i]] : nullptr;
        ChainReq r{};
        r.a = &x;
        r.vbits = x.bits;
        r.n_dev = len;
        if (red) {
            r.has_agg = 1;
            r.agg = red->op;
            r.agg_out = red->d_result;
        }
        switch (st.kind) {
            case AMX_STEP_FILTER:
                r.pred = &st.pred;
                r.mask_out = mask;
                rc = run_chain(r, pws, pwb, s);
                mask_live = true;
                break;
            case AMX_STEP_BINARY: {
                const int b = produced++ & 1;
                amx_column out{w + prog->buf_off[b], n, st.out_format, st.out_bits};
                r.b = &aux;
                r.op = st.op;
                r.vbits = st.value_bits;
                r.out = &out;
                rc = run_chain(r, pws, pwb, s);
                x = out;
                break;
            }
            case AMX_STEP_COMPRESSSTORE: {
                const int b = produced++ & 1;
                amx_column out{w + prog->buf_off[b], n, st.out_format, st.out_bits};
                amx_column faux;
                if (prog->fused_from[i] >= 0) {
                    const amx_step& f = prog->steps[prog->fused_from[i]];
                    faux = f.aux;
                    faux.n = n;
                    r.b = &faux;
                    r.op = f.op;
                    r.vbits = f.value_bits;
                }
                if (prog->pred_from[i] >= 0)
                    r.pred = &prog->steps[prog->pred_from[i]].pred;  // the merged filter's predicate
                else if (mask_live)
                    r.mask_in = mask;
                else
                    r.pred = &st.pred;
                // the survivor count: the caller's result slot when given, else the workspace's
                uint64_t* cnt = st.d_result ? st.d_result : lens + i;
                r.out = &out;
                r.compact = 1;
                r.count_out = cnt;
                rc = run_chain(r, pws, pwb, s);
                x = out;
                len = cnt;
                mask_live = false;
                break;
            }
            case AMX_STEP_REDUCE:
                r.mask_in = mask_live ? mask : nullptr;
                r.has_agg = 1;
                r.agg = st.op;
                r.agg_out = st.d_result;
                rc = run_chain(r, pws, pwb, s);
                break;
            case AMX_STEP_GROUPBY: {
                const amx_column* ok = st.group_keys.data ? &st.group_keys : nullptr;
                const amx_column* os = st.group_sums.data ? &st.group_sums : nullptr;
                const amx_column* oc = st.group_counts.data ? &st.group_counts : nullptr;
                rc = groupby_run(&aux, &x, mask_live ? mask : nullptr, ok, os, oc, st.d_result, w + prog->gb_off[i],
                                 amx_groupby_workspace_bytes(st.aux.bits), stream, len);
                break;
            }
        }
        if (rc) return rc;
    }
    return AMX_OK;
}

amx_status amx_program_output(const amx_program* prog, const void* ws, amx_column* x, const uint64_t** d_len)
{
    if (!prog || !x || !d_len) return fail(AMX_ERR_INVALID_ARG, "program_output: null argument");
    const uint8_t* w = static_cast<const uint8_t*>(ws);
    if (prog->final_buf < 0)
        *x = prog->x;
    else {
        if (!ws) return fail(AMX_ERR_INVALID_ARG, "program_output: null workspace");
        *x = amx_column{const_cast<uint8_t*>(w) + prog->buf_off[prog->final_buf], prog->x.n, prog->final_format,
                        prog->final_bits};
    }
    if (prog->final_len_slot < 0)
        *d_len = nullptr;
    else if (prog->steps[prog->final_len_slot].d_result)
        *d_len = prog->steps[prog->final_len_slot].d_result;
    else
        *d_len = reinterpret_cast<const uint64_t*>(w + prog->len_off) + prog->final_len_slot;
    return AMX_OK;
}

amx_status amx_program_status(const amx_program* prog, const void* ws, void* stream)
{
    if (!prog || !ws) return fail(AMX_ERR_INVALID_ARG, "program_status: null argument");
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "program_status: stream");
    const uint8_t* w = static_cast<const uint8_t*>(ws);
    for (size_t i = 0; i < prog->steps.size(); i++) {
        // the pipeline header this step's launches cleared and may have written an error into
        const amx_step& st = prog->steps[i];
        uint64_t hoff = prog->pipe_off + i * prog->pipe_bytes;
        if (prog->merged[i]) continue;  // launches nothing of its own
        if (st.kind == AMX_STEP_GROUPBY) {
            const uint64_t g = groupby_pipeline_offset(st.aux.bits);
            if (g == ~0ull) continue;  // groups extracted by one CTA: no bounded waits
            hoff = prog->gb_off[i] + g;
        }
        uint32_t err = 0;
        const WsHeader* h = reinterpret_cast<const WsHeader*>(w + hoff);
        e = cudaMemcpy(&err, &h->err, sizeof(err), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) return cuda_fail(e, "program_status: read");
        if (err) return fail((amx_status)err, "program: device-side failure in step %zu (%u)", i, err);
    }
    return AMX_OK;
}

void amx_program_destroy(amx_program* prog) { delete prog; }

amx_status amx_graph_capture(const amx_program* const* progs, void* const* workspaces, const uint64_t* ws_bytes,
                             uint32_t count, uint32_t lanes, amx_graph** graph)
{
    if (!graph) return fail(AMX_ERR_INVALID_ARG, "graph_capture: null output");
    *graph = nullptr;
    if (count && (!progs || !workspaces || !ws_bytes)) return fail(AMX_ERR_INVALID_ARG, "graph_capture: null arrays");
    if (lanes < 1) lanes = 1;
    if (lanes > 64) lanes = 64;
    if (lanes > count && count) lanes = count;
    for (uint32_t i = 0; i < count; i++) {
        if (!progs[i]) return fail(AMX_ERR_INVALID_ARG, "graph_capture: null program %u", i);
        if (ws_bytes[i] < progs[i]->total) return fail(AMX_ERR_WORKSPACE, "graph_capture: workspace %u too small", i);
    }
    // longest programs first, each to the lane with the least planned bytes
    std::vector<uint32_t> order(count);
    for (uint32_t i = 0; i < count; i++) order[i] = i;
    auto work = [&](uint32_t i) {
        const amx_program* p = progs[i];
        return (double)storage_bytes(p->x.format, p->x.bits, p->x.n) * (double)(p->steps.size() + 1);
    };
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return work(a) > work(b); });
    std::vector<double> load(lanes, 0.0);
    std::vector<std::vector<uint32_t>> plan(lanes);
    for (uint32_t i : order) {
        const uint32_t l = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
        plan[l].push_back(i);
        load[l] += work(i);
    }

    std::vector<cudaStream_t> st(lanes, nullptr);
    std::vector<cudaEvent_t> ev(lanes + 1, nullptr);
    amx_status rc = AMX_OK;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaSuccess;
    for (uint32_t l = 0; l < lanes && e == cudaSuccess; l++) e = cudaStreamCreateWithFlags(&st[l], cudaStreamNonBlocking);
    for (uint32_t l = 0; l <= lanes && e == cudaSuccess; l++) e = cudaEventCreateWithFlags(&ev[l], cudaEventDisableTiming);
    if (e != cudaSuccess) rc = cuda_fail(e, "graph_capture: streams");
    bool capturing = false;
    if (!rc) {
        e = cudaStreamBeginCapture(st[0], cudaStreamCaptureModeThreadLocal);
        if (e != cudaSuccess)
            rc = cuda_fail(e, "graph_capture: begin");
        else
            capturing = true;
    }
    if (!rc) {
        e = cudaEventRecord(ev[lanes], st[0]);  // fork
        for (uint32_t l = 1; l < lanes && e == cudaSuccess; l++) e = cudaStreamWaitEvent(st[l], ev[lanes], 0);
        if (e != cudaSuccess) rc = cuda_fail(e, "graph_capture: fork");
    }
    for (uint32_t l = 0; l < lanes && !rc; l++)
        for (uint32_t i : plan[l]) {
            rc = amx_program_run(progs[i], workspaces[i], ws_bytes[i], st[l]);
            if (rc) break;
        }
    if (!rc) {
        for (uint32_t l = 1; l < lanes && e == cudaSuccess; l++) {
            e = cudaEventRecord(ev[l], st[l]);  // join
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st[0], ev[l], 0);
        }
        if (e != cudaSuccess) rc = cuda_fail(e, "graph_capture: join");
    }
    if (capturing) {
        e = cudaStreamEndCapture(st[0], &g);
        if (!rc && e != cudaSuccess) rc = cuda_fail(e, "graph_capture: end");
    }
    amx_graph* out = nullptr;
    if (!rc) {
        out = new (std::nothrow) amx_graph();
        if (!out)
            rc = fail(AMX_ERR_CAPACITY, "graph_capture: out of host memory");
        else {
            out->graph = g;
            e = cudaGraphInstantiate(&out->exec, g, 0);
            if (e != cudaSuccess) {
                rc = cuda_fail(e, "graph_capture: instantiate");
                delete out;
                out = nullptr;
            }
        }
    }
    if (rc && g) cudaGraphDestroy(g);
    for (auto x : ev)
        if (x) cudaEventDestroy(x);
    for (auto x : st)
        if (x) cudaStreamDestroy(x);
    if (rc) {
        cudaGetLastError();  // a failed capture leaves its error pending
        return rc;
    }
    *graph = out;
    return AMX_OK;
}

amx_status amx_graph_launch(const amx_graph* graph, void* stream)
{
    if (!graph) return fail(AMX_ERR_INVALID_ARG, "graph_launch: null graph");
    cudaError_t e = cudaGraphLaunch(graph->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "graph_launch");
    return AMX_OK;
}

void amx_graph_destroy(amx_graph* graph)
{
    if (!graph) return;
    cudaGraphExecDestroy(graph->exec);
    cudaGraphDestroy(graph->graph);
    delete graph;
}

}  // extern "C"
