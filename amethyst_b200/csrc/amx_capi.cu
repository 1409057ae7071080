// amx_capi.cu -- the C ABI of libamethyst_b200.so: argument checks, descriptor set-up,
// workspace clearing and kernel launches for the column operators.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "amx_dispatch.h"

namespace amx {

static thread_local std::string g_last_error;

amx_status fail(amx_status s, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return s;
}

amx_status cuda_fail(cudaError_t e, const char* what)
{
    return fail(AMX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

uint64_t mask_of(uint32_t bits) { return bits >= 64 ? ~0ull : ((1ull << bits) - 1); }

// floor(2^64 / d) + 1 for 2 <= d <= 64 (0 otherwise): exact n / d = umul64hi(n, m) for n < 2^58
uint64_t magic64(uint32_t d) { return d >= 2 ? (uint64_t)(((unsigned __int128)1 << 64) / d) + 1 : 0; }

uint64_t storage_bytes(uint32_t format, uint32_t bits, uint64_t n)
{
    switch (format) {
        case AMX_PLAIN32: return 4 * n;
        case AMX_PLAIN64: return 8 * n;
        case AMX_SLAB: {
            const uint64_t eps = 64 / bits;
            return 8 * ((n + eps - 1) / eps);
        }
        case AMX_NOGAPS: return 8 * ((n * bits + 63) / 64);
    }
    return 0;
}

static bool width_ok(uint32_t format, uint32_t bits)
{
    if (bits < 1) return false;
    switch (format) {
        case AMX_PLAIN32: return bits <= 32;
        case AMX_PLAIN64:
        case AMX_SLAB:
        case AMX_NOGAPS: return bits <= 64;
    }
    return false;
}

amx_status check_column(const amx_column* c, const char* name)
{
    if (!c) return fail(AMX_ERR_INVALID_ARG, "%s: null column", name);
    if (c->format > AMX_NOGAPS) return fail(AMX_ERR_INVALID_ARG, "%s: unknown format %u", name, c->format);
    if (!width_ok(c->format, c->bits))
        return fail(AMX_ERR_INVALID_ARG, "%s: width %u not valid for format %u", name, c->bits, c->format);
    if (c->n > kMaxElements) return fail(AMX_ERR_CAPACITY, "%s: %llu elements exceed 2^40", name, (unsigned long long)c->n);
    if (c->n && !c->data) return fail(AMX_ERR_INVALID_ARG, "%s: null data", name);
    if (((uintptr_t)c->data) & 15) return fail(AMX_ERR_ALIGNMENT, "%s: data not 16-byte aligned", name);
    return AMX_OK;
}

ColDev col_dev(const amx_column* c)
{
    ColDev d{};
    d.data = c->data;
    d.n = c->n;
    d.bytes = storage_bytes(c->format, c->bits, c->n);
    d.mask = mask_of(c->bits);
    d.format = c->format;
    d.bits = c->bits;
    d.eps = c->format == AMX_SLAB ? 64 / c->bits : 0;
    d.magic = d.eps >= 2 ? (uint32_t)((1ull << 32) / d.eps + 1) : 0;
    d.magic64 = magic64(d.eps);
    return d;
}

ColDev mask_dev(const uint32_t* m, uint64_t n)
{
    ColDev d{};
    d.data = m;
    d.n = n;
    d.bytes = 4 * ((n + 31) / 32);
    d.mask = ~0ull;
    d.format = kFmtMask;
    d.bits = 1;
    return d;
}

OutDev out_dev(const amx_column* c)
{
    OutDev o{};
    o.data = c->data;
    o.mask = mask_of(c->bits);
    o.format = c->format;
    o.bits = c->bits;
    o.eps = c->format == AMX_SLAB ? 64 / c->bits : 0;
    o.eps_m64 = magic64(o.eps);
    o.bits_m64 = magic64(o.bits);
    return o;
}

// keep(v) = ((v - lo) <= span) != neg
amx_status normalize_pred(const amx_predicate* p, uint64_t& lo, uint64_t& span, uint32_t& neg)
{
    lo = 0;
    span = ~0ull;
    neg = 0;
    if (!p) return AMX_OK;
    const uint64_t k0 = p->k0, k1 = p->k1;
    switch (p->kind) {
        case AMX_PRED_ALL: break;
        case AMX_PRED_LT:
            if (k0 == 0)
                neg = 1;
            else
                span = k0 - 1;
            break;
        case AMX_PRED_LE: span = k0; break;
        case AMX_PRED_GT:
            span = k0;
            neg = 1;
            break;
        case AMX_PRED_GE:
            if (k0 != 0) {
                span = k0 - 1;
                neg = 1;
            }
            break;
        case AMX_PRED_EQ:
            lo = k0;
            span = 0;
            break;
        case AMX_PRED_NE:
            lo = k0;
            span = 0;
            neg = 1;
            break;
        case AMX_PRED_BETWEEN:
            if (k0 > k1)
                neg = 1;
            else {
                lo = k0;
                span = k1 - k0;
            }
            break;
        case AMX_PRED_NOT_BETWEEN:
            if (k0 <= k1) {
                lo = k0;
                span = k1 - k0;
                neg = 1;
            }
            break;
        case AMX_PRED_HALF:
            if (p->bits < 1 || p->bits > 64) return fail(AMX_ERR_INVALID_ARG, "predicate: HALF needs bits in 1..64");
            span = (1ull << (p->bits - 1)) - 1;
            neg = 1;
            break;
        default: return fail(AMX_ERR_INVALID_ARG, "predicate: unknown kind %u", p->kind);
    }
    return AMX_OK;
}

static int g_sm_count[64];

int sm_count()
{
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return 148;
    if (!g_sm_count[dev]) {
        int c = 0;
        cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
        g_sm_count[dev] = c > 0 ? c : 148;
    }
    return g_sm_count[dev];
}

}  // namespace amx

using namespace amx;

extern "C" {

int amx_version(void) { return AMX_VERSION; }

const char* amx_status_string(amx_status s)
{
    switch (s) {
        case AMX_OK: return "ok";
        case AMX_ERR_INVALID_ARG: return "invalid argument";
        case AMX_ERR_UNSUPPORTED: return "unsupported";
        case AMX_ERR_ALIGNMENT: return "misaligned pointer";
        case AMX_ERR_WORKSPACE: return "workspace too small";
        case AMX_ERR_CUDA: return "CUDA error";
        case AMX_ERR_TIMEOUT: return "device-side wait timed out";
        case AMX_ERR_CAPACITY: return "size exceeds capacity";
    }
    return "unknown status";
}

const char* amx_last_error(void) { return g_last_error.c_str(); }

amx_status amx_set_tuning(const amx_tuning* t)
{
    tuning() = t ? *t : amx_tuning{};
    return AMX_OK;
}

amx_status amx_test_lookback_timeout(uint64_t tile, uint32_t wait_polls)
{
    LookbackFault& f = lookback_fault();
    f.withhold_plus1 = tile == ~0ull ? 0 : tile + 1;
    f.wait_polls = tile == ~0ull ? 0 : wait_polls;
    return AMX_OK;
}

amx_status amx_get_tuning(amx_tuning* t)
{
    if (!t) return fail(AMX_ERR_INVALID_ARG, "get_tuning: null output");
    *t = tuning();
    return AMX_OK;
}

uint64_t amx_storage_bytes(uint32_t format, uint32_t bits, uint64_t n)
{
    if (!width_ok(format, bits)) return 0;
    return storage_bytes(format, bits, n);
}

uint64_t amx_mask_bytes(uint64_t n) { return 4 * ((n + 31) / 32); }

uint32_t amx_binary_out_bits(uint32_t op, uint32_t lb, uint32_t rb)
{
    uint32_t w = 0;
    const uint32_t mx = lb > rb ? lb : rb, mn = lb < rb ? lb : rb;
    switch (op) {
        case AMX_OP_ADD: w = mx + 1; break;
        case AMX_OP_SUB: w = mx; break;
        case AMX_OP_MUL: w = lb + rb; break;
        case AMX_OP_DIV: w = lb; break;
        case AMX_OP_MOD:
        case AMX_OP_MIN:
        case AMX_OP_AND: w = mn; break;
        case AMX_OP_MAX:
        case AMX_OP_OR:
        case AMX_OP_XOR: w = mx; break;
        case AMX_OP_BOOL_OR:
        case AMX_OP_BOOL_XOR:
        case AMX_OP_MATH: w = 1; break;
        case AMX_OP_LHS: w = lb; break;
        default: return 0;
    }
    return w > 64 ? 64 : w;
}

uint64_t amx_workspace_bytes(uint64_t n) { return sizeof(WsHeader) + 8 * ((n + kMinTile - 1) / kMinTile) + 64; }

amx_status amx_workspace_status(const void* workspace, void* stream)
{
    if (!workspace) return fail(AMX_ERR_INVALID_ARG, "workspace_status: null workspace");
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "workspace_status: stream");
    uint32_t err = 0;
    e = cudaMemcpy(&err, &reinterpret_cast<const WsHeader*>(workspace)->err, sizeof(err), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "workspace_status: read");
    if (err) return fail((amx_status)err, "device-side failure recorded in the workspace (%u)", err);
    return AMX_OK;
}

amx_status amx_filter(const amx_column* in, const amx_predicate* pred, uint32_t* d_mask, void* ws, size_t ws_bytes,
                      void* stream)
{
    amx_status st = check_column(in, "filter: in");
    if (st) return st;
    if (!pred) return fail(AMX_ERR_INVALID_ARG, "filter: null predicate");
    if (!d_mask && in->n) return fail(AMX_ERR_INVALID_ARG, "filter: null mask");
    if (((uintptr_t)d_mask) & 15) return fail(AMX_ERR_ALIGNMENT, "filter: mask not 16-byte aligned");
    ChainReq r{};
    r.a = in;
    r.pred = pred;
    r.vbits = in->bits;
    r.mask_out = d_mask;
    return run_chain(r, ws, ws_bytes, (cudaStream_t)stream);
}

amx_status amx_compressstore(const amx_column* in, const uint32_t* d_mask, const amx_column* out, uint64_t* d_count,
                             void* ws, size_t ws_bytes, void* stream)
{
    amx_status st = check_column(in, "compressstore: in");
    if (st) return st;
    if ((st = check_column(out, "compressstore: out"))) return st;
    if (!d_mask && in->n) return fail(AMX_ERR_INVALID_ARG, "compressstore: null mask");
    if (((uintptr_t)d_mask) & 15) return fail(AMX_ERR_ALIGNMENT, "compressstore: mask not 16-byte aligned");
    if (out->n < in->n) return fail(AMX_ERR_INVALID_ARG, "compressstore: output capacity below input length");
    ChainReq r{};
    r.a = in;
    r.mask_in = d_mask;
    r.vbits = in->bits;
    r.out = out;
    r.compact = 1;
    r.count_out = d_count;
    return run_chain(r, ws, ws_bytes, (cudaStream_t)stream);
}

amx_status amx_filter_compressstore(const amx_column* in, const amx_predicate* pred, const amx_column* out,
                                    uint64_t* d_count, void* ws, size_t ws_bytes, void* stream)
{
    amx_status st = check_column(in, "filter_compressstore: in");
    if (st) return st;
    if ((st = check_column(out, "filter_compressstore: out"))) return st;
    if (!pred) return fail(AMX_ERR_INVALID_ARG, "filter_compressstore: null predicate");
    if (out->n < in->n) return fail(AMX_ERR_INVALID_ARG, "filter_compressstore: output capacity below input length");
    ChainReq r{};
    r.a = in;
    r.pred = pred;
    r.vbits = in->bits;
    r.out = out;
    r.compact = 1;
    r.count_out = d_count;
    return run_chain(r, ws, ws_bytes, (cudaStream_t)stream);
}

amx_status amx_binary(uint32_t op, const amx_column* lhs, const amx_column* rhs, const amx_column* out, void* ws,
                      size_t ws_bytes, void* stream)
{
    amx_status st = check_column(lhs, "binary: lhs");
    if (st) return st;
    if ((st = check_column(rhs, "binary: rhs"))) return st;
    if ((st = check_column(out, "binary: out"))) return st;
    if (op > AMX_OP_LHS) return fail(AMX_ERR_INVALID_ARG, "binary: unknown op %u", op);
    if (lhs->n != rhs->n) return fail(AMX_ERR_INVALID_ARG, "binary: lhs and rhs lengths differ");
    if (out->n < lhs->n) return fail(AMX_ERR_INVALID_ARG, "binary: output capacity below input length");
    ChainReq r{};
    r.a = lhs;
    r.b = rhs;
    r.op = op;
    r.vbits = out->bits;
    r.out = out;
    return run_chain(r, ws, ws_bytes, (cudaStream_t)stream);
}

amx_status amx_convert(const amx_column* in, const amx_column* out, void* ws, size_t ws_bytes, void* stream)
{
    amx_status st = check_column(in, "convert: in");
    if (st) return st;
    if ((st = check_column(out, "convert: out"))) return st;
    if (out->n < in->n) return fail(AMX_ERR_INVALID_ARG, "convert: output capacity below input length");
    ChainReq r{};
    r.a = in;
    r.vbits = out->bits;
    r.out = out;
    return run_chain(r, ws, ws_bytes, (cudaStream_t)stream);
}

amx_status amx_reduce(uint32_t agg, const amx_column* in, const uint32_t* d_mask, uint64_t* d_result, void* ws,
                      size_t ws_bytes, void* stream)
{
    amx_status st = check_column(in, "reduce: in");
    if (st) return st;
    if (agg > AMX_AGG_XOR) return fail(AMX_ERR_INVALID_ARG, "reduce: unknown aggregation %u", agg);
    if (!d_result) return fail(AMX_ERR_INVALID_ARG, "reduce: null result");
    if (((uintptr_t)d_mask) & 15) return fail(AMX_ERR_ALIGNMENT, "reduce: mask not 16-byte aligned");
    ChainReq r{};
    r.a = in;
    r.mask_in = d_mask;
    r.vbits = in->bits;
    r.has_agg = 1;
    r.agg = agg;
    r.agg_out = d_result;
    return run_chain(r, ws, ws_bytes, (cudaStream_t)stream);
}

amx_status amx_chain(const amx_chain_desc* desc, const amx_column* lhs, const amx_column* rhs, const amx_column* out,
                     uint32_t* d_mask, uint64_t* d_count, uint64_t* d_agg, void* ws, size_t ws_bytes, void* stream)
{
    if (!desc) return fail(AMX_ERR_INVALID_ARG, "chain: null descriptor");
    amx_status st = check_column(lhs, "chain: lhs");
    if (st) return st;
    if (rhs) {
        if ((st = check_column(rhs, "chain: rhs"))) return st;
        if (rhs->n != lhs->n) return fail(AMX_ERR_INVALID_ARG, "chain: lhs and rhs lengths differ");
        if (desc->op > AMX_OP_LHS) return fail(AMX_ERR_INVALID_ARG, "chain: unknown op %u", desc->op);
    }
    if (out) {
        if ((st = check_column(out, "chain: out"))) return st;
        if (out->n < lhs->n) return fail(AMX_ERR_INVALID_ARG, "chain: output capacity below input length");
    }
    if (desc->value_bits < 1 || desc->value_bits > 64) return fail(AMX_ERR_INVALID_ARG, "chain: value_bits must be 1..64");
    if (desc->agg > AMX_AGG_XOR) return fail(AMX_ERR_INVALID_ARG, "chain: unknown aggregation %u", desc->agg);
    if (((uintptr_t)d_mask) & 15) return fail(AMX_ERR_ALIGNMENT, "chain: mask not 16-byte aligned");
    ChainReq r{};
    r.a = lhs;
    r.b = rhs;
    r.op = desc->op;
    r.vbits = desc->value_bits;
    r.pred = &desc->pred;
    r.out = out;
    r.compact = out ? 1 : 0;
    r.mask_out = d_mask;
    r.count_out = d_count;
    r.has_agg = d_agg ? 1 : 0;
    r.agg = desc->agg;
    r.agg_out = d_agg;
    return run_chain(r, ws, ws_bytes, (cudaStream_t)stream);
}

}  // extern "C"
