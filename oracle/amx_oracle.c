/*
 * amx_oracle.c -- scalar CPU oracle (TEST INFRASTRUCTURE ONLY, see amx_oracle.h).
 *
 * Each routine restates the reference's semantics in plain C and cites the
 * reference file:line it follows (paths inside the Amethyst source tree).
 * Nothing here is shipped: the product library never links this file.
 */
#include "amx_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* gen_bitmask: src/common_code.cuh:38-41 (bits==0 gives 0 here instead of UB) */
uint64_t ora_mask_bits(uint32_t bits)
{
    if (bits == 0) return 0;
    if (bits >= 64) return ~(uint64_t)0;
    return (~(uint64_t)0) >> (64 - bits);
}

/* elems_per_slab = 64 / bits: src/common_code.cuh:46 */
uint32_t ora_elems_per_slab(uint32_t bits) { return 64u / bits; }

uint64_t ora_storage_words(uint32_t format, uint32_t bits, uint64_t n)
{
    switch (format) {
        case ORA_PLAIN32:
        case ORA_PLAIN64: return n;
        case ORA_SLAB: {
            uint64_t eps = ora_elems_per_slab(bits);
            return (n + eps - 1) / eps;
        }
        case ORA_NOGAPS: return (n * bits + 63) / 64;
    }
    return 0;
}

uint64_t ora_storage_bytes(uint32_t format, uint32_t bits, uint64_t n)
{
    return ora_storage_words(format, bits, n) * (format == ORA_PLAIN32 ? 4u : 8u);
}

/* get_elem_nogaps: src/common_code.cuh:100-116 */
static uint64_t nogaps_get(const uint64_t* buf, uint32_t bits, uint64_t idx)
{
    uint64_t slab = (idx * bits) / 64;
    uint64_t offset = (idx * bits) % 64;
    uint64_t remaining = 64 - offset;
    uint64_t elem;
    if (remaining < bits) {
        elem = (buf[slab] >> offset) & ora_mask_bits((uint32_t)remaining);
        uint64_t rest = bits - remaining;
        elem |= (buf[slab + 1] & ora_mask_bits((uint32_t)rest)) << remaining;
    }
    else {
        elem = (buf[slab] >> offset) & ora_mask_bits(bits);
    }
    return elem;
}

/* element accessors: plain = get_element_baseline src/common_code.cuh:51-55,
 * slab = get_element src/common_code.cuh:43-50, nogaps as above. */
uint64_t ora_get(const ora_column* c, uint64_t i)
{
    uint64_t m = ora_mask_bits(c->bits);
    switch (c->format) {
        case ORA_PLAIN32: return ((const uint32_t*)c->data)[i] & m;
        case ORA_PLAIN64: return ((const uint64_t*)c->data)[i] & m;
        case ORA_SLAB: {
            uint64_t eps = ora_elems_per_slab(c->bits);
            uint64_t s = i / eps;
            uint64_t off = (i - s * eps) * c->bits;
            return (((const uint64_t*)c->data)[s] >> off) & m;
        }
        case ORA_NOGAPS: return nogaps_get((const uint64_t*)c->data, c->bits, i);
    }
    return 0;
}

/* Canonical encoding.  Slab writers start every slab accumulator at zero
 * (src/kernels/binary_op_slabs.cuh:48-65), so dead bits and bits past n are 0. */
void ora_encode(uint32_t format, uint32_t bits, const uint64_t* values, uint64_t n, void* out)
{
    uint64_t m = ora_mask_bits(bits);
    memset(out, 0, ora_storage_bytes(format, bits, n));
    switch (format) {
        case ORA_PLAIN32:
            for (uint64_t i = 0; i < n; i++) ((uint32_t*)out)[i] = (uint32_t)(values[i] & m);
            break;
        case ORA_PLAIN64:
            for (uint64_t i = 0; i < n; i++) ((uint64_t*)out)[i] = values[i] & m;
            break;
        case ORA_SLAB: {
            uint64_t eps = ora_elems_per_slab(bits);
            uint64_t* w = (uint64_t*)out;
            for (uint64_t i = 0; i < n; i++) w[i / eps] |= (values[i] & m) << ((i % eps) * bits);
            break;
        }
        case ORA_NOGAPS: {
            uint64_t* w = (uint64_t*)out;
            for (uint64_t i = 0; i < n; i++) {
                uint64_t v = values[i] & m;
                uint64_t pos = i * bits;
                uint64_t off = pos % 64;
                w[pos / 64] |= v << off;
                if (off + bits > 64) w[pos / 64 + 1] |= v >> (64 - off);
            }
            break;
        }
    }
}

void ora_decode(const ora_column* c, uint64_t* values)
{
    for (uint64_t i = 0; i < c->n; i++) values[i] = ora_get(c, i);
}

/* Predicates.  HALF is FILTER_PREDICATE_OP: src/config.cuh:107-113.  The
 * comparison kinds are the runtime predicates the configs need (v < 205,
 * C >= 2^13, per-column thresholds); they have no compile-time counterpart
 * in the reference, which bakes one predicate into each kernel instance. */
int ora_pred_eval(const ora_pred* p, uint64_t v)
{
    switch (p->kind) {
        case ORA_PRED_ALL: return 1;
        case ORA_PRED_LT: return v < p->k0;
        case ORA_PRED_LE: return v <= p->k0;
        case ORA_PRED_GT: return v > p->k0;
        case ORA_PRED_GE: return v >= p->k0;
        case ORA_PRED_EQ: return v == p->k0;
        case ORA_PRED_NE: return v != p->k0;
        case ORA_PRED_BETWEEN: return p->k0 <= v && v <= p->k1;
        case ORA_PRED_NOT_BETWEEN: return !(p->k0 <= v && v <= p->k1);
        case ORA_PRED_HALF: return v >= ((uint64_t)1 << (p->bits - 1));
    }
    return 0;
}

/* Binary operators, each masked to the output width like the reference's
 * op_* templates (src/config.cuh:5-42).  Division or modulo by zero has no
 * defined reference behaviour; here x/0 = all ones and x%0 = x. */
uint64_t ora_binop(uint32_t op, uint64_t l, uint64_t r, uint32_t out_bits)
{
    uint64_t v = 0;
    switch (op) {
        case ORA_OP_ADD: v = l + r; break;
        case ORA_OP_SUB: v = l - r; break;
        case ORA_OP_MUL: v = l * r; break;
        case ORA_OP_DIV: v = r ? l / r : ~(uint64_t)0; break;
        case ORA_OP_MOD: v = r ? l % r : l; break;
        case ORA_OP_MIN: v = l < r ? l : r; break;
        case ORA_OP_MAX: v = l > r ? l : r; break;
        case ORA_OP_AND: v = l & r; break;
        case ORA_OP_OR: v = l | r; break;
        case ORA_OP_XOR: v = l ^ r; break;
        case ORA_OP_BOOL_OR: v = (l || r); break;
        case ORA_OP_BOOL_XOR: v = ((l && !r) || (!l && r)); break;
        case ORA_OP_MATH: {
            uint64_t den = l * l + r * r + 5 * l;
            v = den ? (l * l + r * r + 4 * l) / den : ~(uint64_t)0;
            break;
        }
        case ORA_OP_LHS: v = l; break;
    }
    return v & ora_mask_bits(out_bits);
}

static uint32_t umax32(uint32_t a, uint32_t b) { return a > b ? a : b; }
static uint32_t umin32(uint32_t a, uint32_t b) { return a < b ? a : b; }

/* Output widths that can never truncate.  add/mul/mod follow op_*_outbits
 * (src/config.cuh:44-55) generalised to two input widths. */
uint32_t ora_binop_out_bits(uint32_t op, uint32_t lb, uint32_t rb)
{
    uint32_t w = 0;
    switch (op) {
        case ORA_OP_ADD: w = umax32(lb, rb) + 1; break;
        case ORA_OP_SUB: w = umax32(lb, rb); break;
        case ORA_OP_MUL: w = lb + rb; break;
        case ORA_OP_DIV: w = lb; break;
        case ORA_OP_MOD: w = umin32(lb, rb); break;
        case ORA_OP_MIN: w = umin32(lb, rb); break;
        case ORA_OP_MAX: w = umax32(lb, rb); break;
        case ORA_OP_AND: w = umin32(lb, rb); break;
        case ORA_OP_OR:
        case ORA_OP_XOR: w = umax32(lb, rb); break;
        case ORA_OP_BOOL_OR:
        case ORA_OP_BOOL_XOR:
        case ORA_OP_MATH: w = 1; break;
        case ORA_OP_LHS: w = lb; break;
    }
    return w > 64 ? 64 : w;
}

/* filter: validation loop src/benchs/bench_filter_slabs.cu:38-46; mask bit i is
 * bit i%32 of uint32 word i/32, bits past n are 0 (src/kernels/filter_slabs.cuh:43-55). */
void ora_filter(const ora_column* in, const ora_pred* p, uint32_t* mask)
{
    uint64_t words = (in->n + 31) / 32;
    memset(mask, 0, words * 4);
    for (uint64_t i = 0; i < in->n; i++)
        if (ora_pred_eval(p, ora_get(in, i))) mask[i / 32] |= 1u << (i % 32);
}

/* compressstore: validation walk src/benchs/bench_compressstore_slabs.cu:74-95 */
uint64_t ora_compressstore(const ora_column* in, const uint32_t* mask, ora_column* out)
{
    uint64_t* vals = (uint64_t*)malloc((in->n ? in->n : 1) * sizeof(uint64_t));
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < in->n; i++)
        if ((mask[i / 32] >> (i % 32)) & 1u) vals[cnt++] = ora_get(in, i);
    if (out) ora_encode(out->format, out->bits, vals, cnt, out->data);
    free(vals);
    return cnt;
}

uint64_t ora_filter_compressstore(const ora_column* in, const ora_pred* p, ora_column* out)
{
    uint64_t* vals = (uint64_t*)malloc((in->n ? in->n : 1) * sizeof(uint64_t));
    uint64_t cnt = 0;
    for (uint64_t i = 0; i < in->n; i++) {
        uint64_t v = ora_get(in, i);
        if (ora_pred_eval(p, v)) vals[cnt++] = v;
    }
    if (out) ora_encode(out->format, out->bits, vals, cnt, out->data);
    free(vals);
    return cnt;
}

/* binary op: validation src/benchs/bench_binary_op_slabs.cu:32-41 */
void ora_binary(uint32_t op, const ora_column* l, const ora_column* r, ora_column* out)
{
    uint64_t n = l->n;
    uint64_t* vals = (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < n; i++) vals[i] = ora_binop(op, ora_get(l, i), r ? ora_get(r, i) : 0, out->bits);
    ora_encode(out->format, out->bits, vals, n, out->data);
    free(vals);
}

static uint64_t agg_identity(uint32_t agg)
{
    switch (agg) {
        case ORA_AGG_MIN:
        case ORA_AGG_AND: return ~(uint64_t)0;
        default: return 0;
    }
}

static uint64_t agg_apply(uint32_t agg, uint64_t a, uint64_t v)
{
    switch (agg) {
        case ORA_AGG_SUM: return a + v; /* HOP_OP: src/config.cuh:62-71, wraps mod 2^64 */
        case ORA_AGG_MIN: return v < a ? v : a;
        case ORA_AGG_MAX: return v > a ? v : a;
        case ORA_AGG_AND: return a & v;
        case ORA_AGG_OR: return a | v;
        case ORA_AGG_XOR: return a ^ v;
    }
    return a;
}

/* aggregation: validation src/benchs/bench_hop_slabs.cu:38-51 */
uint64_t ora_reduce(uint32_t agg, const ora_column* in, const uint32_t* mask)
{
    uint64_t a = agg_identity(agg);
    for (uint64_t i = 0; i < in->n; i++) {
        if (mask && !((mask[i / 32] >> (i % 32)) & 1u)) continue;
        a = agg_apply(agg, a, ora_get(in, i));
    }
    return a;
}

ora_chain_result ora_chain_range(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits, const ora_pred* p,
                                 uint32_t agg, uint64_t begin, uint64_t end)
{
    ora_chain_result res = {0, agg_identity(agg)};
    uint64_t m = ora_mask_bits(vbits);
    for (uint64_t i = begin; i < end; i++) {
        uint64_t v = r ? ora_binop(op, ora_get(l, i), ora_get(r, i), vbits) : (ora_get(l, i) & m);
        if (ora_pred_eval(p, v)) {
            res.count++;
            res.agg = agg_apply(agg, res.agg, v);
        }
    }
    return res;
}

ora_chain_result ora_chain(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits, const ora_pred* p,
                           uint32_t agg, ora_column* out)
{
    ora_chain_result res = {0, agg_identity(agg)};
    uint64_t n = l->n;
    uint64_t m = ora_mask_bits(vbits);
    uint64_t* vals = out ? (uint64_t*)malloc((n ? n : 1) * sizeof(uint64_t)) : NULL;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t v = r ? ora_binop(op, ora_get(l, i), ora_get(r, i), vbits) : (ora_get(l, i) & m);
        if (ora_pred_eval(p, v)) {
            if (vals) vals[res.count] = v;
            res.count++;
            res.agg = agg_apply(agg, res.agg, v);
        }
    }
    if (out) {
        ora_encode(out->format, out->bits, vals, res.count, out->data);
        free(vals);
    }
    return res;
}

typedef struct {
    uint32_t op;
    const ora_column* l;
    const ora_column* r;
    uint32_t vbits;
    const ora_pred* p;
    uint32_t agg;
    uint64_t begin, end;
    ora_chain_result res;
} chain_job;

static void* chain_worker(void* arg)
{
    chain_job* j = (chain_job*)arg;
    j->res = ora_chain_range(j->op, j->l, j->r, j->vbits, j->p, j->agg, j->begin, j->end);
    return NULL;
}

ora_chain_result ora_chain_mt(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits, const ora_pred* p,
                              uint32_t agg, int threads)
{
    if (threads < 1) threads = 1;
    chain_job* jobs = (chain_job*)calloc((size_t)threads, sizeof(chain_job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    uint64_t n = l->n;
    for (int t = 0; t < threads; t++) {
        jobs[t] = (chain_job){op, l, r, vbits, p, agg, n * (uint64_t)t / threads, n * (uint64_t)(t + 1) / threads, {0, 0}};
        pthread_create(&th[t], NULL, chain_worker, &jobs[t]);
    }
    ora_chain_result res = {0, agg_identity(agg)};
    for (int t = 0; t < threads; t++) {
        pthread_join(th[t], NULL);
        res.count += jobs[t].res.count;
        res.agg = agg_apply(agg, res.agg, jobs[t].res.agg);
    }
    free(jobs);
    free(th);
    return res;
}

/* ora_chain with the survivors also compacted into `out` (any format, at out->bits), on
 * `threads` threads: each thread keeps the survivors of its element range, the ranges are
 * concatenated in order and encoded.  Same results as ora_chain. */
typedef struct {
    chain_job c;
    uint64_t* vals;
} chainc_job;

static void* chainc_worker(void* arg)
{
    chainc_job* j = (chainc_job*)arg;
    chain_job* c = &j->c;
    ora_chain_result res = {0, agg_identity(c->agg)};
    uint64_t m = ora_mask_bits(c->vbits);
    for (uint64_t i = c->begin; i < c->end; i++) {
        uint64_t v = c->r ? ora_binop(c->op, ora_get(c->l, i), ora_get(c->r, i), c->vbits) : (ora_get(c->l, i) & m);
        if (ora_pred_eval(c->p, v)) {
            j->vals[res.count++] = v;
            res.agg = agg_apply(c->agg, res.agg, v);
        }
    }
    c->res = res;
    return NULL;
}

ora_chain_result ora_chain_compress_mt(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits,
                                       const ora_pred* p, uint32_t agg, const ora_column* out, int threads)
{
    if (threads < 1) threads = 1;
    chainc_job* jobs = (chainc_job*)calloc((size_t)threads, sizeof(chainc_job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    uint64_t n = l->n;
    for (int t = 0; t < threads; t++) {
        uint64_t b = n * (uint64_t)t / threads, e = n * (uint64_t)(t + 1) / threads;
        jobs[t].c = (chain_job){op, l, r, vbits, p, agg, b, e, {0, 0}};
        jobs[t].vals = (uint64_t*)malloc((e - b + 1) * sizeof(uint64_t));
        pthread_create(&th[t], NULL, chainc_worker, &jobs[t]);
    }
    ora_chain_result res = {0, agg_identity(agg)};
    for (int t = 0; t < threads; t++) {
        pthread_join(th[t], NULL);
        res.count += jobs[t].c.res.count;
        res.agg = agg_apply(agg, res.agg, jobs[t].c.res.agg);
    }
    uint64_t* all = (uint64_t*)malloc((res.count + 1) * sizeof(uint64_t));
    uint64_t at = 0;
    for (int t = 0; t < threads; t++) {
        memcpy(all + at, jobs[t].vals, jobs[t].c.res.count * sizeof(uint64_t));
        at += jobs[t].c.res.count;
        free(jobs[t].vals);
    }
    ora_encode(out->format, out->bits, all, res.count, out->data);
    free(all);
    free(jobs);
    free(th);
    return res;
}

/* sort-based group-by for keys of any width up to 32 bits: the (key, value) pairs of the masked
 * elements sorted by key, then reduced by key into ascending keys, uint64 sums and counts -- the
 * reference's radix-sort + reduce-by-key path (src/benchs/bench_groupby_sort_cub.cu:50-63), with
 * full uint64 sums and counts emitted.  Returns the number of groups. */
typedef struct {
    uint64_t key, val;
} kv_pair;

static int kv_cmp(const void* a, const void* b)
{
    const kv_pair* x = (const kv_pair*)a;
    const kv_pair* y = (const kv_pair*)b;
    return x->key < y->key ? -1 : (x->key > y->key ? 1 : 0);
}

uint64_t ora_groupby_sorted(const ora_column* keys, const ora_column* vals, const uint32_t* mask, uint64_t* out_keys,
                            uint64_t* out_sums, uint64_t* out_counts)
{
    kv_pair* kv = (kv_pair*)malloc((keys->n + 1) * sizeof(kv_pair));
    uint64_t m = 0;
    for (uint64_t i = 0; i < keys->n; i++) {
        if (mask && !((mask[i / 32] >> (i % 32)) & 1u)) continue;
        kv[m].key = ora_get(keys, i);
        kv[m].val = ora_get(vals, i);
        m++;
    }
    qsort(kv, m, sizeof(kv_pair), kv_cmp);
    uint64_t g = 0;
    for (uint64_t i = 0; i < m; i++) {
        if (i == 0 || kv[i].key != kv[i - 1].key) {
            out_keys[g] = kv[i].key;
            out_sums[g] = 0;
            out_counts[g] = 0;
            g++;
        }
        out_sums[g - 1] += kv[i].val;
        out_counts[g - 1]++;
    }
    free(kv);
    return g;
}

/* group-by sum/count over a dense key space.  The reference's table
 * (src/kernels/groupby_sm_array.cuh:4-59) truncates sums to the key width and
 * does not emit counts; the dense oracle keeps full uint64 sums and counts. */
uint64_t ora_groupby_dense(const ora_column* keys, const ora_column* vals, uint64_t* sums, uint64_t* counts)
{
    uint64_t space = (uint64_t)1 << keys->bits;
    memset(sums, 0, space * 8);
    memset(counts, 0, space * 8);
    for (uint64_t i = 0; i < keys->n; i++) {
        uint64_t k = ora_get(keys, i);
        sums[k] += ora_get(vals, i);
        counts[k]++;
    }
    uint64_t g = 0;
    for (uint64_t k = 0; k < space; k++) g += counts[k] != 0;
    return g;
}

/* slab matrices pad every row to whole slabs: get_matrix_element
 * src/common_code.cuh:124-129.  Plain and nogaps matrices are dense row-major. */
uint64_t ora_matrix_words(uint32_t format, uint32_t bits, uint64_t rows, uint64_t cols)
{
    if (format == ORA_SLAB) {
        uint64_t eps = ora_elems_per_slab(bits);
        return rows * ((cols + eps - 1) / eps);
    }
    return ora_storage_words(format, bits, rows * cols);
}

uint64_t ora_matrix_get(const ora_column* c, uint64_t rows, uint64_t cols, uint64_t r, uint64_t col)
{
    (void)rows;
    if (c->format == ORA_SLAB) {
        uint64_t eps = ora_elems_per_slab(c->bits);
        uint64_t row_slabs = (cols + eps - 1) / eps;
        return (((const uint64_t*)c->data)[r * row_slabs + col / eps] >> (c->bits * (col % eps))) & ora_mask_bits(c->bits);
    }
    return ora_get(c, r * cols + col);
}

void ora_matrix_encode(uint32_t format, uint32_t bits, const uint64_t* values, uint64_t rows, uint64_t cols, void* out)
{
    if (format != ORA_SLAB) {
        ora_encode(format, bits, values, rows * cols, out);
        return;
    }
    uint64_t eps = ora_elems_per_slab(bits);
    uint64_t row_slabs = (cols + eps - 1) / eps;
    uint64_t m = ora_mask_bits(bits);
    uint64_t* w = (uint64_t*)out;
    memset(w, 0, rows * row_slabs * 8);
    for (uint64_t r = 0; r < rows; r++)
        for (uint64_t c = 0; c < cols; c++)
            w[r * row_slabs + c / eps] |= (values[r * cols + c] & m) << ((c % eps) * bits);
}

typedef struct {
    const ora_column* a;
    const ora_column* b;
    uint64_t m, n, k;
    int64_t* out;
    uint64_t r0, r1;
} mm_job;

static void* mm_worker(void* arg)
{
    mm_job* j = (mm_job*)arg;
    uint64_t* brow = (uint64_t*)malloc(j->n * sizeof(uint64_t));
    uint64_t* arow = (uint64_t*)malloc(j->k * sizeof(uint64_t));
    for (uint64_t r = j->r0; r < j->r1; r++) {
        for (uint64_t kk = 0; kk < j->k; kk++) arow[kk] = ora_matrix_get(j->a, j->m, j->k, r, kk);
        uint64_t* acc = (uint64_t*)calloc(j->n, sizeof(uint64_t));
        for (uint64_t kk = 0; kk < j->k; kk++) {
            uint64_t av = arow[kk];
            if (!av) continue;
            for (uint64_t c = 0; c < j->n; c++) brow[c] = ora_matrix_get(j->b, j->k, j->n, kk, c);
            for (uint64_t c = 0; c < j->n; c++) acc[c] += av * brow[c];
        }
        for (uint64_t c = 0; c < j->n; c++) j->out[r * j->n + c] = (int64_t)acc[c];
        free(acc);
    }
    free(brow);
    free(arow);
    return NULL;
}

/* exact integer matrix product; no reference kernel exists (README.md:20) */
void ora_matmul(const ora_column* a, const ora_column* b, uint64_t m, uint64_t n, uint64_t k, int64_t* out, int threads)
{
    if (threads < 1) threads = 1;
    mm_job* jobs = (mm_job*)calloc((size_t)threads, sizeof(mm_job));
    pthread_t* th = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    for (int t = 0; t < threads; t++) {
        jobs[t] = (mm_job){a, b, m, n, k, out, m * (uint64_t)t / threads, m * (uint64_t)(t + 1) / threads};
        pthread_create(&th[t], NULL, mm_worker, &jobs[t]);
    }
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    free(jobs);
    free(th);
}

/* PCG32 (XSH RR) seeded through splitmix64: the published algorithms that
 * src/fast_prng.cuh:7-36 implements. */
void ora_pcg32_seed(ora_pcg32* g, uint64_t seed)
{
    uint64_t z = seed + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    g->state = z ^ (z >> 31);
    g->inc = 1;
}

uint32_t ora_pcg32_next(ora_pcg32* g)
{
    uint64_t old = g->state;
    g->state = old * 6364136223846793005ull + (g->inc | 1);
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
}

/* input arrays of src/main.cu:242-251: per element, data1 takes two draws
 * (first draw = high half) then data2 two draws; a zero word becomes 1. */
void ora_reference_inputs(uint64_t seed, uint64_t* data1, uint64_t* data2, uint64_t n)
{
    ora_pcg32 g;
    ora_pcg32_seed(&g, seed);
    for (uint64_t i = 0; i < n; i++) {
        uint64_t hi = ora_pcg32_next(&g);
        uint64_t lo = ora_pcg32_next(&g);
        uint64_t a = (hi << 32) | lo;
        data1[i] = a ? a : 1;
        hi = ora_pcg32_next(&g);
        lo = ora_pcg32_next(&g);
        uint64_t b = (hi << 32) | lo;
        data2[i] = b ? b : 1;
    }
}

/* generate_mask_uniform: src/main.cu:33-46 */
void ora_mask_uniform(uint8_t* buf, uint64_t offset, uint64_t length, double selectivity)
{
    uint64_t p = (uint64_t)(selectivity * (double)UINT32_MAX);
    ora_pcg32 g;
    ora_pcg32_seed(&g, 42);
    for (uint64_t i = offset; i < offset + length; i++) {
        uint8_t acc = 0;
        for (int j = 7; j >= 0; j--)
            if (ora_pcg32_next(&g) < p) acc |= (uint8_t)(1u << j);
        buf[i] = acc;
    }
}

/* create_bitmask: src/main.cu:59-108 (float arithmetic as in the reference) */
void ora_mask_clusters(uint8_t* buf, double selectivity, uint64_t cluster_count, uint64_t total)
{
    float sel = (float)selectivity;
    uint64_t set_one = (uint64_t)(sel * (float)total);
    uint64_t cluster_size = set_one / cluster_count;
    uint64_t slice = total / cluster_count;
    memset(buf, 0, total / 8);
    for (uint64_t c = 0; c < cluster_count; c++)
        for (uint64_t k = 0; k < cluster_size; k++) {
            uint64_t i = c * slice + k;
            if (i / 8 < total / 8) buf[i / 8] |= (uint8_t)(1u << (7 - (i % 8)));
        }
}

/* Marsaglia xorshift64 (13, 7, 17) */
uint64_t ora_xorshift64(uint64_t* s)
{
    uint64_t x = *s;
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    *s = x;
    return x;
}

/* uniform values in [0, 2^bits): top `bits` bits of successive xorshift64 draws; the seed
 * is spread over the state word first so that small seeds give full-entropy streams */
void ora_uniform_values(uint64_t seed, uint32_t bits, uint64_t* out, uint64_t n)
{
    uint64_t s = seed * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
    if (!s) s = 0x9E3779B97F4A7C15ull;
    for (uint64_t i = 0; i < n; i++) {
        uint64_t r = ora_xorshift64(&s);
        out[i] = bits >= 64 ? r : (r >> (64 - bits));
    }
}
