/*
 * amx_oracle.h -- scalar CPU oracle for the Amethyst packed-integer operator layer.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * element accessors, validation loops and operator semantics.  Only the test
 * suite, the smoke check and the CPU-baseline leg of the benchmark may load it,
 * and only as the checker.  The product library (libamethyst_b200.so) never
 * links, loads or calls anything in this directory.
 *
 * Parity pins: every routine cites the reference file:line whose semantics it
 * restates (paths relative to the Amethyst source tree).  The restatement is
 * checked against the reference's own host code, compiled from its headers
 * into oracle/_ref/ (see ref_harness.cu), by tests/test_oracle_pins.py.
 */
#ifndef AMX_ORACLE_H
#define AMX_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Storage formats.  The numbering is shared with include/amethyst.h. */
enum {
    ORA_PLAIN32 = 0, /* one uint32 per element, value = word & mask(bits)      */
    ORA_PLAIN64 = 1, /* one uint64 per element: src/common_code.cuh:51-55      */
    ORA_SLAB = 2,    /* floor(64/bits) elements per uint64: common_code.cuh:43-50 */
    ORA_NOGAPS = 3   /* continuous bit stream: common_code.cuh:100-116         */
};

typedef struct {
    void* data;
    uint64_t n;
    uint32_t format;
    uint32_t bits;
} ora_column;

/* Predicate kinds (shared numbering with include/amethyst.h). */
enum {
    ORA_PRED_ALL = 0,
    ORA_PRED_LT = 1,
    ORA_PRED_LE = 2,
    ORA_PRED_GT = 3,
    ORA_PRED_GE = 4,
    ORA_PRED_EQ = 5,
    ORA_PRED_NE = 6,
    ORA_PRED_BETWEEN = 7,     /* k0 <= v <= k1 */
    ORA_PRED_NOT_BETWEEN = 8, /* !(k0 <= v <= k1) */
    ORA_PRED_HALF = 9         /* v >= 2^(bits-1): src/config.cuh:107-113 */
};

typedef struct {
    uint32_t kind;
    uint32_t bits; /* width the HALF predicate refers to */
    uint64_t k0;
    uint64_t k1;
} ora_pred;

/* Binary operators (shared numbering with include/amethyst.h). */
enum {
    ORA_OP_ADD = 0,  /* op_add   src/config.cuh:5-9   */
    ORA_OP_SUB = 1,  /* wrap-around subtraction (no reference counterpart) */
    ORA_OP_MUL = 2,  /* op_mul   src/config.cuh:27-31 */
    ORA_OP_DIV = 3,  /* op_div   src/config.cuh:22-26 */
    ORA_OP_MOD = 4,  /* op_mod   src/config.cuh:17-21 */
    ORA_OP_MIN = 5,
    ORA_OP_MAX = 6,
    ORA_OP_AND = 7,
    ORA_OP_OR = 8,
    ORA_OP_XOR = 9,
    ORA_OP_BOOL_OR = 10,  /* op_bool_simple  src/config.cuh:32-36 */
    ORA_OP_BOOL_XOR = 11, /* op_bool_complex src/config.cuh:38-42 */
    ORA_OP_MATH = 12,     /* op_math         src/config.cuh:11-15 */
    ORA_OP_LHS = 13       /* identity on the left operand (format conversion) */
};

/* Aggregations (shared numbering with include/amethyst.h). */
enum { ORA_AGG_SUM = 0, ORA_AGG_MIN = 1, ORA_AGG_MAX = 2, ORA_AGG_AND = 3, ORA_AGG_OR = 4, ORA_AGG_XOR = 5 };

uint64_t ora_mask_bits(uint32_t bits);
uint32_t ora_elems_per_slab(uint32_t bits);
/* number of storage words (uint32 for PLAIN32, uint64 otherwise) */
uint64_t ora_storage_words(uint32_t format, uint32_t bits, uint64_t n);
uint64_t ora_storage_bytes(uint32_t format, uint32_t bits, uint64_t n);

uint64_t ora_get(const ora_column* c, uint64_t i);
/* canonical encoder: buffer is fully rewritten, dead/tail bits are zero */
void ora_encode(uint32_t format, uint32_t bits, const uint64_t* values, uint64_t n, void* out);
void ora_decode(const ora_column* c, uint64_t* values);

int ora_pred_eval(const ora_pred* p, uint64_t v);
uint64_t ora_binop(uint32_t op, uint64_t l, uint64_t r, uint32_t out_bits);
uint32_t ora_binop_out_bits(uint32_t op, uint32_t lbits, uint32_t rbits);

/* filter -> LSB-first bitmask in uint32 words, bits past n are zero */
void ora_filter(const ora_column* in, const ora_pred* p, uint32_t* mask);
/* compressstore: survivors of the mask, canonical output at out->format/bits */
uint64_t ora_compressstore(const ora_column* in, const uint32_t* mask, ora_column* out);
uint64_t ora_filter_compressstore(const ora_column* in, const ora_pred* p, ora_column* out);
void ora_binary(uint32_t op, const ora_column* l, const ora_column* r, ora_column* out);
uint64_t ora_reduce(uint32_t agg, const ora_column* in, const uint32_t* mask /* may be NULL */);

/* fused chain: v = op(l, r) [r may be NULL -> v = l], keep pred(v),
 * compact survivors into out (may be NULL), aggregate survivors. */
typedef struct {
    uint64_t count;
    uint64_t agg;
} ora_chain_result;
ora_chain_result ora_chain(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits, const ora_pred* p,
                           uint32_t agg, ora_column* out);
/* same, over element range [begin, end) only (no output), for the threaded timer */
ora_chain_result ora_chain_range(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits, const ora_pred* p,
                                 uint32_t agg, uint64_t begin, uint64_t end);
/* threaded CPU baseline: count + aggregate of the chain with `threads` pthreads */
ora_chain_result ora_chain_mt(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits, const ora_pred* p,
                              uint32_t agg, int threads);
/* ora_chain that also writes the survivors to out (capacity >= l->n), multi-threaded */
ora_chain_result ora_chain_compress_mt(uint32_t op, const ora_column* l, const ora_column* r, uint32_t vbits,
                                       const ora_pred* p, uint32_t agg, const ora_column* out, int threads);

/* group-by: dense per-key sums/counts (keys must be < 2^key_bits, key_bits <= 24).
 * Returns the number of distinct keys. */
/* sort-based group-by, keys up to 32 bits (the reference's sort + reduce-by-key path) */
uint64_t ora_groupby_sorted(const ora_column* keys, const ora_column* vals, const uint32_t* mask, uint64_t* out_keys,
                            uint64_t* out_sums, uint64_t* out_counts);
uint64_t ora_groupby_dense(const ora_column* keys, const ora_column* vals, uint64_t* sums, uint64_t* counts);

/* matrix multiply: A (M x K), B (K x N) row-major, out int64 (M x N).
 * Slab format is row-padded: src/common_code.cuh:124-129. */
void ora_matmul(const ora_column* a, const ora_column* b, uint64_t m, uint64_t n, uint64_t k, int64_t* out, int threads);
uint64_t ora_matrix_get(const ora_column* c, uint64_t rows, uint64_t cols, uint64_t r, uint64_t col);
uint64_t ora_matrix_words(uint32_t format, uint32_t bits, uint64_t rows, uint64_t cols);
void ora_matrix_encode(uint32_t format, uint32_t bits, const uint64_t* values, uint64_t rows, uint64_t cols, void* out);

/* fixtures */
typedef struct {
    uint64_t state;
    uint64_t inc;
} ora_pcg32;
void ora_pcg32_seed(ora_pcg32* g, uint64_t seed); /* src/fast_prng.cuh:11-19 */
uint32_t ora_pcg32_next(ora_pcg32* g);           /* src/fast_prng.cuh:21-29 */
/* the reference's input arrays: src/main.cu:242-251 */
void ora_reference_inputs(uint64_t seed, uint64_t* data1, uint64_t* data2, uint64_t n);
/* src/main.cu:33-46 */
void ora_mask_uniform(uint8_t* buf, uint64_t offset, uint64_t length, double selectivity);
/* src/main.cu:59-108 (bit 7-(i%8) of byte i/8, MSB-first as the reference writes it) */
void ora_mask_clusters(uint8_t* buf, double selectivity, uint64_t cluster_count, uint64_t total);
uint64_t ora_xorshift64(uint64_t* state);
void ora_uniform_values(uint64_t seed, uint32_t bits, uint64_t* out, uint64_t n);

#ifdef __cplusplus
}
#endif
#endif
