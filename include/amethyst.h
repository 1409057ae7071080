/*
 * amethyst.h -- C ABI of the B200-native Amethyst operator layer (libamethyst_b200.so).
 *
 * Every operator accepts columns in any storage format and writes any storage format:
 *
 *   AMX_PLAIN32  one uint32 per element, value = word & mask(bits), bits 1..32
 *   AMX_PLAIN64  one uint64 per element, value = word & mask(bits), bits 1..64
 *                (the reference's "baseline" format: src/common_code.cuh:51-55)
 *   AMX_SLAB     floor(64/bits) elements per little-endian uint64 slab, element i in slab
 *                i/eps at bit (i%eps)*bits, dead top bits ignored on read and written 0
 *                (the reference's "slabs" format: src/common_code.cuh:43-50)
 *   AMX_NOGAPS   continuous bit stream, element i at bit i*bits
 *                (the reference's "nogaps" format: src/common_code.cuh:100-116)
 *
 * Bitmasks are LSB-first bit arrays in uint32 words (bit i of the mask = bit i%32 of word
 * i/32), bits past n zero -- the layout the reference's filter writes
 * (src/kernels/filter_slabs.cuh:55) and its compressstore reads (src/bit_iterator.cuh:18-21).
 *
 * Conventions shared by every entry point:
 *   - all data pointers are device pointers aligned to 16 bytes (cudaMalloc gives 256);
 *   - calls are asynchronous on `stream` (a cudaStream_t; NULL = legacy default stream),
 *     never synchronise, and never allocate memory;
 *   - operators that need scratch memory take a caller-owned device workspace of at least
 *     amx_workspace_bytes(n) bytes; the call clears the part it uses with
 *     cudaMemsetAsync on `stream`.  A workspace must not be shared by calls that may
 *     overlap on the GPU;
 *   - results that are scalars (counts, aggregates, group counts) are written to device
 *     memory, so a sequence of calls can be captured into a CUDA graph;
 *   - device-side failures (a bounded wait that ran out) are recorded in the workspace and
 *     read back with amx_workspace_status(), which synchronises the stream.
 * The status codes replace the reference's print-and-exit error handling
 * (src/cuda_try.cuh:8-21).
 */
#ifndef AMETHYST_H
#define AMETHYST_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AMX_VERSION 100

typedef enum {
    AMX_OK = 0,
    AMX_ERR_INVALID_ARG = 1,  /* null pointer, bad width, size mismatch, unknown enum */
    AMX_ERR_UNSUPPORTED = 2,  /* valid request this build does not implement */
    AMX_ERR_ALIGNMENT = 3,    /* a data pointer is not 16-byte aligned */
    AMX_ERR_WORKSPACE = 4,    /* workspace missing or smaller than required */
    AMX_ERR_CUDA = 5,         /* a CUDA runtime call failed (see amx_last_error) */
    AMX_ERR_TIMEOUT = 6,      /* a bounded device-side wait gave up; outputs are invalid */
    AMX_ERR_CAPACITY = 7      /* a size exceeds a documented maximum */
} amx_status;

typedef enum { AMX_PLAIN32 = 0, AMX_PLAIN64 = 1, AMX_SLAB = 2, AMX_NOGAPS = 3 } amx_format;

/* A column: `n` elements of `bits` bits stored at `data` in `format`. */
typedef struct {
    void* data;
    uint64_t n;
    uint32_t format;
    uint32_t bits;
} amx_column;

/* Predicates.  The reference compiles one predicate into each kernel instance
 * (FILTER_PREDICATE_OP, src/config.cuh:107-113); here it is a runtime descriptor.
 * AMX_PRED_HALF is that reference predicate: v >= 2^(bits-1), `bits` taken from the
 * descriptor. */
typedef enum {
    AMX_PRED_ALL = 0,
    AMX_PRED_LT = 1,          /* v <  k0 */
    AMX_PRED_LE = 2,          /* v <= k0 */
    AMX_PRED_GT = 3,          /* v >  k0 */
    AMX_PRED_GE = 4,          /* v >= k0 */
    AMX_PRED_EQ = 5,          /* v == k0 */
    AMX_PRED_NE = 6,          /* v != k0 */
    AMX_PRED_BETWEEN = 7,     /* k0 <= v <= k1 */
    AMX_PRED_NOT_BETWEEN = 8, /* !(k0 <= v <= k1) */
    AMX_PRED_HALF = 9         /* v >= 2^(bits-1) */
} amx_pred_kind;

typedef struct {
    uint32_t kind;
    uint32_t bits;
    uint64_t k0;
    uint64_t k1;
} amx_predicate;

/* Element-wise binary operators; every result is masked to the output column's width like
 * the reference's op_* templates (src/config.cuh:5-42).  x/0 = all ones, x%0 = x. */
typedef enum {
    AMX_OP_ADD = 0,
    AMX_OP_SUB = 1,      /* (l - r) mod 2^out_bits */
    AMX_OP_MUL = 2,
    AMX_OP_DIV = 3,
    AMX_OP_MOD = 4,
    AMX_OP_MIN = 5,
    AMX_OP_MAX = 6,
    AMX_OP_AND = 7,
    AMX_OP_OR = 8,
    AMX_OP_XOR = 9,
    AMX_OP_BOOL_OR = 10,  /* op_bool_simple  */
    AMX_OP_BOOL_XOR = 11, /* op_bool_complex */
    AMX_OP_MATH = 12,     /* op_math: (l*l + r*r + 4l) / (l*l + r*r + 5l) */
    AMX_OP_LHS = 13       /* identity on the left operand */
} amx_binop;

/* Horizontal aggregations ("hop", src/config.cuh:62-71), all into uint64. */
typedef enum { AMX_AGG_SUM = 0, AMX_AGG_MIN = 1, AMX_AGG_MAX = 2, AMX_AGG_AND = 3, AMX_AGG_OR = 4, AMX_AGG_XOR = 5 } amx_agg;

/* ---- sizing and diagnostics --------------------------------------------------------- */
int amx_version(void);
const char* amx_status_string(amx_status s);
/* message of the last failed call on this host thread */
const char* amx_last_error(void);
/* storage bytes of a column of n elements */
uint64_t amx_storage_bytes(uint32_t format, uint32_t bits, uint64_t n);
/* bytes of an n-element bitmask: ceil(n/32) * 4 */
uint64_t amx_mask_bytes(uint64_t n);
/* narrowest output width that never truncates op(lhs, rhs) */
uint32_t amx_binary_out_bits(uint32_t op, uint32_t lhs_bits, uint32_t rhs_bits);
/* workspace bytes needed by the column operators on n elements */
uint64_t amx_workspace_bytes(uint64_t n);
/* synchronises `stream`, then reports a device-side failure recorded in `workspace` by the
 * last call that used it (AMX_OK if none) */
amx_status amx_workspace_status(const void* workspace, void* stream);

/* Launch tuning for the calls this host thread makes next (the autotuner's knobs).  Zero
 * fields mean "automatic".  staged_bytes: input bytes kept staged ahead of the compute warps
 * (sets the depth of the shared-memory ring); compact_stages: ring depth of compacting passes;
 * policy: 0 automatic, 1 the generic runtime-width kernel, 1 + id a compile-time-width kernel
 * (id = slab width for one column); for amx_matmul 2 selects the fused kernel (operands unpacked
 * in shared memory from TMA-staged packed slices, product packed from the accumulators; slab
 * operands of one width) and 3 the same with the packed words read from global memory;
 * max_ctas: cap on the persistent grid of the group-by aggregation (0: every CTA that fits).
 * amx_set_tuning(NULL) restores the defaults. */
typedef struct {
    uint32_t staged_bytes;
    uint32_t compact_stages;
    int32_t policy;
    uint32_t max_ctas;
} amx_tuning;
amx_status amx_set_tuning(const amx_tuning* t);
amx_status amx_get_tuning(amx_tuning* t);

/* Test hook for the failure path (no reference counterpart; the reference prints and exits,
 * src/cuda_try.cuh:8-21).  For the tile-pipeline launches this host thread makes next, the kernel
 * never publishes the look-back count of tile `tile`, and every look-back poll loop gives up after
 * `wait_polls` polls (0: the built-in bound of 2^20).  The waits on that tile then run out: the
 * kernel records AMX_ERR_TIMEOUT, takes the missing count as 0, finishes (its compacted outputs
 * are invalid), and amx_workspace_status() reports the timeout.  Nothing faults or hangs.
 * tile = UINT64_MAX switches the hook off. */
amx_status amx_test_lookback_timeout(uint64_t tile, uint32_t wait_polls);

/* ---- column operators ------------------------------------------------------------------ */

/* filter -> bitmask.  Replaces kernel_filter_{slabs,nogaps,baseline}
 * (src/kernels/filter_slabs.cuh:4-57, filter_nogaps.cuh:4-65, filter_baseline.cuh:9-36). */
amx_status amx_filter(const amx_column* in, const amx_predicate* pred, uint32_t* d_mask, void* workspace,
                      size_t workspace_bytes, void* stream);

/* compressstore: the elements whose mask bit is set, in order, written to `out`
 * (out->n is its capacity and must be >= in->n); the survivor count goes to *d_count.
 * Replaces the popcount -> scan -> write pipeline of bench_compressstore_slabs
 * (src/benchs/bench_compressstore_slabs.cu:38-56, kernels
 * src/kernels/compressstore_slabs.cuh:4-206) and the CUB plain path
 * (src/benchs/bench_compressstore_baseline_cub.cu:35). */
amx_status amx_compressstore(const amx_column* in, const uint32_t* d_mask, const amx_column* out, uint64_t* d_count,
                             void* workspace, size_t workspace_bytes, void* stream);

/* filter fused with compressstore: no mask is materialised. */
amx_status amx_filter_compressstore(const amx_column* in, const amx_predicate* pred, const amx_column* out,
                                    uint64_t* d_count, void* workspace, size_t workspace_bytes, void* stream);

/* filter fused with compressstore for callers that cannot allocate device memory (no
 * counterpart in the reference).  Identical results to amx_filter_compressstore, but it takes no
 * workspace: its scratch is a fixed 1 MiB array inside the library's device memory, held by
 * every GPU that loads the library until the process exits.  Columns longer than 2^29 elements
 * are rejected with AMX_ERR_CAPACITY.  All calls share that array and each call clears what it
 * needs first, so calls ordered on one stream are fine but calls that may overlap on the GPU
 * race.  The first call on a device looks up the array's address there; make it before any
 * stream capture starts.  Calls no cudaMalloc, cudaFree or allocating library routine. */
amx_status amx_filter_compressstore_noalloc(const amx_column* in, const amx_predicate* pred, const amx_column* out,
                                            uint64_t* d_count, void* stream);
/* synchronises `stream`, then reports a device-side failure (AMX_ERR_TIMEOUT: the outputs are
 * invalid) recorded by the last amx_filter_compressstore_noalloc call on the current device;
 * AMX_OK if none.  The next no-alloc call clears the record, so check before making it.  The
 * array's address is looked up once per device: do not call either no-alloc entry point on a
 * device after cudaDeviceReset in the same process. */
amx_status amx_filter_compressstore_noalloc_status(void* stream);

/* element-wise binary op, lhs and rhs may differ in format and width.  Replaces
 * kernel_binary_op_{slabs,nogaps,baseline} (src/kernels/binary_op_slabs.cuh:7-67,
 * binary_op_nogaps.cuh:5-89, binary_op_baseline.cuh:4-13). */
amx_status amx_binary(uint32_t op, const amx_column* lhs, const amx_column* rhs, const amx_column* out,
                      void* workspace, size_t workspace_bytes, void* stream);

/* re-encode a column in another format / width (values masked to out->bits). */
amx_status amx_convert(const amx_column* in, const amx_column* out, void* workspace, size_t workspace_bytes,
                       void* stream);

/* aggregation of all elements (d_mask NULL) or of the masked ones.  Replaces
 * kernel_hop_{slabs,nogaps} (src/kernels/hop.cuh:7-76) and cub::DeviceReduce
 * (src/benchs/bench_hop_baseline_cub.cu:38). */
amx_status amx_reduce(uint32_t agg, const amx_column* in, const uint32_t* d_mask, uint64_t* d_result,
                      void* workspace, size_t workspace_bytes, void* stream);

/* ---- group-by ---------------------------------------------------------------------------- */
/* Group-by sum + count: for every distinct key (ascending) the key, the uint64 sum of its values
 * and its count, compressed into the three output columns (each may be NULL; capacity >=
 * 2^key_bits for keys of at most 24 bits); the number of groups goes to *d_groups.  Keys: any
 * format, at most 32 bits.  Keys of 25..32 bits aggregate into a global hash table whose size the
 * workspace sets (amx_groupby_wide_workspace_bytes(key_bits, max_groups) holds max_groups
 * distinct keys at half load); the groups come out in ascending key order as well, at most as
 * many as the smallest output capacity, and more distinct keys than the table or the outputs
 * hold is reported by amx_groupby_status as AMX_ERR_CAPACITY.
 * Values: any format and width.  Optional d_mask restricts the input to the masked elements.
 * Writing sums into a narrower column masks them, which gives the reference's aggregate
 * (sum masked to the key width).  Replaces kernel_groupby_sm_array_gather/_writeout
 * (src/kernels/groupby_sm_array.cuh:4-81) and the sort-based path
 * (src/benchs/bench_groupby_sort_cub.cu:50-63).  The workspace must be 256-byte aligned. */
uint64_t amx_groupby_workspace_bytes(uint32_t key_bits);  /* keys <= 24 bits; 0 otherwise */
uint64_t amx_groupby_wide_workspace_bytes(uint32_t key_bits, uint64_t max_groups);  /* keys of 25..32 bits */
/* synchronises `stream`, then reports a device-side failure recorded in `workspace` by the last
 * amx_groupby with keys of key_bits (AMX_ERR_CAPACITY: a full table or output; AMX_ERR_TIMEOUT) */
amx_status amx_groupby_status(const void* workspace, uint32_t key_bits, void* stream);
amx_status amx_groupby(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                       const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                       uint64_t* d_groups, void* workspace, size_t workspace_bytes, void* stream);

/* Sort-based group-by: the same results as amx_groupby (ascending keys, uint64 sums, counts) for
 * keys of 1..32 bits and values of 1..64 bits in any format, by an LSD radix sort of the key/value
 * pairs in 8-bit digits followed by a reduce-by-key -- the reference's sort path
 * (src/benchs/bench_groupby_sort_cub.cu:48-66: cub::DeviceRadixSort::SortPairs then
 * cub::DeviceReduce::ReduceByKey).  Its cost does not depend on the number of groups, which has
 * no bound but n.  Outputs hold as many groups as their capacity; more groups record
 * AMX_ERR_CAPACITY (amx_groupby_sort_status).  The workspace (256-byte aligned) holds two copies
 * of the pairs and one of the groups: amx_groupby_sort_workspace_bytes(n, key_bits, value_bits). */
uint64_t amx_groupby_sort_workspace_bytes(uint64_t n, uint32_t key_bits, uint32_t value_bits);
amx_status amx_groupby_sort(const amx_column* keys, const amx_column* vals, const uint32_t* d_mask,
                            const amx_column* out_keys, const amx_column* out_sums, const amx_column* out_counts,
                            uint64_t* d_groups, void* workspace, size_t workspace_bytes, void* stream);
/* synchronises `stream`, then reports a device-side failure recorded by the last amx_groupby_sort
 * that used `workspace` */
amx_status amx_groupby_sort_status(const void* workspace, void* stream);

/* ---- batches of columns ------------------------------------------------------------------ */
/* Filter + compressstore + sum over `ncols` slab columns of any lengths and widths (1..32 bits)
 * in one persistent launch.  Column i keeps the elements that pass preds[i], compacted into
 * outs[i] (slabs of the input width, capacity >= ins[i].n); its survivor count goes to
 * d_counts[i] and the uint64 sum of its survivors to d_sums[i].  The reference launches every
 * operator once per column (src/main.cu:300-340).
 *   amx_batch_prepare   validates the columns, uploads the column table to the workspace and
 *                       fills `plan` (synchronises `stream` once; call it outside graph capture);
 *   amx_batch_run       clears the outputs and launches the batch: stream-ordered, allocation-free
 *                       and capturable into a CUDA graph, replayable as long as the columns and
 *                       the workspace stay in place.
 * Tuning (may be NULL): threads per CTA, CTAs per SM and slab words per thread (the tile size);
 * the autotuner (amethyst_b200/autotune.py) picks them per workload. */
typedef struct {
    uint32_t threads;           /* threads per CTA: 256 or 512 */
    uint32_t ctas_per_sm;       /* 0: as many as fit */
    uint32_t words_per_thread;  /* slab words each thread takes per tile, 1..8 (0: 8); sets the tile size */
    uint32_t reserved;
} amx_batch_tuning;

typedef struct {
    uint32_t ncols;
    uint32_t threads;
    uint32_t grid;
    uint32_t reserved;
    uint64_t items;
    uint64_t workspace_bytes;
} amx_batch_plan;

uint64_t amx_batch_workspace_bytes(const amx_column* ins, uint32_t ncols, const amx_batch_tuning* tuning);
amx_status amx_batch_prepare(const amx_column* ins, const amx_predicate* preds, const amx_column* outs, uint32_t ncols,
                             const amx_batch_tuning* tuning, amx_batch_plan* plan, void* workspace,
                             size_t workspace_bytes, void* stream);
amx_status amx_batch_run(const amx_batch_plan* plan, uint64_t* d_counts, uint64_t* d_sums, void* workspace,
                         size_t workspace_bytes, void* stream);
/* synchronises `stream`, then reports a device-side failure recorded by the last batch run */
amx_status amx_batch_status(const void* workspace, void* stream);

/* ---- matrix op ---------------------------------------------------------------------------- */
/* C (M x N) = A (M x K) * B (K x N) over unsigned entries of at most 8 bits, exact, on the integer
 * tensor cores (u8 x u8 -> int32).  Matrices are columns of M*K, K*N and M*N entries: AMX_SLAB
 * matrices pad every row to whole slabs (get_matrix_element, src/common_code.cuh:124-129), the
 * other formats are row-major.  K * (2^a_bits - 1) * (2^b_bits - 1) must stay below 2^31
 * (AMX_ERR_UNSUPPORTED otherwise).  out->bits == 0 writes C at the narrowest width that holds
 * its largest entry and stores that width in *d_out_bits (device memory, may be NULL); size
 * `out` with amx_matmul_out_bytes(format, 0, ...), the widest possible case.  A nonzero
 * out->bits masks every entry to that width.  The workspace (amx_matmul_workspace_bytes) must be
 * 1024-byte aligned.  By default the operands are unpacked once to u8 in the workspace and the
 * int32 product is packed by a second pass; amx_tuning.policy = 2 or 3 selects the fused kernel
 * (slab operands of one width: unpacked in shared memory, packed from the accumulators, nothing
 * decompressed to HBM), which is bit-identical and measured slower.  The reference has no matrix
 * kernel, only the element accessors (src/common_code.cuh:65-86,118-134). */
uint64_t amx_matmul_workspace_bytes(uint32_t M, uint32_t N, uint32_t K);
uint64_t amx_matmul_out_bytes(uint32_t format, uint32_t out_bits, uint32_t M, uint32_t N, uint32_t K, uint32_t a_bits,
                              uint32_t b_bits);
amx_status amx_matmul(const amx_column* a, const amx_column* b, uint32_t M, uint32_t N, uint32_t K,
                      const amx_column* out, uint32_t* d_out_bits, void* workspace, size_t workspace_bytes,
                      void* stream);
/* synchronises `stream`, then reports a device-side failure recorded by the last amx_matmul that
 * used `workspace` (AMX_OK if none) */
amx_status amx_matmul_status(const void* workspace, void* stream);

/* ---- fused operator chain -------------------------------------------------------------- */
/* v = op(lhs, rhs) masked to value_bits (v = lhs when rhs is NULL), keep the elements with
 * pred(v), then any of: the survivors compacted into `out`, the bitmask of pred(v) into
 * d_mask, the survivor count into *d_count, agg over the survivors into *d_agg.  Each
 * output pointer may be NULL.  One pass over the inputs; no intermediate reaches memory.
 * The reference has no fused chain (src/op_chaining_demo.cu:137-152 runs operators one
 * after another). */
typedef struct {
    uint32_t op;
    uint32_t value_bits;
    amx_predicate pred;
    uint32_t agg;
    uint32_t reserved;
} amx_chain_desc;

amx_status amx_chain(const amx_chain_desc* desc, const amx_column* lhs, const amx_column* rhs, const amx_column* out,
                     uint32_t* d_mask, uint64_t* d_count, uint64_t* d_agg, void* workspace, size_t workspace_bytes,
                     void* stream);

/* ---- operator-chain programs ------------------------------------------------------------- */
/* A program runs a chain of steps over one column x with no host round trip: every length a
 * step produces (a compressstore's survivor count) stays in device memory and the following
 * kernels read it there, so a program is a fixed sequence of stream-ordered launches that can
 * be captured into a CUDA graph.  State: the column x (initially the input), its length len,
 * and the live filter mask (initially none).  Steps:
 *   FILTER         mask = pred(x[0..len))
 *   COMPRESSSTORE  x = the elements of x whose mask bit is set (pred(x) when no mask is live),
 *                  stored as out_format / out_bits; len = their count; no mask is live after it
 *   BINARY         x = op(x, aux[0..len)) masked to value_bits, stored as out_format / out_bits;
 *                  the mask stays live.  out_format AMX_FORMAT_FUSED (only before a
 *                  COMPRESSSTORE) runs the op inside that step's pass: no intermediate
 *   REDUCE         *d_result = op (an amx_agg) over x[0..len) (the masked elements if a mask is
 *                  live)
 *   GROUPBY        group-by sum + count of x[0..len) by the keys aux[0..len) (masked if a mask
 *                  is live) into group_keys / group_sums / group_counts (any may have NULL data;
 *                  capacity >= 2^aux.bits), the number of groups into *d_result; keys <= 24 bits
 * Steps that one pass can serve run as one: a FILTER directly before a COMPRESSSTORE becomes its
 * predicate, and a REDUCE directly after a COMPRESSSTORE, a FILTER, or a BINARY op with no live
 * mask is computed in that step's pass.  AMX_FORMAT_FUSED may also precede FILTER, COMPRESSSTORE.
 * A storage width narrower than the values keeps their low bits: choose one only for values
 * known to fit.  aux columns hold at least x.n elements; the first len of them are used.  The
 * reference runs operators one after another with a host-side count between them
 * (src/op_chaining_demo.cu:137-152, src/benchs/bench_compressstore_slabs.cu:60-62); programs have
 * no reference counterpart. */
typedef enum {
    AMX_STEP_FILTER = 0,
    AMX_STEP_COMPRESSSTORE = 1,
    AMX_STEP_BINARY = 2,
    AMX_STEP_REDUCE = 3,
    AMX_STEP_GROUPBY = 4
} amx_step_kind;

#define AMX_FORMAT_FUSED 0xffu
#define AMX_PROGRAM_MAX_STEPS 32

typedef struct {
    uint32_t kind;
    uint32_t op;          /* BINARY: amx_binop; REDUCE: amx_agg */
    uint32_t value_bits;  /* BINARY: width the result is masked to */
    uint32_t out_format;  /* BINARY, COMPRESSSTORE: storage of the new x (AMX_FORMAT_FUSED: none) */
    uint32_t out_bits;    /* BINARY, COMPRESSSTORE: storage width of the new x */
    uint32_t reserved;
    amx_predicate pred;   /* FILTER; COMPRESSSTORE when no mask is live */
    amx_column aux;       /* BINARY: right operand; GROUPBY: keys */
    uint64_t* d_result;   /* REDUCE: the aggregate; GROUPBY: the number of groups; COMPRESSSTORE: the
                           * survivor count (GROUPBY, COMPRESSSTORE: may be NULL) */
    amx_column group_keys;
    amx_column group_sums;
    amx_column group_counts;
} amx_step;

typedef struct amx_program amx_program;

/* validates the steps and plans the workspace (host only; the step array is copied) */
amx_status amx_program_create(const amx_column* x, const amx_step* steps, uint32_t nsteps, amx_program** prog);
/* device workspace a run needs (256-byte aligned, reusable by consecutive runs on one stream) */
uint64_t amx_program_workspace_bytes(const amx_program* prog);
/* enqueues every step on `stream`: no synchronisation, no allocation, capturable */
amx_status amx_program_run(const amx_program* prog, void* workspace, size_t workspace_bytes, void* stream);
/* the final x of the last run: its column (data inside the workspace or the input's own; n = the
 * capacity) and a device pointer to its length (NULL when no step changes the length: x->n) */
amx_status amx_program_output(const amx_program* prog, const void* workspace, amx_column* x, const uint64_t** d_len);
/* synchronises `stream`, then reports a device-side failure recorded by the last run */
amx_status amx_program_status(const amx_program* prog, const void* workspace, void* stream);
void amx_program_destroy(amx_program* prog);

/* Many programs in one CUDA graph: program i runs on lane i's stream (lanes assigned longest
 * first to the least loaded lane), lanes fork from and join the launching stream, so the
 * programs of different lanes overlap on the GPU.  Each program needs its own workspace.  The
 * capture uses internal streams; launching replays every program with no host work per step. */
typedef struct amx_graph amx_graph;
amx_status amx_graph_capture(const amx_program* const* progs, void* const* workspaces, const uint64_t* workspace_bytes,
                             uint32_t count, uint32_t lanes, amx_graph** graph);
amx_status amx_graph_launch(const amx_graph* graph, void* stream);
void amx_graph_destroy(amx_graph* graph);

/* ---- column statistics ------------------------------------------------------------------- */
/* d_hist[k] += number of elements whose value needs exactly k bits (k = 0 for the value 0),
 * k = 0..64 (65 uint64 counters, caller-cleared) -- the bit-width histogram the format selector
 * reads.  No reference counterpart. */
amx_status amx_bit_histogram(const amx_column* in, uint64_t* d_hist, void* stream);

/* ---- learned format selector ------------------------------------------------------------- */
/* A 16 -> 64 -> 64 -> classes FP32 MLP (ReLU, softmax) that picks storage formats and widths for
 * the intermediate columns of operator chains (amethyst_b200/selector.py builds its features and
 * labels).  Parameters: W1[64][16] b1[64] W2[64][64] b2[64] W3[classes][64] b3[classes], as one
 * float array of amx_mlp_param_count(classes) entries; classes 2..8.  No reference counterpart:
 * the reference fixes every format at compile time (src/main.cu:300-340).
 *   amx_mlp_forward     probabilities [batch][classes] for features [batch][16];
 *   amx_mlp_train_step  one mini-batch of softmax cross-entropy and one Adam step (step >= 1;
 *                       d_adam holds 2 * param_count floats, zero before the first step); the
 *                       mean loss goes to *d_loss (may be NULL).  Deterministic. */
uint32_t amx_mlp_param_count(uint32_t classes);
amx_status amx_mlp_forward(const float* d_params, uint32_t classes, const float* d_x, uint32_t batch, float* d_probs,
                           void* stream);
amx_status amx_mlp_train_step(float* d_params, float* d_adam, uint32_t step, uint32_t classes, const float* d_x,
                              const uint32_t* d_labels, uint32_t batch, float lr, float* d_loss, void* stream);

/* ---- synthetic data (benchmarks and tests; no reference counterpart) --------------------- */
/* element i = top `bits` bits of splitmix64(seed + (i+1)*0x9E3779B97F4A7C15) followed by one
 * xorshift64 (13,7,17) step, written as plain uint32 (elem_bytes 4) or uint64 (8) words */
amx_status amx_fill_uniform(void* d_out, uint64_t n, uint32_t elem_bytes, uint32_t bits, uint64_t seed, void* stream);
/* keys by inverse CDF: u = draw(i) >> 11 scaled to [0,1), key = first k with d_cdf[k] > u
 * (d_cdf: `groups` ascending doubles ending at 1.0) -- e.g. Zipf-distributed group keys */
amx_status amx_fill_from_cdf(uint32_t* d_out, uint64_t n, const double* d_cdf, uint32_t groups, uint64_t seed,
                             void* stream);

#ifdef __cplusplus
}
#endif
#endif
