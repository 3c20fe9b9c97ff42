/*
 * einfold_b200 — a C ABI for einfold's kernel layer on one NVIDIA B200.
 *
 * The entry points replace the four functions that einfold's physical
 * operator calls (crates/einfold-kernels/src/algorithm.rs:52-160):
 *
 *   einfold_fold        <- einfold_kernels::fold        (algorithm.rs:97-133)
 *   einfold_fold_dense  <- einfold_kernels::fold_dense  (algorithm.rs:52-62)
 *   einfold_fold_chain  <- einfold_kernels::fold_chain  (algorithm.rs:76-83)
 *   einfold_pipeline    <- einfold_kernels::pipeline    (algorithm.rs:146-160)
 *   einfold_schema / einfold_pipeline_schema
 *                       <- einfold_kernels::{schema, pipeline_schema}
 *                          (schema.rs:31-36, 155-206)
 *
 * Tables cross the boundary in the Arrow C Data Interface: a relation is its
 * batches, each exported as a struct array (what arrow-rs's
 * `FFI_ArrowArray::new(&StructArray::from(batch).to_data())` and pyarrow's
 * `RecordBatch._export_to_c` give), with the schema exported once. Results
 * come back the same way and are owned by the library until
 * einfold_result_release. Fold and pipeline descriptions are plain structs
 * mirroring crates/einfold-ir (fold.rs:59-416, pipeline.rs:63-201,
 * expression.rs:57-135).
 *
 * The lower entry points (einfold_rank_words, einfold_split_gemm,
 * einfold_fp64_gemm, einfold_attention_*) take device pointers and a CUDA
 * stream; they serve a caller that keeps its data in HBM, such as the
 * torch.autograd.Function in the Python package, and the benchmarks. A
 * NULL stream there means the context's own stream, which is created
 * non-blocking: it does not wait for work queued on the legacy default
 * stream. A caller whose operands are written on the default stream passes
 * cudaStreamLegacy; one that writes them on another stream passes that
 * stream. The Arrow entry points run on the context's stream: operands in
 * HBM must be complete before the call.
 *
 * Every call is synchronous with respect to the host unless it takes a
 * stream. Calls on one context are serialized by the context; contexts on
 * the same device may be used from different threads.
 */
#ifndef EINFOLD_B200_H
#define EINFOLD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Arrow C Data Interface (https://arrow.apache.org/docs/format/CDataInterface.html) ---- */
#ifndef ARROW_C_DATA_INTERFACE
#define ARROW_C_DATA_INTERFACE
#define ARROW_FLAG_DICTIONARY_ORDERED 1
#define ARROW_FLAG_NULLABLE 2
#define ARROW_FLAG_MAP_KEYS_SORTED 4
struct ArrowSchema {
  const char* format;
  const char* name;
  const char* metadata;
  int64_t flags;
  int64_t n_children;
  struct ArrowSchema** children;
  struct ArrowSchema* dictionary;
  void (*release)(struct ArrowSchema*);
  void* private_data;
};
struct ArrowArray {
  int64_t length;
  int64_t null_count;
  int64_t offset;
  int64_t n_buffers;
  int64_t n_children;
  const void** buffers;
  struct ArrowArray** children;
  struct ArrowArray* dictionary;
  void (*release)(struct ArrowArray*);
  void* private_data;
};
#endif

/* ---- Status ---- */
typedef enum {
  EINFOLD_OK = 0,
  /* The kernels' requirements don't hold: the caller runs the host's plan
   * (Ok(None) in the reference). */
  EINFOLD_DECLINED = 1,
  /* The budget refused memory (ArrowError::MemoryError, options.rs:101-108). */
  EINFOLD_BUDGET = 2,
  /* Inputs the fold doesn't fit (ArrowError::InvalidArgumentError, lib.rs:54-56). */
  EINFOLD_INVALID = 3,
  /* A limit of the algorithm (ArrowError::ComputeError, discriminate.rs:383-387). */
  EINFOLD_COMPUTE = 4,
  /* A CUDA error: the device is unusable for this call. */
  EINFOLD_DEVICE = 5,
  /* A bounded device-side wait ran out; the context stays usable. */
  EINFOLD_TIMEOUT = 6
} einfold_status;

/* Which algorithm computed a fold (algorithm.rs:23-36). */
typedef enum { EINFOLD_ALG_NONE = 0, EINFOLD_ALG_DENSE = 1, EINFOLD_ALG_DISCRIMINATE = 2, EINFOLD_ALG_FUSED = 3 } einfold_algorithm;

/* ---- Fold descriptions (crates/einfold-ir/src/fold.rs) ---- */
typedef struct { int32_t dimension; int32_t column; } einfold_key;            /* fold.rs:Key */
typedef struct {                                                              /* fold.rs:Operand */
  int32_t n_keys;
  const einfold_key* keys;
  int32_t factor; /* column index, or -1 for none */
} einfold_operand;
typedef struct {                                                              /* fold.rs:Output */
  int32_t dimension;
  int32_t domain_column;   /* -1 when the fold has no domain */
  int32_t domain_equality; /* 0 '=', 1 IS NOT DISTINCT FROM */
} einfold_output;
typedef struct {                                                              /* fold.rs:Condition */
  int32_t left;
  int32_t comparison; /* 0 <, 1 <=, 2 >, 3 >= */
  int32_t right;
  int32_t pad;
  int64_t offset;     /* left <comparison> right + offset */
} einfold_condition;
typedef struct {                                                              /* fold.rs:Domain */
  int32_t n_carry;
  const int32_t* carry;
  int32_t has_missing;
  int32_t pad;
  double missing;
} einfold_domain;
/* An expression in postfix order (expression.rs:117-135). kind: 0 column
 * (a = operand, b = column), 1 literal (value), 2 unary (a = 0 negate,
 * 1 abs, 2 exp, 3 ln), 3 binary (a = 0 +, 1 -, 2 *, 3 /, 4 power). */
typedef struct { int32_t kind; int32_t a; int32_t b; int32_t pad; double value; } einfold_expr_node;
typedef struct { int32_t n_nodes; const einfold_expr_node* nodes; } einfold_expression;

typedef struct {
  int32_t n_dimensions;
  const int32_t* equality;   /* per dimension: 0 '=', 1 IS NOT DISTINCT FROM */
  int32_t n_operands;
  const einfold_operand* operands;
  int32_t n_outputs;
  const einfold_output* outputs;
  int32_t row_is_expression; /* 0: product of factors; 1: `row` */
  einfold_expression row;
  const einfold_domain* domain; /* NULL: no domain */
  int32_t n_conditions;
  const einfold_condition* conditions;
} einfold_fold_desc;

/* ---- Pipelines (crates/einfold-ir/src/pipeline.rs) ---- */
typedef struct {
  const einfold_fold_desc* producer;
  int32_t weight_is_expression; /* 0: Weight::Exp{scale, shift}; 1: Weight::Of(weight) */
  int32_t scale_kind;           /* 0 One, 1 Times(c), 2 Over(c) */
  double scale_c;
  int32_t shift;                /* 0 None, 1 KeptMaximum */
  int32_t normalizer;           /* 0 KeptGroups, 1 JoinedRows, 2 None */
  einfold_expression weight;    /* reads operand 0, column 0: the score */
  int32_t n_dimensions;         /* the pipeline's own dimensions */
  const int32_t* equality;
  einfold_operand values;
  int32_t n_outputs;
  const int32_t* outputs;
} einfold_pipeline_desc;

/* ---- Relations ---- */
typedef struct {
  const struct ArrowSchema* schema; /* a struct schema: the relation's columns */
  int64_t n_batches;
  struct ArrowArray* const* batches; /* each a struct array of `schema` */
  /* Where the batches' buffers live: -1 host memory; d >= 0 the memory of
   * CUDA device d (the Arrow C Device Data Interface's ARROW_DEVICE_CUDA).
   * Device columns must state their null counts. */
  int32_t device;
  int32_t pad;
} einfold_relation;

/* ---- Options (options.rs:70-84) ---- */
typedef struct {
  int32_t float_keys;  /* 0 Bitwise, 1 SignedZerosEqual (options.rs:14-23) */
  int32_t threads;     /* host threads for staging; results don't depend on it */
  int32_t domain_rows; /* 0 Any, 1 UniqueKeys (options.rs:35-44) */
  /* Dense products: 0 split (int8 slices on the tensor cores, exact integer
   * accumulation, FP64 combine), 1 fp64 (CUDA-core FP64 in the reference's
   * order of additions: the reference's bits). */
  int32_t precision;
  int32_t slices;      /* split products: slices per operand, 0 = default (6) */
  /* 0: result buffers in host memory; 1: in the context's device memory
   * (released with cudaFree by the arrays' release callbacks). */
  int32_t result_on_device;
  /* The budget (options.rs:56-65): grow returns nonzero if `bytes` more may be
   * allocated; shrink gives bytes back. NULL grow = no limit. */
  void* budget_ctx;
  int32_t (*budget_grow)(void* ctx, uint64_t bytes);
  void (*budget_shrink)(void* ctx, uint64_t bytes);
} einfold_options;

/* ---- Results ---- */
typedef struct {
  int32_t status;    /* einfold_status */
  int32_t algorithm; /* einfold_algorithm */
  int64_t n_batches;
  struct ArrowArray* batches; /* n_batches struct arrays, library-owned */
  struct ArrowSchema* schema; /* the result's schema, library-owned */
  uint64_t tiles_visited;     /* pipelines: pairs of tiles computed (fused.rs:114-123) */
  uint64_t tiles;             /* pipelines: pairs of tiles in the same batch */
  /* Device kernels launched and device milliseconds spent, for metrics. */
  uint64_t kernels_launched;
  double device_ms;
  /* The dense products' tensor-core kernels: milliseconds (CUDA events around
   * their launches on the call's stream) and int8 multiply-adds x 2 done. */
  double product_ms;
  double product_ops;
  /* Attention forwards in the split form: how the (query tile, batch) items
   * reached the SMs (0 a block per item, 1 persistent blocks claiming them by
   * key tiles, 2 persistent batch by batch; -1 other calls), picked by timing
   * each on the first call of a padded shape (extents and conditions, whatever
   * the ragged lengths) unless EINFOLD_ATTENTION_SCHEDULE =
   * grid | tiles | batches forces one; and how the tile phase was launched
   * (0 directly: arguments seen for the first time, or EINFOLD_GRAPHS=0;
   * 1 a CUDA graph replayed; seen a second time, 2 one updated with the new
   * arguments or 3 one captured and instantiated). */
  int32_t schedule;
  int32_t graph;
  char message[480];
} einfold_result;

typedef struct einfold_context einfold_context;

/* A context on `device` (one stream). NULL on failure; see einfold_last_error. */
einfold_context* einfold_context_create(int32_t device);
void einfold_context_destroy(einfold_context* ctx);
const char* einfold_last_error(void);
/* The library's version string. */
const char* einfold_version(void);

/* einfold_kernels::fold: dense when its requirements hold, else
 * discrimination. `domain` may be NULL. */
int32_t einfold_fold(einfold_context* ctx, const einfold_fold_desc* fold, const einfold_relation* a,
                     const einfold_relation* b, const einfold_relation* domain, const einfold_options* options,
                     einfold_result* result);
/* einfold_kernels::fold_dense: the dense algorithm or EINFOLD_DECLINED. */
int32_t einfold_fold_dense(einfold_context* ctx, const einfold_fold_desc* fold, const einfold_relation* a,
                           const einfold_relation* b, const einfold_relation* domain,
                           const einfold_options* options, einfold_result* result);
/* einfold_kernels::fold_chain over three operands. */
int32_t einfold_fold_chain(einfold_context* ctx, const einfold_fold_desc* fold, const einfold_relation* operands,
                           const einfold_options* options, einfold_result* result);
/* einfold_kernels::pipeline over q, k and v. Where the reference's
 * placement declines an operand that misses cells (fused.rs:624-664), this
 * accepts ragged groups: every batch (the W dimensions) with its rows
 * present from position 0 to a length of its own along X (q) and along J
 * (k and v, the same length for both), each such row complete, and nothing
 * after; the rows past a batch's length join nothing and give no result
 * rows. Other missing cells decline, as the reference's placement does. */
int32_t einfold_pipeline(einfold_context* ctx, const einfold_pipeline_desc* pipeline,
                         const einfold_relation* operands, const einfold_options* options,
                         einfold_result* result);
/* The gradients of einfold_pipeline's result with respect to q's, k's and
 * v's factor columns, for the attention-shaped pipelines (product scores,
 * Weight::Exp{One or Times(c), KeptMaximum}, normalised over the kept
 * groups; others return EINFOLD_DECLINED). The reference has no backward
 * pass for its fused pipeline (docs/design.md:612); its gradients are
 * gradient SQL the host plan runs, which this computes in one call:
 * d_out holds the result's key columns (the pipeline's outputs, in order)
 * and a DOUBLE gradient per result row (a result row with no d_out row has
 * gradient 0). The forward pass is recomputed for its log-sum-exp, then the
 * backward kernels run (scores recomputed tile by tile from it). results
 * points at three results, d_q, d_k and d_v: a row per placed cell of the
 * operand (ragged groups: the cells present), its key columns as the
 * operand types them and a DOUBLE column "grad", rows in key order. Ragged
 * groups (each batch's rows present from position 0 to its length along X
 * for q, along J for k and v) are accepted, as by einfold_pipeline. */
int32_t einfold_pipeline_backward(einfold_context* ctx, const einfold_pipeline_desc* pipeline,
                                  const einfold_relation* operands, const einfold_relation* d_out,
                                  const einfold_options* options, einfold_result* results);
/* einfold_kernels::schema: the result schema of a fold over `operands`
 * (2 or 3) and an optional domain. On success *out is owned by the caller. */
int32_t einfold_schema(const einfold_fold_desc* fold, const struct ArrowSchema* const* operands,
                       int32_t n_operands, const struct ArrowSchema* domain, struct ArrowSchema* out,
                       char* message, int32_t message_len);
int32_t einfold_pipeline_schema(const einfold_pipeline_desc* pipeline, const struct ArrowSchema* const* inputs,
                                struct ArrowSchema* out, char* message, int32_t message_len);
/* Releases what a result holds. */
void einfold_result_release(einfold_result* result);

/* ---- Device-pointer entry points ---- */

/* Ranks of n 64-bit words in their order (discriminate.rs:280-292): rank[i]
 * for each word, first[r] the smallest index holding rank r; *n_ranks gets
 * the number of distinct words. All pointers are device memory. */
int32_t einfold_rank_words(einfold_context* ctx, const uint64_t* words, int64_t n, uint32_t* rank,
                           uint32_t* first, int64_t* n_ranks, void* stream);

/* The ranks of a relation's key columns (rank_columns,
 * crates/einfold-kernels/src/discriminate.rs:240-277, with ranks and by_bytes
 * at :165-235): rank[i] the number of distinct keys below row i's key in the
 * order of Arrow's row format (NULL first, integers by value, floats in
 * total order, strings and binaries by their bytes, a prefix first; -0.0 and
 * 0.0 one key under float_keys = 1), first[r] the smallest row of rank r;
 * *n_ranks the number of distinct keys. Keys of any length and any number of
 * columns. rank has a slot per row and first one per distinct key (at most
 * the rows); both are host memory for a relation in host memory, device
 * memory of its device for one in HBM. */
int32_t einfold_rank_columns(einfold_context* ctx, const einfold_relation* relation, int32_t n_columns,
                             const int32_t* columns, int32_t float_keys, uint32_t* rank, uint32_t* first,
                             int64_t* n_ranks);

/* C[w] = A[w] · B[w] for w < batches, FP64, all row-major device arrays:
 * A [batches][m][k], B [batches][k][n] (b_transposed = 0) or
 * [batches][n][k] (b_transposed = 1), C [batches][m][n].
 * einfold_split_gemm slices each row of A and column of B into `slices`
 * int8 digits under a power-of-two scale, multiplies them on the tensor
 * cores with exact int32 accumulation and combines the levels in FP64;
 * every input must be finite. einfold_fp64_gemm adds in k order with
 * unfused multiply and add. */
int32_t einfold_split_gemm(einfold_context* ctx, const double* a, const double* b, double* c, int64_t batches,
                           int64_t m, int64_t n, int64_t k, int32_t b_transposed, int32_t slices, void* stream);
int32_t einfold_fp64_gemm(einfold_context* ctx, const double* a, const double* b, double* c, int64_t batches,
                          int64_t m, int64_t n, int64_t k, int32_t b_transposed, void* stream);

/* einfold_split_gemm for callers that can't allocate device memory: an
 * engine that hands every byte of HBM to its own pool, or code running
 * inside an allocator callback or under a memory budget that forbids any
 * allocation outside its pool. It has no counterpart in the reference.
 * Its scratch (the operands' digits and scales) lives in one 64 MiB array in
 * the library's device memory, which every GPU that loads the library holds
 * until the process exits; a product needing more returns EINFOLD_INVALID
 * with the sizes in `message`, and einfold_split_gemm is the one to call.
 * No context: it runs on the calling thread's current device and `stream`
 * (NULL: the legacy default stream) and returns once the product is done.
 * It calls no cudaMalloc or cudaFree. Its first call on a device (in each
 * CUDA context the device gets, e.g. again after cudaDeviceReset) looks up
 * the array's address. Every call shares the array: calls that overlap on
 * the GPU, from two threads or two streams, race and give wrong results;
 * serialize them. */
int32_t einfold_split_gemm_static(const double* a, const double* b, double* c, int64_t batches, int64_t m,
                                  int64_t n, int64_t k, int32_t b_transposed, int32_t slices, void* stream,
                                  char* message, int32_t message_len);

/* ---- A dense backend (DenseBackend, crates/einfold-kernels/src/backend.rs:124-143) ----
 * The two calls a Rust DenseBackend implementation forwards: may_run with a
 * work's kind and shape before einfold packs its operands, run with the
 * packed operands (DenseWork, backend.rs:46-96), which einfold has checked
 * (keys in range, no duplicates, no NULLs, every factor finite). Operands
 * are row-major, batch first, in host memory (device = -1, as the trait
 * hands them; copied over and the result back) or already in the memory
 * of CUDA device `device` (result there too). */
typedef struct {
  int32_t kind;    /* 0 DenseShape::Product, 1 DenseShape::Attention */
  int32_t pad;
  int64_t batches; /* w */
  int64_t rows;    /* product: x, the rows of a and of the result; attention: queries x */
  int64_t inner;   /* product: z, the summed dimension; attention: features e */
  int64_t columns; /* product: y; attention: value columns y */
  int64_t keys;    /* attention: key positions j */
} einfold_dense_shape;
typedef struct {
  einfold_dense_shape shape;
  const double* a;        /* product: a [w][x][z] */
  const double* b;        /* product: b [w][z][y] */
  const double* q;        /* attention: q [w][x][e] */
  const double* kt;       /* attention: the keys transposed, kt [w][e][j] */
  const double* v;        /* attention: v [w][j][y] */
  int32_t scale_kind;     /* attention: 0 One, 1 Times(c), 2 Over(c) */
  int32_t precision;      /* 0 split (int8 slices, exact sums, FP64 combine), 1 FP64 */
  double scale_c;
  const int64_t* allowed; /* attention: per query x, the keys [lo, hi) it joins, the same in every
                           * batch (2·queries values, host memory) */
  int32_t device;         /* -1 host memory; d >= 0 CUDA device d's memory */
  int32_t pad2;
} einfold_dense_work;

/* Whether run may take work of this shape (DenseBackend::may_run): 1 for
 * products and attention of non-negative extents, 0 otherwise. */
int32_t einfold_backend_may_run(const einfold_dense_shape* shape);
/* DenseBackend::run: writes the result [w][x][y] (row-major, batch first;
 * attention rows with no keys are 0) and returns EINFOLD_OK, or
 * EINFOLD_DECLINED (Ok(None): einfold computes the work itself) for a kind
 * it doesn't know, attention ranges that aren't [x + a, x + b) clamped to
 * the keys (the ranges einfold's conditions give), or attention whose sums
 * the reference's guards would refuse. */
int32_t einfold_backend_run(einfold_context* ctx, const einfold_dense_work* work, double* result,
                            einfold_result* info);

/* ---- Attention over device arrays ----
 * The pipeline einfold_pipeline runs for product scores, weights
 * exp(s - MAX(s)) over the kept groups and an average normalised by their
 * sum (fused.rs:694-1019), over placed FP64 device arrays rather than Arrow
 * relations: for w < batches and x < lq,
 *   out[w][x][y] = Σ_j exp(s_xj - m_x) v[w][j][y] / Σ_j exp(s_xj - m_x),
 *   s_xj = scale · (q[w][x] · k[w][j]),  m_x = max_j s_xj,
 * over the j < lk that every condition allows, x <cmp_i> j + off_i (cmp 0 <,
 * 1 <=, 2 >, 3 >=; at most 8; none: every j). q [batches][lq][d], k
 * [batches][lk][d], v [batches][lk][dv], out [batches][lq][dv], lse
 * [batches][lq] (may be NULL) = m_x + ln Σ_j exp(s_xj - m_x); a row with no
 * allowed j is left unwritten. precision 0 runs the split form (int8 digit
 * products on the tensor cores, six slices; `slices` 0 or 6) when every
 * value is finite and d <= 128, else (and for precision 1, or other slice
 * counts) the FP64 tile kernel. Returns EINFOLD_DECLINED where the
 * reference's overflow or underflow guards (fused.rs:1024-1086) would send
 * the pipeline back to the host plan. `info` (may be NULL) receives the
 * message, kernels launched and device times. The reference's pipeline
 * has no device-array entry; these stand where a caller holds the operands
 * as tensors, and for training. */
int32_t einfold_attention_forward(einfold_context* ctx, const double* q, const double* k, const double* v,
                                  double* out, double* lse, int64_t batches, int64_t lq, int64_t lk, int64_t d,
                                  int64_t dv, int32_t n_conditions, const int32_t* comparisons,
                                  const int64_t* offsets, double scale, int32_t precision, int32_t slices,
                                  void* stream, einfold_result* info);

/* The gradients of einfold_attention_forward's out: given its q, k, v, out
 * and lse and the upstream gradient d_out [batches][lq][dv], writes d_q,
 * d_k, d_v (shaped as q, k, v). Scores are recomputed tile by tile from the
 * saved lse: P = exp(s - lse), dV = Pᵀ·dO, dP = dO·Vᵀ, D = rowsum(dO∘O),
 * dS = P∘(dP - D), dQ = scale·dS·K, dK = scale·dSᵀ·Q; each output row is
 * summed by one CTA in a fixed order (no atomics: the same bits on every
 * run). precision 0: the split form (six slices) where every value is
 * finite and d, dv <= 64; otherwise, and for precision 1, FP64. The
 * reference has no backward pass for its fused pipeline: its gradients are
 * gradient SQL that the host plan runs. */
int32_t einfold_attention_backward(einfold_context* ctx, const double* q, const double* k, const double* v,
                                   const double* out, const double* lse, const double* d_out, double* d_q,
                                   double* d_k, double* d_v, int64_t batches, int64_t lq, int64_t lk, int64_t d,
                                   int64_t dv, int32_t n_conditions, const int32_t* comparisons,
                                   const int64_t* offsets, double scale, int32_t precision, void* stream,
                                   einfold_result* info);

/* Ragged batches (groups of different lengths, which the reference's
 * placement declines, fused.rs:624-664): the same operands padded to lq and
 * lk rows, batch w using q_lengths[w] queries and k_lengths[w] keys (device
 * arrays of `batches` int64 values, each in [0, lq] and [0, lk]; NULL:
 * full). A query at or past its batch's length joins nothing (its out and
 * lse rows are left unwritten, its d_q row is zero), a key at or past it is
 * joined by none (its d_k and d_v rows are zero); the padding rows must
 * hold finite values. The forward pass runs all batches in one launch over
 * the query tiles that join some key, the tiles with the most key tiles
 * first. Otherwise as einfold_attention_forward and
 * einfold_attention_backward. */
int32_t einfold_attention_forward_ragged(einfold_context* ctx, const double* q, const double* k, const double* v,
                                         double* out, double* lse, int64_t batches, int64_t lq, int64_t lk,
                                         int64_t d, int64_t dv, const int64_t* q_lengths, const int64_t* k_lengths,
                                         int32_t n_conditions, const int32_t* comparisons, const int64_t* offsets,
                                         double scale, int32_t precision, int32_t slices, void* stream,
                                         einfold_result* info);
int32_t einfold_attention_backward_ragged(einfold_context* ctx, const double* q, const double* k, const double* v,
                                          const double* out, const double* lse, const double* d_out, double* d_q,
                                          double* d_k, double* d_v, int64_t batches, int64_t lq, int64_t lk,
                                          int64_t d, int64_t dv, const int64_t* q_lengths, const int64_t* k_lengths,
                                          int32_t n_conditions, const int32_t* comparisons, const int64_t* offsets,
                                          double scale, int32_t precision, void* stream, einfold_result* info);

/* ---- Device self-checks (no counterpart in the reference: they check two
 * mechanisms the kernels rely on, for a caller's health check and the tests) ---- */

/* One block waits on an mbarrier that nothing arrives on, with the bounded
 * wait every kernel's mbarrier waits use, for at most limit_ns (at most the
 * kernels' own 2 s): the wait runs out, the block records it in a status
 * word and returns, and the call returns EINFOLD_TIMEOUT, as a call whose
 * kernel's wait ran out does; the context stays usable. *waited_ns (may be
 * NULL) gets how long the wait took. */
int32_t einfold_check_wait(einfold_context* ctx, uint64_t limit_ns, uint64_t* waited_ns);

/* y[i] = exp(x[i]) as the softmax weights compute it (Tang's table-driven
 * method), for shift < 0; for 0 <= shift <= 64, 2^shift·exp(x[i]) with x
 * clamped to [-708, 709], the weights' form. Device arrays; returns once
 * done. */
int32_t einfold_exp_weights(einfold_context* ctx, const double* x, double* y, int64_t n, int32_t shift,
                            void* stream);

/* A row expression's value as the pipelines' tile kernels evaluate it
 * (Expression::evaluate, crates/einfold-ir/src/expression.rs), for every
 * pair of a row i of `a` and a row j of `b`: out[i·nb + j], with
 * out_valid[i·nb + j] = 0 (and out 0) where a column the expression reads is
 * NULL. a and b hold `cols` DOUBLE values a row, row-major, with a validity
 * byte each (1: valid); a column node (operand o, column c) reads value c of
 * a's row (o = 0) or b's (o = 1). Device arrays; returns once done. Replaces
 * the host evaluation the reference's row expressions get
 * (tests/expression_vs_sql.rs checks it against SQL). */
int32_t einfold_evaluate_pairs(einfold_context* ctx, const einfold_expression* expression, const double* a,
                               const uint8_t* a_valid, int64_t na, const double* b, const uint8_t* b_valid,
                               int64_t nb, int32_t cols, double* out, uint8_t* out_valid, void* stream);

#ifdef __cplusplus
}
#endif
#endif
