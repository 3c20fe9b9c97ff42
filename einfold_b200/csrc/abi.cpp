// The extern "C" entry points of include/einfold_b200.h.
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <mutex>

#include "attention.cuh"
#include "fold.h"
#include "gemm.cuh"
#include "rank.cuh"

struct einfold_context : ef::Context {};

namespace {

thread_local std::string g_last_error;

void set_message(einfold_result* r, const std::string& m) {
  std::snprintf(r->message, sizeof r->message, "%s", m.c_str());
}

// Runs `body` with the context's lock and device, mapping failures to a status.
template <class F>
int32_t guarded(einfold_context* ctx, einfold_result* result, F&& body) {
  if (result) {
    std::memset(result, 0, sizeof *result);
  }
  if (!ctx) {
    if (result) set_message(result, "no context");
    return EINFOLD_INVALID;
  }
  ef::Context* c = static_cast<ef::Context*>(ctx);
  std::lock_guard<std::mutex> lock(c->lock);
  int32_t status = EINFOLD_OK;
  try {
    ef::DeviceGuard dev(c->device);
    c->kernels = 0;
    c->last_phase = 0;
    c->phase("call");
    c->product_ms = 0;
    c->product_ops = 0;
    c->schedule = -1;
    c->graph = 0;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, c->stream);
    status = body(*c);
    cudaEventRecord(t1, c->stream);
    cudaEventSynchronize(t1);
    float ms = 0;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (result) {
      result->device_ms = ms;
      result->kernels_launched = c->kernels;
      result->product_ms = c->product_ms;
      result->product_ops = c->product_ops;
      result->schedule = c->schedule;
      result->graph = c->graph;
    }
  } catch (const ef::Declined& d) {
    status = EINFOLD_DECLINED;
    if (result) set_message(result, d.why);
  } catch (const ef::Failure& f) {
    status = f.status;
    if (result) set_message(result, f.what());
    g_last_error = f.what();
  } catch (const std::exception& e) {
    status = EINFOLD_COMPUTE;
    if (result) set_message(result, e.what());
    g_last_error = e.what();
  }
  if (status != EINFOLD_OK && result) ef::release_result(result);
  if (result) result->status = status;
  return status;
}

einfold_options defaults(const einfold_options* o) {
  einfold_options d;
  std::memset(&d, 0, sizeof d);
  d.threads = 1;
  return o ? *o : d;
}

int32_t run_fold(einfold_context* ctx, const einfold_fold_desc* fold, const einfold_relation* a,
                 const einfold_relation* b, const einfold_relation* domain, const einfold_options* options,
                 einfold_result* result, bool dense_only) {
  return guarded(ctx, result, [&](ef::Context& c) -> int32_t {
    einfold_options o = defaults(options);
    ef::Budget budget;
    budget.o = &o;
    ef::FoldD f = ef::parse_fold(fold);
    ef::Relation ra = ef::import_relation(a), rb = ef::import_relation(b);
    ef::Relation rd;
    if (domain) rd = ef::import_relation(domain);
    std::vector<const std::vector<ef::Field>*> ops = {&ra.fields, &rb.fields};
    std::vector<ef::Field> schema = ef::fold_schema(f, ops, domain ? &rd.fields : nullptr);
    if (!dense_only && o.domain_rows == 1)
      ef::fail(EINFOLD_INVALID, "only fold_dense checks that a domain's keys are unique");
    ef::FoldOutput out;
    try {
      out = ef::dense_fold(c, f, ra, rb, domain ? &rd : nullptr, schema, o, budget);
    } catch (const ef::Declined& d) {
      if (dense_only) throw;
      if (!f.conditions.empty()) ef::fail(EINFOLD_INVALID, "the discrimination algorithm computes no masks");
      out = ef::discriminate_fold(c, f, ra, rb, domain ? &rd : nullptr, schema, o, budget);
    }
    result->algorithm = out.algorithm;
    ef::export_result(std::move(out.batches), schema, result);
    return EINFOLD_OK;
  });
}

}  // namespace

extern "C" {

const char* einfold_version(void) { return "einfold_b200 0.1.0 (sm_100a)"; }

const char* einfold_last_error(void) { return g_last_error.c_str(); }

einfold_context* einfold_context_create(int32_t device) {
  try {
    auto* c = new einfold_context();
    c->device = device;
    c->tracing = std::getenv("EINFOLD_TRACE") != nullptr;
    ef::DeviceGuard dev(device);
    EF_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    EF_CUDA(cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    // Keep freed blocks in the stream-ordered pool across calls instead of
    // returning them to the driver at every synchronization.
    cudaMemPool_t pool;
    EF_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    uint64_t keep = UINT64_MAX;
    EF_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    return c;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return nullptr;
  }
}

void einfold_context_destroy(einfold_context* ctx) {
  if (!ctx) return;
  {
    ef::DeviceGuard dev(ctx->device);
    if (ctx->stream) {
      cudaStreamSynchronize(ctx->stream);
      if (ctx->aux) {
        cudaStreamSynchronize(ctx->aux);
        ef::device_cache_forget(ctx->aux);
        cudaStreamDestroy(ctx->aux);
      }
      ctx->graphs.clear();
      ef::device_cache_forget(ctx->stream);
      cudaStreamDestroy(ctx->stream);
    }
  }
  delete ctx;
}

int32_t einfold_fold(einfold_context* ctx, const einfold_fold_desc* fold, const einfold_relation* a,
                     const einfold_relation* b, const einfold_relation* domain, const einfold_options* options,
                     einfold_result* result) {
  return run_fold(ctx, fold, a, b, domain, options, result, false);
}

int32_t einfold_fold_dense(einfold_context* ctx, const einfold_fold_desc* fold, const einfold_relation* a,
                           const einfold_relation* b, const einfold_relation* domain,
                           const einfold_options* options, einfold_result* result) {
  return run_fold(ctx, fold, a, b, domain, options, result, true);
}

int32_t einfold_fold_chain(einfold_context* ctx, const einfold_fold_desc* fold, const einfold_relation* operands,
                           const einfold_options* options, einfold_result* result) {
  return guarded(ctx, result, [&](ef::Context& c) -> int32_t {
    einfold_options o = defaults(options);
    ef::Budget budget;
    budget.o = &o;
    ef::FoldD f = ef::parse_fold(fold);
    std::vector<ef::Relation> rels;
    for (int i = 0; i < 3; i++) rels.push_back(ef::import_relation(&operands[i]));
    std::vector<const std::vector<ef::Field>*> ops;
    for (auto& r : rels) ops.push_back(&r.fields);
    if (f.operands.size() != 3) throw ef::Declined{"not three operands"};
    std::vector<ef::Field> schema = ef::fold_schema(f, ops, nullptr);
    std::vector<const ef::Relation*> rp = {&rels[0], &rels[1], &rels[2]};
    ef::FoldOutput out = ef::chain_fold(c, f, rp, schema, o, budget);
    result->algorithm = out.algorithm;
    ef::export_result(std::move(out.batches), schema, result);
    return EINFOLD_OK;
  });
}

int32_t einfold_pipeline(einfold_context* ctx, const einfold_pipeline_desc* pipeline,
                         const einfold_relation* operands, const einfold_options* options,
                         einfold_result* result) {
  return guarded(ctx, result, [&](ef::Context& c) -> int32_t {
    einfold_options o = defaults(options);
    ef::Budget budget;
    budget.o = &o;
    ef::PipelineD p = ef::parse_pipeline(pipeline);
    std::vector<ef::Relation> rels;
    for (int i = 0; i < 3; i++) rels.push_back(ef::import_relation(&operands[i]));
    std::vector<const std::vector<ef::Field>*> ins = {&rels[0].fields, &rels[1].fields, &rels[2].fields};
    std::vector<ef::Field> schema = ef::pipeline_schema(p, ins);
    ef::FoldOutput out = ef::fused_pipeline(c, p, rels[0], rels[1], rels[2], schema, o, budget);
    result->algorithm = EINFOLD_ALG_FUSED;
    result->tiles_visited = out.tiles_visited;
    result->tiles = out.tiles;
    ef::export_result(std::move(out.batches), schema, result);
    return EINFOLD_OK;
  });
}

int32_t einfold_pipeline_backward(einfold_context* ctx, const einfold_pipeline_desc* pipeline,
                                  const einfold_relation* operands, const einfold_relation* d_out,
                                  const einfold_options* options, einfold_result* results) {
  if (results) std::memset(results + 1, 0, 2 * sizeof *results);
  const int32_t st = guarded(ctx, results, [&](ef::Context& c) -> int32_t {
    if (!pipeline || !operands || !d_out || !results) ef::fail(EINFOLD_INVALID, "a NULL argument");
    einfold_options o = defaults(options);
    ef::PipelineD p = ef::parse_pipeline(pipeline);
    std::vector<ef::Relation> rels;
    for (int i = 0; i < 3; i++) rels.push_back(ef::import_relation(&operands[i]));
    ef::Relation rd = ef::import_relation(d_out);
    std::vector<const std::vector<ef::Field>*> ins = {&rels[0].fields, &rels[1].fields, &rels[2].fields};
    ef::pipeline_schema(p, ins);  // the forward pipeline's own validity rules
    ef::GradientOutput g = ef::pipeline_backward(c, p, rels[0], rels[1], rels[2], rd, o);
    for (int i = 0; i < 3; i++) {
      results[i].algorithm = EINFOLD_ALG_FUSED;
      ef::export_result(std::move(g.batches[i]), g.schemas[i], &results[i]);
    }
    return EINFOLD_OK;
  });
  if (results) {
    for (int i = 1; i < 3; i++) {
      if (st != EINFOLD_OK) ef::release_result(&results[i]);
      results[i].status = st;
      std::memcpy(results[i].message, results[0].message, sizeof results[i].message);
    }
  }
  return st;
}

int32_t einfold_schema(const einfold_fold_desc* fold, const struct ArrowSchema* const* operands, int32_t n_operands,
                       const struct ArrowSchema* domain, struct ArrowSchema* out, char* message,
                       int32_t message_len) {
  try {
    ef::FoldD f = ef::parse_fold(fold);
    if (f.row_expr) ef::fail(EINFOLD_INVALID, "EinFold computes SUM of products only");
    std::vector<std::vector<ef::Field>> fields;
    for (int i = 0; i < n_operands; i++) fields.push_back(ef::import_schema(operands[i]));
    std::vector<const std::vector<ef::Field>*> ops;
    for (auto& fl : fields) ops.push_back(&fl);
    std::vector<ef::Field> dom;
    if (domain) dom = ef::import_schema(domain);
    ef::export_schema(ef::fold_schema(f, ops, domain ? &dom : nullptr), out);
    return EINFOLD_OK;
  } catch (const ef::Failure& e) {
    if (message && message_len > 0) std::snprintf(message, (size_t)message_len, "%s", e.what());
    return e.status;
  }
}

int32_t einfold_pipeline_schema(const einfold_pipeline_desc* pipeline, const struct ArrowSchema* const* inputs,
                                struct ArrowSchema* out, char* message, int32_t message_len) {
  try {
    ef::PipelineD p = ef::parse_pipeline(pipeline);
    std::vector<std::vector<ef::Field>> fields;
    for (int i = 0; i < 3; i++) fields.push_back(ef::import_schema(inputs[i]));
    std::vector<const std::vector<ef::Field>*> ins = {&fields[0], &fields[1], &fields[2]};
    ef::export_schema(ef::pipeline_schema(p, ins), out);
    return EINFOLD_OK;
  } catch (const ef::Failure& e) {
    if (message && message_len > 0) std::snprintf(message, (size_t)message_len, "%s", e.what());
    return e.status;
  }
}

void einfold_result_release(einfold_result* result) { ef::release_result(result); }

int32_t einfold_split_gemm(einfold_context* ctx, const double* a, const double* b, double* c, int64_t batches,
                           int64_t m, int64_t n, int64_t k, int32_t b_transposed, int32_t slices, void* stream) {
  einfold_result r;
  return guarded(ctx, &r, [&](ef::Context& cx) -> int32_t {
    cudaStream_t s = stream ? (cudaStream_t)stream : cx.stream;
    ef::split_gemm(cx, a, b, b_transposed == 0, c, batches, m, n, k, slices ? slices : ef::kDefaultSlices, s);
    return EINFOLD_OK;
  });
}

int32_t einfold_rank_words(einfold_context* ctx, const uint64_t* words, int64_t n, uint32_t* rank, uint32_t* first,
                           int64_t* n_ranks, void* stream) {
  einfold_result r;
  return guarded(ctx, &r, [&](ef::Context& cx) -> int32_t {
    cudaStream_t s = stream ? (cudaStream_t)stream : cx.stream;
    int64_t k = ef::rank_keys(cx, words, 1, n, n, rank, first, s);
    if (n_ranks) *n_ranks = k;
    return EINFOLD_OK;
  });
}

int32_t einfold_rank_columns(einfold_context* ctx, const einfold_relation* relation, int32_t n_columns,
                             const int32_t* columns, int32_t float_keys, uint32_t* rank, uint32_t* first,
                             int64_t* n_ranks) {
  einfold_result r;
  const int32_t st = guarded(ctx, &r, [&](ef::Context& cx) -> int32_t {
    if (!relation || n_columns < 0 || (n_columns && !columns)) ef::fail(EINFOLD_INVALID, "no relation or columns");
    ef::Relation rel = ef::import_relation(relation);
    std::vector<int> cols(columns, columns + n_columns);
    const int64_t k = ef::rank_columns(cx, rel, cols, float_keys, rank, first, relation->device >= 0);
    if (n_ranks) *n_ranks = k;
    return EINFOLD_OK;
  });
  if (st != EINFOLD_OK) g_last_error = r.message;
  return st;
}

int32_t einfold_fp64_gemm(einfold_context* ctx, const double* a, const double* b, double* c, int64_t batches,
                          int64_t m, int64_t n, int64_t k, int32_t b_transposed, void* stream) {
  einfold_result r;
  return guarded(ctx, &r, [&](ef::Context& cx) -> int32_t {
    cudaStream_t s = stream ? (cudaStream_t)stream : cx.stream;
    if (!b_transposed) {
      ef::fp64_gemm(cx, a, nullptr, b, c, batches, m, n, k, 0, 0, false, s);
    } else {
      ef::DeviceBuffer<double> bn((size_t)(batches * n * k), s);
      ef::transpose(b, bn.get(), batches, n, k, s);
      ef::fp64_gemm(cx, a, nullptr, bn.get(), c, batches, m, n, k, 0, 0, false, s);
    }
    EF_CUDA(cudaStreamSynchronize(s));
    return EINFOLD_OK;
  });
}

int32_t einfold_backend_may_run(const einfold_dense_shape* shape) {
  if (!shape) return 0;
  if (shape->batches < 0 || shape->rows < 0 || shape->inner < 0 || shape->columns < 0) return 0;
  if (shape->kind == 0) return 1;
  if (shape->kind == 1) return shape->keys >= 0 ? 1 : 0;
  return 0;
}

int32_t einfold_backend_run(einfold_context* ctx, const einfold_dense_work* work, double* result,
                            einfold_result* info) {
  einfold_result local;
  einfold_result* r = info ? info : &local;
  const int32_t st = guarded(ctx, r, [&](ef::Context& c) -> int32_t {
    if (!work || !result) ef::fail(EINFOLD_INVALID, "no work or no result");
    const einfold_dense_shape& sh = work->shape;
    if (!einfold_backend_may_run(&sh)) ef::decline("a kind of work this backend doesn't know");
    cudaStream_t s = c.stream;
    const bool host = work->device < 0;
    if (!host && work->device != c.device)
      ef::fail(EINFOLD_INVALID, "operands on device %d, the context on %d", work->device, c.device);
    const int64_t W = sh.batches;
    // Device copies of host operands (none for operands already in HBM).
    std::vector<ef::DeviceBuffer<double>> keep;
    keep.reserve(3);
    auto on_device = [&](const double* p, int64_t n) -> const double* {
      if (!host || n == 0) return p;
      keep.emplace_back((size_t)n, s);
      EF_CUDA(cudaMemcpyAsync(keep.back().get(), p, (size_t)n * 8, cudaMemcpyHostToDevice, s));
      return keep.back().get();
    };
    ef::DeviceBuffer<double> out;
    if (sh.kind == 0) {
      const int64_t x = sh.rows, z = sh.inner, y = sh.columns;
      const double* a = on_device(work->a, W * x * z);
      const double* b = on_device(work->b, W * z * y);
      double* o = result;
      if (host) {
        out.allocate((size_t)std::max<int64_t>(W * x * y, 1), s);
        o = out.get();
      }
      if (W * x * y > 0) {
        if (z == 0) EF_CUDA(cudaMemsetAsync(o, 0, (size_t)(W * x * y) * 8, s));
        else if (work->precision == 1) ef::fp64_gemm(c, a, nullptr, b, o, W, x, y, z, 0, 0, false, s);
        else ef::split_gemm(c, a, b, true, o, W, x, y, z, ef::kDefaultSlices, s);
        if (host) EF_CUDA(cudaMemcpyAsync(result, o, (size_t)(W * x * y) * 8, cudaMemcpyDeviceToHost, s));
      }
      EF_CUDA(cudaStreamSynchronize(s));
      return EINFOLD_OK;
    }
    // Attention.
    const int64_t x = sh.rows, e = sh.inner, y = sh.columns, j = sh.keys;
    if (!work->allowed && x > 0) ef::fail(EINFOLD_INVALID, "attention without its ranges");
    if (work->scale_kind < 0 || work->scale_kind > 2) ef::fail(EINFOLD_INVALID, "a scale of kind %d", work->scale_kind);
    ef::Mask mask;
    if (!ef::ranges_as_mask(work->allowed, x, j, mask)) ef::decline("ranges that no conditions give");
    const double* q = on_device(work->q, W * x * e);
    const double* kt = on_device(work->kt, W * e * j);
    const double* v = on_device(work->v, W * j * y);
    ef::DeviceBuffer<double> k((size_t)std::max<int64_t>(W * j * e, 1), s);
    if (W * j * e > 0) ef::transpose(kt, k.get(), W, e, j, s);
    double* o = result;
    if (host) {
      out.allocate((size_t)std::max<int64_t>(W * x * y, 1), s);
      o = out.get();
    }
    if (W * x * y > 0) EF_CUDA(cudaMemsetAsync(o, 0, (size_t)(W * x * y) * 8, s));
    ef::AttentionProblem p;
    p.q = q;
    p.k = k.get();
    p.v = v;
    p.out = o;
    p.batches = W;
    p.lnx = x;
    p.lnj = j;
    p.ne = e;
    p.ny = y;
    p.mask = mask;
    p.scale_kind = work->scale_kind;
    p.scale_c = work->scale_c;
    if (W > 0 && x > 0 && y > 0 && j > 0 && e > 0) {
      if (ef::attention_forward(c, p, work->precision, 0, s) == ef::ATTENTION_GUARDED)
        ef::decline("a sum that overflowed or may have underflowed");
    }
    if (host && W * x * y > 0) EF_CUDA(cudaMemcpyAsync(result, o, (size_t)(W * x * y) * 8, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    return EINFOLD_OK;
  });
  if (st != EINFOLD_OK) g_last_error = r->message;
  return st;
}

static ef::AttentionProblem attention_problem(const double* q, const double* k, const double* v, double* out,
                                              double* lse, int64_t batches, int64_t lq, int64_t lk, int64_t d,
                                              int64_t dv, int32_t n_conditions, const int32_t* comparisons,
                                              const int64_t* offsets, double scale) {
  if (batches < 0 || lq < 0 || lk < 0 || d < 0 || dv < 0) ef::fail(EINFOLD_INVALID, "a negative extent");
  if (n_conditions < 0 || n_conditions > ef::kMaxMask)
    ef::fail(EINFOLD_INVALID, "0 to 8 conditions, not %d", n_conditions);
  if (n_conditions && (!comparisons || !offsets)) ef::fail(EINFOLD_INVALID, "conditions without comparisons or offsets");
  if (!std::isfinite(scale)) ef::fail(EINFOLD_INVALID, "a scale that isn't finite");
  ef::AttentionProblem p;
  p.q = q;
  p.k = k;
  p.v = v;
  p.out = out;
  p.lse = lse;
  p.batches = batches;
  p.lnx = lq;
  p.lnj = lk;
  p.ne = d;
  p.ny = dv;
  p.mask.n = n_conditions;
  for (int i = 0; i < n_conditions; i++) {
    if (comparisons[i] < 0 || comparisons[i] > 3) ef::fail(EINFOLD_INVALID, "a comparison of kind %d", comparisons[i]);
    p.mask.cmp[i] = comparisons[i];
    p.mask.off[i] = offsets[i];
  }
  p.mask.lnx = lq > 0 ? lq : 1;
  p.mask.lnj = lk;
  p.scale_kind = scale == 1.0 ? 0 : 1;
  p.scale_c = scale;
  return p;
}

int32_t einfold_attention_forward(einfold_context* ctx, const double* q, const double* k, const double* v,
                                  double* out, double* lse, int64_t batches, int64_t lq, int64_t lk, int64_t d,
                                  int64_t dv, int32_t n_conditions, const int32_t* comparisons,
                                  const int64_t* offsets, double scale, int32_t precision, int32_t slices,
                                  void* stream, einfold_result* info) {
  return guarded(ctx, info, [&](ef::Context& cx) -> int32_t {
    cudaStream_t s = stream ? (cudaStream_t)stream : cx.stream;
    ef::AttentionProblem p =
        attention_problem(q, k, v, out, lse, batches, lq, lk, d, dv, n_conditions, comparisons, offsets, scale);
    const ef::AttentionOutcome r = ef::attention_forward(cx, p, precision, slices, s);
    EF_CUDA(cudaStreamSynchronize(s));
    if (r == ef::ATTENTION_GUARDED) ef::decline("a sum that overflowed or may have underflowed");
    return EINFOLD_OK;
  });
}

int32_t einfold_attention_backward(einfold_context* ctx, const double* q, const double* k, const double* v,
                                   const double* out, const double* lse, const double* d_out, double* d_q,
                                   double* d_k, double* d_v, int64_t batches, int64_t lq, int64_t lk, int64_t d,
                                   int64_t dv, int32_t n_conditions, const int32_t* comparisons,
                                   const int64_t* offsets, double scale, int32_t precision, void* stream,
                                   einfold_result* info) {
  return guarded(ctx, info, [&](ef::Context& cx) -> int32_t {
    cudaStream_t s = stream ? (cudaStream_t)stream : cx.stream;
    ef::AttentionGradients g;
    g.f = attention_problem(q, k, v, nullptr, nullptr, batches, lq, lk, d, dv, n_conditions, comparisons, offsets,
                            scale);
    g.out = out;
    g.lse = lse;
    g.d_out = d_out;
    g.d_q = d_q;
    g.d_k = d_k;
    g.d_v = d_v;
    ef::attention_backward(cx, g, precision, s);
    EF_CUDA(cudaStreamSynchronize(s));
    return EINFOLD_OK;
  });
}

// Ragged lengths: read back, checked against the padded extents, and
// attached to the problem's mask.
static void attach_lengths(ef::AttentionProblem& p, const int64_t* q_lengths, const int64_t* k_lengths,
                           cudaStream_t s) {
  auto fetch = [&](const int64_t* dev, int64_t limit, const char* what, std::vector<int64_t>& host) {
    if (!dev || p.batches == 0) return;
    host.resize((size_t)p.batches);
    EF_CUDA(cudaMemcpyAsync(host.data(), dev, (size_t)p.batches * 8, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    for (int64_t x : host)
      if (x < 0 || x > limit)
        ef::fail(EINFOLD_INVALID, "a %s length of %lld outside [0, %lld]", what, (long long)x, (long long)limit);
  };
  fetch(q_lengths, p.lnx, "query", p.xlen_host);
  fetch(k_lengths, p.lnj, "key", p.jlen_host);
  p.mask.xlen = p.batches ? q_lengths : nullptr;
  p.mask.jlen = p.batches ? k_lengths : nullptr;
}

int32_t einfold_attention_forward_ragged(einfold_context* ctx, const double* q, const double* k, const double* v,
                                         double* out, double* lse, int64_t batches, int64_t lq, int64_t lk,
                                         int64_t d, int64_t dv, const int64_t* q_lengths, const int64_t* k_lengths,
                                         int32_t n_conditions, const int32_t* comparisons, const int64_t* offsets,
                                         double scale, int32_t precision, int32_t slices, void* stream,
                                         einfold_result* info) {
  return guarded(ctx, info, [&](ef::Context& cx) -> int32_t {
    cudaStream_t s = stream ? (cudaStream_t)stream : cx.stream;
    ef::AttentionProblem p =
        attention_problem(q, k, v, out, lse, batches, lq, lk, d, dv, n_conditions, comparisons, offsets, scale);
    attach_lengths(p, q_lengths, k_lengths, s);
    const ef::AttentionOutcome r = ef::attention_forward(cx, p, precision, slices, s);
    EF_CUDA(cudaStreamSynchronize(s));
    if (r == ef::ATTENTION_GUARDED) ef::decline("a sum that overflowed or may have underflowed");
    return EINFOLD_OK;
  });
}

int32_t einfold_attention_backward_ragged(einfold_context* ctx, const double* q, const double* k, const double* v,
                                          const double* out, const double* lse, const double* d_out, double* d_q,
                                          double* d_k, double* d_v, int64_t batches, int64_t lq, int64_t lk,
                                          int64_t d, int64_t dv, const int64_t* q_lengths, const int64_t* k_lengths,
                                          int32_t n_conditions, const int32_t* comparisons, const int64_t* offsets,
                                          double scale, int32_t precision, void* stream, einfold_result* info) {
  return guarded(ctx, info, [&](ef::Context& cx) -> int32_t {
    cudaStream_t s = stream ? (cudaStream_t)stream : cx.stream;
    ef::AttentionGradients g;
    g.f = attention_problem(q, k, v, nullptr, nullptr, batches, lq, lk, d, dv, n_conditions, comparisons, offsets,
                            scale);
    attach_lengths(g.f, q_lengths, k_lengths, s);
    g.out = out;
    g.lse = lse;
    g.d_out = d_out;
    g.d_q = d_q;
    g.d_k = d_k;
    g.d_v = d_v;
    ef::attention_backward(cx, g, precision, s);
    EF_CUDA(cudaStreamSynchronize(s));
    return EINFOLD_OK;
  });
}

}  // extern "C"
