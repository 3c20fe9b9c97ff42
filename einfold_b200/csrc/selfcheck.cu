// Checks of two device-side mechanisms every kernel relies on, callable by a
// caller's health check and by the tests:
//  - the bounded wait: one block waits on an mbarrier nothing arrives on,
//    with the same bounded wait (ptx::mbar_wait_for) the kernels' mbarrier
//    waits use, under a limit the caller gives; the wait runs out, sets the
//    status word and the block returns, so the call reports EINFOLD_TIMEOUT
//    as a kernel's timed-out wait does, and the context stays usable;
//  - the exponential of the softmax weights (exp_tang, exp_weight), over an
//    array of arguments, so its error can be measured against the math
//    library's exp;
//  - the row-expression interpreter the tile kernels run (eval), over every
//    pair of rows of two tables, as Expression::evaluate defines a row
//    expression's value (expression.rs), NULL where a column it reads is.
#include <vector>

#include "common.h"
#include "expr.cuh"
#include "fastexp.cuh"
#include "ptx.cuh"

namespace ef {
namespace {

__global__ void wait_on_nothing(uint64_t limit_ns, int* status, unsigned long long* waited) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    ptx::mbar_init(&bar, 1);
    ptx::mbar_fence_init();
  }
  __syncthreads();
  const uint64_t t0 = ptx::now_ns();
  // Nothing arrives on `bar`: phase 0 never completes.
  const bool done = ptx::mbar_wait_for(&bar, 0, limit_ns, true);
  const uint64_t t1 = ptx::now_ns();
  if (!done) atomicOr(status, 2);
  if (threadIdx.x == 0) *waited = t1 - t0;
}

__global__ void exp_array(const double* __restrict__ x, double* __restrict__ y, int64_t n, int shift,
                          const double* __restrict__ table) {
  __shared__ double t[64];
  if (threadIdx.x < 64) t[threadIdx.x] = table[threadIdx.x];
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] = shift < 0 ? exp_tang(x[i], t) : exp_weight(x[i], t, shift);
}

// out[i·nb + j]: the expression over row i of a and row j of b (slot c < cols
// reads a[i][c], slot cols + c reads b[j][c]); valid where every slot the
// expression reads is (`reads`: the slots' bits, up to 64 slots).
__global__ void evaluate_pairs_kernel(const ExprNode* __restrict__ nodes, int n_nodes, const double* __restrict__ a,
                                      const uint8_t* __restrict__ a_valid, int64_t na, const double* __restrict__ b,
                                      const uint8_t* __restrict__ b_valid, int64_t nb, int cols, uint64_t reads,
                                      double* __restrict__ out, uint8_t* __restrict__ out_valid) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < na * nb; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = p / nb, j = p % nb;
    bool valid = true;
    for (int c = 0; c < 2 * cols; c++)
      if ((reads >> c) & 1) valid = valid && (c < cols ? a_valid[i * cols + c] : b_valid[j * cols + c - cols]) != 0;
    const double v = eval<64>(nodes, n_nodes, [&](int k) { return k < cols ? a[i * cols + k] : b[j * cols + k - cols]; });
    out[p] = valid ? v : 0.0;
    out_valid[p] = valid;
  }
}

}  // namespace
}  // namespace ef

struct einfold_context : ef::Context {};

extern "C" int32_t einfold_evaluate_pairs(einfold_context* ctx, const einfold_expression* expression, const double* a,
                                          const uint8_t* a_valid, int64_t na, const double* b, const uint8_t* b_valid,
                                          int64_t nb, int32_t cols, double* out, uint8_t* out_valid, void* stream) {
  using namespace ef;
  if (!ctx) return EINFOLD_INVALID;
  Context& c = *ctx;
  std::lock_guard<std::mutex> lock(c.lock);
  try {
    DeviceGuard dev(c.device);
    if (!expression || expression->n_nodes < 1 || expression->n_nodes > 4096 || !expression->nodes)
      fail(EINFOLD_INVALID, "no expression, or one of more than 4096 nodes");
    if (na < 0 || nb < 0 || cols < 1 || cols > 32) fail(EINFOLD_INVALID, "na or nb < 0, or cols outside 1..32");
    if (na > 0 && nb > INT64_MAX / na) fail(EINFOLD_INVALID, "na·nb overflows");
    // The postfix nodes, checked as a pipeline's are: every operation finds
    // its operands, one value is left, the stack never deeper than 60.
    std::vector<ExprNode> nodes;
    uint64_t reads = 0;
    int depth = 0;
    for (int32_t i = 0; i < expression->n_nodes; i++) {
      const einfold_expr_node& e = expression->nodes[i];
      ExprNode x{e.kind, e.a, e.b, e.value};
      if (e.kind == 0) {
        if (e.a < 0 || e.a > 1 || e.b < 0 || e.b >= cols) fail(EINFOLD_INVALID, "a column outside the tables");
        x.a = e.a * cols + e.b;
        reads |= 1ull << x.a;
        depth++;
      } else if (e.kind == 1) {
        depth++;
      } else if (e.kind == 2) {
        if (depth < 1 || e.a < 0 || e.a > 3) fail(EINFOLD_INVALID, "a malformed expression");
      } else if (e.kind == 3) {
        if (depth < 2 || e.a < 0 || e.a > 4) fail(EINFOLD_INVALID, "a malformed expression");
        depth--;
      } else {
        fail(EINFOLD_INVALID, "an expression node of kind %d", e.kind);
      }
      if (depth > 60) fail(EINFOLD_INVALID, "an expression deeper than 60");
      nodes.push_back(x);
    }
    if (depth != 1) fail(EINFOLD_INVALID, "a malformed expression");
    cudaStream_t s = stream ? (cudaStream_t)stream : c.stream;
    const uint64_t pairs = (uint64_t)na * (uint64_t)nb;
    if (pairs) {
      DeviceBuffer<ExprNode> d(nodes.size(), s);
      EF_CUDA(cudaMemcpyAsync(d.get(), nodes.data(), nodes.size() * sizeof(ExprNode), cudaMemcpyHostToDevice, s));
      evaluate_pairs_kernel<<<blocks_for(pairs, 256), 256, 0, s>>>(d.get(), (int)nodes.size(), a, a_valid, na, b, b_valid,
                                                                   nb, cols, reads, out, out_valid);
      EF_LAUNCH_CHECK();
      EF_CUDA(cudaStreamSynchronize(s));  // `nodes` is a host temporary
    }
    EF_CUDA(cudaStreamSynchronize(s));
    return EINFOLD_OK;
  } catch (const Failure& f) {
    return f.status;
  }
}

extern "C" int32_t einfold_check_wait(einfold_context* ctx, uint64_t limit_ns, uint64_t* waited_ns) {
  using namespace ef;
  if (!ctx) return EINFOLD_INVALID;
  Context& c = *ctx;
  std::lock_guard<std::mutex> lock(c.lock);
  try {
    DeviceGuard dev(c.device);
    if (limit_ns > ptx::kWaitNs) fail(EINFOLD_INVALID, "a limit above the kernels' own (%llu ns)",
                                      (unsigned long long)ptx::kWaitNs);
    cudaStream_t s = c.stream;
    DeviceBuffer<int> status(1, s);
    DeviceBuffer<unsigned long long> waited(1, s);
    status.zero();
    waited.zero();
    wait_on_nothing<<<1, 32, 0, s>>>(limit_ns, status.get(), waited.get());
    EF_LAUNCH_CHECK();
    int st = 0;
    unsigned long long w = 0;
    EF_CUDA(cudaMemcpyAsync(&st, status.get(), 4, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaMemcpyAsync(&w, waited.get(), 8, cudaMemcpyDeviceToHost, s));
    EF_CUDA(cudaStreamSynchronize(s));
    if (waited_ns) *waited_ns = w;
    return (st & 2) ? EINFOLD_TIMEOUT : EINFOLD_OK;
  } catch (const Failure& f) {
    return f.status;
  }
}

extern "C" int32_t einfold_exp_weights(einfold_context* ctx, const double* x, double* y, int64_t n, int32_t shift,
                                       void* stream) {
  using namespace ef;
  if (!ctx) return EINFOLD_INVALID;
  Context& c = *ctx;
  std::lock_guard<std::mutex> lock(c.lock);
  try {
    DeviceGuard dev(c.device);
    if (n < 0 || shift > 64) fail(EINFOLD_INVALID, "n < 0 or a shift above 64");
    cudaStream_t s = stream ? (cudaStream_t)stream : c.stream;
    if (n) {
      exp_array<<<blocks_for((uint64_t)n, 256), 256, 0, s>>>(x, y, n, shift, exp_table(c.device));
      EF_LAUNCH_CHECK();
    }
    EF_CUDA(cudaStreamSynchronize(s));
    return EINFOLD_OK;
  } catch (const Failure& f) {
    return f.status;
  }
}
