// Checks of two device-side mechanisms every kernel relies on, callable by a
// caller's health check and by the tests:
//  - the bounded wait: one block waits on an mbarrier nothing arrives on,
//    with the same bounded wait (ptx::mbar_wait_for) the kernels' mbarrier
//    waits use, under a limit the caller gives; the wait runs out, sets the
//    status word and the block returns, so the call reports EINFOLD_TIMEOUT
//    as a kernel's timed-out wait does, and the context stays usable;
//  - the exponential of the softmax weights (exp_tang, exp_weight), over an
//    array of arguments, so its error can be measured against the math
//    library's exp.
#include "common.h"
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

}  // namespace
}  // namespace ef

struct einfold_context : ef::Context {};

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
