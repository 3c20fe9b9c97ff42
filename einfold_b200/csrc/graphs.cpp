// The context's CUDA graph cache (common.h).
#include "common.h"

namespace ef {

int GraphCache::run(const std::vector<uint8_t>& shape, const std::vector<uint8_t>& key, cudaStream_t stream,
                    const std::function<void(cudaStream_t)>& enqueue) {
  clock++;
  for (Entry& e : entries)
    if (e.key == key && e.shape == shape) {
      e.used = clock;
      EF_CUDA(cudaGraphLaunch(e.exec, stream));
      return 1;
    }
  if (key != seen_key || shape != seen_shape) {
    seen_shape = shape;
    seen_key = key;
    enqueue(stream);
    return 0;
  }
  // Captured on a stream of the cache's own: the caller's may be the
  // legacy default stream, which cannot be captured. Capturing records the
  // launches without running them.
  if (!capture) EF_CUDA(cudaStreamCreateWithFlags(&capture, cudaStreamNonBlocking));
  cudaStream_t cs = capture;
  cudaGraph_t graph = nullptr;
  EF_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  try {
    enqueue(cs);
  } catch (...) {
    cudaStreamEndCapture(cs, &graph);
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    throw;
  }
  EF_CUDA(cudaStreamEndCapture(cs, &graph));
  int how = 3;
  Entry* slot = nullptr;
  for (Entry& e : entries)
    if (e.shape == shape) {
      cudaGraphExecUpdateResultInfo info;
      if (cudaGraphExecUpdate(e.exec, graph, &info) == cudaSuccess) {
        slot = &e;
        how = 2;
      } else {
        // Not updatable: replaced below.
        cudaGetLastError();
        cudaGraphExecDestroy(e.exec);
        e.exec = nullptr;
      }
      break;
    }
  if (!slot) {
    cudaGraphExec_t exec = nullptr;
    const cudaError_t err = cudaGraphInstantiate(&exec, graph, 0);
    if (err != cudaSuccess) cudaGraphDestroy(graph);
    EF_CUDA(err);
    for (size_t i = 0; i < entries.size();)
      if (!entries[i].exec) entries.erase(entries.begin() + (int64_t)i);
      else i++;
    if (entries.size() >= kMaxEntries) {
      size_t oldest = 0;
      for (size_t i = 1; i < entries.size(); i++)
        if (entries[i].used < entries[oldest].used) oldest = i;
      cudaGraphExecDestroy(entries[oldest].exec);
      entries.erase(entries.begin() + (int64_t)oldest);
    }
    entries.push_back(Entry{shape, key, exec, 0});
    slot = &entries.back();
  }
  cudaGraphDestroy(graph);
  slot->key = key;
  slot->used = clock;
  EF_CUDA(cudaGraphLaunch(slot->exec, stream));
  return how;
}

void GraphCache::clear() {
  for (Entry& e : entries)
    if (e.exec) cudaGraphExecDestroy(e.exec);
  entries.clear();
  if (capture) cudaStreamDestroy(capture);
  capture = nullptr;
}

}  // namespace ef
