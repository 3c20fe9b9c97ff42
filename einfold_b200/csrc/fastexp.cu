// The table of exp_tang, one per device.
#include <cmath>
#include <mutex>

#include "common.h"
#include "fastexp.cuh"

namespace ef {

const double* exp_table(int device) {
  constexpr int kDevices = 64;
  static std::once_flag once[kDevices];
  static double* tables[kDevices] = {};
  if (device < 0 || device >= kDevices) fail(EINFOLD_INVALID, "device %d out of range", device);
  std::call_once(once[device], [&] {
    double host[64];
    for (int j = 0; j < 64; j++) host[j] = (double)std::exp2l((long double)j / 64.0L);
    double* dev = nullptr;
    EF_CUDA(cudaMalloc(&dev, sizeof host));
    EF_CUDA(cudaMemcpy(dev, host, sizeof host, cudaMemcpyHostToDevice));
    tables[device] = dev;
  });
  if (!tables[device]) fail(EINFOLD_DEVICE, "the exp table of device %d could not be set up", device);
  return tables[device];
}

}  // namespace ef
