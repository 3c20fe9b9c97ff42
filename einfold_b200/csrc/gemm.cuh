// Dense products for the dense fold and the device entry points.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "common.h"

namespace ef {

constexpr int kDefaultSlices = 6;
constexpr int kMinSlices = 2;
constexpr int kMaxSlices = 7;

// C[w] = A[w] · B[w] for w < batches: A [batches][m][k] row-major, B either
// natural [batches][k][n] (b_natural) or transposed [batches][n][k], C
// [batches][m][n]. Every value of A and B must be finite: each row of A and
// each column of B is cut into `slices` int8 digits under a power-of-two
// scale, the digit products are summed exactly in int32 on the tensor cores,
// level by level, and the levels are combined in FP64.
void split_gemm(Context& ctx, const double* a, const double* b, bool b_natural, double* c, int64_t batches,
                int64_t m, int64_t n, int64_t k, int slices, cudaStream_t stream);

// C[w] = A[w] · B[w] in FP64 on the CUDA cores, B natural [batches][k][n],
// each cell's terms added in k order from +0.0 with unfused multiply and add,
// skipping cells of A whose 2-bit `held` code (16 per word, if given) isn't 2.
// With zblock > 0, the terms of each block of `zblock` values of k are summed
// apart and the blocks added in order (the reference's accumulate for small
// outputs, dense.rs:752-768).
void fp64_gemm(Context& ctx, const double* a, const uint32_t* held, const double* b, double* c, int64_t batches,
               int64_t m, int64_t n, int64_t k, int64_t batch_of_row, int64_t zblock, bool fused_multiply_add,
               cudaStream_t stream);

// BT[w][j][i] = B[w][i][j] for a [batches][rows][cols] array.
void transpose(const double* b, double* bt, int64_t batches, int64_t rows, int64_t cols, cudaStream_t stream);

}  // namespace ef
