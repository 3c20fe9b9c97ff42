// Dense products for the dense fold and the device entry points.
#pragma once

#include <cuda.h>
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

// The split product's operand slicing, for kernels that stage digits
// themselves. Rows of x [batches][rows][k] (leading dimension ld) become S
// int8 digit planes digits[(w·S + s)][r][kk] for r < rows_pad, kk < k_pad
// (zeros beyond), each row under a power-of-two scale 2^e with e in
// e_out[w·rows_pad + r]; status bit 1 if a value isn't finite. With
// `lens` (device, one per batch), rows at or past lens[w] are not read and
// slice to zeros; with skip_padding as well, their digits (rows at or past
// `rows` too) are not written at all, for a caller that reads none of them
// (their exponents are still 0).
void slice_rows_into(int S, const double* x, int64_t batches, int64_t rows, int64_t k, int64_t ld, int64_t rows_pad,
                     int64_t k_pad, int32_t* e_out, int8_t* digits, int* status, cudaStream_t stream,
                     const int64_t* lens = nullptr, bool skip_padding = false);
// Columns of x [batches][k][n] become K-major digit planes
// digits[(w·S + s)][col][kk] for col < n_pad and kk < k_pad (both multiples
// of 64), each column under its own power of two, e_out[w·n_pad + col];
// colmax is scratch of batches·n words; with `lens`, rows of x (positions
// along k) at or past lens[w] count as zeros and are not read.
void slice_cols_into(int S, const double* x, int64_t batches, int64_t k, int64_t n, int64_t n_pad, int64_t k_pad,
                     unsigned long long* colmax, int32_t* e_out, int8_t* digits, int* status, cudaStream_t stream,
                     const int64_t* lens = nullptr);
// out[0] = max e[i] and out[1] = max -e[i] over n exponents, folded into
// what out already holds (INT_MIN for a fresh pair).
void exponent_range(const int32_t* e, int64_t n, int* out, cudaStream_t stream);
// A TMA map over digit planes [planes][rows][k_pad] (uint8), boxes of 64
// bytes of k by box_rows rows by box_planes planes, 64-byte swizzle.
CUtensorMap digit_planes_map(const int8_t* digits, int64_t k_pad, int64_t rows, int64_t planes, int box_rows,
                             int box_planes);

// A TMA map over doubles [batches][rows][cols] (cols a multiple of 2),
// boxes of box_cols (at most 16) by box_rows in the 128-byte swizzle.
CUtensorMap f64_boxes_map(const double* x, int64_t cols, int64_t rows, int64_t batches, int box_cols, int box_rows);

// BT[w][j][i] = B[w][i][j] for a [batches][rows][cols] array.
void transpose(const double* b, double* bt, int64_t batches, int64_t rows, int64_t cols, cudaStream_t stream);

}  // namespace ef
