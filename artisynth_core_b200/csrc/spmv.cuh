// spmv.cuh -- warp-per-block-row 3x3 block SpMV shared by the PCG and the
// standalone SpMV kernel.
#pragma once

#include <cuda_runtime.h>

namespace b200fem {

// y_row = (S x)_row by one warp: lane k takes blocks p0+k, p0+k+32, ...
// (block column, its 9 values and the 3 x entries are all independent
// loads, so a row costs two dependent L2 round trips), then a fixed
// butterfly reduction.
template <typename MT>
__device__ __forceinline__ void warp_row_spmv(int row, const int* __restrict__ rowptr,
                                              const int* __restrict__ col, const MT* __restrict__ S,
                                              const double* __restrict__ x, int lane, double* y) {
  const int p0 = rowptr[row], p1 = rowptr[row + 1];
  double a0 = 0, a1 = 0, a2 = 0;
  for (int p = p0 + lane; p < p1; p += 32) {
    const int c = col[p];
    const MT* B = S + (size_t)p * 9;
    double b[9];
#pragma unroll
    for (int k = 0; k < 9; k++) b[k] = (double)B[k];
    const double x0 = x[3 * (size_t)c], x1 = x[3 * (size_t)c + 1], x2 = x[3 * (size_t)c + 2];
    a0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
    a1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
    a2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, off);
    a1 += __shfl_xor_sync(0xffffffffu, a1, off);
    a2 += __shfl_xor_sync(0xffffffffu, a2, off);
  }
  y[0] = a0;
  y[1] = a1;
  y[2] = a2;
}

}  // namespace b200fem
