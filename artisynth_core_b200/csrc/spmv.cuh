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

// The NODAL dilational term of the factored solve matrix,
//   S v = S1 v + sum_n t_n d_n,  t_n = c_m kp_n (d_n . v),
// with d_n the divBlk row of node n (one 3-vector per neighbour slot) and
// c_m = h^2 + h beta of its model (computeNodalIncompressibility,
// FemModel3d.java:2632-2669, with the addPosJacobian / addVelJacobian
// scales).  dil_node_t forms t_n of one node (slots a0 .. a1 of nbr_row and
// divblk; fixed neighbours have row -1); the rows then add t_n d_n(i) over
// their own entries.  Plain loads: v is rewritten between the PCG's grid
// barriers.
__device__ __forceinline__ double dil_node_t(int a0, int a1, const int* nbr_row, const double* divblk,
                                             const double* v) {
  double s = 0;
  for (int a = a0; a < a1; a++) {
    const int r = nbr_row[a];
    if (r < 0) continue;
    const double* g = divblk + 3 * (size_t)a;
    const double* x = v + 3 * (size_t)r;
    s += g[0] * x[0] + g[1] * x[1] + g[2] * x[2];
  }
  return s;
}

}  // namespace b200fem
