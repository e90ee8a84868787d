// point_cons.cu -- ConstrainedBackwardEuler with LinearPointConstraints:
// bilateral constraints that couple several nodes (LinearPointConstraint.java:
// constraint c holds sum_i w_i x_i = target_c, one row per axis).
//
// The velocity solve is the KKT system [S G^T; G 0][v; lam] = [b; 0]
// (MechSystemSolver.KKTFactorAndSolve, MechSystemSolver.java:2865-2990, with
// zero compliance and gdot: setBilateralOffsets :2697-2721).  It is solved
// by its Schur complement on the device PCG: u0 = S^-1 b and Y_k = S^-1 G_k^T
// for the m constraint rows (m + 1 PCG solves), then (G Y) lam = G u0 by
// dense elimination in one CTA and v = u0 - Y lam.  After x1 = x0 + h v1
// the GlobalMass position correction (applyPosCorrection) moves the nodes
// by dx = M^-1 G^T mu with (G M^-1 G^T) mu = -(G x1 - target).  Every sum
// runs in a fixed order, so steps are bit-reproducible.
#include <cuda_runtime.h>

#include "engine.h"

namespace b200fem {

// rhs = G_k^T for constraint row k = 3 c + d (the rows of every point with a
// solve index get w on component d), summed in entry order by one thread
__global__ void pc_rhs_kernel(double* __restrict__ rhs, const int* __restrict__ ptr, const int* __restrict__ row,
                              const double* __restrict__ w, int k) {
  if (threadIdx.x != 0) return;
  const int c = k / 3, d = k % 3;
  for (int q = ptr[c]; q < ptr[c + 1]; q++)
    if (row[q] >= 0) rhs[3 * (size_t)row[q] + d] += w[q];
}

// a solve that missed its tolerance marks the step as not converged
__global__ void pc_status_kernel(const double* __restrict__ model_out, int n_models, int* __restrict__ flags) {
  for (int m = threadIdx.x; m < n_models; m += blockDim.x)
    if (model_out[(size_t)m * 4 + 2] == 0.0) atomicExch(&flags[2], 1);
}

// In place, one CTA: solve A x = r (m x m, row-major) by Gaussian
// elimination with partial pivoting; r receives x.  A singular pivot sets
// flags[0] and leaves x zero.
__device__ void pc_dense_solve(double* A, double* r, int m, int* flags) {
  __shared__ int s_piv;
  __shared__ int s_bad;
  if (threadIdx.x == 0) s_bad = 0;
  __syncthreads();
  for (int j = 0; j < m; j++) {
    if (threadIdx.x == 0) {
      int best = j;
      for (int i = j + 1; i < m; i++)
        if (fabs(A[(size_t)i * m + j]) > fabs(A[(size_t)best * m + j])) best = i;
      s_piv = best;
      if (A[(size_t)best * m + j] == 0.0) s_bad = 1;
    }
    __syncthreads();
    if (s_bad) break;
    const int pv = s_piv;
    if (pv != j) {
      for (int c = threadIdx.x; c < m; c += blockDim.x) {
        const double t = A[(size_t)j * m + c];
        A[(size_t)j * m + c] = A[(size_t)pv * m + c];
        A[(size_t)pv * m + c] = t;
      }
      if (threadIdx.x == 0) {
        const double t = r[j];
        r[j] = r[pv];
        r[pv] = t;
      }
    }
    __syncthreads();
    const double dj = A[(size_t)j * m + j];
    for (int i = j + 1 + threadIdx.x; i < m; i += blockDim.x) {
      const double f = A[(size_t)i * m + j] / dj;
      for (int c = j; c < m; c++) A[(size_t)i * m + c] -= f * A[(size_t)j * m + c];
      r[i] -= f * r[j];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    if (s_bad) {
      atomicExch(flags, B200FEM_ERR_INVALID_ARG);
      for (int i = 0; i < m; i++) r[i] = 0;
    } else {
      for (int i = m - 1; i >= 0; i--) {
        double t = r[i];
        for (int c = i + 1; c < m; c++) t -= A[(size_t)i * m + c] * r[c];
        r[i] = t / A[(size_t)i * m + i];
      }
    }
  }
  __syncthreads();
}

// A = G Y, r = G u0, then lam = A^-1 r (into r)
__global__ void pc_schur_kernel(int m, int R, const int* __restrict__ ptr, const int* __restrict__ row,
                                const double* __restrict__ w, const double* __restrict__ Y,
                                const double* __restrict__ u0, double* __restrict__ A, double* __restrict__ r,
                                int* __restrict__ flags) {
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int k = t / m, l = t % m, c = k / 3, d = k % 3;
    const double* yl = Y + (size_t)l * 3 * R;
    double s = 0;
    for (int q = ptr[c]; q < ptr[c + 1]; q++)
      if (row[q] >= 0) s += w[q] * yl[3 * (size_t)row[q] + d];
    A[t] = s;
  }
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    const int c = k / 3, d = k % 3;
    double s = 0;
    for (int q = ptr[c]; q < ptr[c + 1]; q++)
      if (row[q] >= 0) s += w[q] * u0[3 * (size_t)row[q] + d];
    r[k] = s;
  }
  __syncthreads();
  pc_dense_solve(A, r, m, flags);
}

// v = u0 - sum_k lam_k Y_k (k ascending)
__global__ void pc_velocity_kernel(int m, int R, const double* __restrict__ Y, const double* __restrict__ lam,
                                   double* __restrict__ v) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 3LL * R) return;
  double s = v[q];
  for (int k = 0; k < m; k++) s -= lam[k] * Y[(size_t)k * 3 * R + q];
  v[q] = s;
}

// GlobalMass position correction, one CTA: dist = G x - target over every
// point of each constraint, P = G M^-1 G^T over the points with a solve
// index, P mu = -dist, x += M^-1 G^T mu
__global__ void pc_correct_kernel(int ncons, const int* __restrict__ ptr, const int* __restrict__ node,
                                  const int* __restrict__ row, const double* __restrict__ w,
                                  const double* __restrict__ target, const double* __restrict__ mass,
                                  double* __restrict__ x, double* __restrict__ P, double* __restrict__ g,
                                  int* __restrict__ flags) {
  const int m = 3 * ncons;
  for (int k = threadIdx.x; k < m; k += blockDim.x) {
    const int c = k / 3, d = k % 3;
    double dist = -target[k];
    for (int q = ptr[c]; q < ptr[c + 1]; q++) dist += w[q] * x[3 * (size_t)node[q] + d];
    g[k] = -dist;
  }
  for (int t = threadIdx.x; t < m * m; t += blockDim.x) {
    const int k = t / m, l = t % m, c = k / 3, d = k % 3, c2 = l / 3, d2 = l % 3;
    double s = 0;
    if (d == d2)
      for (int q = ptr[c]; q < ptr[c + 1]; q++) {
        if (row[q] < 0) continue;
        for (int q2 = ptr[c2]; q2 < ptr[c2 + 1]; q2++)
          if (node[q2] == node[q]) s += w[q] * w[q2] / mass[node[q]];
      }
    P[t] = s;
  }
  __syncthreads();
  pc_dense_solve(P, g, m, flags);
  if (threadIdx.x == 0)
    for (int c = 0; c < ncons; c++)
      for (int q = ptr[c]; q < ptr[c + 1]; q++) {
        if (row[q] < 0) continue;
        for (int d = 0; d < 3; d++) x[3 * (size_t)node[q] + d] += w[q] * g[3 * c + d] / mass[node[q]];
      }
}

// The step's solve with LinearPointConstraints (replaces launch_solve for
// the ConstrainedBackwardEuler integrator); capturable: no host
// synchronisation.
cudaError_t launch_solve_points(Engine& eng, int max_iter) {
  DevPack& d = eng.d;
  const PointCons& pc = eng.pcons;
  const int m = 3 * pc.n, R = d.n_rows;
  const size_t vbytes = sizeof(double) * 3 * (size_t)R;
  cudaError_t e = launch_pcg_on(eng, max_iter, false, d.b, d.sol, 0.0, d.model_scal);
  if (e != cudaSuccess) return e;
  pc_status_kernel<<<1, 128, 0, eng.stream>>>(d.model_scal, d.n_models, d.flags);
  for (int k = 0; k < m && e == cudaSuccess; k++) {
    double* yk = d.pc_Y + (size_t)k * 3 * R;
    if ((e = cudaMemsetAsync(d.pc_rhs, 0, vbytes, eng.stream)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(yk, 0, vbytes, eng.stream)) != cudaSuccess) return e;
    pc_rhs_kernel<<<1, 32, 0, eng.stream>>>(d.pc_rhs, d.pc_ptr, d.pc_row, d.pc_w, k);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = launch_pcg_on(eng, max_iter, false, d.pc_rhs, yk, 0.0, d.model_scal);
    if (e == cudaSuccess) pc_status_kernel<<<1, 128, 0, eng.stream>>>(d.model_scal, d.n_models, d.flags);
  }
  if (e != cudaSuccess) return e;
  pc_schur_kernel<<<1, 256, 0, eng.stream>>>(m, R, d.pc_ptr, d.pc_row, d.pc_w, d.pc_Y, d.sol, d.pc_A, d.pc_lam,
                                            d.flags);
  pc_velocity_kernel<<<(unsigned)((3LL * R + 255) / 256), 256, 0, eng.stream>>>(m, R, d.pc_Y, d.pc_lam, d.sol);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = launch_state_update(eng, d.sol)) != cudaSuccess) return e;
  pc_correct_kernel<<<1, 256, 0, eng.stream>>>(pc.n, d.pc_ptr, d.pc_node, d.pc_row, d.pc_w, d.pc_target, d.mass,
                                              d.x, d.pc_A, d.pc_lam, d.flags);
  return cudaGetLastError();
}

}  // namespace b200fem
