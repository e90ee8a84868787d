// pcg_cluster.cu -- block-Jacobi PCG for packs of many models, one
// thread-block cluster per model.
//
// The persistent grid-wide PCG (pcg.cu) spreads every model over the whole
// GPU and pays a grid barrier per iteration; in a pack of uneven models the
// last iterations of the slowest model leave most CTAs waiting at those
// barriers.  Here each model of the pack is solved by one cluster of
// kClusterCtas CTAs: the cluster takes the next model from a queue (largest
// first), solves S v = b for it with classic preconditioned CG
// (CGSolver.java:42-134 with the block-Jacobi preconditioner of the
// persistent PCG) and takes the next model, so no SM waits for another
// model.  The CTAs of a cluster share each reduction through distributed
// shared memory and meet at hardware cluster barriers, two per iteration;
// there is no spin-wait on memory.
//
// Per iteration k (p_{k-1} in one of two buffers, z_{k-1} final):
//   rows pass:   p_k = z + beta p_{k-1} (first iteration: z), stored in the
//                other buffer; q = S p_k with every neighbour's p_k formed
//                the same way from its z and p_{k-1}; partial p.q
//   barrier:     alpha = r.z / p.q
//   update pass: x += alpha p, r -= alpha q, z = D^-1 r; partials r.z, r.r
//   barrier:     beta, convergence of the recurrence residual
// When the recurrence converges, the true residual b - S x decides; a model
// that misses the tolerance restarts from it (at most kMaxRestartsCl times,
// within max_iter iterations in all).  Reductions run in a fixed order, so
// results are bit-reproducible for a given cluster size.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "device_math.cuh"
#include "engine.h"

namespace cg = cooperative_groups;

namespace b200fem {

constexpr int kClusterCtas = 8;
constexpr int kClThreads = 512;
constexpr int kClLanes = 8;  // lanes per block row
constexpr int kClGroups = kClThreads / kClLanes;
constexpr int kMaxRestartsCl = 10;

struct ClusterPcgArgs {
  int n_models;
  const int* order;      // models in the order the clusters take them
  int* queue;            // next position in `order` (zero at launch)
  const int* model_row;  // model m owns block rows [model_row[m], model_row[m + 1])
  const int* rowptr;
  const int* col;
  const int* blk_diag;
  const void* S;
  double* Dinv;
  const double* b;
  double* x;
  double* r;
  double* z;
  double* pbuf0;
  double* pbuf1;
  double* q;
  const double* step;
  double tol_override;
  double* model_out;  // per model: iterations, true relative residual, converged
  const int* model_active;
  const double* row_nrm;
  const double* row_off;
  int max_iter;
  int update_state;
  double* xpos;
  double* vel;
  double* vprev;
  double* vprev2;
  double* vprev3;
  double* vprev4;
  const int* act_node;
  int* flags;
};

__device__ __forceinline__ void cl_mul33(double* y, const double* D, const double* v) {
#pragma unroll
  for (int c = 0; c < 3; c++) y[c] = D[3 * c] * v[0] + D[3 * c + 1] * v[1] + D[3 * c + 2] * v[2];
}

__device__ __forceinline__ double cl_dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ void cl_project(const double* nrm, int row, double* y) {
  if (!nrm) return;
  const double* n = nrm + 3 * (size_t)row;
  const double d = n[0] * y[0] + n[1] * y[1] + n[2] * y[2];
  y[0] -= n[0] * d;
  y[1] -= n[1] * d;
  y[2] -= n[2] * d;
}

__device__ __forceinline__ void cl_load3(double* d, const double* v, int row) {
  d[0] = __ldcg(v + 3 * (size_t)row);
  d[1] = __ldcg(v + 3 * (size_t)row + 1);
  d[2] = __ldcg(v + 3 * (size_t)row + 2);
}

__device__ __forceinline__ void cl_store3(double* v, int row, const double* d) {
  v[3 * (size_t)row] = d[0];
  v[3 * (size_t)row + 1] = d[1];
  v[3 * (size_t)row + 2] = d[2];
}

// the search direction of a neighbour row: z + beta p_prev (first: z)
__device__ __forceinline__ void cl_dir(double* pv, const double* z, const double* pprev, int row, double beta,
                                       bool first) {
  cl_load3(pv, z, row);
  if (!first) {
    double po[3];
    cl_load3(po, pprev, row);
#pragma unroll
    for (int c = 0; c < 3; c++) pv[c] = fma(beta, po[c], pv[c]);
  }
}

// y = (S v)_row on a group of kClLanes lanes (all lanes get the sum); the
// vector is formed per neighbour by vec(pv, j).  Every lane of the warp
// calls it together (the group sums are warp shuffles over the full mask); a
// group whose row is past its range passes valid = false and adds nothing.
template <typename MT, typename Vec>
__device__ __forceinline__ void cl_row_spmv(const ClusterPcgArgs& a, int row, bool valid, int gl, Vec vec,
                                            double* y) {
  const MT* S = (const MT*)a.S;
  double acc[3] = {0, 0, 0};
  const int p0 = valid ? a.rowptr[row] : 0, p1 = valid ? a.rowptr[row + 1] : 0;
  for (int p = p0 + gl; p < p1; p += kClLanes) {
    const int j = a.col[p];
    double v[3];
    vec(v, j);
    const MT* B = S + (size_t)p * 9;
#pragma unroll
    for (int i = 0; i < 3; i++)
      acc[i] += (double)B[3 * i] * v[0] + (double)B[3 * i + 1] * v[1] + (double)B[3 * i + 2] * v[2];
  }
#pragma unroll
  for (int off = kClLanes / 2; off > 0; off >>= 1)
#pragma unroll
    for (int i = 0; i < 3; i++) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], off);
  y[0] = acc[0];
  y[1] = acc[1];
  y[2] = acc[2];
}

// Sum of ND per-thread values over the cluster, in a fixed order: warps by
// butterfly, the CTA's warps in order, then the CTAs in rank order through
// distributed shared memory.  Every thread of the cluster gets the sums.
// `slot` alternates between the two partial buffers (a CTA may write the
// next reduction's partial while a slower one still reads this one).
template <int ND>
__device__ __forceinline__ void cl_reduce(cg::cluster_group& cluster, double (*part)[4], double (*wsum)[4],
                                          double* tot, int& slot, double* v) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < ND; k++) v[k] += __shfl_xor_sync(0xffffffffu, v[k], off);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < ND; k++) wsum[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[ND];
#pragma unroll
    for (int k = 0; k < ND; k++) s[k] = 0;
    for (int w = 0; w < kClThreads / 32; w++)
#pragma unroll
      for (int k = 0; k < ND; k++) s[k] += wsum[w][k];
#pragma unroll
    for (int k = 0; k < ND; k++) part[slot][k] = s[k];
  }
  cluster.sync();
  if (threadIdx.x == 0) {
    double s[ND];
#pragma unroll
    for (int k = 0; k < ND; k++) s[k] = 0;
    for (int c = 0; c < kClusterCtas; c++) {
      const double* rp = cluster.map_shared_rank(&part[slot][0], c);
#pragma unroll
      for (int k = 0; k < ND; k++) s[k] += rp[k];
    }
#pragma unroll
    for (int k = 0; k < ND; k++) tot[k] = s[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < ND; k++) v[k] = tot[k];
  slot ^= 1;
}

template <typename MT>
__global__ void __launch_bounds__(kClThreads) pcg_cluster_kernel(ClusterPcgArgs a) {
  cg::cluster_group cluster = cg::this_cluster();
  const int rank = (int)cluster.block_rank();
  __shared__ double part[2][4];
  __shared__ double wsum[kClThreads / 32][4];
  __shared__ double tot[4];
  __shared__ int s_next;
  const int grp = threadIdx.x / kClLanes, gl = threadIdx.x % kClLanes;
  constexpr int kWarpGroups = 32 / kClLanes;
  const int wgrp = grp % kWarpGroups, wbase = grp - wgrp;  // group within the warp, warp's first group
  const bool leader = gl == 0;
  int slot = 0;
  for (;;) {
    // ---- the next model: rank 0 takes it from the queue, every CTA reads it
    if (rank == 0 && threadIdx.x == 0) {
      const int k = atomicAdd(a.queue, 1);
      s_next = k < a.n_models ? a.order[k] : -1;
    }
    cluster.sync();
    const int m = *cluster.map_shared_rank(&s_next, 0);
    cluster.sync();  // every CTA has read rank 0's s_next before it changes
    if (m < 0) break;
    const int R0 = a.model_row[m], R1 = a.model_row[m + 1];
    const bool off = a.model_active && !a.model_active[m];
    if (off || R1 <= R0) {
      if (rank == 0 && threadIdx.x == 0) {
        a.model_out[(size_t)m * 4] = 0;
        a.model_out[(size_t)m * 4 + 1] = 0;
        a.model_out[(size_t)m * 4 + 2] = 1.0;
      }
      continue;
    }
    // this CTA's rows
    const int nrow = R1 - R0;
    const int c0 = R0 + (int)((long long)nrow * rank / kClusterCtas);
    const int c1 = R0 + (int)((long long)nrow * (rank + 1) / kClusterCtas);
    const double tol = a.tol_override > 0 ? a.tol_override : a.step[(size_t)m * 8 + 6];

    // ---- block-Jacobi inverse, r = b - S x0, z = D^-1 r; ||b||^2, r.z, r.r
    double v3[3] = {0, 0, 0};
    // (loops with a shuffle run over warp-uniform bases: the warp's four
    // groups take rows base .. base + 3)
    for (int base = c0 + wbase; base < c1; base += kClGroups) {
      const int row = base + wgrp;
      const bool valid = row < c1;
      double Ax[3];
      cl_row_spmv<MT>(a, row, valid, gl, [&](double* pv, int j) { cl_load3(pv, a.x, j); }, Ax);
      if (leader && valid) {
        const MT* Db = (const MT*)a.S + (size_t)a.blk_diag[row] * 9;
        double d[9], inv[9];
#pragma unroll
        for (int k = 0; k < 9; k++) d[k] = (double)Db[k];
        if (invert3(inv, d) == 0.0) {
          atomicExch(a.flags, B200FEM_ERR_INVALID_ARG);
#pragma unroll
          for (int k = 0; k < 9; k++) inv[k] = 0;
        }
        if (a.row_nrm) {
          // P D^-1 P with P = I - n n^T
          const double* n = a.row_nrm + 3 * (size_t)row;
          double t[9];
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              t[3 * i + j] = inv[3 * i + j] - n[i] * (n[0] * inv[j] + n[1] * inv[3 + j] + n[2] * inv[6 + j]);
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++)
              inv[3 * i + j] = t[3 * i + j] - (t[3 * i] * n[0] + t[3 * i + 1] * n[1] + t[3 * i + 2] * n[2]) * n[j];
        }
#pragma unroll
        for (int k = 0; k < 9; k++) a.Dinv[(size_t)row * 9 + k] = inv[k];
        double bv[3], rr[3], zz[3];
        cl_load3(bv, a.b, row);
#pragma unroll
        for (int c = 0; c < 3; c++) rr[c] = bv[c] - Ax[c];
        cl_project(a.row_nrm, row, rr);
        cl_project(a.row_nrm, row, bv);
        cl_mul33(zz, inv, rr);
        cl_store3(a.r, row, rr);
        cl_store3(a.z, row, zz);
        v3[0] += cl_dot3(bv, bv);
        v3[1] += cl_dot3(rr, zz);
        v3[2] += cl_dot3(rr, rr);
      }
    }
    cl_reduce<3>(cluster, part, wsum, tot, slot, v3);
    const double bb = v3[0];
    double rz = v3[1], rr2 = v3[2];
    const double thr2 = tol * tol * (bb > 0 ? bb : 1.0);
    int it = 0, restarts = 0;
    double rel = 0;
    bool ok = false;
    for (;;) {
      // ---- CG iterations from r, z (first direction p = z)
      bool first = true;
      double beta = 0;
      double* pold = a.pbuf0;
      double* pnew = a.pbuf1;
      bool conv = rr2 <= thr2;
      while (!conv && it < a.max_iter) {
        double v1[1] = {0};
        for (int base = c0 + wbase; base < c1; base += kClGroups) {
          const int row = base + wgrp;
          const bool valid = row < c1;
          double qv[3];
          cl_row_spmv<MT>(a, row, valid, gl, [&](double* pv, int j) { cl_dir(pv, a.z, pold, j, beta, first); },
                          qv);
          if (leader && valid) {
            double pv[3];
            cl_dir(pv, a.z, pold, row, beta, first);
            cl_project(a.row_nrm, row, qv);
            cl_store3(pnew, row, pv);
            cl_store3(a.q, row, qv);
            v1[0] += cl_dot3(pv, qv);
          }
        }
        cl_reduce<1>(cluster, part, wsum, tot, slot, v1);
        const double alpha = v1[0] != 0.0 ? rz / v1[0] : 0.0;
        double v2[2] = {0, 0};
        for (int row = c0 + grp; row < c1; row += kClGroups) {
          if (!leader) continue;
          double pv[3], qv[3], xv[3], rv[3], zz[3];
          cl_load3(pv, pnew, row);
          cl_load3(qv, a.q, row);
          cl_load3(xv, a.x, row);
          cl_load3(rv, a.r, row);
#pragma unroll
          for (int c = 0; c < 3; c++) {
            xv[c] = fma(alpha, pv[c], xv[c]);
            rv[c] = fma(-alpha, qv[c], rv[c]);
          }
          cl_mul33(zz, a.Dinv + (size_t)row * 9, rv);
          cl_store3(a.x, row, xv);
          cl_store3(a.r, row, rv);
          cl_store3(a.z, row, zz);
          v2[0] += cl_dot3(rv, zz);
          v2[1] += cl_dot3(rv, rv);
        }
        cl_reduce<2>(cluster, part, wsum, tot, slot, v2);
        beta = rz != 0.0 ? v2[0] / rz : 0.0;
        rz = v2[0];
        rr2 = v2[1];
        it++;
        conv = rr2 <= thr2;
        first = false;
        double* t = pold;
        pold = pnew;
        pnew = t;
      }
      // ---- the true residual decides (restart state if it misses)
      double v1[2] = {0, 0};
      for (int base = c0 + wbase; base < c1; base += kClGroups) {
        const int row = base + wgrp;
        const bool valid = row < c1;
        double Ax[3];
        cl_row_spmv<MT>(a, row, valid, gl, [&](double* pv, int j) { cl_load3(pv, a.x, j); }, Ax);
        if (leader && valid) {
          double bv[3], rv[3], zz[3];
          cl_load3(bv, a.b, row);
#pragma unroll
          for (int c = 0; c < 3; c++) rv[c] = bv[c] - Ax[c];
          cl_project(a.row_nrm, row, rv);
          cl_mul33(zz, a.Dinv + (size_t)row * 9, rv);
          cl_store3(a.r, row, rv);
          cl_store3(a.z, row, zz);
          v1[0] += cl_dot3(rv, rv);
          v1[1] += cl_dot3(rv, zz);
        }
      }
      cl_reduce<2>(cluster, part, wsum, tot, slot, v1);
      rel = bb > 0 ? sqrt(v1[0] / bb) : sqrt(v1[0]);
      ok = rel <= tol || v1[0] == 0.0;
      if (ok || restarts >= kMaxRestartsCl || it >= a.max_iter) break;
      restarts++;
      rz = v1[1];
      rr2 = v1[0];
    }
    if (rank == 0 && threadIdx.x == 0) {
      a.model_out[(size_t)m * 4] = it;
      a.model_out[(size_t)m * 4 + 1] = rel;
      a.model_out[(size_t)m * 4 + 2] = ok ? 1.0 : 0.0;
    }
    if (a.update_state) {
      // setActiveVelState, x1 = x0 + h v1 (MechSystemSolver.java:2465-2475),
      // and the velocity history of the warm start
      const double h = a.step[(size_t)m * 8];
      for (int row = c0 + threadIdx.x; row < c1; row += kClThreads) {
        const int n = a.act_node[row];
        double xn[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
          const double vn = a.x[3 * (size_t)row + c];
          a.vprev4[3 * (size_t)n + c] = a.vprev3[3 * (size_t)n + c];
          a.vprev3[3 * (size_t)n + c] = a.vprev2[3 * (size_t)n + c];
          a.vprev2[3 * (size_t)n + c] = a.vprev[3 * (size_t)n + c];
          a.vprev[3 * (size_t)n + c] = a.vel[3 * (size_t)n + c];
          a.vel[3 * (size_t)n + c] = vn;
          xn[c] = a.xpos[3 * (size_t)n + c] + h * vn;
        }
        if (a.row_nrm) {
          const double* nq = a.row_nrm + 3 * (size_t)row;
          const double dist = nq[0] * xn[0] + nq[1] * xn[1] + nq[2] * xn[2] - a.row_off[row];
#pragma unroll
          for (int c = 0; c < 3; c++) xn[c] -= nq[c] * dist;
        }
#pragma unroll
        for (int c = 0; c < 3; c++) a.xpos[3 * (size_t)n + c] = xn[c];
      }
    }
  }
  cluster.sync();  // no CTA leaves while another may still read its shared memory
}

// clusters that fit on the device at once (0 when clusters are unavailable)
int pcg_cluster_capacity(bool fp32) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(kClusterCtas * 64);
  cfg.blockDim = dim3(kClThreads);
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kClusterCtas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  cudaError_t e = fp32 ? cudaOccupancyMaxActiveClusters(&n, pcg_cluster_kernel<float>, &cfg)
                       : cudaOccupancyMaxActiveClusters(&n, pcg_cluster_kernel<double>, &cfg);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

// One solve of every model of the pack with one cluster per model (the
// step's solve when the pack uses the cluster split).  The queue counter is
// cleared on the stream first, so the launch is capturable.
cudaError_t launch_pcg_cluster(Engine& eng, int max_iter, bool update_state, const double* rhs, double* xsol,
                               double tol_override, double* model_out) {
  DevPack& d = eng.d;
  cudaError_t e = cudaMemsetAsync(d.cl_queue, 0, sizeof(int), eng.stream);
  if (e != cudaSuccess) return e;
  ClusterPcgArgs a;
  a.n_models = d.n_models;
  a.order = d.cl_order;
  a.queue = d.cl_queue;
  a.model_row = d.model_row;
  a.rowptr = d.blk_rowptr;
  a.col = d.blk_col;
  a.blk_diag = d.blk_diag;
  const bool fp32 = eng.precision == B200FEM_PREC_MIXED;
  a.S = fp32 ? (const void*)d.S_f : (const void*)d.S;
  a.Dinv = d.Dinv;
  a.b = rhs;
  a.x = xsol;
  a.r = d.r;
  a.z = d.z;
  a.pbuf0 = d.p;
  a.pbuf1 = d.u;
  a.q = d.q;
  a.step = d.step;
  a.tol_override = tol_override;
  a.model_out = model_out;
  a.model_active = eng.any_inactive ? d.model_active : nullptr;
  a.row_nrm = (update_state && eng.integrator == B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER && d.row_nrm)
                  ? d.row_nrm
                  : nullptr;
  a.row_off = a.row_nrm ? d.row_off : nullptr;
  a.max_iter = max_iter;
  a.update_state = update_state ? 1 : 0;
  a.xpos = d.x;
  a.vel = d.v;
  a.vprev = d.vprev;
  a.vprev2 = d.vprev2;
  a.vprev3 = d.vprev3;
  a.vprev4 = d.vprev4;
  a.act_node = d.act_node;
  a.flags = d.flags;
  cudaLaunchConfig_t cfg = {};
  const int clusters = std::max(1, std::min(eng.cl_clusters, d.n_models));
  cfg.gridDim = dim3(kClusterCtas * clusters);
  cfg.blockDim = dim3(kClThreads);
  cfg.stream = eng.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kClusterCtas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return fp32 ? cudaLaunchKernelEx(&cfg, pcg_cluster_kernel<float>, a)
              : cudaLaunchKernelEx(&cfg, pcg_cluster_kernel<double>, a);
}

}  // namespace b200fem
