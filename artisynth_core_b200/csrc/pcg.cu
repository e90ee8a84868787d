// pcg.cu -- persistent cooperative block-Jacobi PCG for the BackwardEuler
// system S v = b (replaces the reference's direct PARDISO / cuDSS solve,
// MechSystemSolver.java:2397-2444, and its CGSolver, CGSolver.java:42-134).
//
// The iteration is the pipelined preconditioned CG of Ghysels & Vanroose
// (2014): the dot products of an iteration and the SpMV of the next search
// direction share one grid-wide synchronisation, so each iteration costs a
// single grid barrier.  After convergence of the recurrence residual the
// true residual b - S x is formed; if it exceeds the tolerance the
// recurrences are restarted from it (residual replacement).
//
// Work split: every CTA owns a contiguous range of block rows, cut into
// "pieces" at model boundaries (a pack may hold many models).  Dot products
// are reduced per piece in a fixed order (warp shuffles, then shared
// memory), partial sums are written to a double-buffered table, and each
// model's scalars are summed from its pieces in a fixed order after the
// barrier: results are bit-reproducible and independent of timing.
#include <cuda_runtime.h>

#include "device_math.cuh"
#include "engine.h"
#include "spmv.cuh"

namespace b200fem {

constexpr int kPcgThreads = 1024;
constexpr int kRowChunk = 512;
constexpr int kMaxCtaPieces = 48;
constexpr int kMaxRestarts = 3;
constexpr unsigned long long kBarrierTimeoutNs = 5000000000ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ unsigned atom_add_release_u32(unsigned* p, unsigned v) {
  unsigned o;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(o) : "l"(p), "r"(v) : "memory");
  return o;
}

// Grid-wide barrier of a cooperative launch (all CTAs co-resident) on a
// monotonically increasing arrival counter: arrival k of a round sees
// count = round*G + k and waits for count >= (round+1)*G.  Release on the
// arrival and acquire on the poll order every CTA's prior global writes
// before every CTA's later reads.  The wait is bounded: after
// kBarrierTimeoutNs the CTA records B200FEM_ERR_TIMEOUT in flags[0] and
// returns false, and every CTA leaves the kernel at its next barrier.
// The counter must be zero when the kernel starts.
__device__ bool grid_barrier(unsigned* count, int* flags) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int* err = flags;
    const unsigned G = gridDim.x;
    const unsigned arrived = atom_add_release_u32(count, 1u) + 1u;
    const unsigned goal = ((arrived + G - 1u) / G) * G;
    int ok = 1;
    const unsigned long long t0 = global_ns();
    while ((int)(ld_acquire_u32(count) - goal) < 0) {
      if (*err != 0) {
        ok = 0;
        break;
      }
      if (global_ns() - t0 > kBarrierTimeoutNs) {
        atomicExch(flags, B200FEM_ERR_TIMEOUT);
        ok = 0;
        break;
      }
    }
    if (*err != 0) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

struct PcgArgs {
  int n_rows, n_pieces;
  const int* rowptr;
  const int* col;
  const int* blk_diag;
  const void* S;
  double* Dinv;
  const double* b;
  double *x, *r, *u, *w, *m0, *m1, *z, *q, *s, *p;
  const int* piece_row;
  const int* piece_model;
  const int* model_piece;
  const int* cta_piece;
  double* partials;  // [2][n_pieces][4]
  const double* step;
  double* model_out;  // n_models * 4: iterations, true rel residual, converged
  unsigned* barrier;
  int* flags;
  int* unconv;  // per iteration: some model still unconverged
  int max_iter;
  int update_state;
  double* xpos;
  double* vel;
  const int* act_node;
  const int* row_model;
};

struct CtaView {
  int pc0, pc1;
};

// Reduce ND per-row values over this CTA's pieces in a fixed order and write
// partials[buf][piece][k].  fn(row, lane, vals) runs per row, either by a
// whole warp (WARP_ROWS) or by one thread.
template <int ND, bool WARP_ROWS, typename Fn>
__device__ void cta_row_pass(const PcgArgs& a, CtaView cv, int buf, double (*rowbuf)[3], double (*pacc)[3],
                             Fn fn) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int npc = cv.pc1 - cv.pc0;
  for (int j = threadIdx.x; j < npc * 3; j += blockDim.x) pacc[j / 3][j % 3] = 0;
  const int r0 = a.piece_row[cv.pc0], r1 = a.piece_row[cv.pc1];
  for (int c0 = r0; c0 < r1; c0 += kRowChunk) {
    const int c1 = min(c0 + kRowChunk, r1);
    __syncthreads();
    if (WARP_ROWS) {
      for (int row = c0 + warp; row < c1; row += nwarps) {
        double vals[3] = {0, 0, 0};
        fn(row, lane, vals);
        if (lane == 0)
#pragma unroll
          for (int k = 0; k < ND; k++) rowbuf[row - c0][k] = vals[k];
      }
    } else {
      for (int row = c0 + (int)threadIdx.x; row < c1; row += blockDim.x) {
        double vals[3] = {0, 0, 0};
        fn(row, 0, vals);
#pragma unroll
        for (int k = 0; k < ND; k++) rowbuf[row - c0][k] = vals[k];
      }
    }
    __syncthreads();
    for (int j = warp; j < npc; j += nwarps) {
      const int pr0 = max(a.piece_row[cv.pc0 + j], c0), pr1 = min(a.piece_row[cv.pc0 + j + 1], c1);
      if (pr0 >= pr1) continue;
      double sm[3] = {0, 0, 0};
      for (int row = pr0 + lane; row < pr1; row += 32)
#pragma unroll
        for (int k = 0; k < ND; k++) sm[k] += rowbuf[row - c0][k];
#pragma unroll
      for (int k = 0; k < ND; k++)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) sm[k] += __shfl_xor_sync(0xffffffffu, sm[k], off);
      if (lane == 0)
#pragma unroll
        for (int k = 0; k < ND; k++) pacc[j][k] += sm[k];
    }
  }
  __syncthreads();
  double* out = a.partials + (size_t)buf * a.n_pieces * 4;
  for (int j = threadIdx.x; j < npc; j += blockDim.x)
#pragma unroll
    for (int k = 0; k < ND; k++) out[(size_t)(cv.pc0 + j) * 4 + k] = pacc[j][k];
}

// Per local piece: sum of the partials of its model (warp per piece, fixed
// lane striding and butterfly order).
template <int ND>
__device__ void model_sums(const PcgArgs& a, CtaView cv, int buf, double (*out)[3]) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const double* src = a.partials + (size_t)buf * a.n_pieces * 4;
  for (int j = warp; j < cv.pc1 - cv.pc0; j += nwarps) {
    const int m = a.piece_model[cv.pc0 + j];
    const int q0 = a.model_piece[m], q1 = a.model_piece[m + 1];
    double sm[3] = {0, 0, 0};
    for (int qq = q0 + lane; qq < q1; qq += 32)
#pragma unroll
      for (int k = 0; k < ND; k++) sm[k] += __ldcg(&src[(size_t)qq * 4 + k]);
#pragma unroll
    for (int k = 0; k < ND; k++)
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) sm[k] += __shfl_xor_sync(0xffffffffu, sm[k], off);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < ND; k++) out[j][k] = sm[k];
  }
  __syncthreads();
}

__device__ __forceinline__ int piece_of_row(const PcgArgs& a, CtaView cv, int row) {
  int j = 0;
  while (cv.pc0 + j + 1 < cv.pc1 && a.piece_row[cv.pc0 + j + 1] <= row) j++;
  return j;
}

__device__ __forceinline__ void load3(double* d, const double* src, int row) {
  d[0] = src[3 * (size_t)row];
  d[1] = src[3 * (size_t)row + 1];
  d[2] = src[3 * (size_t)row + 2];
}
__device__ __forceinline__ void store3(double* dst, int row, const double* v) {
  dst[3 * (size_t)row] = v[0];
  dst[3 * (size_t)row + 1] = v[1];
  dst[3 * (size_t)row + 2] = v[2];
}
__device__ __forceinline__ void mul33(double* y, const double* D, const double* v) {
#pragma unroll
  for (int c = 0; c < 3; c++) y[c] = D[3 * c] * v[0] + D[3 * c + 1] * v[1] + D[3 * c + 2] * v[2];
}
__device__ __forceinline__ double dot3(const double* a, const double* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

template <typename MT>
__global__ void __launch_bounds__(kPcgThreads) pcg_kernel(PcgArgs a) {
  __shared__ double rowbuf[kRowChunk][3];
  __shared__ double sn[kRowChunk][3];
  __shared__ double pacc[kMaxCtaPieces][3];
  __shared__ double sums[kMaxCtaPieces][3];
  __shared__ double s_bb[kMaxCtaPieces], s_tol[kMaxCtaPieces], s_alpha[kMaxCtaPieces],
      s_beta[kMaxCtaPieces], s_gold[kMaxCtaPieces], s_aold[kMaxCtaPieces];
  __shared__ int s_conv[kMaxCtaPieces], s_iters[kMaxCtaPieces], s_first[kMaxCtaPieces];
  __shared__ int s_restart;
  const MT* S = (const MT*)a.S;
  CtaView cv{a.cta_piece[blockIdx.x], a.cta_piece[blockIdx.x + 1]};
  const int npc = cv.pc1 - cv.pc0;
  int ph = 0;

  // ---- P0: block-Jacobi inverse, r = b - S x, u = Dinv r, ||b||^2
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i <= a.max_iter + 1; i += blockDim.x) a.unconv[i] = 0;
  cta_row_pass<1, true>(a, cv, ph & 1, rowbuf, pacc, [&](int row, int lane, double* vals) {
    double Ax[3];
    warp_row_spmv<MT>(row, a.rowptr, a.col, S, a.x, lane, Ax);
    if (lane == 0) {
      const MT* Db = S + (size_t)a.blk_diag[row] * 9;
      double d[9], inv[9];
#pragma unroll
      for (int i = 0; i < 9; i++) d[i] = (double)Db[i];
      if (invert3(inv, d) == 0.0) {
        atomicExch(a.flags, B200FEM_ERR_INVALID_ARG);
#pragma unroll
        for (int i = 0; i < 9; i++) inv[i] = 0;
      }
#pragma unroll
      for (int i = 0; i < 9; i++) a.Dinv[(size_t)row * 9 + i] = inv[i];
      double bv[3], r[3], u[3];
      load3(bv, a.b, row);
#pragma unroll
      for (int c = 0; c < 3; c++) r[c] = bv[c] - Ax[c];
      mul33(u, inv, r);
      store3(a.r, row, r);
      store3(a.u, row, u);
      vals[0] = dot3(bv, bv);
    }
  });
  if (!grid_barrier(a.barrier, a.flags)) return;
  model_sums<1>(a, cv, ph & 1, sums);
  for (int j = threadIdx.x; j < npc; j += blockDim.x) {
    const int m = a.piece_model[cv.pc0 + j];
    s_bb[j] = sums[j][0];
    s_tol[j] = a.step[(size_t)m * 8 + 6];
    s_conv[j] = 0;
    s_iters[j] = 0;
  }
  ph++;

  int total_it = 0;
  for (int restart = 0;; restart++) {
    // ---- P1: w = S u, m = Dinv w; dots gamma = r.u, delta = w.u, rho = r.r
    for (int j = threadIdx.x; j < npc; j += blockDim.x) s_first[j] = 1;
    cta_row_pass<3, true>(a, cv, ph & 1, rowbuf, pacc, [&](int row, int lane, double* vals) {
      if (s_conv[piece_of_row(a, cv, row)]) return;
      double Au[3];
      warp_row_spmv<MT>(row, a.rowptr, a.col, S, a.u, lane, Au);
      if (lane == 0) {
        double r[3], u[3], m[3], zero[3] = {0, 0, 0};
        load3(r, a.r, row);
        load3(u, a.u, row);
        mul33(m, a.Dinv + (size_t)row * 9, Au);
        store3(a.w, row, Au);
        store3(a.m0, row, m);
        store3(a.z, row, zero);
        store3(a.q, row, zero);
        store3(a.s, row, zero);
        store3(a.p, row, zero);
        vals[0] = dot3(r, u);
        vals[1] = dot3(Au, u);
        vals[2] = dot3(r, r);
      }
    });
    if (!grid_barrier(a.barrier, a.flags)) return;
    int mbuf = 0;  // m0 holds the current m

    for (int it = 0;; it++) {
      const int idx = total_it + it;
      const double* mc = mbuf ? a.m1 : a.m0;
      double* mn = mbuf ? a.m0 : a.m1;
      // The SpMV n = S m does not depend on this iteration's scalars, so it
      // runs on the first warps while the last warps reduce the scalars.
      const int nsumw = min(max(npc, 1), 8);
      const int nroww = (blockDim.x >> 5) - nsumw;
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int r0 = a.piece_row[cv.pc0], r1 = a.piece_row[cv.pc1];
      for (int j = threadIdx.x; j < npc * 3; j += blockDim.x) pacc[j / 3][j % 3] = 0;
      bool stop = false;
      for (int c0 = r0, first = 1; c0 < r1 || first; c0 += kRowChunk, first = 0) {
        const int c1 = min(c0 + kRowChunk, r1);
        if (warp < nroww) {
          for (int row = c0 + warp; row < c1; row += nroww) {
            double n[3];
            warp_row_spmv<MT>(row, a.rowptr, a.col, S, mc, lane, n);
            if (lane == 0) {
              sn[row - c0][0] = n[0];
              sn[row - c0][1] = n[1];
              sn[row - c0][2] = n[2];
            }
          }
        } else if (first) {
          const int sw = warp - nroww;
          const double* src = a.partials + (size_t)(ph & 1) * a.n_pieces * 4;
          for (int j = sw; j < npc; j += nsumw) {
            const int m = a.piece_model[cv.pc0 + j];
            const int q0 = a.model_piece[m], q1 = a.model_piece[m + 1];
            double sm[3] = {0, 0, 0};
            for (int qq = q0 + lane; qq < q1; qq += 32)
#pragma unroll
              for (int k = 0; k < 3; k++) sm[k] += __ldcg(&src[(size_t)qq * 4 + k]);
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
              for (int off = 16; off > 0; off >>= 1) sm[k] += __shfl_xor_sync(0xffffffffu, sm[k], off);
            if (lane == 0) {
              sums[j][0] = sm[0];
              sums[j][1] = sm[1];
              sums[j][2] = sm[2];
            }
          }
        }
        __syncthreads();
        if (first) {
          // scalars; convergence on the recurrence residual
          for (int j = threadIdx.x; j < npc; j += blockDim.x) {
            if (s_conv[j]) continue;
            const double gam = sums[j][0], del = sums[j][1], rho = sums[j][2];
            if (sqrt(rho) <= s_tol[j] * sqrt(s_bb[j]) || rho == 0.0) {
              s_conv[j] = 1;
              continue;
            }
            double beta = 0, alpha;
            if (s_first[j]) {
              alpha = gam / del;
              s_first[j] = 0;
            } else {
              beta = gam / s_gold[j];
              alpha = gam / (del - beta * gam / s_aold[j]);
            }
            s_beta[j] = beta;
            s_alpha[j] = alpha;
            s_gold[j] = gam;
            s_aold[j] = alpha;
            s_iters[j]++;
            const int m = a.piece_model[cv.pc0 + j];
            if (cv.pc0 + j == a.model_piece[m + 1] - 1) a.unconv[idx] = 1;
          }
          __syncthreads();
          if (idx >= a.max_iter) {
            stop = true;
            break;
          }
        }
        // z = n + beta z; q = m + beta q; s = w + beta s; p = u + beta p;
        // x += alpha p; r -= alpha s; u -= alpha q; w -= alpha z; m' = Dinv w
        for (int row = c0 + (int)threadIdx.x; row < c1; row += blockDim.x) {
          const int j = piece_of_row(a, cv, row);
          double v3[3] = {0, 0, 0};
          if (!s_conv[j]) {
            const double al = s_alpha[j], be = s_beta[j];
            double x[3], r[3], u[3], w[3], z[3], q[3], sv[3], p[3], mm[3], D[9];
            load3(x, a.x, row);
            load3(r, a.r, row);
            load3(u, a.u, row);
            load3(w, a.w, row);
            load3(z, a.z, row);
            load3(q, a.q, row);
            load3(sv, a.s, row);
            load3(p, a.p, row);
            load3(mm, mc, row);
#pragma unroll
            for (int i = 0; i < 9; i++) D[i] = a.Dinv[(size_t)row * 9 + i];
#pragma unroll
            for (int c = 0; c < 3; c++) {
              z[c] = sn[row - c0][c] + be * z[c];
              q[c] = mm[c] + be * q[c];
              sv[c] = w[c] + be * sv[c];
              p[c] = u[c] + be * p[c];
              x[c] += al * p[c];
              r[c] -= al * sv[c];
              u[c] -= al * q[c];
              w[c] -= al * z[c];
            }
            double mnew[3];
            mul33(mnew, D, w);
            store3(a.x, row, x);
            store3(a.r, row, r);
            store3(a.u, row, u);
            store3(a.w, row, w);
            store3(a.z, row, z);
            store3(a.q, row, q);
            store3(a.s, row, sv);
            store3(a.p, row, p);
            store3(mn, row, mnew);
            v3[0] = dot3(r, u);
            v3[1] = dot3(w, u);
            v3[2] = dot3(r, r);
          }
          rowbuf[row - c0][0] = v3[0];
          rowbuf[row - c0][1] = v3[1];
          rowbuf[row - c0][2] = v3[2];
        }
        __syncthreads();
        for (int j = warp; j < npc; j += (blockDim.x >> 5)) {
          const int pr0 = max(a.piece_row[cv.pc0 + j], c0), pr1 = min(a.piece_row[cv.pc0 + j + 1], c1);
          if (pr0 >= pr1) continue;
          double sm[3] = {0, 0, 0};
          for (int row = pr0 + lane; row < pr1; row += 32)
#pragma unroll
            for (int k = 0; k < 3; k++) sm[k] += rowbuf[row - c0][k];
#pragma unroll
          for (int k = 0; k < 3; k++)
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) sm[k] += __shfl_xor_sync(0xffffffffu, sm[k], off);
          if (lane == 0)
#pragma unroll
            for (int k = 0; k < 3; k++) pacc[j][k] += sm[k];
        }
        __syncthreads();
      }
      if (stop) {
        total_it += it;
        break;
      }
      ph++;
      {
        double* out = a.partials + (size_t)(ph & 1) * a.n_pieces * 4;
        for (int j = threadIdx.x; j < npc; j += blockDim.x)
#pragma unroll
          for (int k = 0; k < 3; k++) out[(size_t)(cv.pc0 + j) * 4 + k] = pacc[j][k];
      }
      if (!grid_barrier(a.barrier, a.flags)) return;
      mbuf ^= 1;
      if (__ldcg(&a.unconv[idx]) == 0) {
        total_it += it;
        break;
      }
    }
    ph++;

    // ---- true residual r = b - S x; restart from it when it misses the
    // tolerance although the recurrence converged
    cta_row_pass<1, true>(a, cv, ph & 1, rowbuf, pacc, [&](int row, int lane, double* vals) {
      double Ax[3];
      warp_row_spmv<MT>(row, a.rowptr, a.col, S, a.x, lane, Ax);
      if (lane == 0) {
        double bv[3], r[3];
        load3(bv, a.b, row);
#pragma unroll
        for (int c = 0; c < 3; c++) r[c] = bv[c] - Ax[c];
        vals[0] = dot3(r, r);
        if (!s_conv[piece_of_row(a, cv, row)]) return;
        double u[3];
        mul33(u, a.Dinv + (size_t)row * 9, r);
        store3(a.r, row, r);
        store3(a.u, row, u);
      }
    });
    if (!grid_barrier(a.barrier, a.flags)) return;
    model_sums<1>(a, cv, ph & 1, sums);
    ph++;
    if (threadIdx.x == 0) s_restart = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < npc; j += blockDim.x) {
      const double rel = s_bb[j] > 0 ? sqrt(sums[j][0] / s_bb[j]) : sqrt(sums[j][0]);
      const bool ok = rel <= s_tol[j] || sums[j][0] == 0.0;
      if (s_conv[j] && !ok && restart < kMaxRestarts && total_it < a.max_iter) {
        s_conv[j] = 0;  // residual replacement for this model
        s_restart = 1;
      }
      const int m = a.piece_model[cv.pc0 + j];
      if (cv.pc0 + j == a.model_piece[m + 1] - 1) {
        double* o = a.model_out + (size_t)m * 4;
        o[0] = s_iters[j];
        o[1] = rel;
        o[2] = (s_conv[j] && ok) ? 1.0 : 0.0;
      }
    }
    __syncthreads();
    // every CTA must agree on a restart: publish and read after a barrier
    if (s_restart && threadIdx.x == 0) a.unconv[a.max_iter + 1] = restart + 1;
    if (!grid_barrier(a.barrier, a.flags)) return;
    if (__ldcg(&a.unconv[a.max_iter + 1]) != restart + 1) break;
  }

  if (a.update_state) {
    const int r0 = a.piece_row[cv.pc0], r1 = a.piece_row[cv.pc1];
    for (int row = r0 + threadIdx.x; row < r1; row += blockDim.x) {
      const int n = a.act_node[row];
      const double h = a.step[(size_t)a.row_model[row] * 8];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double vn = a.x[3 * (size_t)row + c];
        a.vel[3 * (size_t)n + c] = vn;
        a.xpos[3 * (size_t)n + c] += h * vn;
      }
    }
  }
}

cudaError_t launch_pcg(Engine& eng, int max_iter, bool update_state, int init_zero) {
  DevPack& d = eng.d;
  cudaError_t e;
  if (init_zero) {
    if ((e = cudaMemsetAsync(d.sol, 0, sizeof(double) * 3 * (size_t)d.n_rows, eng.stream)) != cudaSuccess) return e;
  }
  if ((e = cudaMemsetAsync(d.barrier, 0, sizeof(unsigned), eng.stream)) != cudaSuccess) return e;
  PcgArgs a;
  a.n_rows = d.n_rows;
  a.n_pieces = d.n_pieces;
  a.rowptr = d.blk_rowptr;
  a.col = d.blk_col;
  a.blk_diag = d.blk_diag;
  a.S = d.S;
  a.Dinv = d.Dinv;
  a.b = d.b;
  a.x = d.sol;
  a.r = d.r;
  a.u = d.u;
  a.w = d.w;
  a.m0 = d.m0;
  a.m1 = d.m1;
  a.z = d.z;
  a.q = d.q;
  a.s = d.s;
  a.p = d.p;
  a.piece_row = d.piece_row;
  a.piece_model = d.piece_model;
  a.model_piece = d.model_piece;
  a.cta_piece = d.cta_piece;
  a.partials = d.partials;
  a.step = d.step;
  a.model_out = d.model_scal;
  a.barrier = d.barrier;
  a.flags = d.flags;
  a.unconv = d.unconv;
  a.max_iter = max_iter;
  a.update_state = update_state ? 1 : 0;
  a.xpos = d.x;
  a.vel = d.v;
  a.act_node = d.act_node;
  a.row_model = d.row_model;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(eng.pcg_grid);
  cfg.blockDim = dim3(kPcgThreads);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = eng.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, pcg_kernel<double>, a);
}

int pcg_threads() { return kPcgThreads; }
int pcg_max_cta_pieces() { return kMaxCtaPieces; }

int pcg_max_grid(int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<double>, kPcgThreads, 0);
  return sms * (per_sm > 0 ? per_sm : 1);
}

}  // namespace b200fem
