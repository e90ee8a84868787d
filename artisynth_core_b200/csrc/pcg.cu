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
// Work split: every CTA owns a list of "pieces" (row ranges of one model).
// In the contiguous split the pieces of a CTA are adjacent (a contiguous row
// range cut at model boundaries), which lets the row state and the CTA's
// slice of S live in shared memory; in the strided split, for packs too
// large for that, every model is cut into short pieces dealt over all CTAs.
// Passes over rows skip the models that have converged.  Dot products
// are reduced per piece in a fixed order (warp shuffles, then shared
// memory), partial sums are written to a double-buffered table, and each
// model's scalars are summed from its pieces in a fixed order after the
// barrier: results are bit-reproducible and independent of timing.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "device_math.cuh"
#include "engine.h"
#include "spmv.cuh"

namespace b200fem {

// Threads per CTA: the strided split (every SM holds thousands of rows in
// its bulk phase) wants many loads in flight; the resident form (a few
// hundred rows per CTA at most, latency-bound) runs 512 threads with up to
// 128 registers each, free of spills.  Measured on the 40x10x10 hex beam:
// 4.7 us per iteration at 512 threads, 5.6 at 1024; on the 256-beam strided
// pack 1024 threads stay faster (9.6 against 12.7 ms of PCG per step).
constexpr int kPcgThreads = 1024;
constexpr int kPcgThreadsResident = 512;
__host__ __device__ constexpr int pcg_block(bool resident) { return resident ? kPcgThreadsResident : kPcgThreads; }
constexpr int kRowChunk = 512;
// lanes per row in the SpMV passes outside the iteration (P0, P1, classic
// phase A, true residual): several rows per warp, a group leader per row
constexpr int kPassLanes = 8;
constexpr int kMaxCtaPieces = 48;
constexpr int kMaxRestarts = 10;
// auto variant: iterations of one round (pipelined, then classic after the
// first restart) before the true residual is checked and the recurrences
// restart from it
constexpr int kRoundCap = 400;
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
__device__ __forceinline__ void red_add_release_u32(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" : : "l"(p), "r"(v) : "memory");
}

// Grid-wide barrier of a cooperative launch (all CTAs co-resident) on a
// monotonically increasing arrival counter.  Every CTA passes the same
// sequence of barriers and counts them in *round (shared memory, read and
// written by thread 0 only, zero at kernel start), so barrier k is complete
// when the counter reaches k*G: the arrival is a fire-and-forget reduction
// (no round trip for its old value) and the poll starts at once.  Release
// on the arrival and acquire on the poll order every CTA's prior global
// writes before every CTA's later reads.  The wait is bounded: after
// timeout_ns (B200FEM_OPT_BARRIER_TIMEOUT_MS, default kBarrierTimeoutNs)
// the CTA records B200FEM_ERR_TIMEOUT in flags[0] and returns false, and
// every CTA leaves the kernel at its next barrier.  skip_cta >= 0 is the
// failure-detection test's knob: that CTA does not arrive at the first
// barrier (it still waits, bounded like the others), so every wait of that
// barrier runs out.  The counter must be zero when the kernel starts.
__device__ bool grid_barrier(unsigned* count, int* flags, unsigned* round, unsigned long long timeout_ns,
                             int skip_cta) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile int* err = flags;
    const unsigned r = ++*round;
    const unsigned goal = r * gridDim.x;
    if (!(r == 1u && (int)blockIdx.x == skip_cta)) red_add_release_u32(count, 1u);
    int ok = 1;
    const unsigned long long t0 = global_ns();
    while ((int)(ld_acquire_u32(count) - goal) < 0) {
      if (*err != 0) {
        ok = 0;
        break;
      }
      if (global_ns() - t0 > timeout_ns) {
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
  const int* cta_piece;  // CTA c owns entries [cta_piece[c], cta_piece[c+1]) of cta_plist
  const int* cta_plist;  // global piece indices, CTA-major
  double* partials;  // [2][n_pieces][4]
  const double* step;
  double tol_override;  // > 0: the tolerance of every model (refinement corrections)
  double* model_out;  // n_models * 4: iterations, true rel residual, converged
  int resident;       // row-local vectors and Dinv live in shared memory
  int cached;         // the CTA's slice of S (values, columns, row offsets) is copied to shared memory
  int nloc_max;       // max rows of one CTA
  int nb_max;         // max blocks of one CTA
  unsigned* barrier;
  int* flags;
  unsigned long long barrier_timeout_ns;  // bound of every grid-barrier wait
  int skip_arrival_cta;  // test knob: this CTA skips its first arrival (-1: none)
  int* unconv;  // per iteration: some model still unconverged
  int max_iter;
  int variant;  // 0 auto (pipelined, classic after a residual replacement), 1 classic, 2 pipelined
  int row_lanes;  // lanes per block row in the iteration SpMV (4, 8, 16, 32)
  int update_state;
  double* xpos;
  double* vprev;  // receives the velocity before the update
  double* vprev2;  // receives vprev before the update
  double* vprev3;  // receives vprev2 before the update
  double* vprev4;  // receives vprev3 before the update
  double* vel;
  const int* act_node;
  const int* row_model;
  const int* model_active;  // per model: 0 = not solved in this call (or null: all)
  // one model whose rows every CTA holds: every CTA computes the same
  // scalars and takes the same decisions (loop exits, restarts) without
  // agreeing through global memory
  int single_model;
  // plane constraints (ConstrainedBackwardEuler), or null: per row the unit
  // normal (zero for rows without a constraint) and the plane's offset
  const double* row_nrm;
  const double* row_off;
  // the factored NODAL solve matrix (null dil_rptr: S is the whole matrix):
  // per row its (node, divBlk slot) entries, the dilational nodes with their
  // neighbour slots' rows, and t_n of the SpMV in progress
  const int* dil_rptr;
  const int* dil_node;
  const int* dil_slot;
  const int* dil_nodes;
  int n_dil_nodes;
  const int* nbr_ptr;
  const int* nbr_row;
  const double* divblk;
  const double* node_kp;
  const int* node_model;
  double* dil_t;
};

// Plane constraints: the constrained velocities of a row lie on its plane,
// so every residual and SpMV output is projected onto it (y -= n (n . y));
// rows without a constraint have n = 0 and stay as they are.  With the
// projected block-Jacobi inverse P D^-1 P every search direction stays on
// the planes, and the PCG solves the KKT system [S G^T; G 0] for v.
__device__ __forceinline__ void project_row(const double* nrm, int row, double* y) {
  if (!nrm) return;
  const double* q = nrm + 3 * (size_t)row;
  const double d = q[0] * y[0] + q[1] * y[1] + q[2] * y[2];
  y[0] -= q[0] * d;
  y[1] -= q[1] * d;
  y[2] -= q[2] * d;
}

// The rows a CTA owns: its local pieces j = 0..npc-1 (global piece gp[j],
// first global row grow[j]) laid end to end in a local row space
// [0, nloc); local piece j covers local rows [lst0[j], lst0[j+1]).  In the
// contiguous split the pieces are adjacent global row ranges (row = r0 + i);
// in the strided split they are short row ranges of different models,
// spread over the CTAs so that every model's rows are shared by many SMs.
// A view may leave pieces out (those of converged models): its row space
// lays only the remaining pieces end to end (lst), so passes over it cost
// in proportion to the rows still iterating.
struct CtaRows {
  const int* gp;
  const int* lst;   // start of piece j in this view's row space
  const int* lst0;  // start of piece j in the local row space
  const int* grow;
  int npc, nloc;
  // the piece holding view row i: the last j with lst[j] <= i (left-out
  // pieces have zero length and are never returned for a valid row)
  __device__ __forceinline__ int piece(int i) const {
    int lo = 0, hi = npc - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (lst[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    return lo;
  }
  __device__ __forceinline__ int row(int i, int j) const { return grow[j] + (i - lst[j]); }
  __device__ __forceinline__ int local(int i, int j) const { return lst0[j] + (i - lst[j]); }
};

// Butterfly sum of ND values over the warp (every lane gets the sums).  The
// levels are the outer loop, so the ND chains interleave: their shuffles
// are in flight together instead of one chain after another.
template <int ND>
__device__ __forceinline__ void warp_sum(double* sm) {
#pragma unroll
  for (int off = 16; off > 0; off >>= 1)
#pragma unroll
    for (int k = 0; k < ND; k++) sm[k] += __shfl_xor_sync(0xffffffffu, sm[k], off);
}

// Reduce ND per-row values over the view's pieces in a fixed order and write
// partials[buf][piece][k] for every local piece (zero for pieces the view
// leaves out).  Per row (local row i, global row `row`, local piece j) either
// fn(i, row, j, lane, valid, vals) runs on a group of kPassLanes lanes
// (WARP_ROWS: every lane of the warp calls it, `valid` false for a group
// without a row, and the group's first lane holds the row's values) or
// fn(i, row, j, 0, vals) on one thread.
template <int ND, bool WARP_ROWS, typename Fn>
__device__ void cta_row_pass(const PcgArgs& a, const CtaRows& cr, int buf, double (*rowbuf)[3],
                             double (*pacc)[3], Fn fn) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const int npc = cr.npc;
  for (int j = threadIdx.x; j < npc * 3; j += blockDim.x) pacc[j / 3][j % 3] = 0;
  for (int c0 = 0; c0 < cr.nloc; c0 += kRowChunk) {
    const int c1 = min(c0 + kRowChunk, cr.nloc);
    __syncthreads();
    if constexpr (WARP_ROWS) {
      constexpr int G = 32 / kPassLanes;
      for (int base = c0 + warp * G; base < c1; base += nwarps * G) {
        const int ia = base + lane / kPassLanes;
        const bool valid = ia < c1;
        int j = 0, li = 0, row = 0;
        if (valid) {
          j = cr.piece(ia);
          li = cr.local(ia, j);
          row = cr.row(ia, j);
        }
        double vals[3] = {0, 0, 0};
        fn(li, row, j, lane, valid, vals);
        if (valid && (lane & (kPassLanes - 1)) == 0)
#pragma unroll
          for (int k = 0; k < ND; k++) rowbuf[ia - c0][k] = vals[k];
      }
    } else {
      for (int i = c0 + (int)threadIdx.x; i < c1; i += blockDim.x) {
        const int j = cr.piece(i);
        double vals[3] = {0, 0, 0};
        fn(cr.local(i, j), cr.row(i, j), j, 0, vals);
#pragma unroll
        for (int k = 0; k < ND; k++) rowbuf[i - c0][k] = vals[k];
      }
    }
    __syncthreads();
    for (int j = warp; j < npc; j += nwarps) {
      const int pr0 = max(cr.lst[j], c0), pr1 = min(cr.lst[j + 1], c1);
      if (pr0 >= pr1) continue;
      double sm[3] = {0, 0, 0};
      for (int i = pr0 + lane; i < pr1; i += 32)
#pragma unroll
        for (int k = 0; k < ND; k++) sm[k] += rowbuf[i - c0][k];
      warp_sum<ND>(sm);
      if (lane == 0)
#pragma unroll
        for (int k = 0; k < ND; k++) pacc[j][k] += sm[k];
    }
  }
  __syncthreads();
  double* out = a.partials + (size_t)buf * a.n_pieces * 4;
  for (int j = threadIdx.x; j < npc; j += blockDim.x)
#pragma unroll
    for (int k = 0; k < ND; k++) out[(size_t)cr.gp[j] * 4 + k] = pacc[j][k];
}

// One lane's share of a model's partials: the sum over pieces q = q0 + lane,
// q0 + lane + 32, ... < q1 of src[q][0..ND), added in increasing q.  The
// loads of U pieces are issued before their sums, so a lane waits for one
// L2 round trip per U pieces instead of one per piece (U = 5 covers a
// model cut into one piece per SM in a single round trip).
template <int ND, int U = 5>
__device__ __forceinline__ void lane_partials(const double* src, int q0, int q1, int lane, double* sm) {
  for (int qq = q0 + lane; qq < q1; qq += 32 * U) {
    double v[U][ND];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int q = qq + 32 * u;
#pragma unroll
      for (int k = 0; k < ND; k++) v[u][k] = q < q1 ? __ldcg(&src[(size_t)q * 4 + k]) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < U; u++)
#pragma unroll
      for (int k = 0; k < ND; k++) sm[k] += v[u][k];
  }
}

// Per local piece: sum of the partials of its model, whose pieces are
// [q0[j], q1[j]) (warp per piece, fixed lane striding and butterfly order);
// pieces with skip[j] set are left out.
template <int ND>
__device__ void model_sums(const PcgArgs& a, const CtaRows& cr, const int* q0s, const int* q1s, int buf,
                           double (*out)[3], const int* skip) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
  const double* src = a.partials + (size_t)buf * a.n_pieces * 4;
  for (int j = warp; j < cr.npc; j += nwarps) {
    if (skip && skip[j]) continue;
    const int q0 = q0s[j], q1 = q1s[j];
    double sm[3] = {0, 0, 0};
    lane_partials<ND>(src, q0, q1, lane, sm);
    warp_sum<ND>(sm);
    if (lane == 0)
#pragma unroll
      for (int k = 0; k < ND; k++) out[j][k] = sm[k];
  }
  __syncthreads();
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

// Row-local PCG state: the vectors x r u w z q s p and the block-Jacobi
// inverse of the CTA's own rows.  In resident mode they live in shared
// memory for the whole solve (only the owning CTA ever touches them) and
// are indexed by local row; otherwise they are the global vectors indexed by
// global row.  The search-direction vectors read by neighbouring rows (u at
// the start, m in the iteration, x for the true residual) are published to
// global memory.
struct RowState {
  double* v[9];
  double* D;
  int res;
  __device__ __forceinline__ double* at(int k, int i, int row) const {
    return res ? v[k] + 3 * i : v[k] + 3 * (size_t)row;
  }
  __device__ __forceinline__ double* dinv(int i, int row) const {
    return res ? D + 9 * i : D + 9 * (size_t)row;
  }
};
enum { VX = 0, VR, VU, VW, VZ, VQ, VS, VP, VM };

// In the contiguous split a CTA's rows own the contiguous block range
// [pbase, pend): when it fits, the values, block columns and row offsets
// are copied to shared memory once per solve and every SpMV of the solve
// reads them there (indexed by local row).
template <typename MT>
struct MatView {
  const int* rowptr;
  const int* col;
  const MT* S;
  const int* ro_s;
  const int* col_s;
  const MT* S_s;
  int cached;
  // factored NODAL term (dil_rptr null: none): y_row += sum t_n d_n(row)
  const int* dil_rptr;
  const int* dil_node;
  const int* dil_slot;
  const double* divblk;
  const double* dil_t;
};

// The dilational entries e0, e0 + stride, ... < e1 of one row, added to a
// lane's partial sums before the row's shuffle reduction.
template <typename MT>
__device__ __forceinline__ void dil_row_walk(const MatView<MT>& mv, int e0, int e1, int stride, double& a0,
                                             double& a1, double& a2) {
  for (int e = e0; e < e1; e += stride) {
    const double tn = mv.dil_t[mv.dil_node[e]];
    const double* g = mv.divblk + 3 * (size_t)mv.dil_slot[e];
    a0 += tn * g[0];
    a1 += tn * g[1];
    a2 += tn * g[2];
  }
}

// the FP64-value walk of block_row_walk (below)
__device__ __forceinline__ void block_row_walk_f64(const int* col, const double* S, const double* x, int p, int p1,
                                                   int stride, double& a0, double& a1, double& a2) {
  for (; p < p1; p += 2 * stride) {
    const int pb = p + stride;
    const bool hb = pb < p1;
    const int ca = col[p];
    const int cb = hb ? col[pb] : ca;
    const double xa0 = x[3 * (size_t)ca], xa1 = x[3 * (size_t)ca + 1], xa2 = x[3 * (size_t)ca + 2];
    double xb0 = 0, xb1 = 0, xb2 = 0;
    if (hb) {
      xb0 = x[3 * (size_t)cb];
      xb1 = x[3 * (size_t)cb + 1];
      xb2 = x[3 * (size_t)cb + 2];
    }
    {
      const double* b = S + (size_t)p * 9;
      a0 += b[0] * xa0 + b[1] * xa1 + b[2] * xa2;
      a1 += b[3] * xa0 + b[4] * xa1 + b[5] * xa2;
      a2 += b[6] * xa0 + b[7] * xa1 + b[8] * xa2;
    }
    if (hb) {
      const double* b = S + (size_t)pb * 9;
      a0 += b[0] * xb0 + b[1] * xb1 + b[2] * xb2;
      a1 += b[3] * xb0 + b[4] * xb1 + b[5] * xb2;
      a2 += b[6] * xb0 + b[7] * xb1 + b[8] * xb2;
    }
  }
}
__device__ __forceinline__ void block_row_walk_f64(const int*, const float*, const double*, int, int, int, double&,
                                                   double&, double&) {}

// One lane's walk over blocks p, p + stride, ... < p1 of a block row:
// a += S_p x_col(p), blocks added in increasing p.  FP32 values: per step
// of two blocks the column indices and both blocks' values are loaded
// together (the values do not depend on the columns: streamed from HBM they
// overlap the index loads), then the two x gathers, so a lane waits for one
// HBM and one L2 round trip per two blocks; a missing second block reloads
// the first block's values and is not added.  FP64 values (18 more
// registers than the 1024-thread kernel has to spare): the x gathers of the
// two blocks are issued together, then each block's values.
template <typename MT>
__device__ __forceinline__ void block_row_walk(const int* col, const MT* S, const double* x, int p, int p1,
                                               int stride, double& a0, double& a1, double& a2) {
  if constexpr (sizeof(MT) == 8) {
    block_row_walk_f64(col, S, x, p, p1, stride, a0, a1, a2);
    return;
  }
  for (; p < p1; p += 2 * stride) {
    const int pb = p + stride;
    const bool hb = pb < p1;
    const int ca = col[p];
    const int cb = hb ? col[pb] : ca;
    MT ba[9], bb[9];
    {
      const MT* A = S + (size_t)p * 9;
      const MT* B = S + (size_t)(hb ? pb : p) * 9;
#pragma unroll
      for (int k = 0; k < 9; k++) ba[k] = A[k];
#pragma unroll
      for (int k = 0; k < 9; k++) bb[k] = B[k];
    }
    const double xa0 = x[3 * (size_t)ca], xa1 = x[3 * (size_t)ca + 1], xa2 = x[3 * (size_t)ca + 2];
    double xb0 = 0, xb1 = 0, xb2 = 0;
    if (hb) {
      xb0 = x[3 * (size_t)cb];
      xb1 = x[3 * (size_t)cb + 1];
      xb2 = x[3 * (size_t)cb + 2];
    }
    {
      double b[9];
#pragma unroll
      for (int k = 0; k < 9; k++) b[k] = (double)ba[k];
      a0 += b[0] * xa0 + b[1] * xa1 + b[2] * xa2;
      a1 += b[3] * xa0 + b[4] * xa1 + b[5] * xa2;
      a2 += b[6] * xa0 + b[7] * xa1 + b[8] * xa2;
    }
    if (hb) {
      double b[9];
#pragma unroll
      for (int k = 0; k < 9; k++) b[k] = (double)bb[k];
      a0 += b[0] * xb0 + b[1] * xb1 + b[2] * xb2;
      a1 += b[3] * xb0 + b[4] * xb1 + b[5] * xb2;
      a2 += b[6] * xb0 + b[7] * xb1 + b[8] * xb2;
    }
  }
}

// The vectors these SpMVs read (the search direction m, the iterate x) are
// rewritten by other CTAs between grid barriers, so they are read with plain
// coherent loads: no __restrict__/read-only-cache path, which is only valid
// for data that stays unchanged for the whole launch.
template <typename MT>
__device__ __forceinline__ void view_row_spmv(const MatView<MT>& mv, int i, int row, const double* x, int lane,
                                              double* y) {
  int p0, p1;
  const int* col;
  const MT* S;
  if (mv.cached) {
    p0 = mv.ro_s[i];
    p1 = mv.ro_s[i + 1];
    col = mv.col_s;
    S = mv.S_s;
  } else {
    p0 = mv.rowptr[row];
    p1 = mv.rowptr[row + 1];
    col = mv.col;
    S = mv.S;
  }
  double a0 = 0, a1 = 0, a2 = 0;
  block_row_walk<MT>(col, S, x, p0 + lane, p1, 32, a0, a1, a2);
  if (mv.dil_rptr) dil_row_walk(mv, mv.dil_rptr[row] + lane, mv.dil_rptr[row + 1], 32, a0, a1, a2);
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

// Several rows per warp: lanes are split into groups of L (8, 16 or 32);
// each group walks one row's blocks with stride L and reduces with
// shuffles inside the group, so 32/L rows are in flight per warp.  Groups
// whose row is past the end contribute nothing.
template <typename MT, int L>
__device__ __forceinline__ void view_rows_spmv_group(const MatView<MT>& mv, int i, int row, bool valid,
                                                     const double* x, int lane, double* y) {
  int p0 = 0, p1 = 0;
  const int* col;
  const MT* S;
  if (mv.cached) {
    col = mv.col_s;
    S = mv.S_s;
    if (valid) {
      p0 = mv.ro_s[i];
      p1 = mv.ro_s[i + 1];
    }
  } else {
    col = mv.col;
    S = mv.S;
    if (valid) {
      p0 = mv.rowptr[row];
      p1 = mv.rowptr[row + 1];
    }
  }
  const int gl = lane & (L - 1);
  double a0 = 0, a1 = 0, a2 = 0;
  block_row_walk<MT>(col, S, x, p0 + gl, p1, L, a0, a1, a2);
  if (mv.dil_rptr && valid) dil_row_walk(mv, mv.dil_rptr[row] + gl, mv.dil_rptr[row + 1], L, a0, a1, a2);
#pragma unroll
  for (int off = L / 2; off > 0; off >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, off);
    a1 += __shfl_xor_sync(0xffffffffu, a1, off);
    a2 += __shfl_xor_sync(0xffffffffu, a2, off);
  }
  y[0] = a0;
  y[1] = a1;
  y[2] = a2;
}

// n = S x for the rows [c0, c1) of the view `ar` into sn.
template <typename MT, int L>
__device__ __forceinline__ void spmv_rows_to_smem(const MatView<MT>& mv, const CtaRows& ar, const double* x,
                                                  int c0, int c1, int warp, int nroww, int lane,
                                                  double (*sn)[3]) {
  constexpr int G = 32 / L;
  for (int base = c0 + warp * G; base < c1; base += nroww * G) {
    const int ia = base + lane / L;
    const bool valid = ia < c1;
    int row = 0, i = 0;
    if (valid) {
      const int j = ar.piece(ia);
      row = ar.row(ia, j);
      i = ar.local(ia, j);
    }
    double n[3];
    view_rows_spmv_group<MT, L>(mv, i, row, valid, x, lane, n);
    if (valid && (lane & (L - 1)) == 0) {
      sn[ia - c0][0] = n[0];
      sn[ia - c0][1] = n[1];
      sn[ia - c0][2] = n[2];
    }
  }
}

// One pipelined-CG row update fused with the SpMV that feeds it, for the
// rows [c0, c1) of the view: a group of L lanes forms n = S m for its row;
// lanes 0..2 of the group then update the row's vector components
//   z = n + beta z; q = m + beta q; s = w + beta s; p = u + beta p;
//   x += alpha p; r -= alpha s; u -= alpha q; w -= alpha z; m' = Dinv w
// (one component each, w shared by shuffles for m'), and the group's dot
// products r.u, w.u, r.r go to rowbuf[row - c0] (zero for converged rows).
template <typename MT, int L>
__device__ __forceinline__ void fused_rows(const PcgArgs& a, const MatView<MT>& mv, const CtaRows& ar,
                                           const RowState& st, bool res, const double* mc, double* mn, int c0,
                                           int c1, int warp, int nw, int lane, const int* conv,
                                           const double* alpha, const double* beta, double (*rowbuf)[3]) {
  static_assert(L >= 4, "three lanes per row update the vector components");
  constexpr int G = 32 / L;
  const int gl = lane & (L - 1);
  const int g0 = lane & ~(L - 1);
  for (int base = c0 + warp * G; base < c1; base += nw * G) {
    const int ia = base + lane / L;
    const bool valid = ia < c1;
    int row = 0, i = 0, j = 0;
    if (valid) {
      j = ar.piece(ia);
      row = ar.row(ia, j);
      i = ar.local(ia, j);
    }
    double n[3];
    view_rows_spmv_group<MT, L>(mv, i, row, valid, mc, lane, n);
    if (valid) project_row(a.row_nrm, row, n);
    const bool upd = valid && !conv[j] && gl < 3;
    double wc = 0, ru = 0, wu = 0, rr = 0;
    if (upd) {
      const int c = gl;
      const double al = alpha[j], be = beta[j];
      double* px = st.at(VX, i, row) + c;
      double* pr = st.at(VR, i, row) + c;
      double* pu = st.at(VU, i, row) + c;
      double* pw = st.at(VW, i, row) + c;
      double* pz = st.at(VZ, i, row) + c;
      double* pq = st.at(VQ, i, row) + c;
      double* ps = st.at(VS, i, row) + c;
      double* pp = st.at(VP, i, row) + c;
      const double mm = res ? st.at(VM, i, row)[c] : mc[3 * (size_t)row + c];
      const double nc = c == 0 ? n[0] : (c == 1 ? n[1] : n[2]);
      const double z = nc + be * *pz;
      const double q = mm + be * *pq;
      const double sv = *pw + be * *ps;
      const double p = *pu + be * *pp;
      *px += al * p;
      const double r = *pr - al * sv;
      const double u = *pu - al * q;
      const double w = *pw - al * z;
      *pz = z;
      *pq = q;
      *ps = sv;
      *pp = p;
      *pr = r;
      *pu = u;
      *pw = w;
      wc = w;
      ru = r * u;
      wu = w * u;
      rr = r * r;
    }
    const double w0 = __shfl_sync(0xffffffffu, wc, g0);
    const double w1 = __shfl_sync(0xffffffffu, wc, g0 + 1);
    const double w2 = __shfl_sync(0xffffffffu, wc, g0 + 2);
    if (upd) {
      const int c = gl;
      const double* D = st.dinv(i, row) + 3 * c;
      const double mnew = D[0] * w0 + D[1] * w1 + D[2] * w2;
      mn[3 * (size_t)row + c] = mnew;
      if (res) st.at(VM, i, row)[c] = mnew;
    }
#pragma unroll
    for (int off = 2; off > 0; off >>= 1) {
      ru += __shfl_xor_sync(0xffffffffu, ru, off);
      wu += __shfl_xor_sync(0xffffffffu, wu, off);
      rr += __shfl_xor_sync(0xffffffffu, rr, off);
    }
    if (valid && gl == 0) {
      rowbuf[ia - c0][0] = ru;
      rowbuf[ia - c0][1] = wu;
      rowbuf[ia - c0][2] = rr;
    }
  }
}

// Warp 0 only: lay the rows of the pieces whose flag is clear end to end
// (prefix sum over at most 64 pieces, two per lane).  The caller orders the
// flag writes before this call and this call before any read of alst with
// __syncthreads.
static_assert(kMaxCtaPieces <= 64, "active_scan covers two pieces per lane");
__device__ __forceinline__ void active_scan(int npc, int lane, const int* flag, const int* lst, int* alst) {
  const int j0 = 2 * lane, j1 = 2 * lane + 1;
  const int c0 = (j0 < npc && !flag[j0]) ? lst[j0 + 1] - lst[j0] : 0;
  const int c1 = (j1 < npc && !flag[j1]) ? lst[j1 + 1] - lst[j1] : 0;
  int incl = c0 + c1;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, off);
    if (lane >= off) incl += t;
  }
  const int excl = incl - c0 - c1;
  if (j0 < npc) alst[j0] = excl;
  if (j1 < npc) alst[j1] = excl + c0;
  if (lane == 31) alst[npc] = incl;
}

// dynamic shared memory layout of the PCG kernel
__host__ __device__ inline size_t pcg_align16(size_t b) { return (b + 15) & ~(size_t)15; }
template <typename MT>
__host__ __device__ inline void pcg_smem_layout(int nloc_max, int nb_max, int res, int cached, size_t* off_vec,
                                                size_t* off_ro, size_t* off_col, size_t* off_S, size_t* total) {
  size_t o = 0;
  *off_vec = o;
  if (res) o += pcg_align16(sizeof(double) * (size_t)nloc_max * (9 * 3 + 9));
  *off_ro = o;
  if (cached) o += pcg_align16(sizeof(int) * (size_t)(nloc_max + 1));
  *off_col = o;
  if (cached) o += pcg_align16(sizeof(int) * (size_t)nb_max);
  *off_S = o;
  if (cached) o += pcg_align16(sizeof(MT) * (size_t)nb_max * 9);
  *total = o;
}

// RES: compiled for shared-memory resident row state (the contiguous split
// of packs that fit); otherwise residency is the runtime flag (zero in the
// strided split), which keeps the register pressure of each form low.
// Factored NODAL solve matrix: t_n = (h^2 + h beta) kp_n (d_n . v) of every
// dilational node.  A group of kDilLanes lanes takes one node, its lanes
// the node's neighbour slots with that stride (so a node costs one round of
// independent loads instead of a chain over its ~15 slots), then a
// shuffle reduction; the nodes are dealt over all warps of the launch.  v
// is a published vector; a grid barrier follows before any row reads t.
constexpr int kDilLanes = 8;
__device__ __forceinline__ void dil_phase(const PcgArgs& a, const double* v) {
  constexpr int G = kDilLanes, per_warp = 32 / G;
  const int lane = threadIdx.x & 31, gl = lane & (G - 1);
  const int gwarp = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
  // warp-uniform loop: every lane of the warp takes part in the shuffles
  for (int base = gwarp * per_warp; base < a.n_dil_nodes; base += nwarps * per_warp) {
    const int k = base + lane / G;
    const bool valid = k < a.n_dil_nodes;
    int n = 0;
    double s = 0;
    if (valid) {
      n = a.dil_nodes[k];
      const int q1 = a.nbr_ptr[n + 1];
      for (int q = a.nbr_ptr[n] + gl; q < q1; q += G) {
        const int r = a.nbr_row[q];
        if (r < 0) continue;
        const double* g = a.divblk + 3 * (size_t)q;
        const double* x = v + 3 * (size_t)r;
        s += g[0] * x[0] + g[1] * x[1] + g[2] * x[2];
      }
    }
#pragma unroll
    for (int off = G / 2; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (valid && gl == 0) {
      const double* sp = a.step + (size_t)a.node_model[n] * 8;
      a.dil_t[n] = (sp[0] * sp[0] + sp[0] * sp[2]) * a.node_kp[n] * s;
    }
  }
}

// DIL: the factored NODAL solve matrix (a separate instantiation, so the
// 64-register form of the plain matrix keeps its registers)
template <typename MT, bool RES, bool DIL = false>
__global__ void __launch_bounds__(pcg_block(RES)) pcg_kernel(PcgArgs a) {
  __shared__ double rowbuf[kRowChunk][3];
  __shared__ double sn[kRowChunk][3];
  __shared__ double pacc[kMaxCtaPieces][3];
  __shared__ double sums[kMaxCtaPieces][3];
  // s_thr: the pipelined test's bound tol * ||b||, fixed for the solve
  __shared__ double s_thr[kMaxCtaPieces];
  __shared__ double s_bb[kMaxCtaPieces], s_tol[kMaxCtaPieces], s_alpha[kMaxCtaPieces],
      s_beta[kMaxCtaPieces], s_gold[kMaxCtaPieces], s_aold[kMaxCtaPieces];
  __shared__ int s_conv[kMaxCtaPieces], s_iters[kMaxCtaPieces], s_first[kMaxCtaPieces];
  // the model's solve is final (its true residual was checked and it was
  // not restarted): later passes leave its rows alone
  __shared__ int s_done[kMaxCtaPieces];
  __shared__ int s_gp[kMaxCtaPieces], s_lst[kMaxCtaPieces + 1], s_grow[kMaxCtaPieces];
  // the pieces [s_q0, s_q1) of each local piece's model (global piece numbers;
  // read here once instead of from global memory in every reduction)
  __shared__ int s_q0[kMaxCtaPieces], s_q1[kMaxCtaPieces];
  // row space of the pieces still iterating (see active_scan)
  __shared__ int s_alst[kMaxCtaPieces + 1];
  __shared__ int s_restart;
  __shared__ int s_unc[2];  // see the pipelined iteration
  // a model's convergence flag changed in this pipelined iteration: the
  // active view is laid out again at its end (otherwise it stays as it is)
  __shared__ int s_conv_dirty;
  if (threadIdx.x == 0) s_conv_dirty = 0;
  extern __shared__ __align__(16) unsigned char dyn[];
  const bool res = RES || a.resident;
  const int pc0 = a.cta_piece[blockIdx.x];
  const int npc = a.cta_piece[blockIdx.x + 1] - pc0;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int ph = 0;
  __shared__ unsigned s_bar_round;  // grid barriers passed (see grid_barrier)
  if (threadIdx.x == 0) s_bar_round = 0;

  for (int j = threadIdx.x; j < npc; j += blockDim.x) {
    const int g = a.cta_plist[pc0 + j];
    s_gp[j] = g;
    s_grow[j] = a.piece_row[g];
    const int m = a.piece_model[g];
    s_q0[j] = a.model_piece[m];
    s_q1[j] = a.model_piece[m + 1];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int acc = 0;
    for (int j = 0; j < npc; j++) {
      s_lst[j] = acc;
      acc += a.piece_row[s_gp[j] + 1] - s_grow[j];
    }
    s_lst[npc] = acc;
  }
  __syncthreads();
  const CtaRows cr{s_gp, s_lst, s_lst, s_grow, npc, s_lst[npc]};  // all local rows
  const int nloc = cr.nloc;
  // the rows of the pieces whose flag is clear, after rescan(flag)
  auto active_view = [&]() { return CtaRows{s_gp, s_alst, s_lst, s_grow, npc, s_alst[npc]}; };
  auto rescan = [&](const int* flag) {
    __syncthreads();  // the flag writes of every thread come first
    if (warp == 0) active_scan(npc, lane, flag, s_lst, s_alst);
    __syncthreads();
  };
  // the last piece of a model owns the model's flags and outputs
  auto owner = [&](int j) { return s_gp[j] == s_q1[j] - 1; };

  size_t off_vec, off_ro, off_col, off_S, total;
  pcg_smem_layout<MT>(a.nloc_max, a.nb_max, res, a.cached, &off_vec, &off_ro, &off_col, &off_S, &total);
  RowState st;
  st.res = res;
  if (res) {
    double* base = (double*)(dyn + off_vec);
    for (int k = 0; k < 9; k++) st.v[k] = base + (size_t)k * a.nloc_max * 3;
    st.D = base + (size_t)9 * a.nloc_max * 3;
  } else {
    st.v[VX] = a.x; st.v[VR] = a.r; st.v[VU] = a.u; st.v[VW] = a.w;
    st.v[VZ] = a.z; st.v[VQ] = a.q; st.v[VS] = a.s; st.v[VP] = a.p;
    st.v[VM] = nullptr;  // m is read from the published buffer
    st.D = a.Dinv;
  }
  MatView<MT> mv;
  mv.rowptr = a.rowptr;
  mv.col = a.col;
  mv.S = (const MT*)a.S;
  mv.cached = a.cached;
  mv.ro_s = (const int*)(dyn + off_ro);
  mv.col_s = (const int*)(dyn + off_col);
  mv.S_s = (const MT*)(dyn + off_S);
  mv.dil_rptr = DIL ? a.dil_rptr : nullptr;
  mv.dil_node = DIL ? a.dil_node : nullptr;
  mv.dil_slot = DIL ? a.dil_slot : nullptr;
  mv.divblk = DIL ? a.divblk : nullptr;
  mv.dil_t = DIL ? a.dil_t : nullptr;
  // every CTA takes the factored term's extra phase and grid barrier before
  // each SpMV alike (the same instantiation for the whole launch)
  constexpr bool dil = DIL;
  // residency and caching are planned only for the contiguous split, where
  // local row i is global row r0 + i
  const int r0 = npc > 0 ? s_grow[0] : 0;
  const int pbase = a.rowptr[r0];
  if (a.cached) {
    const int nb = a.rowptr[r0 + nloc] - pbase;
    int* ro = (int*)(dyn + off_ro);
    int* cs = (int*)(dyn + off_col);
    MT* Ss = (MT*)(dyn + off_S);
    for (int i = threadIdx.x; i <= nloc; i += blockDim.x) ro[i] = a.rowptr[r0 + i] - pbase;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) cs[i] = a.col[pbase + i];
    const MT* Sg = (const MT*)a.S + (size_t)pbase * 9;
    // resident form: eight loads in flight per thread before their stores
    // (the 64-register form copies one value at a time)
    const int nv = nb * 9, stride = blockDim.x;
    constexpr int U = RES ? 8 : 1;
    for (int i0 = threadIdx.x; i0 < nv; i0 += U * stride) {
      MT v[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u * stride;
        v[u] = i < nv ? Sg[i] : MT(0);
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int i = i0 + u * stride;
        if (i < nv) Ss[i] = v[u];
      }
    }
  }
  // the per-iteration flags are cleared two iterations ahead of their use
  // (iteration idx clears idx + 2, ordered before any write to it by the
  // barriers of iterations idx and idx + 1); the first two and the restart
  // slot here, before the first barrier
  if (blockIdx.x == 0 && threadIdx.x < 3) a.unconv[threadIdx.x < 2 ? threadIdx.x : a.max_iter + 1] = 0;
  // models left out of this call are final from the start
  for (int j = threadIdx.x; j < npc; j += blockDim.x) {
    const int m = a.piece_model[s_gp[j]];
    const int off = a.model_active && !a.model_active[m];
    s_tol[j] = a.tol_override > 0 ? a.tol_override : a.step[(size_t)m * 8 + 6];
    s_conv[j] = off;
    s_done[j] = off;
    s_iters[j] = 0;
    s_bb[j] = 0;
    if (off && owner(j)) {
      double* o = a.model_out + (size_t)m * 4;
      o[0] = 0;
      o[1] = 0;
      o[2] = 1.0;
    }
  }
  rescan(s_done);
  if (dil) {
    dil_phase(a, a.x);
    if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
  }

  // ---- P0: block-Jacobi inverse, r = b - S x0, u = Dinv r (published to
  // m1 for the next SpMV), ||b||^2
  cta_row_pass<1, true>(a, active_view(), ph & 1, rowbuf, pacc,
                        [&](int i, int row, int, int ln, bool valid, double* vals) {
    double Ax[3];
    view_rows_spmv_group<MT, kPassLanes>(mv, i, row, valid, a.x, ln, Ax);
    if (valid && (ln & (kPassLanes - 1)) == 0) {
      const MT* Db = (const MT*)a.S + (size_t)a.blk_diag[row] * 9;
      if (a.cached) Db = mv.S_s + (size_t)(a.blk_diag[row] - pbase) * 9;
      double d[9], inv[9];
#pragma unroll
      for (int k = 0; k < 9; k++) d[k] = (double)Db[k];
      if (dil) {
        // the dilational term's diagonal block: sum_n c kp_n d_n(row) d_n(row)^T
        const double* sp = a.step + (size_t)a.row_model[row] * 8;
        const double cm = sp[0] * sp[0] + sp[0] * sp[2];
        for (int e = a.dil_rptr[row]; e < a.dil_rptr[row + 1]; e++) {
          const double* g = a.divblk + 3 * (size_t)a.dil_slot[e];
          const double ck = cm * a.node_kp[a.dil_node[e]];
#pragma unroll
          for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) d[3 * r + c] += ck * g[r] * g[c];
        }
      }
      if (invert3(inv, d) == 0.0) {
        atomicExch(a.flags, B200FEM_ERR_INVALID_ARG);
#pragma unroll
        for (int k = 0; k < 9; k++) inv[k] = 0;
      }
      if (a.row_nrm) {
        // P D^-1 P with P = I - n n^T
        const double* q = a.row_nrm + 3 * (size_t)row;
        double t[9];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++)
            t[3 * r + c] = inv[3 * r + c] - q[r] * (q[0] * inv[c] + q[1] * inv[3 + c] + q[2] * inv[6 + c]);
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++)
            inv[3 * r + c] = t[3 * r + c] - (t[3 * r] * q[0] + t[3 * r + 1] * q[1] + t[3 * r + 2] * q[2]) * q[c];
      }
      double* D = st.dinv(i, row);
#pragma unroll
      for (int k = 0; k < 9; k++) D[k] = inv[k];
      double bv[3], r[3], u[3], x0[3];
      load3(bv, a.b, row);
      load3(x0, a.x, row);
#pragma unroll
      for (int c = 0; c < 3; c++) r[c] = bv[c] - Ax[c];
      project_row(a.row_nrm, row, r);
      project_row(a.row_nrm, row, bv);
      mul33(u, inv, r);
      store3(st.at(VR, i, row), 0, r);
      store3(st.at(VU, i, row), 0, u);
      if (res) store3(st.at(VX, i, row), 0, x0);
      store3(a.m1, row, u);
      vals[0] = dot3(bv, bv);
    }
  });
  if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
  model_sums<1>(a, cr, s_q0, s_q1, ph & 1, sums, s_done);
  for (int j = threadIdx.x; j < npc; j += blockDim.x)
    if (!s_done[j]) {
      s_bb[j] = sums[j][0];
      s_thr[j] = s_tol[j] * sqrt(s_bb[j]);
    }
  ph++;

  int total_it = 0;
  bool classic = a.variant == 1;
  for (int restart = 0;; restart++) {
    if (classic) {
      // ---- classic PCG (two grid barriers per iteration), from the state
      // P0 or the true-residual pass left: r, z = Dinv r (resident) and z
      // published in m1.  rho = r.z, ||r||^2 first.
      rescan(s_conv);
      cta_row_pass<2, false>(a, active_view(), ph & 1, rowbuf, pacc, [&](int i, int row, int j, int, double* vals) {
        if (s_conv[j]) return;
        double r[3], z[3], zero[3] = {0, 0, 0};
        load3(r, st.at(VR, i, row), 0);
        load3(z, st.at(VU, i, row), 0);
        store3(st.at(VP, i, row), 0, zero);
        store3(st.at(VQ, i, row), 0, zero);
        vals[0] = dot3(r, z);
        vals[1] = dot3(r, r);
      });
      if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
      model_sums<2>(a, cr, s_q0, s_q1, ph & 1, sums, s_conv);
      ph++;
      for (int j = threadIdx.x; j < npc; j += blockDim.x) {
        if (s_conv[j]) continue;
        s_gold[j] = sums[j][0];  // rho
        if (sqrt(sums[j][1]) <= s_tol[j] * sqrt(s_bb[j]) || sums[j][1] == 0.0) s_conv[j] = 1;
        s_first[j] = 1;
      }
      rescan(s_conv);
      for (int it = 0;; it++) {
        const int idx = total_it + it;
        if (blockIdx.x == 0 && threadIdx.x == 0 && idx + 2 <= a.max_iter) a.unconv[idx + 2] = 0;
        // phase A: p = z + beta p; q = S z + beta q (z complete); p.q
        for (int j = threadIdx.x; j < npc; j += blockDim.x) {
          if (s_conv[j]) continue;
          s_beta[j] = s_first[j] ? 0.0 : s_gold[j] / s_aold[j];
          s_first[j] = 0;
          if (owner(j)) a.unconv[idx] = 1;
        }
        __syncthreads();
        if (idx >= a.max_iter || (a.variant == 0 && it >= kRoundCap)) {
          total_it += it;
          break;
        }
        if (dil) {
          dil_phase(a, a.m1);
          if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
        }
        cta_row_pass<1, true>(a, active_view(), ph & 1, rowbuf, pacc,
                              [&](int i, int row, int j, int ln, bool valid, double* vals) {
          const bool act = valid && !s_conv[j];
          double Az[3];
          view_rows_spmv_group<MT, kPassLanes>(mv, i, row, act, a.m1, ln, Az);
          if (act && (ln & (kPassLanes - 1)) == 0) {
            project_row(a.row_nrm, row, Az);
            const double be = s_beta[j];
            double* pz = st.at(VU, i, row);
            double* pp = st.at(VP, i, row);
            double* pq = st.at(VQ, i, row);
            double pqv = 0;
#pragma unroll
            for (int c = 0; c < 3; c++) {
              pp[c] = pz[c] + be * pp[c];
              pq[c] = Az[c] + be * pq[c];
              pqv += pp[c] * pq[c];
            }
            vals[0] = pqv;
          }
        });
        if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
        if (__ldcg(&a.unconv[idx]) == 0) {
          total_it += it;
          break;
        }
        model_sums<1>(a, cr, s_q0, s_q1, ph & 1, sums, s_conv);
        ph++;
        for (int j = threadIdx.x; j < npc; j += blockDim.x)
          s_alpha[j] = s_conv[j] ? 0.0 : s_gold[j] / sums[j][0];
        __syncthreads();
        // phase B: x += alpha p; r -= alpha q; z = Dinv r (published); r.z, r.r
        cta_row_pass<2, false>(a, active_view(), ph & 1, rowbuf, pacc, [&](int i, int row, int j, int, double* vals) {
          if (s_conv[j]) return;
          const double al = s_alpha[j];
          double* px = st.at(VX, i, row);
          double* pr = st.at(VR, i, row);
          double* pz = st.at(VU, i, row);
          const double* pp = st.at(VP, i, row);
          const double* pq = st.at(VQ, i, row);
          double r[3], z[3];
#pragma unroll
          for (int c = 0; c < 3; c++) {
            px[c] += al * pp[c];
            r[c] = pr[c] - al * pq[c];
            pr[c] = r[c];
          }
          mul33(z, st.dinv(i, row), r);
          store3(pz, 0, z);
          store3(a.m1, row, z);
          vals[0] = dot3(r, z);
          vals[1] = dot3(r, r);
        });
        if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
        model_sums<2>(a, cr, s_q0, s_q1, ph & 1, sums, s_conv);
        ph++;
        for (int j = threadIdx.x; j < npc; j += blockDim.x) {
          if (s_conv[j]) continue;
          s_aold[j] = s_gold[j];  // rho of the previous iteration
          s_gold[j] = sums[j][0];
          s_iters[j]++;
          if (sqrt(sums[j][1]) <= s_tol[j] * sqrt(s_bb[j]) || sums[j][1] == 0.0) s_conv[j] = 1;
        }
        rescan(s_conv);
      }
    } else {
    // ---- P1: w = S u, m = Dinv w (published to m0); dots r.u, w.u, r.r
    for (int j = threadIdx.x; j < npc; j += blockDim.x) s_first[j] = 1;
    rescan(s_conv);
    if (dil) {
      dil_phase(a, a.m1);
      if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
    }
    cta_row_pass<3, true>(a, active_view(), ph & 1, rowbuf, pacc,
                          [&](int i, int row, int j, int ln, bool valid, double* vals) {
      const bool act = valid && !s_conv[j];
      double Au[3];
      view_rows_spmv_group<MT, kPassLanes>(mv, i, row, act, a.m1, ln, Au);
      if (act && (ln & (kPassLanes - 1)) == 0) {
        project_row(a.row_nrm, row, Au);
        double r[3], u[3], m[3], zero[3] = {0, 0, 0};
        load3(r, st.at(VR, i, row), 0);
        load3(u, st.at(VU, i, row), 0);
        mul33(m, st.dinv(i, row), Au);
        store3(st.at(VW, i, row), 0, Au);
        store3(a.m0, row, m);
        if (res) store3(st.at(VM, i, row), 0, m);
        store3(st.at(VZ, i, row), 0, zero);
        store3(st.at(VQ, i, row), 0, zero);
        store3(st.at(VS, i, row), 0, zero);
        store3(st.at(VP, i, row), 0, zero);
        vals[0] = dot3(r, u);
        vals[1] = dot3(Au, u);
        vals[2] = dot3(r, r);
      }
    });
    if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
    int mbuf = 0;  // m0 holds the current m

    for (int it = 0;; it++) {
      const int idx = total_it + it;
      if (blockIdx.x == 0 && threadIdx.x == 0 && idx + 2 <= a.max_iter) a.unconv[idx + 2] = 0;
      const double* mc = mbuf ? a.m1 : a.m0;
      double* mn = mbuf ? a.m0 : a.m1;
      if (dil) {
        dil_phase(a, mc);
        if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
      }
      // The SpMV n = S m does not depend on this iteration's scalars, so it
      // runs on the first warps while the last warps reduce the scalars.
      // Both work on the rows of the models unconverged when the iteration
      // began (the view laid out at the end of the previous iteration).
      const int nsumw = min(max(npc, 1), 8);
      const int nroww = (blockDim.x >> 5) - nsumw;
      for (int j = threadIdx.x; j < npc * 3; j += blockDim.x) pacc[j / 3][j % 3] = 0;
      bool stop = false, conv_exit = false;
      const CtaRows ar = active_view();
      const int nact = ar.nloc;
      for (int c0 = 0, first = 1; c0 < nact || first; c0 += kRowChunk, first = 0) {
        const int c1 = min(c0 + kRowChunk, nact);
        if (first) {
          if (warp < nroww) {
            if (a.row_lanes == 4) spmv_rows_to_smem<MT, 4>(mv, ar, mc, c0, c1, warp, nroww, lane, sn);
            else if (a.row_lanes == 8) spmv_rows_to_smem<MT, 8>(mv, ar, mc, c0, c1, warp, nroww, lane, sn);
            else if (a.row_lanes == 16) spmv_rows_to_smem<MT, 16>(mv, ar, mc, c0, c1, warp, nroww, lane, sn);
            else spmv_rows_to_smem<MT, 32>(mv, ar, mc, c0, c1, warp, nroww, lane, sn);
          } else if (first) {
            // reduce this iteration's scalars and form alpha, beta; the
            // convergence test is on the recurrence residual
            const int sw = warp - nroww;
            const double* src = a.partials + (size_t)(ph & 1) * a.n_pieces * 4;
            // unconv[idx - 1] is final (its barrier has passed); it is
            // loaded here, next to the partials, and tested after this
            // iteration's barrier instead of costing a round trip after
            // every barrier.  Two slots: the next write to this one comes
            // after the next barrier's __syncthreads.
            const int unc = (sw == 0 && lane == 0 && it > 0) ? __ldcg(&a.unconv[idx - 1]) : 1;
            for (int j = sw; j < npc; j += nsumw) {
              if (s_conv[j]) continue;
              const int q0 = s_q0[j], q1 = s_q1[j];
              // the reciprocals of the previous gamma and alpha do not
              // depend on the partials: they are formed while the loads are
              // in flight, which leaves one division after the sums
              const double rg = 1.0 / s_gold[j], ra = 1.0 / s_aold[j];
              double sm[3] = {0, 0, 0};
              lane_partials<3>(src, q0, q1, lane, sm);
              warp_sum<3>(sm);
              if (lane == 0) {
                const double gam = sm[0], del = sm[1], rho = sm[2];
                if (sqrt(rho) <= s_thr[j] || rho == 0.0) {
                  s_conv[j] = 1;
                  s_conv_dirty = 1;
                } else {
                  double beta = 0, alpha;
                  if (s_first[j]) {
                    alpha = gam / del;
                    s_first[j] = 0;
                  } else {
                    beta = gam * rg;
                    alpha = gam / (del - beta * gam * ra);
                  }
                  s_beta[j] = beta;
                  s_alpha[j] = alpha;
                  s_gold[j] = gam;
                  s_aold[j] = alpha;
                  s_iters[j]++;
                  if (owner(j)) a.unconv[idx] = 1;
                }
              }
            }
            if (sw == 0 && lane == 0) s_unc[it & 1] = unc;
          }
          __syncthreads();
          if (first && (idx >= a.max_iter || (a.variant == 0 && it >= kRoundCap))) {
            stop = true;
            break;
          }
          if (first && a.single_model && s_conv[0]) {
            // the model met the recurrence test at this iteration: the
            // iterate is final, and every CTA leaves here alike
            conv_exit = true;
            break;
          }
          // z = n + beta z; q = m + beta q; s = w + beta s; p = u + beta p;
          // x += alpha p; r -= alpha s; u -= alpha q; w -= alpha z; m' = Dinv w
          // (resident form, one piece: each thread sums its rows' dot-product
          // terms, each warp reduces them and the per-warp sums go to
          // rowbuf[warp]; the 64-register strided form keeps rowbuf rows)
          const bool regsum = RES && npc == 1;
          double acc3[3] = {0, 0, 0};
          for (int ia = c0 + (int)threadIdx.x; ia < c1; ia += blockDim.x) {
            const int j = ar.piece(ia);
            double v3[3] = {0, 0, 0};
            if (!s_conv[j]) {
              const int i = ar.local(ia, j);
              const int row = ar.row(ia, j);
              const double al = s_alpha[j], be = s_beta[j];
              double* px = st.at(VX, i, row);
              double* pr = st.at(VR, i, row);
              double* pu = st.at(VU, i, row);
              double* pw = st.at(VW, i, row);
              double* pz = st.at(VZ, i, row);
              double* pq = st.at(VQ, i, row);
              double* ps = st.at(VS, i, row);
              double* pp = st.at(VP, i, row);
              const double* D = st.dinv(i, row);
              double mm[3], w[3], r[3], u[3];
              if (res) load3(mm, st.at(VM, i, row), 0);
              else load3(mm, mc, row);
              double nn[3] = {sn[ia - c0][0], sn[ia - c0][1], sn[ia - c0][2]};
              project_row(a.row_nrm, row, nn);
#pragma unroll
              for (int c = 0; c < 3; c++) {
                const double z = nn[c] + be * pz[c];
                const double q = mm[c] + be * pq[c];
                const double sv = pw[c] + be * ps[c];
                const double p = pu[c] + be * pp[c];
                px[c] += al * p;
                r[c] = pr[c] - al * sv;
                u[c] = pu[c] - al * q;
                w[c] = pw[c] - al * z;
                pz[c] = z;
                pq[c] = q;
                ps[c] = sv;
                pp[c] = p;
                pr[c] = r[c];
                pu[c] = u[c];
                pw[c] = w[c];
              }
              double mnew[3];
              mul33(mnew, D, w);
              store3(mn, row, mnew);
              if (res) store3(st.at(VM, i, row), 0, mnew);
              v3[0] = dot3(r, u);
              v3[1] = dot3(w, u);
              v3[2] = dot3(r, r);
            }
            if (regsum) {
#pragma unroll
              for (int k = 0; k < 3; k++) acc3[k] += v3[k];
            } else {
              rowbuf[ia - c0][0] = v3[0];
              rowbuf[ia - c0][1] = v3[1];
              rowbuf[ia - c0][2] = v3[2];
            }
          }
          if (regsum) {
            warp_sum<3>(acc3);
            if (lane == 0)
#pragma unroll
              for (int k = 0; k < 3; k++) rowbuf[warp][k] = acc3[k];
          }
        } else {
          // later chunks: all warps, SpMV and update fused per row
          const int nw = blockDim.x >> 5;
          if (a.row_lanes == 4) fused_rows<MT, 4>(a, mv, ar, st, res, mc, mn, c0, c1, warp, nw, lane, s_conv, s_alpha, s_beta, rowbuf);
          else if (a.row_lanes == 8) fused_rows<MT, 8>(a, mv, ar, st, res, mc, mn, c0, c1, warp, nw, lane, s_conv, s_alpha, s_beta, rowbuf);
          else if (a.row_lanes == 16) fused_rows<MT, 16>(a, mv, ar, st, res, mc, mn, c0, c1, warp, nw, lane, s_conv, s_alpha, s_beta, rowbuf);
          else fused_rows<MT, 32>(a, mv, ar, st, res, mc, mn, c0, c1, warp, nw, lane, s_conv, s_alpha, s_beta, rowbuf);
        }
        __syncthreads();
        if (RES && npc == 1 && first) {
          // one piece: the per-warp sums in warp order
          if (threadIdx.x == 0) {
            const int nw = blockDim.x >> 5;
            for (int w = 0; w < nw; w++)
#pragma unroll
              for (int k = 0; k < 3; k++) pacc[0][k] += rowbuf[w][k];
          }
          continue;
        }
        if (npc == 1 && c1 - c0 <= 32) {
          // one piece, one warp of rows: reduce in warp 0 without a second pass
          if (warp == 0) {
            double sm[3] = {0, 0, 0};
            if (c0 + lane < c1)
#pragma unroll
              for (int k = 0; k < 3; k++) sm[k] = rowbuf[lane][k];
            warp_sum<3>(sm);
            if (lane == 0)
#pragma unroll
              for (int k = 0; k < 3; k++) pacc[0][k] += sm[k];
          }
          continue;
        }
        for (int j = warp; j < npc; j += (blockDim.x >> 5)) {
          const int pr0 = max(s_alst[j], c0), pr1 = min(s_alst[j + 1], c1);
          if (pr0 >= pr1 || s_conv[j]) continue;
          double sm[3] = {0, 0, 0};
          for (int i = pr0 + lane; i < pr1; i += 32)
#pragma unroll
            for (int k = 0; k < 3; k++) sm[k] += rowbuf[i - c0][k];
          warp_sum<3>(sm);
          if (lane == 0)
#pragma unroll
            for (int k = 0; k < 3; k++) pacc[j][k] += sm[k];
        }
        __syncthreads();
      }
      if (stop || conv_exit) {
        total_it += it;
        break;
      }
      ph++;
      {
        double* out = a.partials + (size_t)(ph & 1) * a.n_pieces * 4;
        for (int j = threadIdx.x; j < npc; j += blockDim.x)
#pragma unroll
          for (int k = 0; k < 3; k++) out[(size_t)s_gp[j] * 4 + k] = pacc[j][k];
      }
      // the next iteration works on the models still unconverged; the
      // resident form lays the view out again only when a flag changed
      // (every thread read s_conv_dirty after the first chunk's barrier; it
      // is cleared after the rescan's closing barrier)
      if (!RES || s_conv_dirty) {
        rescan(s_conv);
        if (threadIdx.x == 0) s_conv_dirty = 0;
      }
      if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
      mbuf ^= 1;
      // every model still iterating at idx - 1 converged there: iteration
      // idx had no rows to work on and is not counted
      if (s_unc[it & 1] == 0) {
        total_it += it - 1;
        break;
      }
    }
    ph++;
    }  // pipelined

    // ---- publish x, then the true residual r = b - S x of the models not
    // yet final; restart from it when it misses the tolerance
    if (res)
      for (int i = threadIdx.x; i < nloc; i += blockDim.x) store3(a.x, r0 + i, st.at(VX, i, r0 + i));
    rescan(s_done);
    if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
    if (dil) {
      dil_phase(a, a.x);
      if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
    }
    cta_row_pass<1, true>(a, active_view(), ph & 1, rowbuf, pacc,
                          [&](int i, int row, int, int ln, bool valid, double* vals) {
      double Ax[3];
      view_rows_spmv_group<MT, kPassLanes>(mv, i, row, valid, a.x, ln, Ax);
      if (valid && (ln & (kPassLanes - 1)) == 0) {
        double bv[3], r[3];
        load3(bv, a.b, row);
#pragma unroll
        for (int c = 0; c < 3; c++) r[c] = bv[c] - Ax[c];
        project_row(a.row_nrm, row, r);
        vals[0] = dot3(r, r);
        // restart state (used only if the model restarts)
        double u[3];
        mul33(u, st.dinv(i, row), r);
        store3(st.at(VR, i, row), 0, r);
        store3(st.at(VU, i, row), 0, u);
        store3(a.m1, row, u);
      }
    });
    if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
    model_sums<1>(a, cr, s_q0, s_q1, ph & 1, sums, s_done);
    ph++;
    if (threadIdx.x == 0) s_restart = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < npc; j += blockDim.x) {
      if (s_done[j]) continue;
      const double rel = s_bb[j] > 0 ? sqrt(sums[j][0] / s_bb[j]) : sqrt(sums[j][0]);
      const bool ok = rel <= s_tol[j] || sums[j][0] == 0.0;
      // the true residual decides: a model whose true residual meets the
      // tolerance is done.  Otherwise residual replacement when the
      // recurrence converged; in auto mode also when the round hit its cap
      // unconverged (classic PCG continues from the true residual)
      const bool capped = !s_conv[j] && a.variant == 0;
      const bool again = !ok && (s_conv[j] || capped) && restart < kMaxRestarts && total_it < a.max_iter;
      if (again) {
        s_conv[j] = 0;
        s_restart = 1;
      }
      if (owner(j)) {
        double* o = a.model_out + (size_t)a.piece_model[s_gp[j]] * 4;
        o[0] = s_iters[j];
        o[1] = rel;
        o[2] = ok ? 1.0 : 0.0;
      }
      if (!again) {
        s_done[j] = 1;
        s_conv[j] = 1;  // no further iterations for this model
      }
    }
    __syncthreads();
    // every CTA must agree on a restart: publish and read after a barrier
    // (one model held by every CTA: each reached the same decision)
    if (a.single_model) {
      if (!s_restart) break;
    } else {
      if (s_restart && threadIdx.x == 0) a.unconv[a.max_iter + 1] = restart + 1;
      if (!grid_barrier(a.barrier, a.flags, &s_bar_round, a.barrier_timeout_ns, a.skip_arrival_cta)) return;
      if (__ldcg(&a.unconv[a.max_iter + 1]) != restart + 1) break;
    }
    // continue with classic PCG, whose attainable accuracy is better than
    // that of the pipelined recurrences
    if (a.variant == 0) classic = true;
  }

  if (a.update_state) {
    for (int i = threadIdx.x; i < nloc; i += blockDim.x) {
      const int row = cr.row(i, cr.piece(i));
      if (a.model_active && !a.model_active[a.row_model[row]]) continue;
      const int n = a.act_node[row];
      const double h = a.step[(size_t)a.row_model[row] * 8];
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
        // GlobalMass position correction of a single-particle plane
        // constraint: the node moves onto its plane along the normal
        const double* q = a.row_nrm + 3 * (size_t)row;
        const double dist = q[0] * xn[0] + q[1] * xn[1] + q[2] * xn[2] - a.row_off[row];
#pragma unroll
        for (int c = 0; c < 3; c++) xn[c] -= q[c] * dist;
      }
#pragma unroll
      for (int c = 0; c < 3; c++) a.xpos[3 * (size_t)n + c] = xn[c];
    }
  }
}

// Solve S x = b with the persistent PCG on the given right-hand side and
// iterate (x in/out); tol_override > 0 replaces every model's tolerance;
// per-model results go to model_out.
cudaError_t launch_pcg_on(Engine& eng, int max_iter, bool update_state, const double* rhs, double* xsol,
                          double tol_override, double* model_out) {
  if (eng.pcg_cluster) return launch_pcg_cluster(eng, max_iter, update_state, rhs, xsol, tol_override, model_out);
  DevPack& d = eng.d;
  cudaError_t e;
  if ((e = cudaMemsetAsync(d.barrier, 0, sizeof(unsigned), eng.stream)) != cudaSuccess) return e;
  PcgArgs a;
  a.n_rows = d.n_rows;
  a.n_pieces = d.n_pieces;
  a.rowptr = d.blk_rowptr;
  a.col = d.blk_col;
  a.blk_diag = d.blk_diag;
  a.S = d.S;
  a.Dinv = d.Dinv;
  a.b = rhs;
  a.x = xsol;
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
  a.cta_plist = d.cta_plist;
  a.partials = d.partials;
  a.step = d.step;
  a.model_out = model_out;
  a.tol_override = tol_override;
  a.barrier = d.barrier;
  a.flags = d.flags;
  a.barrier_timeout_ns = 1000000ull * (unsigned long long)eng.barrier_timeout_ms;
  a.skip_arrival_cta = eng.test_skip_arrival - 1;
  a.unconv = d.unconv;
  a.max_iter = max_iter;
  a.variant = eng.pcg_variant;
  a.row_lanes = eng.pcg_row_lanes;
  a.update_state = update_state ? 1 : 0;
  a.xpos = d.x;
  a.vel = d.v;
  a.vprev = d.vprev;
  a.vprev2 = d.vprev2;
  a.vprev3 = d.vprev3;
  a.vprev4 = d.vprev4;
  a.act_node = d.act_node;
  a.row_model = d.row_model;
  a.model_active = eng.any_inactive ? d.model_active : nullptr;
  a.single_model = (d.n_models == 1 && eng.pcg_every_cta_rows) ? 1 : 0;
  // constraints belong to the ConstrainedBackwardEuler step's solve only
  a.row_nrm = (update_state && eng.integrator == B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER && d.row_nrm)
                  ? d.row_nrm
                  : nullptr;
  a.row_off = a.row_nrm ? d.row_off : nullptr;
  a.dil_rptr = nullptr;
  if (eng.factored) {
    a.rowptr = d.s1_rowptr;
    a.col = d.s1_col;
    a.blk_diag = d.s1_diag;
    a.S = d.S1;
    if (d.n_dil_nodes > 0) a.dil_rptr = d.dil_rptr;
    a.dil_node = d.dil_node;
    a.dil_slot = d.dil_slot;
    a.dil_nodes = d.dil_nodes;
    a.n_dil_nodes = d.n_dil_nodes;
    a.nbr_ptr = d.nbr_ptr;
    a.nbr_row = d.nbr_row;
    a.divblk = d.divblk;
    a.node_kp = d.node_kp;
    a.node_model = d.node_model;
    a.dil_t = d.dil_t;
  }
  a.resident = eng.pcg_resident;
  a.cached = eng.pcg_cached;
  a.nloc_max = eng.pcg_nloc_max;
  a.nb_max = eng.pcg_nb_max;
  size_t ov, oro, oc, oS, total;
  if (eng.precision == B200FEM_PREC_MIXED)
    pcg_smem_layout<float>(a.nloc_max, a.nb_max, a.resident, a.cached, &ov, &oro, &oc, &oS, &total);
  else
    pcg_smem_layout<double>(a.nloc_max, a.nb_max, a.resident, a.cached, &ov, &oro, &oc, &oS, &total);
  if ((int)total > eng.pcg_attr_smem) return cudaErrorInvalidConfiguration;  // prepare_pcg not run
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(eng.pcg_grid);
  cfg.blockDim = dim3(pcg_block(a.resident != 0));
  cfg.dynamicSmemBytes = total;
  cfg.stream = eng.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (eng.precision == B200FEM_PREC_MIXED) {
    a.S = eng.factored ? (const void*)d.S1_f : (const void*)d.S_f;
    if (a.dil_rptr)
      return a.resident ? cudaLaunchKernelEx(&cfg, pcg_kernel<float, true, true>, a)
                        : cudaLaunchKernelEx(&cfg, pcg_kernel<float, false, true>, a);
    return a.resident ? cudaLaunchKernelEx(&cfg, pcg_kernel<float, true>, a)
                      : cudaLaunchKernelEx(&cfg, pcg_kernel<float, false>, a);
  }
  if (a.dil_rptr)
    return a.resident ? cudaLaunchKernelEx(&cfg, pcg_kernel<double, true, true>, a)
                      : cudaLaunchKernelEx(&cfg, pcg_kernel<double, false, true>, a);
  return a.resident ? cudaLaunchKernelEx(&cfg, pcg_kernel<double, true>, a)
                    : cudaLaunchKernelEx(&cfg, pcg_kernel<double, false>, a);
}

cudaError_t launch_pcg(Engine& eng, int max_iter, bool update_state, int init_zero) {
  DevPack& d = eng.d;
  if (init_zero) {
    cudaError_t e = cudaMemsetAsync(d.sol, 0, sizeof(double) * 3 * (size_t)d.n_rows, eng.stream);
    if (e != cudaSuccess) return e;
  }
  return launch_pcg_on(eng, max_iter, update_state, d.b, d.sol, 0.0, d.model_scal);
}

int pcg_threads() { return kPcgThreads; }

// The dynamic shared-memory opt-in of pcg_kernel is process-wide per
// function: raise it monotonically so one caller never lowers it below what
// another needs.
static std::mutex g_pcg_attr_mu;
static int g_pcg_attr_bytes[2][64] = {{0}};

static cudaError_t ensure_pcg_smem(int device, size_t bytes, bool fp32 = false) {
  std::lock_guard<std::mutex> lk(g_pcg_attr_mu);
  const int d = (device >= 0 && device < 64) ? device : 0;
  int& cur = g_pcg_attr_bytes[fp32 ? 1 : 0][d];
  if ((int)bytes <= cur) return cudaSuccess;
  const cudaFuncAttribute at = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = fp32 ? cudaFuncSetAttribute(pcg_kernel<float, false>, at, (int)bytes)
                       : cudaFuncSetAttribute(pcg_kernel<double, false>, at, (int)bytes);
  if (e == cudaSuccess)
    e = fp32 ? cudaFuncSetAttribute(pcg_kernel<float, true>, at, (int)bytes)
             : cudaFuncSetAttribute(pcg_kernel<double, true>, at, (int)bytes);
  if (e == cudaSuccess)
    e = fp32 ? cudaFuncSetAttribute(pcg_kernel<float, false, true>, at, (int)bytes)
             : cudaFuncSetAttribute(pcg_kernel<double, false, true>, at, (int)bytes);
  if (e == cudaSuccess)
    e = fp32 ? cudaFuncSetAttribute(pcg_kernel<float, true, true>, at, (int)bytes)
             : cudaFuncSetAttribute(pcg_kernel<double, true, true>, at, (int)bytes);
  if (e == cudaSuccess) cur = (int)bytes;
  return e;
}

cudaError_t prepare_pcg(Engine& eng) {
  size_t ov, oro, oc, oS, total;
  const bool fp32 = eng.precision == B200FEM_PREC_MIXED;
  if (fp32)
    pcg_smem_layout<float>(eng.pcg_nloc_max, eng.pcg_nb_max, eng.pcg_resident, eng.pcg_cached, &ov, &oro, &oc, &oS,
                           &total);
  else
    pcg_smem_layout<double>(eng.pcg_nloc_max, eng.pcg_nb_max, eng.pcg_resident, eng.pcg_cached, &ov, &oro, &oc, &oS,
                            &total);
  cudaError_t e = ensure_pcg_smem(eng.device, total, fp32);
  if (e == cudaSuccess) eng.pcg_attr_smem = (int)total;
  return e;
}

// Decide shared-memory residency of the PCG row state and of the S slice
// for the given per-CTA maxima (rows, blocks) within the device's opt-in
// shared memory per block.
void pcg_plan_smem(int device, int nloc_max, int nb_max, int* resident, int* cached, bool fp32) {
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  cudaFuncAttributes fa;
  cudaFuncAttributes fb;
  if (fp32) {
    cudaFuncGetAttributes(&fa, pcg_kernel<float, false>);
    cudaFuncGetAttributes(&fb, pcg_kernel<float, true>);
  } else {
    cudaFuncGetAttributes(&fa, pcg_kernel<double, false>);
    cudaFuncGetAttributes(&fb, pcg_kernel<double, true>);
  }
  fa.sharedSizeBytes = std::max(fa.sharedSizeBytes, fb.sharedSizeBytes);
  const long long budget = (long long)optin - (long long)fa.sharedSizeBytes - 1024;
  size_t ov, oro, oc, oS, total;
  *resident = 0;
  *cached = 0;
  auto layout = [&](int res, int cac) {
    if (fp32) pcg_smem_layout<float>(nloc_max, nb_max, res, cac, &ov, &oro, &oc, &oS, &total);
    else pcg_smem_layout<double>(nloc_max, nb_max, res, cac, &ov, &oro, &oc, &oS, &total);
  };
  layout(1, 0);
  if ((long long)total <= budget) *resident = 1;
  layout(*resident, 1);
  if ((long long)total <= budget) *cached = 1;
}
int pcg_max_cta_pieces() { return kMaxCtaPieces; }

int pcg_max_grid(int device) {
  int sms = 0, per_sm = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pcg_kernel<double, false>, kPcgThreads, 0);
  return sms * (per_sm > 0 ? per_sm : 1);
}


// ---------------------------------------------------------------------------
// Allocation-free PCG (b200fem_pcg_solve_noalloc)
//
// For callers that cannot allocate device memory: hosts whose device memory
// is owned entirely by another allocator or pool (a framework's caching
// allocator, a JVM-side arena handed out by the application), and real-time
// or embedded hosts that fix their device footprint at start-up and forbid
// allocation afterwards.  They pass their own device buffers for the matrix,
// right-hand side and solution; every other buffer the solve needs comes
// from the file-scope array below, which every device that loads the
// library holds until the process exits.
// ---------------------------------------------------------------------------
constexpr int kNoAllocMaxRows = B200FEM_NOALLOC_MAX_ROWS;
constexpr int kNoAllocMaxIter = B200FEM_NOALLOC_MAX_ITER;
constexpr int kNoAllocMaxGrid = 1024;

constexpr size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

struct NoAllocLayout {
  // byte offsets inside the scratch array, each 256-byte aligned
  static constexpr size_t dinv = 0;
  static constexpr size_t vec = al256(dinv + sizeof(double) * 9 * (size_t)kNoAllocMaxRows);  // r u w z q s p m0 m1
  static constexpr size_t partials = al256(vec + sizeof(double) * 9 * 3 * (size_t)kNoAllocMaxRows);
  static constexpr size_t step = al256(partials + sizeof(double) * 2 * 4 * (size_t)kNoAllocMaxGrid);
  static constexpr size_t model_out = al256(step + sizeof(double) * 8);
  static constexpr size_t blk_diag = al256(model_out + sizeof(double) * 4);
  static constexpr size_t piece_row = al256(blk_diag + sizeof(int) * (size_t)kNoAllocMaxRows);
  static constexpr size_t piece_model = al256(piece_row + sizeof(int) * (kNoAllocMaxGrid + 1));
  static constexpr size_t model_piece = al256(piece_model + sizeof(int) * kNoAllocMaxGrid);
  static constexpr size_t cta_piece = al256(model_piece + sizeof(int) * 2);
  static constexpr size_t unconv = al256(cta_piece + sizeof(int) * (kNoAllocMaxGrid + 1));
  static constexpr size_t flags = al256(unconv + sizeof(int) * (kNoAllocMaxIter + 2));
  static constexpr size_t barrier = al256(flags + sizeof(int) * 4);
  static constexpr size_t total = al256(barrier + sizeof(unsigned) * 2);
};

static __device__ __align__(256) unsigned char g_noalloc_scratch[NoAllocLayout::total];

// per-device set-up: the device address of the scratch array (host code
// cannot use the symbol itself) and the launch geometry
struct NoAllocDevice {
  bool ready = false;
  unsigned char* base = nullptr;
  int sms = 0;
};
static std::mutex g_noalloc_mu;
static NoAllocDevice g_noalloc_dev[64];

__global__ void noalloc_diag_kernel(int n_rows, const int* __restrict__ rowptr, const int* __restrict__ col,
                                    int* __restrict__ blk_diag, int* __restrict__ flags) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= n_rows) return;
  int d = -1;
  for (int p = rowptr[row]; p < rowptr[row + 1]; p++)
    if (col[p] == row) d = p;
  blk_diag[row] = d < 0 ? rowptr[row] : d;
  if (d < 0) atomicExch(flags, B200FEM_ERR_INVALID_ARG);
}

int pcg_solve_noalloc(int n_rows, const int* rowptr, const int* col, const double* vals, const double* b, double* x,
                      double tol, int max_iter, void* stream_ptr, int* iterations, double* rel_residual,
                      const char** err) {
  cudaStream_t stream = (cudaStream_t)stream_ptr;
  if (n_rows < 1 || max_iter < 1) {
    *err = "n_rows and max_iter must be at least 1";
    return B200FEM_ERR_INVALID_ARG;
  }
  if (n_rows > kNoAllocMaxRows) {
    *err = "n_rows exceeds B200FEM_NOALLOC_MAX_ROWS";
    return B200FEM_ERR_BUDGET;
  }
  if (max_iter > kNoAllocMaxIter) {
    *err = "max_iter exceeds B200FEM_NOALLOC_MAX_ITER";
    return B200FEM_ERR_BUDGET;
  }
  if (!rowptr || !col || !vals || !b || !x || !(tol > 0)) {
    *err = "null device pointer or non-positive tolerance";
    return B200FEM_ERR_INVALID_ARG;
  }
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess || device < 0 || device >= 64) {
    *err = "no current CUDA device";
    return B200FEM_ERR_CUDA;
  }
  NoAllocDevice nd;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice& dev = g_noalloc_dev[device];
    if (!dev.ready) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
        *err = "cudaGetSymbolAddress of the scratch array failed";
        return B200FEM_ERR_CUDA;
      }
      dev.base = (unsigned char*)p;
      if (cudaDeviceGetAttribute(&dev.sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess) {
        *err = "cudaDeviceGetAttribute failed";
        return B200FEM_ERR_CUDA;
      }
      dev.ready = true;
    }
    nd = dev;
  }
  using LY = NoAllocLayout;
  unsigned char* base = nd.base;
  // even split of the rows over the CTAs, one piece each (single model)
  const int G = min(min(nd.sms, kNoAllocMaxGrid), (n_rows + 31) / 32);
  int piece_row[kNoAllocMaxGrid + 1], cta_piece[kNoAllocMaxGrid + 1], piece_model[kNoAllocMaxGrid];
  int model_piece[2] = {0, G};
  for (int c = 0; c <= G; c++) {
    piece_row[c] = (int)((long long)n_rows * c / G);
    cta_piece[c] = c;
  }
  for (int c = 0; c < G; c++) piece_model[c] = 0;
  double step[8] = {0, 0, 0, 0, 0, 0, tol, 0};
  const int nloc_max = (n_rows + G - 1) / G + 1;
  int resident = 0, cached = 0;
  pcg_plan_smem(device, nloc_max, 0, &resident, &cached, false);
  cached = 0;
  size_t ov, oro, oc, oS, dyn;
  pcg_smem_layout<double>(nloc_max, 0, resident, 0, &ov, &oro, &oc, &oS, &dyn);
  cudaError_t e;
  if ((e = ensure_pcg_smem(device, dyn)) != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return B200FEM_ERR_CUDA;
  }
  // the array keeps the previous call's contents: clear what must start at
  // zero (barrier counter, error/status words, model outputs)
  e = cudaMemsetAsync(base + LY::barrier, 0, sizeof(unsigned) * 2, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + LY::flags, 0, sizeof(int) * 4, stream);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + LY::model_out, 0, sizeof(double) * 4, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + LY::piece_row, piece_row, sizeof(int) * (G + 1), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + LY::cta_piece, cta_piece, sizeof(int) * (G + 1), cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + LY::piece_model, piece_model, sizeof(int) * G, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + LY::model_piece, model_piece, sizeof(int) * 2, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(base + LY::step, step, sizeof(step), cudaMemcpyHostToDevice, stream);
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return B200FEM_ERR_CUDA;
  }
  noalloc_diag_kernel<<<(n_rows + 255) / 256, 256, 0, stream>>>(n_rows, rowptr, col, (int*)(base + LY::blk_diag),
                                                               (int*)(base + LY::flags));
  // a row without a diagonal block has no valid blk_diag entry (the
  // stand-in rowptr[row] can lie past the caller's vals for an empty last
  // row): refuse the matrix before the PCG reads any block
  {
    int diag_flag = 0;
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&diag_flag, base + LY::flags, sizeof(int), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
      *err = cudaGetErrorString(e);
      return B200FEM_ERR_CUDA;
    }
    if (diag_flag != 0) {
      *err = "a block row has no diagonal block";
      return B200FEM_ERR_INVALID_ARG;
    }
  }
  double* vec = (double*)(base + LY::vec);
  const size_t V = 3 * (size_t)kNoAllocMaxRows;
  PcgArgs a;
  a.n_rows = n_rows;
  a.n_pieces = G;
  a.rowptr = rowptr;
  a.col = col;
  a.blk_diag = (const int*)(base + LY::blk_diag);
  a.S = vals;
  a.Dinv = (double*)(base + LY::dinv);
  a.b = b;
  a.x = x;
  a.r = vec + 0 * V;
  a.u = vec + 1 * V;
  a.w = vec + 2 * V;
  a.z = vec + 3 * V;
  a.q = vec + 4 * V;
  a.s = vec + 5 * V;
  a.p = vec + 6 * V;
  a.m0 = vec + 7 * V;
  a.m1 = vec + 8 * V;
  a.piece_row = (const int*)(base + LY::piece_row);
  a.piece_model = (const int*)(base + LY::piece_model);
  a.model_piece = (const int*)(base + LY::model_piece);
  a.cta_piece = (const int*)(base + LY::cta_piece);
  // one piece per CTA, numbered like the CTAs: the identity table cta_piece
  // doubles as the piece list
  a.cta_plist = a.cta_piece;
  a.partials = (double*)(base + LY::partials);
  a.step = (const double*)(base + LY::step);
  a.model_out = (double*)(base + LY::model_out);
  a.resident = resident;
  a.cached = 0;
  a.nloc_max = nloc_max;
  a.nb_max = 0;
  a.barrier = (unsigned*)(base + LY::barrier);
  a.flags = (int*)(base + LY::flags);
  a.barrier_timeout_ns = kBarrierTimeoutNs;
  a.skip_arrival_cta = -1;
  a.unconv = (int*)(base + LY::unconv);
  a.max_iter = max_iter;
  a.variant = 0;
  a.row_lanes = 16;
  a.update_state = 0;
  a.vprev = nullptr;
  a.vprev2 = nullptr;
  a.vprev3 = nullptr;
  a.vprev4 = nullptr;
  a.xpos = nullptr;
  a.vel = nullptr;
  a.act_node = nullptr;
  a.row_model = nullptr;
  a.model_active = nullptr;
  a.single_model = 0;
  a.row_nrm = nullptr;
  a.row_off = nullptr;
  a.dil_rptr = nullptr;
  a.tol_override = 0;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(G);
  cfg.blockDim = dim3(pcg_block(a.resident != 0));
  cfg.dynamicSmemBytes = dyn;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  e = resident ? cudaLaunchKernelEx(&cfg, pcg_kernel<double, true>, a)
               : cudaLaunchKernelEx(&cfg, pcg_kernel<double, false>, a);
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return B200FEM_ERR_CUDA;
  }
  double out[4];
  int flags[4];
  e = cudaMemcpyAsync(out, base + LY::model_out, sizeof(out), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaMemcpyAsync(flags, base + LY::flags, sizeof(flags), cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e != cudaSuccess) {
    *err = cudaGetErrorString(e);
    return B200FEM_ERR_CUDA;
  }
  if (iterations) *iterations = (int)out[0];
  if (rel_residual) *rel_residual = out[1];
  if (flags[0] == B200FEM_ERR_TIMEOUT) {
    *err = "PCG grid barrier timed out";
    return B200FEM_ERR_TIMEOUT;
  }
  if (flags[0] != 0) {
    *err = "missing or singular diagonal block";
    return B200FEM_ERR_INVALID_ARG;
  }
  if (out[2] == 0.0) {
    *err = "PCG did not reach the tolerance within max_iter iterations";
    return B200FEM_ERR_NO_CONVERGE;
  }
  return B200FEM_OK;
}

}  // namespace b200fem
