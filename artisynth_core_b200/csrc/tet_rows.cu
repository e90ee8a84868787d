// tet_rows.cu -- node-row assembly of tetrahedral packs (non-linear
// materials) for the BackwardEuler step.
//
// The element-and-gather path writes every element's ten upper tangent
// blocks and four nodal forces to HBM and reads them back at scattered
// positions (FemModel3d.computeStressAndStiffness, FemModel3d.java:
// 3333-3666, followed by the block scatter of FemNodeNeighbor.addSolveBlocks,
// FemNodeNeighbor.java:159-187).  Here one warp owns a task: a few
// consecutive block rows of one model whose node incidences (elements in
// element order) fit CAP lanes.  Each lane recomputes one incident
// tetrahedron -- kinematics, material point, its force at the row's node and
// the four blocks of the row's node against the element's nodes -- from the
// positions and rest data, so each tetrahedron is evaluated once per active
// node (four times) and nothing element-sized goes through HBM.  The lane's
// blocks go to the warp's shared-memory stage; then every block of the
// task's rows sums its contributions (stage entries named by a per-block
// byte list, in element order), adds the NODAL dilational term, applies the
// BackwardEuler coefficients S = (h^2 + h beta) K + (1 + h alpha) M
// (MechSystemSolver.java:2277,2312,2334) and is stored with the task's
// other blocks as contiguous lines; every row sums its forces (incidence
// order) and forms the right-hand side b = M v + h (m g + f_ext - f_int)
// and the PCG's initial guess.
//
// The arithmetic is the element-and-gather path's, expression for
// expression (the same element code, blocks of the upper pair transposed
// for the lower position, the same summation orders), so S and b agree with
// that path's to rounding (the compiler may contract a different product of
// an expression into an FMA in the two kernels).
#include <cuda_runtime.h>

#include "device_math.cuh"
#include "engine.h"

namespace b200fem {

// dN/ds of the four tet nodes (TetElement: N = 1 - s0 - s1 - s2, s0, s1, s2)
__constant__ double c_rows_tet_gns[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};

constexpr int kRowsWarps = 4;  // warps (tasks) per CTA
constexpr int kIncOffR = 0, kIncNodalR = 1, kIncElementR = 2;

struct TetRowArgs {
  int t0, t1;                  // tasks of this launch
  const int* task_row;         // first block row of each task (+1 entry)
  const int* row_incptr;       // per block row: offset of its incidences in row_inc (+1 entry)
  const int* row_inc;          // (element << 3) | (local node << 1) | records the element's statistics
  const int* rowptr;           // block-row offsets
  const int* blk_row;
  const int* blk_diag;
  const int* mirror;           // block at the transposed position
  const int* cptr;             // per block: contribution offsets
  const unsigned char* cbyte;  // per contribution: stage entry (incidence in task * 4 + column node)
  const int* dptr;             // NODAL dilational triples per block (or null)
  const int* didx;
  const double* divblk;
  const double* node_kp;
  const int* conn;
  const int* elem_model;
  const int* elem_mat;  // per element: its row of mat
  const double* x;
  const double* invJ0;
  const double* mat;
  const double* node_p;
  const double* elem_p;
  const double* elem_r;
  const int* row_model;
  const int* act_node;
  const double* mass;
  const double* step;
  const int* active;
  const double* v;
  const double* fext;
  const double* vprev;
  const double* vprev2;
  const double* vprev3;
  const double* vprev4;
  const double* row_nrm;
  void* out;     // S in the storage precision
  double* b;
  double* sol0;
  double* fint;  // per node (rows' nodes only)
  int* flags;
  long long* mindet;
};

__device__ __forceinline__ long long rows_dbl_order(double v) {
  long long i = __double_as_longlong(v);
  return i >= 0 ? i : (i ^ 0x7fffffffffffffffll);
}

// per-warp shared memory: CAP incidences x 4 blocks of 9, CAP forces of 3
// (FP64), and 32 blocks of output staging
template <typename T, int CAP>
struct RowsSmem {
  static constexpr size_t stage = sizeof(T) * (size_t)CAP * 4 * 9;
  static constexpr size_t force = sizeof(double) * (size_t)CAP * 3;
  static constexpr size_t ostage = sizeof(T) * 32 * 9;
  static constexpr size_t per_warp = stage + force + ostage;
  static constexpr size_t bytes() { return per_warp * kRowsWarps; }
};

template <int MAT, int INC, typename T, int CAP>
__global__ void __launch_bounds__(32 * kRowsWarps) tet_rows_kernel(TetRowArgs a) {
  extern __shared__ __align__(16) unsigned char rows_smem[];
  using SM = RowsSmem<T, CAP>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = a.t0 + blockIdx.x * kRowsWarps + warp;
  if (t >= a.t1) return;  // the whole warp (no block-wide barrier below)
  const int r0 = a.task_row[t], r1 = a.task_row[t + 1];
  if (a.active && !a.active[a.row_model[r0]]) return;  // a task's rows are one model's
  unsigned char* base = rows_smem + SM::per_warp * warp;
  T* stage = (T*)base;
  double* fst = (double*)(base + SM::stage);
  T* ost = (T*)(base + SM::stage + SM::force);
  const int i0 = a.row_incptr[r0];
  const int ninc = a.row_incptr[r1] - i0;
  double mydet = 1.0e300;
  int myinv = 0;
#pragma unroll 1
  for (int q = lane; q < ninc; q += 32) {
    const int code = a.row_inc[i0 + q];
    const int e = code >> 3, am = (code >> 1) & 3;
    const int* nodes = a.conn + (size_t)e * 4;
    int nd[4];
#pragma unroll
    for (int n = 0; n < 4; n++) nd[n] = nodes[n];
    // IntegrationPoint3d.computeJacobian and FemDeformedPoint
    // (IntegrationPoint3d.java:190-201, FemDeformedPoint.java:60-97)
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const double g0 = c_rows_tet_gns[3 * n], g1 = c_rows_tet_gns[3 * n + 1], g2 = c_rows_tet_gns[3 * n + 2];
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const double xr = a.x[3 * (size_t)nd[n] + r];
        J[3 * r] += xr * g0;
        J[3 * r + 1] += xr * g1;
        J[3 * r + 2] += xr * g2;
      }
    }
    double iJ0[9], F[9], invJ[9];
#pragma unroll
    for (int i = 0; i < 9; i++) iJ0[i] = a.invJ0[(size_t)e * 9 + i];
    matmul3(F, J, iJ0);
    const double detF = det3(F);
    const double detJ = invert3(invJ, J);
    if (code & 1) {
      myinv |= !(detJ > 0.0);
      mydet = fmin(mydet, detJ);
    }
    const double dv = detJ * (1.0 / 6.0);
    double g[4][3];
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const double g0 = c_rows_tet_gns[3 * n], g1 = c_rows_tet_gns[3 * n + 1], g2 = c_rows_tet_gns[3 * n + 2];
#pragma unroll
      for (int c = 0; c < 3; c++) g[n][c] = invJ[c] * g0 + invJ[3 + c] * g1 + invJ[6 + c] * g2;
    }
    const double* mp = a.mat + (size_t)a.elem_mat[e] * kMatParams;
    double sig[6];
    T Dt[MAT == B200FEM_MAT_NEOHOOKEAN ? 2 : 36];
    if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) {
      double ca, cb;
      neohookean_point<double>(sig, &ca, &cb, mp[0], mp[1], F, detF);
      Dt[0] = (T)ca;
      Dt[1] = (T)cb;
    } else {
      double pr = 0;
      if constexpr (INC == kIncNodalR)
        pr = 0.25 * (a.node_p[nd[0]] + a.node_p[nd[1]] + a.node_p[nd[2]] + a.node_p[nd[3]]);
      else if constexpr (INC == kIncElementR)
        pr = a.elem_p[e];
      double D[36];
      material_point<MAT, double>(sig, D, mp, F, detF, pr);
#pragma unroll
      for (int i = 0; i < 36; i++) Dt[i] = (T)D[i];
    }
    // FemUtilities.addStressForce (FemUtilities.java:40-49), FP64
    double gam[3];
#pragma unroll
    for (int c = 0; c < 3; c++) gam[c] = am == 0 ? g[0][c] : am == 1 ? g[1][c] : am == 2 ? g[2][c] : g[3][c];
    {
      double f[3] = {0, 0, 0};
      add_stress_force(f, gam, sig, dv);
      fst[3 * q] = f[0];
      fst[3 * q + 1] = f[1];
      fst[3 * q + 2] = f[2];
    }
    // the four blocks (am, bn): the upper pair's block, transposed when
    // am > bn (FemModel3d.java:3003-3026 mirrors the upper triangle)
    T gt[4][3], st[6];
    const T dvt = (T)dv;
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
      for (int c = 0; c < 3; c++) gt[n][c] = (T)g[n][c];
#pragma unroll
    for (int i = 0; i < 6; i++) st[i] = (T)sig[i];
    T rinv = T(0);
    if constexpr (INC == kIncElementR) rinv = (T)(a.elem_r[e] * dv * dv);
    T* sq = stage + (size_t)q * 36;
#pragma unroll
    for (int bn = 0; bn < 4; bn++) {
      const int lo = am < bn ? am : bn, hi = am < bn ? bn : am;
      T glo[3], ghi[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        glo[c] = lo == 0 ? gt[0][c] : lo == 1 ? gt[1][c] : lo == 2 ? gt[2][c] : gt[3][c];
        ghi[c] = hi == 0 ? gt[0][c] : hi == 1 ? gt[1][c] : hi == 2 ? gt[2][c] : gt[3][c];
      }
      T K[9];
#pragma unroll
      for (int i = 0; i < 9; i++) K[i] = T(0);
      if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) add_bdb_iso(K, glo, Dt[0], Dt[1], ghi, dvt);
      else add_bdb(K, glo, Dt, ghi, dvt);
      add_geometric(K, glo, st, ghi, dvt);
      if constexpr (INC == kIncElementR) {
        // ELEMENT dilational stiffness Rinv (g_a dv)(g_b dv)^T
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) K[3 * i + j] += rinv * glo[i] * ghi[j];
      }
      if (am > bn) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) sq[9 * bn + 3 * i + j] = K[3 * j + i];
      } else {
#pragma unroll
        for (int i = 0; i < 9; i++) sq[9 * bn + i] = K[i];
      }
    }
  }
  // inverted elements and smallest detJ, one atomic per warp
  {
    const int tot = __reduce_add_sync(0xffffffffu, myinv);
    double dm = mydet;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) dm = fmin(dm, __shfl_xor_sync(0xffffffffu, dm, off));
    if (lane == 0) {
      if (tot) atomicAdd(&a.flags[1], tot);
      if (dm < 1.0e300) atomicMin(a.mindet, rows_dbl_order(dm));
    }
  }
  __syncwarp();
  // blocks of the task's rows
  const int p0 = a.rowptr[r0], p1 = a.rowptr[r1];
  T* out = (T*)a.out;
#pragma unroll 1
  for (int pb = p0; pb < p1; pb += 32) {
    const int p = pb + lane;
    if (p < p1) {
      double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const int c1 = a.cptr[p + 1];
      for (int c = a.cptr[p]; c < c1; c++) {
        const T* B = stage + (size_t)a.cbyte[c] * 9;
#pragma unroll
        for (int k = 0; k < 9; k++) s[k] += (double)B[k];
      }
      const int row = a.blk_row[p];
      if (a.dptr) {
        // NODAL dilational term sum_n kp_n divBlk(n,i) divBlk(n,j)^T over
        // the upper block's list (FemModel3d.java:2632-2669); a lower block
        // takes its mirror's sum, transposed
        const int mp = a.mirror[p];
        const bool lower = mp >= 0 && mp < p;
        const int pu = lower ? mp : p;
        double sd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const int d1 = a.dptr[pu + 1];
        for (int tr_i = a.dptr[pu]; tr_i < d1; tr_i++) {
          const int* tr = a.didx + 3 * (size_t)tr_i;
          const double kp = a.node_kp[tr[2]];
          const double* di = a.divblk + 3 * (size_t)tr[0];
          const double* dj = a.divblk + 3 * (size_t)tr[1];
#pragma unroll
          for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) sd[3 * r + c] += kp * di[r] * dj[c];
        }
        if (lower) {
#pragma unroll
          for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) s[3 * r + c] += sd[3 * c + r];
        } else {
#pragma unroll
          for (int k = 0; k < 9; k++) s[k] += sd[k];
        }
      }
      const double* sp = a.step + (size_t)a.row_model[row] * 8;
      const double h = sp[0], al = sp[1], be = sp[2];
      const double cm = p == a.blk_diag[row] ? (1.0 + h * al) * a.mass[a.act_node[row]] : 0.0;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        double val = (h * h + h * be) * s[k];
        if (k % 4 == 0) val += cm;
        ost[9 * lane + k] = (T)val;
      }
    }
    __syncwarp();
    const int nv = (p1 - pb < 32 ? p1 - pb : 32) * 9;
    T* o = out + (size_t)pb * 9;
    for (int i = lane; i < nv; i += 32) o[i] = ost[i];
    __syncwarp();
  }
  // rows: internal force (incidence order), right-hand side, initial guess
  for (int r = r0 + lane; r < r1; r += 32) {
    double f[3] = {0, 0, 0};
    const int q1 = a.row_incptr[r + 1] - i0;
    for (int q = a.row_incptr[r] - i0; q < q1; q++) {
#pragma unroll
      for (int c = 0; c < 3; c++) f[c] += fst[3 * q + c];
    }
    const int n = a.act_node[r];
    if (a.fint) {
#pragma unroll
      for (int c = 0; c < 3; c++) a.fint[3 * (size_t)n + c] = f[c];
    }
    const double* sp = a.step + (size_t)a.row_model[r] * 8;
    const double h = sp[0], m = a.mass[n];
#pragma unroll
    for (int c = 0; c < 3; c++)
      a.b[3 * (size_t)r + c] = m * a.v[3 * (size_t)n + c] + h * (m * sp[3 + c] + a.fext[3 * (size_t)n + c] - f[c]);
    double s0[3];
#pragma unroll
    for (int c = 0; c < 3; c++) {
      const size_t k = 3 * (size_t)n + c;
      const double vc = a.v[k];
      if (a.vprev4)
        s0[c] = 5.0 * (vc - a.vprev3[k]) + 10.0 * (a.vprev2[k] - a.vprev[k]) + a.vprev4[k];
      else if (a.vprev3)
        s0[c] = 4.0 * (vc + a.vprev2[k]) - 6.0 * a.vprev[k] - a.vprev3[k];
      else if (a.vprev2)
        s0[c] = 3.0 * (vc - a.vprev[k]) + a.vprev2[k];
      else
        s0[c] = a.vprev ? 2.0 * vc - a.vprev[k] : vc;
    }
    if (a.row_nrm) {
      const double* qn = a.row_nrm + 3 * (size_t)r;
      const double d = qn[0] * s0[0] + qn[1] * s0[1] + qn[2] * s0[2];
#pragma unroll
      for (int c = 0; c < 3; c++) s0[c] -= qn[c] * d;
    }
#pragma unroll
    for (int c = 0; c < 3; c++) a.sol0[3 * (size_t)r + c] = s0[c];
  }
}

template <int MAT, int INC, typename T, int CAP>
static cudaError_t launch_rows_cap(const TetRowArgs& a, cudaStream_t st, bool attr_only) {
  constexpr size_t smem = RowsSmem<T, CAP>::bytes();
  if (attr_only)
    return cudaFuncSetAttribute(tet_rows_kernel<MAT, INC, T, CAP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem);
  const int n = a.t1 - a.t0;
  if (n <= 0) return cudaSuccess;
  tet_rows_kernel<MAT, INC, T, CAP><<<(n + kRowsWarps - 1) / kRowsWarps, 32 * kRowsWarps, smem, st>>>(a);
  return cudaGetLastError();
}

template <int MAT, int INC, typename T>
static cudaError_t launch_rows_mat(const TetRowArgs& a, int cap, cudaStream_t st, bool attr_only) {
  return cap <= 32 ? launch_rows_cap<MAT, INC, T, 32>(a, st, attr_only)
                   : launch_rows_cap<MAT, INC, T, 64>(a, st, attr_only);
}

template <typename T>
static cudaError_t launch_rows_group(const TetRowArgs& a, const ElemGroup& g, int cap, cudaStream_t st,
                                     bool attr_only) {
  constexpr int NH = B200FEM_MAT_NEOHOOKEAN, MR = B200FEM_MAT_MOONEYRIVLIN, SV = B200FEM_MAT_STVK;
  const int inc = g.nodal ? kIncNodalR : g.elem_inc ? kIncElementR : kIncOffR;
  switch (g.mat_kind) {
    case NH:
      return launch_rows_mat<NH, kIncOffR, T>(a, cap, st, attr_only);
    case SV:
      return launch_rows_mat<SV, kIncOffR, T>(a, cap, st, attr_only);
    case MR:
      if (inc == kIncNodalR) return launch_rows_mat<MR, kIncNodalR, T>(a, cap, st, attr_only);
      if (inc == kIncElementR) return launch_rows_mat<MR, kIncElementR, T>(a, cap, st, attr_only);
      return launch_rows_mat<MR, kIncOffR, T>(a, cap, st, attr_only);
    default:
      return cudaErrorInvalidValue;
  }
}

// The step's assembly on the node-row path: one launch per element group
// (runs of models with one material kind and soft incompressibility) over
// its tasks; attr_only sets the kernels' shared-memory opt-in.
cudaError_t launch_tet_rows(Engine& eng, bool attr_only) {
  DevPack& d = eng.d;
  const bool fp32 = eng.precision == B200FEM_PREC_MIXED;
  TetRowArgs a;
  a.task_row = d.task_row;
  a.row_incptr = d.row_incptr;
  a.row_inc = d.row_inc;
  a.rowptr = d.blk_rowptr;
  a.blk_row = d.blk_row;
  a.blk_diag = d.blk_diag;
  a.mirror = d.blk_mirror;
  a.cptr = d.contrib_ptr;
  a.cbyte = d.contrib_byte;
  a.dptr = d.dil_ptr;
  a.didx = d.dil_idx;
  a.divblk = d.divblk;
  a.node_kp = d.node_kp;
  a.conn = d.conn;
  a.elem_model = d.elem_model;
  a.elem_mat = d.elem_mat;
  a.x = d.x;
  a.invJ0 = d.invJ0;
  a.mat = d.mat;
  a.node_p = d.node_p;
  a.elem_p = d.elem_p;
  a.elem_r = d.elem_r;
  a.row_model = d.row_model;
  a.act_node = d.act_node;
  a.mass = d.mass;
  a.step = d.step;
  a.active = eng.any_inactive ? d.model_active : nullptr;
  a.v = d.v;
  a.fext = d.fext;
  a.vprev = eng.opt_warm_start >= 1 ? d.vprev : nullptr;
  a.vprev2 = eng.opt_warm_start >= 2 ? d.vprev2 : nullptr;
  a.vprev3 = eng.opt_warm_start >= 3 ? d.vprev3 : nullptr;
  a.vprev4 = eng.opt_warm_start == 4 ? d.vprev4 : nullptr;
  a.row_nrm = (eng.integrator == B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER && d.row_nrm) ? d.row_nrm : nullptr;
  a.out = fp32 ? (void*)d.S_f : (void*)d.S;
  a.b = d.b;
  a.sol0 = d.sol;
  a.fint = d.fint;
  a.flags = d.flags;
  a.mindet = (long long*)d.dmin;
  for (size_t gi = 0; gi < eng.groups.size(); gi++) {
    const ElemGroup& g = eng.groups[gi];
    a.t0 = eng.rows_task_off[gi];
    a.t1 = eng.rows_task_off[gi + 1];
    cudaError_t e = fp32 ? launch_rows_group<float>(a, g, eng.rows_cap, eng.stream, attr_only)
                         : launch_rows_group<double>(a, g, eng.rows_cap, eng.stream, attr_only);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace b200fem
