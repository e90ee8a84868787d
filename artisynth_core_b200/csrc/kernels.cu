// kernels.cu -- sm_100a kernels of the FEM hot path:
//
//   elem_tet_kernel   tetrahedra, non-linear materials: one thread per
//                     element in registers -- kinematics, stress and nodal
//                     forces in FP64, the ten upper pair blocks in the
//                     storage precision, warp-staged contiguous stores
//   elem_nonlinear_kernel / elem_linear_kernel
//                     every element type (hex, wedge, pyramid, quadratic tet
//                     and hex; tets on request) through the shape traits
//                     below: coordinates staged
//                     through shared memory, per-integration-point kinematics
//                     and material (F, sigma, D), then one thread per element
//                     node pair forms the 3x3 tangent block and one per node
//                     the stress force (FemModel3d.computeStressAndStiffness,
//                     FemModel3d.java:3333-3666)
//   elem_force_kernel FP64 nodal forces of the mixed form (multi-point elements)
//   gather_block_kernel
//                     deterministic, atomic-free scatter: every 3x3 block sums
//                     its precomputed contribution list (element pair,
//                     transposed flag) in element order and applies the
//                     BackwardEuler coefficients S = (h^2+h beta)K + (1+h alpha)M
//   fused_block_kernel  optional fused row-chunk assembly (no element blocks
//                     in HBM)
//   rows_kernel       nodal internal force gather and BackwardEuler RHS
//   elem_kv_kernel, refine_*  iterative refinement of the mixed form
//   (pcg_kernel lives in pcg.cu)
//
// All reductions are in a fixed order: results are bit-reproducible run to run.
#include <cuda_runtime.h>

#include <cstdio>
#include <type_traits>

#include "device_math.cuh"
#include "spmv.cuh"
#include "engine.h"

namespace b200fem {

// ---------------------------------------------------------------------------
// constant shape tables
// ---------------------------------------------------------------------------
__constant__ double c_tet_gns[12];
__constant__ double c_hex_gns[8 * 8 * 3];  // [ip][node][3]
__constant__ double c_hex_wgns[8 * 3];     // warping point (centre)
__constant__ float c_tet_gns_f[12];
__constant__ float c_hex_gns_f[8 * 8 * 3];
__constant__ int c_pair_a[36], c_pair_b[36];
// wedges and pyramids: [ip][node][3] and the warping point [node][3]
__constant__ double c_wed_gns[6 * 6 * 3], c_wed_wgns[6 * 3];
__constant__ double c_pyr_gns[5 * 5 * 3], c_pyr_wgns[5 * 3];
__constant__ float c_wed_gns_f[6 * 6 * 3], c_pyr_gns_f[5 * 5 * 3];
// quadratic tets: 4 points x 10 nodes, warping point
__constant__ double c_qtet_gns[4 * 10 * 3], c_qtet_wgns[10 * 3];
__constant__ float c_qtet_gns_f[4 * 10 * 3];
// quadratic hexes: 14 points x 20 nodes, warping point
__constant__ double c_qhex_gns[14 * 20 * 3], c_qhex_wgns[20 * 3];
__constant__ float c_qhex_gns_f[14 * 20 * 3];
// quadratic wedges (9 points x 15 nodes) and pyramids (5 points x 13 nodes)
__constant__ double c_qwed_gns[9 * 15 * 3], c_qwed_wgns[15 * 3];
__constant__ double c_qpyr_gns[5 * 13 * 3], c_qpyr_wgns[13 * 3];
__constant__ float c_qwed_gns_f[9 * 15 * 3], c_qpyr_gns_f[5 * 13 * 3];

// ELEMENT soft incompressibility with several pressure values: pressure
// weights H [ip][value] and the weight matrix W (quadratic hexes: 4 values,
// quadratic wedges: 2)
__constant__ double c_qhex_H[14 * 4], c_qhex_W[4 * 4];
__constant__ double c_qwed_H[9 * 2], c_qwed_W[2 * 2];

static bool g_const_ready[64] = {false};

static cudaError_t ensure_constants(int device) {
  if (device >= 0 && device < 64 && g_const_ready[device]) return cudaSuccess;
  double tet[12] = {-1, -1, -1, 1, 0, 0, 0, 1, 0, 0, 0, 1};
  static const double node[8][3] = {{-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
                                    {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}};
  double hex[8 * 8 * 3], hexw[24];
  const double q = 1.0 / sqrt(3.0);
  auto grad = [&](double* g, int i, double s0, double s1, double s2) {
    double a = node[i][0], b = node[i][1], c = node[i][2];
    g[0] = 0.125 * a * (1 + b * s1) * (1 + c * s2);
    g[1] = 0.125 * (1 + a * s0) * b * (1 + c * s2);
    g[2] = 0.125 * (1 + a * s0) * (1 + b * s1) * c;
  };
  for (int k = 0; k < 8; k++)
    for (int i = 0; i < 8; i++) grad(&hex[(k * 8 + i) * 3], i, node[k][0] * q, node[k][1] * q, node[k][2] * q);
  for (int i = 0; i < 8; i++) grad(&hexw[i * 3], i, 0, 0, 0);
  float tetf[12], hexf[192];
  for (int i = 0; i < 12; i++) tetf[i] = (float)tet[i];
  for (int i = 0; i < 192; i++) hexf[i] = (float)hex[i];
  int pa[36], pb[36], w = 0;
  for (int a = 0; a < 8; a++)
    for (int b = a; b < 8; b++) { pa[w] = a; pb[w] = b; w++; }
  // wedge and pyramid tables from the host shape functions
  double wed[6 * 6 * 3], wedw[18], pyr[5 * 5 * 3], pyrw[15], wt;
  float wedf[108], pyrf[75];
  for (int k = 0; k < 6; k++) shape_grads(B200FEM_ELEM_WEDGE, k, &wed[k * 18], &wt);
  shape_grads(B200FEM_ELEM_WEDGE, -1, wedw, &wt);
  for (int k = 0; k < 5; k++) shape_grads(B200FEM_ELEM_PYRAMID, k, &pyr[k * 15], &wt);
  shape_grads(B200FEM_ELEM_PYRAMID, -1, pyrw, &wt);
  double qt[120], qtw[30];
  float qtf[120];
  for (int k = 0; k < 4; k++) shape_grads(B200FEM_ELEM_QUADTET, k, &qt[k * 30], &wt);
  shape_grads(B200FEM_ELEM_QUADTET, -1, qtw, &wt);
  for (int i = 0; i < 120; i++) qtf[i] = (float)qt[i];
  static double qh[840], qhw[60];
  static float qhf[840];
  for (int k = 0; k < 14; k++) shape_grads(B200FEM_ELEM_QUADHEX, k, &qh[k * 60], &wt);
  shape_grads(B200FEM_ELEM_QUADHEX, -1, qhw, &wt);
  for (int i = 0; i < 840; i++) qhf[i] = (float)qh[i];
  static double qw[405], qww[45], qp[195], qpw[39];
  static float qwf[405], qpf[195];
  for (int k = 0; k < 9; k++) shape_grads(B200FEM_ELEM_QUADWEDGE, k, &qw[k * 45], &wt);
  shape_grads(B200FEM_ELEM_QUADWEDGE, -1, qww, &wt);
  for (int k = 0; k < 5; k++) shape_grads(B200FEM_ELEM_QUADPYRAMID, k, &qp[k * 39], &wt);
  shape_grads(B200FEM_ELEM_QUADPYRAMID, -1, qpw, &wt);
  for (int i = 0; i < 405; i++) qwf[i] = (float)qw[i];
  for (int i = 0; i < 195; i++) qpf[i] = (float)qp[i];
  for (int i = 0; i < 108; i++) wedf[i] = (float)wed[i];
  for (int i = 0; i < 75; i++) pyrf[i] = (float)pyr[i];
  cudaError_t e;
  if ((e = cudaMemcpyToSymbol(c_qwed_gns, qw, sizeof(qw))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qwed_wgns, qww, sizeof(qww))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qwed_gns_f, qwf, sizeof(qwf))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qpyr_gns, qp, sizeof(qp))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qpyr_wgns, qpw, sizeof(qpw))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qpyr_gns_f, qpf, sizeof(qpf))) != cudaSuccess) return e;
  {
    double hh[14 * 4], hw[16], wh[9 * 2], ww[4];
    pressure_tables(B200FEM_ELEM_QUADHEX, hh, hw);
    pressure_tables(B200FEM_ELEM_QUADWEDGE, wh, ww);
    if ((e = cudaMemcpyToSymbol(c_qhex_H, hh, sizeof(hh))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_qhex_W, hw, sizeof(hw))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_qwed_H, wh, sizeof(wh))) != cudaSuccess) return e;
    if ((e = cudaMemcpyToSymbol(c_qwed_W, ww, sizeof(ww))) != cudaSuccess) return e;
  }
  if ((e = cudaMemcpyToSymbol(c_qhex_gns, qh, sizeof(qh))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qhex_wgns, qhw, sizeof(qhw))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qhex_gns_f, qhf, sizeof(qhf))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qtet_gns, qt, sizeof(qt))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qtet_wgns, qtw, sizeof(qtw))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_qtet_gns_f, qtf, sizeof(qtf))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_wed_gns, wed, sizeof(wed))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_wed_wgns, wedw, sizeof(wedw))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_pyr_gns, pyr, sizeof(pyr))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_pyr_wgns, pyrw, sizeof(pyrw))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_wed_gns_f, wedf, sizeof(wedf))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_pyr_gns_f, pyrf, sizeof(pyrf))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_tet_gns, tet, sizeof(tet))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_hex_gns, hex, sizeof(hex))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_hex_wgns, hexw, sizeof(hexw))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_tet_gns_f, tetf, sizeof(tetf))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_hex_gns_f, hexf, sizeof(hexf))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_pair_a, pa, sizeof(pa))) != cudaSuccess) return e;
  if ((e = cudaMemcpyToSymbol(c_pair_b, pb, sizeof(pb))) != cudaSuccess) return e;
  if (device >= 0 && device < 64) g_const_ready[device] = true;
  return cudaSuccess;
}

// pair index w of (a, b), a <= b, enumerated row-major over the upper
// triangle of the nen x nen element matrix
template <int NEN>
__device__ __forceinline__ void pair_of(int w, int& a, int& b) {
  if constexpr (NEN == 8) {
    a = c_pair_a[w];
    b = c_pair_b[w];
  } else if constexpr (NEN == 4) {
    // 4-node table: (0,0)(0,1)(0,2)(0,3)(1,1)(1,2)(1,3)(2,2)(2,3)(3,3)
    const int ta[10] = {0, 0, 0, 0, 1, 1, 1, 2, 2, 3};
    const int tb[10] = {0, 1, 2, 3, 1, 2, 3, 2, 3, 3};
    a = ta[w];
    b = tb[w];
  } else {
    // row a of the upper triangle holds NEN - a pairs
    a = 0;
    while (w >= NEN - a) {
      w -= NEN - a;
      a++;
    }
    b = a + w;
  }
}

// dN_n/ds component c at integration point k
template <typename T, int TYPE>
__device__ __forceinline__ T gns(int k, int n, int c) {
  if constexpr (TYPE == B200FEM_ELEM_TET) {
    if constexpr (sizeof(T) == 8) return c_tet_gns[3 * n + c];
    else return c_tet_gns_f[3 * n + c];
  } else if constexpr (TYPE == B200FEM_ELEM_HEX) {
    if constexpr (sizeof(T) == 8) return c_hex_gns[(k * 8 + n) * 3 + c];
    else return c_hex_gns_f[(k * 8 + n) * 3 + c];
  } else if constexpr (TYPE == B200FEM_ELEM_WEDGE) {
    if constexpr (sizeof(T) == 8) return c_wed_gns[(k * 6 + n) * 3 + c];
    else return c_wed_gns_f[(k * 6 + n) * 3 + c];
  } else if constexpr (TYPE == B200FEM_ELEM_QUADTET) {
    if constexpr (sizeof(T) == 8) return c_qtet_gns[(k * 10 + n) * 3 + c];
    else return c_qtet_gns_f[(k * 10 + n) * 3 + c];
  } else if constexpr (TYPE == B200FEM_ELEM_QUADHEX) {
    if constexpr (sizeof(T) == 8) return c_qhex_gns[(k * 20 + n) * 3 + c];
    else return c_qhex_gns_f[(k * 20 + n) * 3 + c];
  } else if constexpr (TYPE == B200FEM_ELEM_QUADWEDGE) {
    if constexpr (sizeof(T) == 8) return c_qwed_gns[(k * 15 + n) * 3 + c];
    else return c_qwed_gns_f[(k * 15 + n) * 3 + c];
  } else if constexpr (TYPE == B200FEM_ELEM_QUADPYRAMID) {
    if constexpr (sizeof(T) == 8) return c_qpyr_gns[(k * 13 + n) * 3 + c];
    else return c_qpyr_gns_f[(k * 13 + n) * 3 + c];
  } else {
    if constexpr (sizeof(T) == 8) return c_pyr_gns[(k * 5 + n) * 3 + c];
    else return c_pyr_gns_f[(k * 5 + n) * 3 + c];
  }
}

// dN_n/ds at the warping point (StiffnessWarper3d: TetElement integration
// point 0, HexElement centre, WedgeElement (1/3, 1/3, 0), PyramidElement
// (0, 0, -1/2), QuadtetElement the linear tet's gradients on its corners)
template <int TYPE>
__device__ __forceinline__ double wgns(int n, int c) {
  if constexpr (TYPE == B200FEM_ELEM_TET) return c_tet_gns[3 * n + c];
  else if constexpr (TYPE == B200FEM_ELEM_HEX) return c_hex_wgns[3 * n + c];
  else if constexpr (TYPE == B200FEM_ELEM_WEDGE) return c_wed_wgns[3 * n + c];
  else if constexpr (TYPE == B200FEM_ELEM_QUADTET) return c_qtet_wgns[3 * n + c];
  else if constexpr (TYPE == B200FEM_ELEM_QUADHEX) return c_qhex_wgns[3 * n + c];
  else if constexpr (TYPE == B200FEM_ELEM_QUADWEDGE) return c_qwed_wgns[3 * n + c];
  else if constexpr (TYPE == B200FEM_ELEM_QUADPYRAMID) return c_qpyr_wgns[3 * n + c];
  else return c_pyr_wgns[3 * n + c];
}

// integration weight of point k (TetElement 1/6; HexElement Gauss 1;
// WedgeElement 1/6; PyramidElement 81/100 for the four base points, 125/27
// for the fifth; QuadtetElement 0.25/6; QuadhexElement 0.335180055401662 at
// the eight corner points, 0.886426592797784 at the six face points)
template <typename T, int TYPE>
__device__ __forceinline__ T ip_weight(int k) {
  if constexpr (TYPE == B200FEM_ELEM_TET || TYPE == B200FEM_ELEM_WEDGE) return T(1.0 / 6.0);
  else if constexpr (TYPE == B200FEM_ELEM_QUADTET) return T(0.25 / 6.0);
  else if constexpr (TYPE == B200FEM_ELEM_QUADHEX) return k < 8 ? T(0.335180055401662) : T(0.886426592797784);
  else if constexpr (TYPE == B200FEM_ELEM_QUADWEDGE) return k < 6 ? T(5 / 54.0) : T(8 / 54.0);
  else if constexpr (TYPE == B200FEM_ELEM_QUADPYRAMID) return k < 4 ? T(81 / 100.0) : T(125 / 27.0);
  else if constexpr (TYPE == B200FEM_ELEM_HEX) return T(1);
  else return k < 4 ? T(81 / 100.0) : T(125 / 27.0);
}

// lanes per element in the FP64 force kernel
__host__ __device__ constexpr int force_slot(int type) {
  return elem_nip(type) > 8 ? 16 : (elem_nip(type) > 1 ? 8 : 1);
}

// calls f(std::integral_constant<int, TYPE>) for the run-time element type
// pressure weight H_l at integration point k and weight-matrix entry W_ij
// of a multi-pressure element type (1 for the one-pressure types)
template <int TYPE>
__device__ __forceinline__ double press_H(int k, int l) {
  if constexpr (TYPE == B200FEM_ELEM_QUADHEX) return c_qhex_H[k * 4 + l];
  else if constexpr (TYPE == B200FEM_ELEM_QUADWEDGE) return c_qwed_H[k * 2 + l];
  else return 1.0;
}
template <int TYPE>
__device__ __forceinline__ double press_W(int i, int j) {
  if constexpr (TYPE == B200FEM_ELEM_QUADHEX) return c_qhex_W[i * 4 + j];
  else if constexpr (TYPE == B200FEM_ELEM_QUADWEDGE) return c_qwed_W[i * 2 + j];
  else return 1.0;
}
// the pressure at integration point k: sum_l H_l p_l over the element's
// values (FemModel3d.java:3465-3471); one value: the element's pressure
template <int TYPE>
__device__ __forceinline__ double elem_point_pressure(const double* elem_p, int e, int k) {
  constexpr int NPV = elem_npv(TYPE);
  if constexpr (NPV == 1) {
    return elem_p[e];
  } else {
    double pr = 0;
#pragma unroll
    for (int l = 0; l < NPV; l++) pr += press_H<TYPE>(k, l) * elem_p[(size_t)e * NPV + l];
    return pr;
  }
}

template <typename F>
static cudaError_t by_elem_type(int type, F&& f) {
  switch (type) {
    case B200FEM_ELEM_TET: return f(std::integral_constant<int, B200FEM_ELEM_TET>{});
    case B200FEM_ELEM_HEX: return f(std::integral_constant<int, B200FEM_ELEM_HEX>{});
    case B200FEM_ELEM_WEDGE: return f(std::integral_constant<int, B200FEM_ELEM_WEDGE>{});
    case B200FEM_ELEM_PYRAMID: return f(std::integral_constant<int, B200FEM_ELEM_PYRAMID>{});
    case B200FEM_ELEM_QUADTET: return f(std::integral_constant<int, B200FEM_ELEM_QUADTET>{});
    case B200FEM_ELEM_QUADHEX: return f(std::integral_constant<int, B200FEM_ELEM_QUADHEX>{});
    case B200FEM_ELEM_QUADWEDGE: return f(std::integral_constant<int, B200FEM_ELEM_QUADWEDGE>{});
    case B200FEM_ELEM_QUADPYRAMID: return f(std::integral_constant<int, B200FEM_ELEM_QUADPYRAMID>{});
    default: return cudaErrorInvalidValue;
  }
}

// ordered-bits min for doubles (atomicMin on the int64 image of a double
// works for non-negative and negative values with this mapping)
__device__ __forceinline__ long long dbl_order(double v) {
  long long i = __double_as_longlong(v);
  return i >= 0 ? i : (i ^ 0x7fffffffffffffffll);
}

// Inverted-element count and smallest detJ, aggregated over a warp before
// the atomics: every element thread updating the same two words would
// serialise on them.  All 32 lanes of the warp call it.
__device__ __forceinline__ void warp_record_det(int* flags, long long* mindet, double det, int inv) {
  const int tot = __reduce_add_sync(0xffffffffu, inv);
  double d = det;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) d = fmin(d, __shfl_xor_sync(0xffffffffu, d, off));
  if ((threadIdx.x & 31) == 0) {
    if (tot) atomicAdd(&flags[1], tot);
    if (d < 1.0e300) atomicMin(mindet, dbl_order(d));
  }
}

// soft incompressibility of an element group (template argument INC)
constexpr int kIncOff = 0, kIncNodal = 1, kIncElement = 2;

struct ElemArgs;
__device__ bool block_inactive(const ElemArgs& a, int ebase, int epb);

struct ElemArgs {
  int e0, e1;
  const int* conn;
  const int* elem_model;
  const int* elem_mat;     // per element: its row of mat
  const double* x;
  const double* invJ0;
  const float* invJ0_f;
  const double* winvJ0;
  const double* K0;
  const double* f0;
  const int* sidx;
  const double* mat;       // kMatParams per row
  const double* node_p;    // NODAL pressures (or null)
  const double* elem_p;    // ELEMENT pressures (or null)
  const double* elem_r;    // ELEMENT Rinv = effective modulus / rest volume (or null)
  const int* active;       // per model: 0 = left out of this assembly (or null: all)
  void* elemK;             // T* E*npair*9
  void* elemF;             // T* E*nen*3
  int* flags;              // [err, inverted]
  long long* mindet;       // ordered bits
  int det_stats;           // the FP64 force kernel records inverted elements / min detJ
};

// Whole-block exit when none of the block's elements belongs to an active
// model (elements of a group are in model order, so blocks rarely mix).
// Called before any shared-memory use; the block returns as a whole.
__device__ bool block_inactive(const ElemArgs& a, int ebase, int epb) {
  if (!a.active) return false;
  bool mine = false;
  for (int t = threadIdx.x; t < epb; t += blockDim.x) {
    const int e = ebase + t;
    mine |= e < a.e1 && a.active[a.elem_model[e]] != 0;
  }
  return !__syncthreads_or(mine);
}

// ---------------------------------------------------------------------------
// non-linear materials (NeoHookean, MooneyRivlin, StVenantKirchhoff), every
// element type
// ---------------------------------------------------------------------------
// Shared-memory layout of the non-linear element kernel (one record per
// integration point: shape gradients, dv, stress, tangent).
template <int TYPE, int MAT, typename T, int EPB>
struct ElemSmem {
  static constexpr int NEN = elem_nen(TYPE);
  static constexpr int NIP = elem_nip(TYPE);
  static constexpr int DS = MAT == B200FEM_MAT_NEOHOOKEAN ? 2 : 36;
  static constexpr int NREC = EPB * NIP;
  static constexpr size_t bytes() {
    return sizeof(T) * ((size_t)EPB * NEN * 3 + (size_t)NREC * (NEN * 3 + 1 + 6 + DS)) + sizeof(int) * EPB * NEN;
  }
};

// two CTAs per SM (128 registers) except for FP64 quadratic hexes and
// wedges (20 and 15 nodes), whose point records and pair sums spilled 100 to
// 1,000 bytes at 128: one CTA per SM and up to 255 registers (update of a
// 24x6x6 beam, B200: quadratic hex MooneyRivlin with four pressure values
// 138 -> 108 us, NeoHookean 61 -> 57 us, quadratic wedge 92 -> 89 us).  The
// 10- and 13-node elements keep two CTAs: quadratic tets measured the same
// either way, quadratic pyramids 53 us at two CTAs against 58 at one.
template <int TYPE, int MAT, int INC, typename T>
constexpr int elem_min_ctas() {
  return (elem_nen(TYPE) >= 15 && sizeof(T) == 8) ? 1 : 2;
}

template <int TYPE, int MAT, int INC, typename T, int EPB>
__global__ void __launch_bounds__(256, (elem_min_ctas<TYPE, MAT, INC, T>())) elem_nonlinear_kernel(ElemArgs a) {
  using SM = ElemSmem<TYPE, MAT, T, EPB>;
  constexpr int NEN = SM::NEN;
  constexpr int NIP = SM::NIP;
  constexpr int NPAIR = NEN * (NEN + 1) / 2;
  constexpr int DS = SM::DS;
  constexpr int NREC = SM::NREC;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T(*sx)[NEN][3] = reinterpret_cast<T(*)[NEN][3]>(smem_raw);
  T(*sg)[NEN][3] = reinterpret_cast<T(*)[NEN][3]>(smem_raw + sizeof(T) * EPB * NEN * 3);
  T* sdv = reinterpret_cast<T*>(smem_raw + sizeof(T) * ((size_t)EPB * NEN * 3 + (size_t)NREC * NEN * 3));
  T(*ssig)[6] = reinterpret_cast<T(*)[6]>(sdv + NREC);
  T(*sD)[DS] = reinterpret_cast<T(*)[DS]>(sdv + NREC + NREC * 6);
  int(*snode)[NEN] = reinterpret_cast<int(*)[NEN]>(sdv + NREC + NREC * 6 + NREC * DS);
  const int ebase = a.e0 + blockIdx.x * EPB;
  if (block_inactive(a, ebase, EPB)) return;
  // stage 0: coalesced connectivity + coordinate loads.  In FP32 the
  // coordinates are taken relative to the element's first node in FP64 so
  // the Jacobian keeps full single precision.
  for (int t = threadIdx.x; t < EPB * NEN; t += blockDim.x) {
    int el = t / NEN, n = t % NEN, e = ebase + el;
    if (e < a.e1) snode[el][n] = a.conn[(size_t)e * NEN + n];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < EPB * NEN * 3; t += blockDim.x) {
    int el = t / (NEN * 3), r = t % (NEN * 3), n = r / 3, c = r % 3, e = ebase + el;
    if (e < a.e1) {
      double v = a.x[3 * (size_t)snode[el][n] + c];
      if constexpr (sizeof(T) == 4) v -= a.x[3 * (size_t)snode[el][0] + c];
      sx[el][n][c] = (T)v;
    }
  }
  __syncthreads();
  // stage 1: one thread per (element, integration point)
  double mydet = 1.0e300;
  int myinv = 0;
  for (int t = threadIdx.x; t < EPB * NIP; t += blockDim.x) {
    int el = t / NIP, k = t % NIP, e = ebase + el;
    if (e >= a.e1) continue;
    T J[9];
#pragma unroll
    for (int i = 0; i < 9; i++) J[i] = T(0);
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      T g0 = gns<T, TYPE>(k, n, 0), g1 = gns<T, TYPE>(k, n, 1), g2 = gns<T, TYPE>(k, n, 2);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        T p = sx[el][n][r];
        J[3 * r] += p * g0;
        J[3 * r + 1] += p * g1;
        J[3 * r + 2] += p * g2;
      }
    }
    T iJ0[9];
    if constexpr (sizeof(T) == 8) {
#pragma unroll
      for (int i = 0; i < 9; i++) iJ0[i] = a.invJ0[((size_t)e * NIP + k) * 9 + i];
    } else {
#pragma unroll
      for (int i = 0; i < 9; i++) iJ0[i] = a.invJ0_f[((size_t)e * NIP + k) * 9 + i];
    }
    T F[9], invJ[9];
    matmul3(F, J, iJ0);
    T detF = det3(F);
    T detJ = invert3(invJ, J);
    myinv += !(detJ > T(0));
    mydet = fmin(mydet, (double)detJ);
    const T w = ip_weight<T, TYPE>(k);
    T dv = detJ * w;
    sdv[t] = dv;
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      T g0 = gns<T, TYPE>(k, n, 0), g1 = gns<T, TYPE>(k, n, 1), g2 = gns<T, TYPE>(k, n, 2);
#pragma unroll
      for (int c = 0; c < 3; c++) sg[t][n][c] = invJ[c] * g0 + invJ[3 + c] * g1 + invJ[6 + c] * g2;
    }
    const double* mp = a.mat + (size_t)a.elem_mat[e] * kMatParams;
    if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) {
      T aa, bb;
      neohookean_point<T>(ssig[t], &aa, &bb, (T)mp[0], (T)mp[1], F, detF);
      sD[t][0] = aa;
      sD[t][1] = bb;
    } else {
      T pr = T(0);
      if constexpr (INC == kIncNodal) {
        if (TYPE == B200FEM_ELEM_TET) {
          double s = 0;
#pragma unroll
          for (int n = 0; n < NEN; n++) s += a.node_p[snode[el][n]];
          pr = (T)(s / NEN);
        } else {
          pr = (T)a.node_p[snode[el][k]];
        }
      } else if constexpr (INC == kIncElement) {
        pr = (T)elem_point_pressure<TYPE>(a.elem_p, e, k);
      }
      T mpt[8];
#pragma unroll
      for (int i = 0; i < 8; i++) mpt[i] = (T)mp[i];
      material_point<MAT, T>(ssig[t], sD[t], mpt, F, detF, pr);
    }
  }
  warp_record_det(a.flags, a.mindet, mydet, myinv);
  __syncthreads();
  // stage 2: one thread per element pair block, then per node force (the
  // FP32 form leaves the forces to the FP64 force kernel)
  constexpr int NF = sizeof(T) == 8 ? NEN : 0;
  T* elemK = (T*)a.elemK;
  double* elemF = (double*)a.elemF;
  for (int t = threadIdx.x; t < EPB * (NPAIR + NF); t += blockDim.x) {
    int el = t / (NPAIR + NF), w = t % (NPAIR + NF), e = ebase + el;
    if (e >= a.e1) continue;
    if (w < NPAIR) {
      int ia, ib;
      pair_of<NEN>(w, ia, ib);
      T K[9];
#pragma unroll
      for (int i = 0; i < 9; i++) K[i] = T(0);
#pragma unroll
      for (int k = 0; k < NIP; k++) {
        int s = el * NIP + k;
        if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN)
          add_bdb_iso(K, sg[s][ia], sD[s][0], sD[s][1], sg[s][ib], sdv[s]);
        else
          add_bdb(K, sg[s][ia], sD[s], sg[s][ib], sdv[s]);
        add_geometric(K, sg[s][ia], ssig[s], sg[s][ib], sdv[s]);
      }
      if constexpr (INC == kIncElement && elem_npv(TYPE) == 1) {
        // ELEMENT dilational stiffness Rinv c_a c_b^T, c = sum_k GNx dv
        // (FemModel3d.java:3650-3663, FemUtilities.addToIncompressConstraints)
        T ca[3] = {T(0), T(0), T(0)}, cb[3] = {T(0), T(0), T(0)};
#pragma unroll
        for (int k = 0; k < NIP; k++) {
          const int s = el * NIP + k;
#pragma unroll
          for (int c = 0; c < 3; c++) {
            ca[c] += sg[s][ia][c] * sdv[s];
            cb[c] += sg[s][ib][c] * sdv[s];
          }
        }
        const T r = (T)a.elem_r[e];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) K[3 * i + j] += r * ca[i] * cb[j];
      } else if constexpr (INC == kIncElement) {
        // several pressure values: constraints c^l = sum_k H_l GNx dv
        // (3 x npv per node) and K_ab += c_a Rinv c_b^T, formed as
        // X = Rinv c_b^T, K += c_a X (FemUtilities.addDilationalStiffness,
        // FemUtilities.java:317-342)
        constexpr int NPV = elem_npv(TYPE);
        T ca[3][NPV], cb[3][NPV];
#pragma unroll
        for (int c = 0; c < 3; c++)
#pragma unroll
          for (int l = 0; l < NPV; l++) ca[c][l] = cb[c][l] = T(0);
#pragma unroll
        for (int k = 0; k < NIP; k++) {
          const int s = el * NIP + k;
#pragma unroll
          for (int l = 0; l < NPV; l++) {
            const T hd = (T)press_H<TYPE>(k, l) * sdv[s];
#pragma unroll
            for (int c = 0; c < 3; c++) {
              ca[c][l] += hd * sg[s][ia][c];
              cb[c][l] += hd * sg[s][ib][c];
            }
          }
        }
        const double* Rv = a.elem_r + (size_t)e * NPV * NPV;
#pragma unroll
        for (int q = 0; q < 3; q++) {
          T X[NPV];
#pragma unroll
          for (int l = 0; l < NPV; l++) {
            T xq = T(0);
#pragma unroll
            for (int m = 0; m < NPV; m++) xq += (T)Rv[l * NPV + m] * cb[q][m];
            X[l] = xq;
          }
#pragma unroll
          for (int r = 0; r < 3; r++) {
            T acc = T(0);
#pragma unroll
            for (int l = 0; l < NPV; l++) acc += ca[r][l] * X[l];
            K[3 * r + q] += acc;
          }
        }
      }
      T* out = elemK + ((size_t)e * NPAIR + w) * 9;
#pragma unroll
      for (int i = 0; i < 9; i++) out[i] = K[i];
    } else {
      int n = w - NPAIR;
      T f[3] = {T(0), T(0), T(0)};
#pragma unroll
      for (int k = 0; k < NIP; k++) {
        int s = el * NIP + k;
        add_stress_force(f, sg[s][n], ssig[s], sdv[s]);
      }
      double* out = elemF + ((size_t)e * NEN + n) * 3;
      out[0] = f[0];
      out[1] = f[1];
      out[2] = f[2];
    }
  }
}

// ---------------------------------------------------------------------------
// linear materials (corotated or not): cached rest stiffness K0, force
// R (K0 R^T x - f0) and stiffness R K0 R^T (StiffnessWarper3d.java:154-307)
// ---------------------------------------------------------------------------
template <int TYPE, typename T>
__global__ void __launch_bounds__(256) elem_linear_kernel(ElemArgs a, int corotated) {
  constexpr int NEN = elem_nen(TYPE);
  constexpr int NPAIR = NEN * (NEN + 1) / 2;
  constexpr int EPB = TYPE == B200FEM_ELEM_TET ? 32 : 8;
  __shared__ double sx[EPB][NEN][3];
  __shared__ double sR[EPB][9];
  __shared__ int snode[EPB][NEN];
  const int ebase = a.e0 + blockIdx.x * EPB;
  if (block_inactive(a, ebase, EPB)) return;
  for (int t = threadIdx.x; t < EPB * NEN; t += blockDim.x) {
    int el = t / NEN, n = t % NEN, e = ebase + el;
    if (e < a.e1) snode[el][n] = a.conn[(size_t)e * NEN + n];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < EPB * NEN * 3; t += blockDim.x) {
    int el = t / (NEN * 3), r = t % (NEN * 3), n = r / 3, c = r % 3, e = ebase + el;
    if (e < a.e1) sx[el][n][c] = a.x[3 * (size_t)snode[el][n] + c];
  }
  __syncthreads();
  for (int el = threadIdx.x; el < EPB; el += blockDim.x) {
    int e = ebase + el;
    if (e >= a.e1) continue;
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (corotated) {
      // F at the warping point (TetElement: integration point 0; HexElement:
      // centre) -- StiffnessWarper3d.computeWarpingRotation (:154-159)
      double J[9];
#pragma unroll
      for (int i = 0; i < 9; i++) J[i] = 0;
#pragma unroll
      for (int n = 0; n < NEN; n++) {
        const double g0 = wgns<TYPE>(n, 0), g1 = wgns<TYPE>(n, 1), g2 = wgns<TYPE>(n, 2);
#pragma unroll
        for (int r = 0; r < 3; r++) {
          J[3 * r] += sx[el][n][r] * g0;
          J[3 * r + 1] += sx[el][n][r] * g1;
          J[3 * r + 2] += sx[el][n][r] * g2;
        }
      }
      double W[9], F[9];
#pragma unroll
      for (int i = 0; i < 9; i++) W[i] = a.winvJ0[(size_t)e * 9 + i];
      matmul3(F, J, W);
      polar_rotation(F, R);
    }
#pragma unroll
    for (int i = 0; i < 9; i++) sR[el][i] = R[i];
  }
  __syncthreads();
  T* elemK = (T*)a.elemK;
  double* elemF = (double*)a.elemF;
  for (int t = threadIdx.x; t < EPB * (NPAIR + NEN); t += blockDim.x) {
    int el = t / (NPAIR + NEN), w = t % (NPAIR + NEN), e = ebase + el;
    if (e >= a.e1) continue;
    const double* R = sR[el];
    const double* K0 = a.K0 + (size_t)e * NEN * NEN * 9;
    if (w < NPAIR) {
      int ia, ib;
      pair_of<NEN>(w, ia, ib);
      const double* Kab = K0 + (ia * NEN + ib) * 9;
      double out9[9];
      if (corotated) {
        // R K R^T (StiffnessWarper3d.rotateStiffness, :219-222)
        double Tm[9];
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++)
            Tm[3 * i + j] = Kab[3 * i] * R[3 * j] + Kab[3 * i + 1] * R[3 * j + 1] + Kab[3 * i + 2] * R[3 * j + 2];
        matmul3(out9, R, Tm);
      } else {
#pragma unroll
        for (int i = 0; i < 9; i++) out9[i] = Kab[i];
      }
      T* out = elemK + ((size_t)e * NPAIR + w) * 9;
#pragma unroll
      for (int i = 0; i < 9; i++) out[i] = (T)out9[i];
    } else {
      int n = w - NPAIR;
      double acc[3] = {0, 0, 0};
      if (a.sidx[snode[el][n]] >= 0) {
        for (int j = 0; j < NEN; j++) {
          double pos[3];
          if (corotated) {
#pragma unroll
            for (int r = 0; r < 3; r++)
              pos[r] = R[r] * sx[el][j][0] + R[3 + r] * sx[el][j][1] + R[6 + r] * sx[el][j][2];
          } else {
            pos[0] = sx[el][j][0]; pos[1] = sx[el][j][1]; pos[2] = sx[el][j][2];
          }
          const double* Kij = K0 + (n * NEN + j) * 9;
#pragma unroll
          for (int r = 0; r < 3; r++) acc[r] += Kij[3 * r] * pos[0] + Kij[3 * r + 1] * pos[1] + Kij[3 * r + 2] * pos[2];
        }
        const double* f0 = a.f0 + ((size_t)e * NEN + n) * 3;
#pragma unroll
        for (int r = 0; r < 3; r++) acc[r] -= f0[r];
        if (corotated) {
          double t2[3];
#pragma unroll
          for (int r = 0; r < 3; r++) t2[r] = R[3 * r] * acc[0] + R[3 * r + 1] * acc[1] + R[3 * r + 2] * acc[2];
          acc[0] = t2[0]; acc[1] = t2[1]; acc[2] = t2[2];
        }
      }
      double* out = elemF + ((size_t)e * NEN + n) * 3;
      out[0] = acc[0];
      out[1] = acc[1];
      out[2] = acc[2];
    }
  }
}

// ---------------------------------------------------------------------------
// block gather: one thread per upper block (diagonal included), taken from
// the list of the pattern's upper blocks, so every lane of a warp sums a
// block.  The sums: the contribution list in element order, then the NODAL
// dilational triples node-ascending.  The matrix is symmetric: a lower
// block's list holds the same contributions in the same order, transposed,
// so each upper block also writes its transpose to the mirror position
// (FemModel3d.java:3003-3026) and lower blocks are never summed.
// ---------------------------------------------------------------------------
template <typename TK, typename TO>
__global__ void __launch_bounds__(256) gather_block_kernel(
    long long n_up, const int* __restrict__ up, const int* __restrict__ cptr, const int* __restrict__ cidx,
    const TK* __restrict__ elemK, const int* __restrict__ blk_row, const int* __restrict__ blk_diag,
    const int* __restrict__ row_model, const int* __restrict__ act_node, const double* __restrict__ mass,
    const double* __restrict__ step, int mode, TO* __restrict__ out, const int* __restrict__ dptr,
    const int* __restrict__ didx, const double* __restrict__ divblk, const double* __restrict__ node_kp,
    const int* __restrict__ active, const int* __restrict__ mirror, const int* __restrict__ dst,
    const int* __restrict__ mdst) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n_up) return;
  const int p = up[q];
  const int row = blk_row[p];
  if (active && !active[row_model[row]]) return;  // blocks of models left out stay
  // output positions: the block's own and its transpose's, or (the factored
  // NODAL solve matrix) their places in S1
  const int op = dst ? dst[q] : p;
  const int mp = dst ? mdst[q] : mirror[p];
  double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const int c1 = cptr[p + 1];
  for (int c = cptr[p]; c < c1; c++) {
    const int code = cidx[c];
    const TK* B = elemK + (size_t)(code >> 1) * 9;
    double b[9];
#pragma unroll
    for (int k = 0; k < 9; k++) b[k] = (double)B[k];
    if (code & 1) {
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) s[3 * i + j] += b[3 * j + i];
    } else {
#pragma unroll
      for (int k = 0; k < 9; k++) s[k] += b[k];
    }
  }
  if (dptr) {
    // NODAL dilational term sum_n kp_n divBlk(n,i) divBlk(n,j)^T, n ascending
    // (FemModel3d.computeNodalIncompressibility, FemModel3d.java:2632-2669)
    double sd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int d1 = dptr[p + 1];
    for (int t = dptr[p]; t < d1; t++) {
      const int* tr = didx + 3 * (size_t)t;
      const double kp = node_kp[tr[2]];
      const double* di = divblk + 3 * (size_t)tr[0];
      const double* dj = divblk + 3 * (size_t)tr[1];
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) sd[3 * r + c] += kp * di[r] * dj[c];
    }
#pragma unroll
    for (int k = 0; k < 9; k++) s[k] += sd[k];
  }
  TO v[9];
  if (mode == 0) {
#pragma unroll
    for (int k = 0; k < 9; k++) v[k] = (TO)s[k];  // plain stiffness K
  } else {
    const double* sp = step + (size_t)row_model[row] * 8;
    const double h = sp[0], al = sp[1], be = sp[2];
    // addPosJacobian (h^2 K), addVelJacobian (h beta K + h alpha M),
    // addActiveMassMatrix (M)  (MechSystemSolver.java:2277,2312,2334)
    const double cm = p == blk_diag[row] ? (1.0 + h * al) * mass[act_node[row]] : 0.0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double val = (h * h + h * be) * s[k];
      if (k % 4 == 0) val += cm;
      v[k] = (TO)val;
    }
  }
  TO* o = out + (size_t)op * 9;
#pragma unroll
  for (int k = 0; k < 9; k++) o[k] = v[k];
  if (mp != op) {
    // off-diagonal: no mass term; the mirror is the transpose
    TO* t = out + (size_t)mp * 9;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) t[3 * i + j] = v[3 * j + i];
  }
}

// ---------------------------------------------------------------------------
// block gather for matrices that stay in L2: one thread per block, the warp's
// 32 consecutive blocks staged in shared memory and stored as contiguous lines
// (the threads of lower blocks only store).
// Same sums in the same order as one thread per entry: the contribution list
// in element order, then the NODAL dilational triples node-ascending.  The
// matrix is symmetric: a lower block's list holds the same contributions in
// the same order, transposed, so each upper block also writes its transpose
// to the mirror position (FemModel3d.java:3003-3026) and lower blocks are
// not summed.
// ---------------------------------------------------------------------------
template <typename TK, typename TO>
__global__ void __launch_bounds__(256) gather_staged_kernel(
    long long nnzb, const int* __restrict__ cptr, const int* __restrict__ cidx, const TK* __restrict__ elemK,
    const int* __restrict__ blk_row, const int* __restrict__ blk_diag, const int* __restrict__ row_model,
    const int* __restrict__ act_node, const double* __restrict__ mass, const double* __restrict__ step, int mode,
    TO* __restrict__ out, const int* __restrict__ dptr, const int* __restrict__ didx,
    const double* __restrict__ divblk, const double* __restrict__ node_kp, const int* __restrict__ active,
    const int* __restrict__ mirror) {
  __shared__ TO stage[8][32 * 9];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long wbase = ((long long)blockIdx.x * 8 + warp) * 32;
  const long long p = wbase + lane;
  TO* my = stage[warp] + lane * 9;
  bool live = p < nnzb;
  int row = 0, mp = -1;
  if (live) {
    row = blk_row[p];
    mp = mirror[p];
    if (active && !active[row_model[row]]) live = false;
  }
  const bool lower = mp >= 0 && mp < p;  // written by its upper block
  if (live && !lower) {
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int c1 = cptr[p + 1];
    for (int c = cptr[p]; c < c1; c++) {
      const int code = cidx[c];
      const TK* B = elemK + (size_t)(code >> 1) * 9;
      double b[9];
#pragma unroll
      for (int k = 0; k < 9; k++) b[k] = (double)B[k];
      if (code & 1) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) s[3 * i + j] += b[3 * j + i];
      } else {
#pragma unroll
        for (int k = 0; k < 9; k++) s[k] += b[k];
      }
    }
    if (dptr) {
      // NODAL dilational term sum_n kp_n divBlk(n,i) divBlk(n,j)^T, n ascending
      // (FemModel3d.computeNodalIncompressibility, FemModel3d.java:2632-2669)
      double sd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      const int d1 = dptr[p + 1];
      for (int t = dptr[p]; t < d1; t++) {
        const int* tr = didx + 3 * (size_t)t;
        const double kp = node_kp[tr[2]];
        const double* di = divblk + 3 * (size_t)tr[0];
        const double* dj = divblk + 3 * (size_t)tr[1];
#pragma unroll
        for (int r = 0; r < 3; r++)
#pragma unroll
          for (int c = 0; c < 3; c++) sd[3 * r + c] += kp * di[r] * dj[c];
      }
#pragma unroll
      for (int k = 0; k < 9; k++) s[k] += sd[k];
    }
    if (mode == 0) {
#pragma unroll
      for (int k = 0; k < 9; k++) my[k] = (TO)s[k];  // plain stiffness K
      if (mp != p) {
        TO* t = out + (size_t)mp * 9;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) t[3 * i + j] = (TO)s[3 * j + i];
      }
    } else {
      const double* sp = step + (size_t)row_model[row] * 8;
      const double h = sp[0], al = sp[1], be = sp[2];
      // addPosJacobian (h^2 K), addVelJacobian (h beta K + h alpha M),
      // addActiveMassMatrix (M)  (MechSystemSolver.java:2277,2312,2334)
      const double cm = p == blk_diag[row] ? (1.0 + h * al) * mass[act_node[row]] : 0.0;
#pragma unroll
      for (int k = 0; k < 9; k++) {
        double val = (h * h + h * be) * s[k];
        if (k % 4 == 0) val += cm;
        my[k] = (TO)val;
      }
      if (mp != p) {
        // off-diagonal: no mass term; the mirror is the transpose
        TO* t = out + (size_t)mp * 9;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) t[3 * i + j] = my[3 * j + i];
      }
    }
  }
  __syncwarp();
  // contiguous stores of the warp's blocks (blocks of models left out stay)
  const long long nv = nnzb - wbase < 32 ? nnzb - wbase : 32;
  if (nv <= 0) return;
  TO* o = out + (size_t)wbase * 9;
  for (int i = lane; i < nv * 9; i += 32) {
    const long long q = wbase + i / 9;
    if (active && !active[row_model[blk_row[q]]]) continue;
    const int mq = mirror[q];
    if (mq >= 0 && mq < q) continue;  // lower block: written by its mirror
    o[i] = stage[warp][i];
  }
}

// ---------------------------------------------------------------------------
// nodal forces and BackwardEuler right-hand side
//   f_int(n) = sum of element stress forces at n
//   b = M v0 + h (m g + f_ext - f_int)
// (the mass- and stiffness-damping terms of updateNodeForces and the
// b += (h alpha M + h beta K) v0 term of backwardEuler cancel exactly,
// MechSystemSolver.java:2194-2301, FemModel3d.java:2783-2843)
// ---------------------------------------------------------------------------
template <typename TF>
__global__ void rows_kernel(int N, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx,
                            const TF* __restrict__ elemF, const int* __restrict__ sidx,
                            const int* __restrict__ node_model, const double* __restrict__ mass,
                            const double* __restrict__ v, const double* __restrict__ fext,
                            const double* __restrict__ step, double* __restrict__ fint,
                            double* __restrict__ b, double* __restrict__ sol0, const int* __restrict__ active,
                            const double* __restrict__ vprev, const double* __restrict__ vprev2,
                            const double* __restrict__ vprev3, const double* __restrict__ vprev4,
                            const double* __restrict__ row_nrm) {
  int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  if (active && !active[node_model[n]]) return;  // model left out of this step
  double f[3] = {0, 0, 0};
  const int i0 = inc_ptr[n], i1 = inc_ptr[n + 1];
  // four incidences per round: their index and force loads are independent
  for (int i = i0; i < i1; i += 4) {
    int idx[4];
#pragma unroll
    for (int k = 0; k < 4; k++) idx[k] = (i + k < i1) ? inc_idx[i + k] : -1;
    double g[4][3];
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int c = 0; c < 3; c++) g[k][c] = idx[k] >= 0 ? (double)elemF[(size_t)idx[k] * 3 + c] : 0.0;
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int c = 0; c < 3; c++) f[c] += g[k][c];
  }
  if (fint) {
    fint[3 * (size_t)n] = f[0];
    fint[3 * (size_t)n + 1] = f[1];
    fint[3 * (size_t)n + 2] = f[2];
  }
  int r = sidx[n];
  if (b && r >= 0) {
    const double* sp = step + (size_t)node_model[n] * 8;
    double h = sp[0], m = mass[n];
#pragma unroll
    for (int c = 0; c < 3; c++)
      b[3 * (size_t)r + c] = m * v[3 * (size_t)n + c] + h * (m * sp[3 + c] + fext[3 * (size_t)n + c] - f[c]);
    // the PCG starts from the current velocity, or from its extrapolation
    // v + (v - v_prev) over the last two steps
    if (sol0) {
      double s0[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const double vc = v[3 * (size_t)n + c];
        if (vprev4)  // quartic through the last five velocities
          s0[c] = 5.0 * (vc - vprev3[3 * (size_t)n + c]) + 10.0 * (vprev2[3 * (size_t)n + c] - vprev[3 * (size_t)n + c]) +
                  vprev4[3 * (size_t)n + c];
        else if (vprev3)  // cubic through the last four velocities
          s0[c] = 4.0 * (vc + vprev2[3 * (size_t)n + c]) - 6.0 * vprev[3 * (size_t)n + c] - vprev3[3 * (size_t)n + c];
        else if (vprev2)  // quadratic through the last three velocities
          s0[c] = 3.0 * (vc - vprev[3 * (size_t)n + c]) + vprev2[3 * (size_t)n + c];
        else
          s0[c] = vprev ? 2.0 * vc - vprev[3 * (size_t)n + c] : vc;
      }
      if (row_nrm) {
        // plane constraint: the initial guess lies on the plane
        const double* q = row_nrm + 3 * (size_t)r;
        const double d = q[0] * s0[0] + q[1] * s0[1] + q[2] * s0[2];
#pragma unroll
        for (int c = 0; c < 3; c++) s0[c] -= q[c] * d;
      }
#pragma unroll
      for (int c = 0; c < 3; c++) sol0[3 * (size_t)r + c] = s0[c];
    }
  }
}

// ---------------------------------------------------------------------------
// block SpMV helpers
// ---------------------------------------------------------------------------
template <typename MT>
__global__ void spmv_kernel(int n_rows, const int* rowptr, const int* col, const MT* S, const double* x,
                            double* y) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= n_rows) return;
  double out[3];
  warp_row_spmv<MT>(warp, rowptr, col, S, x, lane, out);
  if (lane == 0) {
    y[3 * (size_t)warp] = out[0];
    y[3 * (size_t)warp + 1] = out[1];
    y[3 * (size_t)warp + 2] = out[2];
  }
}

// factored NODAL solve matrix, outside the PCG: t_n of every dilational
// node, then each row adds sum t_n d_n(row) over its entries (node order)
__global__ void dil_t_kernel(int nd, const int* __restrict__ nodes, const int* __restrict__ nbr_ptr,
                             const int* __restrict__ nbr_row, const double* __restrict__ divblk,
                             const double* __restrict__ node_kp, const int* __restrict__ node_model,
                             const double* __restrict__ step, const double* __restrict__ v, double* __restrict__ t) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nd) return;
  const int n = nodes[k];
  const double* sp = step + (size_t)node_model[n] * 8;
  const double c = sp[0] * sp[0] + sp[0] * sp[2];
  t[n] = c * node_kp[n] * dil_node_t(nbr_ptr[n], nbr_ptr[n + 1], nbr_row, divblk, v);
}

__global__ void dil_add_kernel(int n_rows, const int* __restrict__ dil_rptr, const int* __restrict__ dil_node,
                               const int* __restrict__ dil_slot, const double* __restrict__ divblk,
                               const double* __restrict__ t, double* __restrict__ y) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_rows) return;
  double a0 = 0, a1 = 0, a2 = 0;
  for (int e = dil_rptr[r]; e < dil_rptr[r + 1]; e++) {
    const double tn = t[dil_node[e]];
    const double* g = divblk + 3 * (size_t)dil_slot[e];
    a0 += tn * g[0];
    a1 += tn * g[1];
    a2 += tn * g[2];
  }
  y[3 * (size_t)r] += a0;
  y[3 * (size_t)r + 1] += a1;
  y[3 * (size_t)r + 2] += a2;
}

// full-partition scalar CRS export: value of block p entry (r, c) goes to
// slot rowoff(3*row + r) + 3*k + c, k = position of p in its block row
__global__ void crs_export_kernel(long long nnzb, const int* blk_row, const int* rowptr,
                                  const double* vals, double* crs) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nnzb * 9) return;
  long long p = t / 9;
  int q = (int)(t - p * 9), r = q / 3, c = q % 3;
  int row = blk_row[p];
  long long p0 = rowptr[row];
  long long nb = rowptr[row + 1] - p0;
  long long slot = 9 * p0 + r * 3 * nb + 3 * (p - p0) + c;
  crs[slot] = vals[t];
}

// ---------------------------------------------------------------------------
// host launchers
// ---------------------------------------------------------------------------
// p + off, or null for an array the pack does not hold
template <typename T>
static T* at(T* p, long long off) {
  return p ? p + off : nullptr;
}

// The group's elements as 0 .. e1-e0-1: every per-element array starts at
// the group's first element (ElemGroup offsets), so the type-specialised
// kernels index them with their own constant strides.
static ElemArgs elem_args(Engine& eng, const ElemGroup& g, bool fp32) {
  DevPack& d = eng.d;
  ElemArgs a;
  a.e0 = 0;
  a.e1 = g.e1 - g.e0;
  a.conn = at(d.conn, g.c0);
  a.elem_model = at(d.elem_model, g.e0);
  a.elem_mat = at(d.elem_mat, g.e0);
  a.active = eng.any_inactive ? d.model_active : nullptr;
  a.x = d.x;
  a.invJ0 = at(d.invJ0, 9 * g.ip0);
  a.invJ0_f = at(d.invJ0_f, 9 * g.ip0);
  a.winvJ0 = at(d.winvJ0, 9LL * g.e0);
  a.K0 = at(d.K0, 9 * g.sq0);
  a.f0 = at(d.f0, 3 * g.c0);
  a.sidx = d.sidx;
  a.mat = d.mat;
  a.node_p = d.node_p;
  a.elem_p = at(d.elem_p, g.pv0);
  a.elem_r = at(d.elem_r, g.pv20);
  a.elemK = fp32 ? (void*)at(d.elemK_f, 9 * g.pr0) : (void*)at(d.elemK, 9 * g.pr0);
  a.elemF = (void*)at(d.elemF, 3 * g.c0);  // nodal forces are FP64 in both forms
  a.flags = d.flags;
  a.mindet = (long long*)d.dmin;
  a.det_stats = 0;
  return a;
}

template <int TYPE, int MAT, int INC, typename T, int EPB>
static cudaError_t launch_nonlinear(const ElemArgs& a, int ne, cudaStream_t st) {
  using SM = ElemSmem<TYPE, MAT, T, EPB>;
  auto kern = elem_nonlinear_kernel<TYPE, MAT, INC, T, EPB>;
  const size_t smem = SM::bytes();
  // the opt-in size is a per-function attribute: set it once per process
  // (it is not a stream operation, so it must not run inside graph capture)
  static bool attr_set = false;
  if (ne < 0) {  // preparation call (outside any stream capture)
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) attr_set = true;
    return e;
  }
  if (!attr_set) return cudaErrorInvalidConfiguration;
  kern<<<(ne + EPB - 1) / EPB, 256, smem, st>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// FP64 element forces of the mixed form (non-linear materials): the force
// residual keeps FP64 -- coordinates, shape gradients, F, stress and the
// nodal forces f_a = sum_ip sigma g_a dv -- while the tangent blocks come
// from the FP32 element kernel.  Nodal forces nearly cancel the external
// load, so their small net value needs FP64 terms.  One thread per element
// (tets) or per integration point: an element of several points holds 8
// consecutive lanes (lanes past its points idle), reduced in a fixed
// butterfly order.
// ---------------------------------------------------------------------------
template <int TYPE, int MAT, int INC>
__global__ void __launch_bounds__(128) elem_force_kernel(ElemArgs a) {
  constexpr int NEN = elem_nen(TYPE);
  constexpr int NIP = elem_nip(TYPE);
  constexpr int SLOT = force_slot(TYPE);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int e = a.e0 + (int)(t / SLOT);
  const int k = (int)(t % SLOT);
  bool live = e < a.e1 && k < NIP;
  if (live && a.active && !a.active[a.elem_model[e]]) live = false;
  double mydet = 1.0e300;
  int myinv = 0;
  double fl[NEN][3];
#pragma unroll
  for (int n = 0; n < NEN; n++) fl[n][0] = fl[n][1] = fl[n][2] = 0;
  if (live) {
    const int* nodes = a.conn + (size_t)e * NEN;
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      const double* xn = a.x + 3 * (size_t)nodes[n];
      const double g0 = gns<double, TYPE>(k, n, 0), g1 = gns<double, TYPE>(k, n, 1), g2 = gns<double, TYPE>(k, n, 2);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        const double xr = xn[r];
        J[3 * r] += xr * g0;
        J[3 * r + 1] += xr * g1;
        J[3 * r + 2] += xr * g2;
      }
    }
    double iJ0[9], F[9], invJ[9];
#pragma unroll
    for (int i = 0; i < 9; i++) iJ0[i] = a.invJ0[((size_t)e * NIP + k) * 9 + i];
    matmul3(F, J, iJ0);
    const double detF = det3(F);
    const double detJ = invert3(invJ, J);
    const double dv = detJ * ip_weight<double, TYPE>(k);
    myinv = !(detJ > 0.0);
    mydet = detJ;
    const double* mp = a.mat + (size_t)a.elem_mat[e] * kMatParams;
    double sig[6];
    if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) {
      double aa, bb;
      neohookean_point<double>(sig, &aa, &bb, mp[0], mp[1], F, detF);
    } else {
      double pr = 0;
      if constexpr (INC == kIncNodal) {
        if (TYPE == B200FEM_ELEM_TET) {
          double s = 0;
#pragma unroll
          for (int n = 0; n < NEN; n++) s += a.node_p[nodes[n]];
          pr = s / NEN;
        } else {
          pr = a.node_p[nodes[k]];
        }
      } else if constexpr (INC == kIncElement) {
        pr = elem_point_pressure<TYPE>(a.elem_p, e, k);
      }
      double D[36];
      material_point<MAT, double>(sig, D, mp, F, detF, pr);
    }
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      const double g0 = gns<double, TYPE>(k, n, 0), g1 = gns<double, TYPE>(k, n, 1), g2 = gns<double, TYPE>(k, n, 2);
      double g[3];
#pragma unroll
      for (int c = 0; c < 3; c++) g[c] = invJ[c] * g0 + invJ[3 + c] * g1 + invJ[6 + c] * g2;
      add_stress_force(fl[n], g, sig, dv);
    }
  }
  if (a.det_stats) warp_record_det(a.flags, a.mindet, mydet, myinv);
  if constexpr (NIP > 1) {
    // sum the points of one element: SLOT consecutive lanes hold its points
#pragma unroll
    for (int n = 0; n < NEN; n++)
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int off = SLOT / 2; off > 0; off >>= 1) fl[n][c] += __shfl_xor_sync(0xffffffffu, fl[n][c], off);
    if (!live || k != 0) return;
  }
  if (!live) return;
  double* out = (double*)a.elemF + (size_t)e * NEN * 3;
#pragma unroll
  for (int n = 0; n < NEN; n++)
#pragma unroll
    for (int c = 0; c < 3; c++) out[3 * n + c] = fl[n][c];
}

// ---------------------------------------------------------------------------
// Tetrahedra, non-linear materials: one thread per element, everything in
// registers.  Kinematics, stress and the nodal forces in FP64 (the force
// residual); the ten upper pair blocks B_a^T D B_b + (g_a^T sigma g_b) I in
// the storage precision T.  A warp stages its 32 element records in shared
// memory and writes them as contiguous lines (records of consecutive
// elements are adjacent in elemK / elemF).
// ---------------------------------------------------------------------------
// warps per CTA of elem_tet_kernel: the staging buffers (32 element records
// per warp) stay within the static shared-memory limit
template <typename T>
__host__ __device__ constexpr int tet_wpb() { return sizeof(T) == 8 ? 1 : 2; }

template <int MAT, int INC, typename T>
__global__ void __launch_bounds__(64) elem_tet_kernel(ElemArgs a) {
  constexpr int NPAIR = 10, KW = NPAIR * 9, FW = 12, WPB = tet_wpb<T>();
  __shared__ T sk[WPB][32 * KW];
  __shared__ double sf[WPB][32 * FW];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int wbase = a.e0 + (blockIdx.x * WPB + warp) * 32;
  const int e = wbase + lane;
  bool live = e < a.e1;
  if (live && a.active && !a.active[a.elem_model[e]]) live = false;
  T* kout = sk[warp] + lane * KW;
  double* fout = sf[warp] + lane * FW;
  double mydet = 1.0e300;
  int myinv = 0;
  if (live) {
    const int* nodes = a.conn + (size_t)e * 4;
    int nd[4];
#pragma unroll
    for (int n = 0; n < 4; n++) nd[n] = nodes[n];
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const double g0 = c_tet_gns[3 * n], g1 = c_tet_gns[3 * n + 1], g2 = c_tet_gns[3 * n + 2];
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
    myinv = !(detJ > 0.0);
    mydet = detJ;
    const double dv = detJ * (1.0 / 6.0);
    double g[4][3];
#pragma unroll
    for (int n = 0; n < 4; n++) {
      const double g0 = c_tet_gns[3 * n], g1 = c_tet_gns[3 * n + 1], g2 = c_tet_gns[3 * n + 2];
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
      if constexpr (INC == kIncNodal) pr = 0.25 * (a.node_p[nd[0]] + a.node_p[nd[1]] + a.node_p[nd[2]] + a.node_p[nd[3]]);
      else if constexpr (INC == kIncElement) pr = a.elem_p[e];
      double D[36];
      material_point<MAT, double>(sig, D, mp, F, detF, pr);
#pragma unroll
      for (int i = 0; i < 36; i++) Dt[i] = (T)D[i];
    }
    // nodal forces (FP64)
#pragma unroll
    for (int n = 0; n < 4; n++) {
      double f[3] = {0, 0, 0};
      add_stress_force(f, g[n], sig, dv);
      fout[3 * n] = f[0];
      fout[3 * n + 1] = f[1];
      fout[3 * n + 2] = f[2];
    }
    // pair blocks (storage precision)
    T gt[4][3], st[6];
    const T dvt = (T)dv;
#pragma unroll
    for (int n = 0; n < 4; n++)
#pragma unroll
      for (int c = 0; c < 3; c++) gt[n][c] = (T)g[n][c];
#pragma unroll
    for (int i = 0; i < 6; i++) st[i] = (T)sig[i];
    int w = 0;
#pragma unroll
    for (int ia = 0; ia < 4; ia++)
#pragma unroll
      for (int ib = ia; ib < 4; ib++, w++) {
        T K[9];
#pragma unroll
        for (int i = 0; i < 9; i++) K[i] = T(0);
        if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) add_bdb_iso(K, gt[ia], Dt[0], Dt[1], gt[ib], dvt);
        else add_bdb(K, gt[ia], Dt, gt[ib], dvt);
        add_geometric(K, gt[ia], st, gt[ib], dvt);
        if constexpr (INC == kIncElement) {
          // ELEMENT dilational stiffness Rinv (g_a dv)(g_b dv)^T (one point)
          const T r = (T)(a.elem_r[e] * dv * dv);
#pragma unroll
          for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) K[3 * i + j] += r * gt[ia][i] * gt[ib][j];
        }
#pragma unroll
        for (int i = 0; i < 9; i++) kout[9 * w + i] = K[i];
      }
  }
  warp_record_det(a.flags, a.mindet, mydet, myinv);
  __syncwarp();
  // contiguous stores of the warp's element records
  const int nv = min(32, a.e1 - wbase);
  if (nv <= 0) return;
  T* K = (T*)a.elemK + (size_t)wbase * KW;
  for (int i = lane; i < nv * KW; i += 32) {
    const int el = i / KW;
    if (a.active && !a.active[a.elem_model[wbase + el]]) continue;
    K[i] = sk[warp][i];
  }
  double* Fo = (double*)a.elemF + (size_t)wbase * FW;
  for (int i = lane; i < nv * FW; i += 32) {
    const int el = i / FW;
    if (a.active && !a.active[a.elem_model[wbase + el]]) continue;
    Fo[i] = sf[warp][i];
  }
}

template <int MAT, int INC, typename T>
static cudaError_t launch_tet(const ElemArgs& a, int ne, cudaStream_t st) {
  constexpr int TPB = 32 * tet_wpb<T>();
  elem_tet_kernel<MAT, INC, T><<<(ne + TPB - 1) / TPB, TPB, 0, st>>>(a);
  return cudaGetLastError();
}

template <int TYPE, int MAT, int INC>
static cudaError_t launch_force(const ElemArgs& a, int ne, cudaStream_t st) {
  const long long threads = (long long)ne * force_slot(TYPE);
  elem_force_kernel<TYPE, MAT, INC><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Fused element-to-block assembly of the BackwardEuler matrix (non-linear
// materials without NODAL incompressibility).  Each CTA owns a chunk of
// consecutive block rows: it first computes, for every element incident to
// those rows, the integration-point records (shape gradients, dv, stress,
// tangent coefficients) into shared memory, then forms each of its blocks by
// walking the block's contribution list in element order -- the same sums,
// in the same order, as the element kernel + gather pair, without the element
// blocks' round trip through HBM.  Elements on a chunk boundary are computed
// by every chunk they touch.
// ---------------------------------------------------------------------------
struct FusedArgs {
  const int* chunk_row;   // [chunks + 1] block-row range of each chunk
  const int* chunk_eptr;  // [chunks + 1]
  const int* chunk_elem;  // element ids of each chunk, ascending
  const int* contrib_ptr;
  const int* contrib_loc;  // (chunk-local element * npair + pair) << 1 | transposed
  const int* rowptr;
  const int* blk_row;
  const int* blk_diag;
  const int* row_model;
  const int* act_node;
  const double* mass;
  const double* step;
  const int* conn;
  const int* elem_model;
  const int* elem_mat;
  const int* active;
  const double* x;
  const double* invJ0;
  const float* invJ0_f;
  const double* mat;
  void* out;  // S (TO)
};

template <int TYPE, int MAT, typename T>
struct FusedSmem {
  static_assert(TYPE == B200FEM_ELEM_TET || TYPE == B200FEM_ELEM_HEX, "fused assembly: tets and hexes");
  static constexpr int NEN = elem_nen(TYPE);
  static constexpr int NIP = elem_nip(TYPE);
  static constexpr int DS = MAT == B200FEM_MAT_NEOHOOKEAN ? 2 : 36;
  static constexpr size_t per_elem() { return sizeof(T) * (size_t)NIP * (NEN * 3 + 1 + 6 + DS); }
};

template <int TYPE, int MAT, typename T, typename TO>
__global__ void __launch_bounds__(256) fused_block_kernel(FusedArgs a) {
  using SM = FusedSmem<TYPE, MAT, T>;
  constexpr int NEN = SM::NEN, NIP = SM::NIP, DS = SM::DS;
  constexpr int NPAIR = NEN * (NEN + 1) / 2;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int c = blockIdx.x;
  const int e0 = a.chunk_eptr[c], ne = a.chunk_eptr[c + 1] - e0;
  const int nrec = ne * NIP;
  T(*sg)[NEN][3] = reinterpret_cast<T(*)[NEN][3]>(smem_raw);
  T* sdv = reinterpret_cast<T*>(smem_raw + sizeof(T) * (size_t)nrec * NEN * 3);
  T(*ssig)[6] = reinterpret_cast<T(*)[6]>(sdv + nrec);
  T(*sD)[DS] = reinterpret_cast<T(*)[DS]>(sdv + nrec + (size_t)nrec * 6);
  // stage 1: one thread per (element, integration point)
  for (int t = threadIdx.x; t < nrec; t += blockDim.x) {
    const int le = t / NIP, k = t % NIP;
    const int e = a.chunk_elem[e0 + le];
    if (a.active && !a.active[a.elem_model[e]]) continue;
    const int* nodes = a.conn + (size_t)e * NEN;
    T J[9];
#pragma unroll
    for (int i = 0; i < 9; i++) J[i] = T(0);
    const int n0 = nodes[0];
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      const int nd = nodes[n];
      const T g0 = gns<T, TYPE>(k, n, 0), g1 = gns<T, TYPE>(k, n, 1), g2 = gns<T, TYPE>(k, n, 2);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        double v = a.x[3 * (size_t)nd + r];
        if constexpr (sizeof(T) == 4) v -= a.x[3 * (size_t)n0 + r];  // FP32: relative to node 0, in FP64
        const T p = (T)v;
        J[3 * r] += p * g0;
        J[3 * r + 1] += p * g1;
        J[3 * r + 2] += p * g2;
      }
    }
    T iJ0[9];
    if constexpr (sizeof(T) == 8) {
#pragma unroll
      for (int i = 0; i < 9; i++) iJ0[i] = a.invJ0[((size_t)e * NIP + k) * 9 + i];
    } else {
#pragma unroll
      for (int i = 0; i < 9; i++) iJ0[i] = a.invJ0_f[((size_t)e * NIP + k) * 9 + i];
    }
    T F[9], invJ[9];
    matmul3(F, J, iJ0);
    const T detF = det3(F);
    const T detJ = invert3(invJ, J);
    const T w = TYPE == B200FEM_ELEM_TET ? T(1.0 / 6.0) : T(1);
    sdv[t] = detJ * w;
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      const T g0 = gns<T, TYPE>(k, n, 0), g1 = gns<T, TYPE>(k, n, 1), g2 = gns<T, TYPE>(k, n, 2);
#pragma unroll
      for (int cc = 0; cc < 3; cc++) sg[t][n][cc] = invJ[cc] * g0 + invJ[3 + cc] * g1 + invJ[6 + cc] * g2;
    }
    const double* mp = a.mat + (size_t)a.elem_mat[e] * kMatParams;
    if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) {
      T aa, bb;
      neohookean_point<T>(ssig[t], &aa, &bb, (T)mp[0], (T)mp[1], F, detF);
      sD[t][0] = aa;
      sD[t][1] = bb;
    } else {
      T mpt[8];
#pragma unroll
      for (int i = 0; i < 8; i++) mpt[i] = (T)mp[i];
      material_point<MAT, T>(ssig[t], sD[t], mpt, F, detF, T(0));
    }
  }
  __syncthreads();
  // stage 2: one thread per block of the chunk's rows
  const int r0 = a.chunk_row[c], r1 = a.chunk_row[c + 1];
  const int pb0 = a.rowptr[r0], pb1 = a.rowptr[r1];
  TO* out = (TO*)a.out;
  for (int p = pb0 + threadIdx.x; p < pb1; p += blockDim.x) {
    const int row = a.blk_row[p];
    const int m = a.row_model[row];
    if (a.active && !a.active[m]) continue;
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const int q1 = a.contrib_ptr[p + 1];
    for (int q = a.contrib_ptr[p]; q < q1; q++) {
      const int code = a.contrib_loc[q];
      const int lw = code >> 1;
      const int le = lw / NPAIR, wp = lw - le * NPAIR;
      int ia, ib;
      pair_of<NEN>(wp, ia, ib);
      T K[9];
#pragma unroll
      for (int i = 0; i < 9; i++) K[i] = T(0);
#pragma unroll
      for (int k = 0; k < NIP; k++) {
        const int s = le * NIP + k;
        if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN)
          add_bdb_iso(K, sg[s][ia], sD[s][0], sD[s][1], sg[s][ib], sdv[s]);
        else
          add_bdb(K, sg[s][ia], sD[s], sg[s][ib], sdv[s]);
        add_geometric(K, sg[s][ia], ssig[s], sg[s][ib], sdv[s]);
      }
      if (code & 1) {
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
          for (int j = 0; j < 3; j++) acc[3 * i + j] += (double)K[3 * j + i];
      } else {
#pragma unroll
        for (int i = 0; i < 9; i++) acc[i] += (double)K[i];
      }
    }
    // S = (h^2 + h beta) K + (1 + h alpha) M  (addPosJacobian, addVelJacobian,
    // addActiveMassMatrix; MechSystemSolver.java:2277,2312,2334)
    const double* sp = a.step + (size_t)m * 8;
    const double h = sp[0], al = sp[1], be = sp[2];
    const double cm = p == a.blk_diag[row] ? (1.0 + h * al) * a.mass[a.act_node[row]] : 0.0;
    TO* o = out + (size_t)p * 9;
#pragma unroll
    for (int i = 0; i < 9; i++) o[i] = (TO)((h * h + h * be) * acc[i] + ((i % 4 == 0) ? cm : 0.0));
  }
}

// shared-memory budget of one chunk: tets two CTAs per SM, hexes (eight
// integration points per element) one
size_t fused_smem_budget(int elem_type) { return elem_type == B200FEM_ELEM_TET ? 100 * 1024 : 200 * 1024; }

template <int TYPE, int MAT, typename T, typename TO>
static cudaError_t launch_fused(const FusedArgs& fa, int chunks, int emax, cudaStream_t st) {
  using SM = FusedSmem<TYPE, MAT, T>;
  auto kern = fused_block_kernel<TYPE, MAT, T, TO>;
  const size_t smem = SM::per_elem() * (size_t)emax;
  static bool attr_set = false;
  if (chunks < 0) {  // preparation call (outside any stream capture): the
    // attribute is process-wide, so it is set to the full budget, which
    // covers every engine's chunks
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)fused_smem_budget(TYPE));
    if (e == cudaSuccess) attr_set = true;
    return e;
  }
  if (!attr_set) return cudaErrorInvalidConfiguration;
  if (chunks == 0) return cudaSuccess;
  kern<<<chunks, 256, smem, st>>>(fa);
  return cudaGetLastError();
}

template <int TYPE, typename T>
static cudaError_t launch_group(Engine& eng, const ElemGroup& g, bool fp32) {
  ElemArgs a = elem_args(eng, g, fp32);
  int ne = g.e1 - g.e0;
  if (ne == 0) return cudaSuccess;
  if (g.mat_kind == B200FEM_MAT_LINEAR) {
    if (ne < 0) return cudaSuccess;
    constexpr int EPB = TYPE == B200FEM_ELEM_TET ? 32 : 8;
    // the corotation and K0 products run in FP64; the mixed form stores
    // the element outputs in FP32
    elem_linear_kernel<TYPE, T><<<(ne + EPB - 1) / EPB, 256, 0, eng.stream>>>(a, g.corotated);
    return cudaGetLastError();
  }
  // elements per CTA (one thread per integration point in stage 1): a
  // large and a small tile per material; the small one gives more CTAs
  // per SM and fewer idle threads in the pair stage on small groups
  // (elements of more than ten nodes: a point record holds 13-20 gradients)
  constexpr int NH_L = TYPE == B200FEM_ELEM_TET ? 256 : (elem_nen(TYPE) > 10 ? 8 : 32), NH_S = NH_L / 2;
  constexpr int MR_L = TYPE == B200FEM_ELEM_TET ? 128 : (elem_nen(TYPE) > 10 ? 8 : 16), MR_S = MR_L / 2;
  // StVenantKirchhoff has the general 6x6 tangent: MooneyRivlin's tiles
  constexpr int NH = B200FEM_MAT_NEOHOOKEAN, MR = B200FEM_MAT_MOONEYRIVLIN, SV = B200FEM_MAT_STVK;
  cudaStream_t st = eng.stream;
  if (ne < 0) {  // preparation: both tiles
    cudaError_t e;
    if (g.mat_kind == NH) {
      e = launch_nonlinear<TYPE, NH, kIncOff, T, NH_L>(a, ne, st);
      return e != cudaSuccess ? e : launch_nonlinear<TYPE, NH, kIncOff, T, NH_S>(a, ne, st);
    }
    if (g.mat_kind == SV) {
      e = launch_nonlinear<TYPE, SV, kIncOff, T, MR_L>(a, ne, st);
      return e != cudaSuccess ? e : launch_nonlinear<TYPE, SV, kIncOff, T, MR_S>(a, ne, st);
    }
    if (g.nodal) {
      e = launch_nonlinear<TYPE, MR, kIncNodal, T, MR_L>(a, ne, st);
      return e != cudaSuccess ? e : launch_nonlinear<TYPE, MR, kIncNodal, T, MR_S>(a, ne, st);
    }
    if (g.elem_inc) {
      e = launch_nonlinear<TYPE, MR, kIncElement, T, MR_L>(a, ne, st);
      return e != cudaSuccess ? e : launch_nonlinear<TYPE, MR, kIncElement, T, MR_S>(a, ne, st);
    }
    e = launch_nonlinear<TYPE, MR, kIncOff, T, MR_L>(a, ne, st);
    return e != cudaSuccess ? e : launch_nonlinear<TYPE, MR, kIncOff, T, MR_S>(a, ne, st);
  }
  const bool small = eng.elem_tile_small;
  cudaError_t e;
  if (TYPE == B200FEM_ELEM_TET && !eng.elem_staged) {
    // one thread per tetrahedron (FP64 forces in the same pass)
    if (g.mat_kind == NH) return launch_tet<NH, kIncOff, T>(a, ne, st);
    if (g.mat_kind == SV) return launch_tet<SV, kIncOff, T>(a, ne, st);
    if (g.nodal) return launch_tet<MR, kIncNodal, T>(a, ne, st);
    if (g.elem_inc) return launch_tet<MR, kIncElement, T>(a, ne, st);
    return launch_tet<MR, kIncOff, T>(a, ne, st);
  }
  if (g.mat_kind == NH) {
    e = small ? launch_nonlinear<TYPE, NH, kIncOff, T, NH_S>(a, ne, st) : launch_nonlinear<TYPE, NH, kIncOff, T, NH_L>(a, ne, st);
    if (e == cudaSuccess && fp32) e = launch_force<TYPE, NH, kIncOff>(a, ne, st);
  } else if (g.mat_kind == SV) {
    e = small ? launch_nonlinear<TYPE, SV, kIncOff, T, MR_S>(a, ne, st) : launch_nonlinear<TYPE, SV, kIncOff, T, MR_L>(a, ne, st);
    if (e == cudaSuccess && fp32) e = launch_force<TYPE, SV, kIncOff>(a, ne, st);
  } else if (g.nodal) {
    e = small ? launch_nonlinear<TYPE, MR, kIncNodal, T, MR_S>(a, ne, st) : launch_nonlinear<TYPE, MR, kIncNodal, T, MR_L>(a, ne, st);
    if (e == cudaSuccess && fp32) e = launch_force<TYPE, MR, kIncNodal>(a, ne, st);
  } else if (g.elem_inc) {
    e = small ? launch_nonlinear<TYPE, MR, kIncElement, T, MR_S>(a, ne, st)
              : launch_nonlinear<TYPE, MR, kIncElement, T, MR_L>(a, ne, st);
    if (e == cudaSuccess && fp32) e = launch_force<TYPE, MR, kIncElement>(a, ne, st);
  } else {
    e = small ? launch_nonlinear<TYPE, MR, kIncOff, T, MR_S>(a, ne, st) : launch_nonlinear<TYPE, MR, kIncOff, T, MR_L>(a, ne, st);
    if (e == cudaSuccess && fp32) e = launch_force<TYPE, MR, kIncOff>(a, ne, st);
  }
  return e;
}

// ---------------------------------------------------------------------------
// NODAL soft incompressibility
// ---------------------------------------------------------------------------
// One incidence's share of its node's volume: tets give V_e/4 (det(J)/24),
// other elements the dv of the integration point a that maps to the node.
template <int TYPE>
__device__ __forceinline__ double nodal_vol_share(const int* __restrict__ nodes, int a,
                                                  const double* __restrict__ x) {
  constexpr int NEN = elem_nen(TYPE);
  double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < NEN; k++) {
    const double* pk = x + 3 * (size_t)nodes[k];
    const double g0 = gns<double, TYPE>(a, k, 0), g1 = gns<double, TYPE>(a, k, 1), g2 = gns<double, TYPE>(a, k, 2);
#pragma unroll
    for (int r = 0; r < 3; r++) {
      J[3 * r] += pk[r] * g0;
      J[3 * r + 1] += pk[r] * g1;
      J[3 * r + 2] += pk[r] * g2;
    }
  }
  return TYPE == B200FEM_ELEM_TET ? det3(J) / 6 / 4 : det3(J) * ip_weight<double, TYPE>(a);
}

// p_n = K(V_n/V0_n - 1) (QUADRATIC) or K ln(J)/J (LOGARITHMIC) for active
// nodes, and kp_n = K_eff / V0_n (computeNodalIncompressibility, :2632-2669)
__device__ __forceinline__ void nodal_pressure_store(int n, double v, const int* __restrict__ sidx,
                                                     const double* __restrict__ rest_vol,
                                                     const double* __restrict__ mat_node, double* __restrict__ vol,
                                                     double* __restrict__ pres, double* __restrict__ kp) {
  vol[n] = v;
  double p = 0, k = 0;
  if (sidx[n] >= 0) {
    const double K = mat_node[2 * (size_t)n], J = v / rest_vol[n];
    if (mat_node[2 * (size_t)n + 1] == 0) {
      p = K * (J - 1);
      k = K;
    } else {
      p = K * log(J) / J;
      k = K * (1 - log(J)) / (J * J);
    }
    k /= rest_vol[n];
  }
  pres[n] = p;
  kp[n] = k;
}

// Nodal volumes and pressures (updateNodalPressures, FemModel3d.java:2471-2515),
// one thread per node over its incidences in element order.
template <int TYPE>
__global__ void nodal_pressure_kernel(int N, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx,
                                      const int* __restrict__ conn, const double* __restrict__ x,
                                      const int* __restrict__ sidx, const double* __restrict__ rest_vol,
                                      const double* __restrict__ mat_node, double* __restrict__ vol,
                                      double* __restrict__ pres, double* __restrict__ kp) {
  constexpr int NEN = elem_nen(TYPE);
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double v = 0;
  for (int i = inc_ptr[n]; i < inc_ptr[n + 1]; i++) {
    const int a = inc_idx[i] % NEN;
    v += nodal_vol_share<TYPE>(conn + (inc_idx[i] - a), a, x);
  }
  nodal_pressure_store(n, v, sidx, rest_vol, mat_node, vol, pres, kp);
}

// the same for a pack of several element types: each incidence carries its
// element's type and local node ((type << 8) | a), the node slot inc_idx
// gives the element's first slot (inc_idx - a)
__global__ void nodal_pressure_mixed_kernel(int N, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx,
                                            const int* __restrict__ inc_tl, const int* __restrict__ conn,
                                            const double* __restrict__ x, const int* __restrict__ sidx,
                                            const double* __restrict__ rest_vol, const double* __restrict__ mat_node,
                                            double* __restrict__ vol, double* __restrict__ pres,
                                            double* __restrict__ kp) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double v = 0;
  for (int i = inc_ptr[n]; i < inc_ptr[n + 1]; i++) {
    const int t = inc_tl[i] >> 8, a = inc_tl[i] & 255;
    const int* nodes = conn + (inc_idx[i] - a);
    switch (t) {
      case B200FEM_ELEM_TET: v += nodal_vol_share<B200FEM_ELEM_TET>(nodes, a, x); break;
      case B200FEM_ELEM_HEX: v += nodal_vol_share<B200FEM_ELEM_HEX>(nodes, a, x); break;
      case B200FEM_ELEM_WEDGE: v += nodal_vol_share<B200FEM_ELEM_WEDGE>(nodes, a, x); break;
      default: v += nodal_vol_share<B200FEM_ELEM_PYRAMID>(nodes, a, x); break;
    }
  }
  nodal_pressure_store(n, v, sidx, rest_vol, mat_node, vol, pres, kp);
}

// divBlk(n, m) = dV_n/dx_m, one incidence's terms (FemModel3d.java:3604-3648):
// tets add -1/12 of the area-weighted normal of the face opposite m
// (TetElement.java:333-362); other elements add dv_k GNx_m at the
// integration point k that maps to n.  slot[j]: node j's entry in nbr(n).
template <int TYPE>
__device__ __forceinline__ void divblk_add(const int* __restrict__ nodes, int a, const int* __restrict__ slot,
                                           const double* __restrict__ x, double* __restrict__ out) {
  constexpr int NEN = elem_nen(TYPE);
  if constexpr (TYPE == B200FEM_ELEM_TET) {
    const double* P[4];
#pragma unroll
    for (int k = 0; k < 4; k++) P[k] = x + 3 * (size_t)nodes[k];
    // faces opposite nodes 0..3: (1,2,3), (0,3,2), (0,1,3), (0,2,1)
    const int f[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const double *q0 = P[f[j][0]], *q1 = P[f[j][1]], *q2 = P[f[j][2]];
      const double ux = q1[0] - q0[0], uy = q1[1] - q0[1], uz = q1[2] - q0[2];
      const double vx = q2[0] - q0[0], vy = q2[1] - q0[1], vz = q2[2] - q0[2];
      double* o = out + 3 * slot[j];
      o[0] += 0.5 * (uy * vz - uz * vy) * (-1 / 12.0);
      o[1] += 0.5 * (uz * vx - ux * vz) * (-1 / 12.0);
      o[2] += 0.5 * (ux * vy - uy * vx) * (-1 / 12.0);
    }
  } else {
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, iJ[9];
#pragma unroll
    for (int k = 0; k < NEN; k++) {
      const double* pk = x + 3 * (size_t)nodes[k];
#pragma unroll
      for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) J[3 * r + c] += pk[r] * gns<double, TYPE>(a, k, c);
    }
    const double dv = invert3(iJ, J) * ip_weight<double, TYPE>(a);
#pragma unroll
    for (int k = 0; k < NEN; k++) {
      const double g0 = gns<double, TYPE>(a, k, 0), g1 = gns<double, TYPE>(a, k, 1), g2 = gns<double, TYPE>(a, k, 2);
      double* o = out + 3 * slot[k];
#pragma unroll
      for (int c = 0; c < 3; c++) o[c] += dv * (iJ[c] * g0 + iJ[3 + c] * g1 + iJ[6 + c] * g2);
    }
  }
}

// divBlk per node, accumulated over its incidences in element order
template <int TYPE>
__global__ void divblk_kernel(int N, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx,
                              const int* __restrict__ inc_slot, const int* __restrict__ conn,
                              const double* __restrict__ x, const int* __restrict__ sidx,
                              const int* __restrict__ nbr_ptr, double* __restrict__ divblk) {
  constexpr int NEN = elem_nen(TYPE);
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double* out = divblk + 3 * (size_t)nbr_ptr[n];
  const int ns = nbr_ptr[n + 1] - nbr_ptr[n];
  for (int s = 0; s < 3 * ns; s++) out[s] = 0;
  if (sidx[n] < 0) return;
  for (int i = inc_ptr[n]; i < inc_ptr[n + 1]; i++) {
    const int a = inc_idx[i] % NEN;
    divblk_add<TYPE>(conn + (inc_idx[i] - a), a, inc_slot + (size_t)i * NEN, x, out);
  }
}

// divBlk per node with the node's sums in shared memory (nodes of at most
// kDivSmemSlots direct neighbours): the same terms added in the same order as
// divblk_kernel, but each += is a shared-memory update instead of a global
// load-add-store chain.  Slot s, component c of thread t lives at
// acc[(3 s + c) * blockDim + t], so a warp's threads touch consecutive words.
constexpr int kDivSmemSlots = 32;
constexpr int kDivSmemThreads = 64;
template <int TYPE>
__global__ void __launch_bounds__(kDivSmemThreads) divblk_smem_kernel(
    int N, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx, const int* __restrict__ inc_slot,
    const int* __restrict__ conn, const double* __restrict__ x, const int* __restrict__ sidx,
    const int* __restrict__ nbr_ptr, double* __restrict__ divblk) {
  constexpr int NEN = elem_nen(TYPE);
  __shared__ double acc[3 * kDivSmemSlots * kDivSmemThreads];
  const int t = threadIdx.x;
  const int n = blockIdx.x * kDivSmemThreads + t;
  if (n >= N) return;  // no block-wide barrier below
  const int ns = nbr_ptr[n + 1] - nbr_ptr[n];
  auto A = [&](int slot, int c) -> double& { return acc[(3 * slot + c) * kDivSmemThreads + t]; };
  for (int q = 0; q < ns; q++) A(q, 0) = A(q, 1) = A(q, 2) = 0;
  if (sidx[n] >= 0) {
    for (int i = inc_ptr[n]; i < inc_ptr[n + 1]; i++) {
      const int a = inc_idx[i] % NEN;
      const int* nodes = conn + (inc_idx[i] - a);
      const int* slot = inc_slot + (size_t)i * NEN;
      if constexpr (TYPE == B200FEM_ELEM_TET) {
        const double* P[4];
#pragma unroll
        for (int k = 0; k < 4; k++) P[k] = x + 3 * (size_t)nodes[k];
        // faces opposite nodes 0..3: (1,2,3), (0,3,2), (0,1,3), (0,2,1)
        const int f[4][3] = {{1, 2, 3}, {0, 3, 2}, {0, 1, 3}, {0, 2, 1}};
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const double *q0 = P[f[j][0]], *q1 = P[f[j][1]], *q2 = P[f[j][2]];
          const double ux = q1[0] - q0[0], uy = q1[1] - q0[1], uz = q1[2] - q0[2];
          const double vx = q2[0] - q0[0], vy = q2[1] - q0[1], vz = q2[2] - q0[2];
          const int sj = slot[j];
          A(sj, 0) += 0.5 * (uy * vz - uz * vy) * (-1 / 12.0);
          A(sj, 1) += 0.5 * (uz * vx - ux * vz) * (-1 / 12.0);
          A(sj, 2) += 0.5 * (ux * vy - uy * vx) * (-1 / 12.0);
        }
      } else {
        double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, iJ[9];
#pragma unroll
        for (int k = 0; k < NEN; k++) {
          const double* pk = x + 3 * (size_t)nodes[k];
#pragma unroll
          for (int r = 0; r < 3; r++)
#pragma unroll
            for (int c = 0; c < 3; c++) J[3 * r + c] += pk[r] * gns<double, TYPE>(a, k, c);
        }
        const double dv = invert3(iJ, J) * ip_weight<double, TYPE>(a);
#pragma unroll
        for (int k = 0; k < NEN; k++) {
          const double g0 = gns<double, TYPE>(a, k, 0), g1 = gns<double, TYPE>(a, k, 1),
                       g2 = gns<double, TYPE>(a, k, 2);
          const int sk = slot[k];
#pragma unroll
          for (int c = 0; c < 3; c++) A(sk, c) += dv * (iJ[c] * g0 + iJ[3 + c] * g1 + iJ[6 + c] * g2);
        }
      }
    }
  }
  double* out = divblk + 3 * (size_t)nbr_ptr[n];
  for (int q = 0; q < ns; q++) {
    out[3 * q] = A(q, 0);
    out[3 * q + 1] = A(q, 1);
    out[3 * q + 2] = A(q, 2);
  }
}

// the same for a pack of several element types (nm slots per incidence)
__global__ void divblk_mixed_kernel(int N, int nm, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx,
                                    const int* __restrict__ inc_tl, const int* __restrict__ inc_slot,
                                    const int* __restrict__ conn, const double* __restrict__ x,
                                    const int* __restrict__ sidx, const int* __restrict__ nbr_ptr,
                                    double* __restrict__ divblk) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  double* out = divblk + 3 * (size_t)nbr_ptr[n];
  const int ns = nbr_ptr[n + 1] - nbr_ptr[n];
  for (int s = 0; s < 3 * ns; s++) out[s] = 0;
  if (sidx[n] < 0) return;
  for (int i = inc_ptr[n]; i < inc_ptr[n + 1]; i++) {
    const int t = inc_tl[i] >> 8, a = inc_tl[i] & 255;
    const int* nodes = conn + (inc_idx[i] - a);
    const int* slot = inc_slot + (size_t)i * nm;
    switch (t) {
      case B200FEM_ELEM_TET: divblk_add<B200FEM_ELEM_TET>(nodes, a, slot, x, out); break;
      case B200FEM_ELEM_HEX: divblk_add<B200FEM_ELEM_HEX>(nodes, a, slot, x, out); break;
      case B200FEM_ELEM_WEDGE: divblk_add<B200FEM_ELEM_WEDGE>(nodes, a, slot, x, out); break;
      default: divblk_add<B200FEM_ELEM_PYRAMID>(nodes, a, slot, x, out); break;
    }
  }
}

cudaError_t launch_nodal_pressure(Engine& eng) {
  DevPack& d = eng.d;
  if (!d.has_nodal) return cudaSuccess;
  const int threads = 128, blocks = (d.n_nodes + threads - 1) / threads;
  if (eng.elem_type == kElemMixed) {
    nodal_pressure_mixed_kernel<<<blocks, threads, 0, eng.stream>>>(d.n_nodes, d.inc_ptr, d.inc_idx, d.inc_tl,
                                                                    d.conn, d.x, d.sidx, d.node_rest_vol,
                                                                    d.mat_node, d.node_vol, d.node_p, d.node_kp);
    return cudaGetLastError();
  }
  return by_elem_type(eng.elem_type, [&](auto tag) {
    constexpr int TY = decltype(tag)::value;
    // NODAL: tets, or elements whose integration points sit at their nodes
    if constexpr (TY != B200FEM_ELEM_TET && !elem_ip_at_nodes(TY)) {
      return cudaErrorNotSupported;
    } else {
      nodal_pressure_kernel<TY><<<blocks, threads, 0, eng.stream>>>(
          d.n_nodes, d.inc_ptr, d.inc_idx, d.conn, d.x, d.sidx, d.node_rest_vol, d.mat_node, d.node_vol, d.node_p,
          d.node_kp);
      return cudaGetLastError();
    }
  });
}

cudaError_t launch_divblk(Engine& eng) {
  DevPack& d = eng.d;
  if (!d.has_nodal) return cudaSuccess;
  const int threads = 128, blocks = (d.n_nodes + threads - 1) / threads;
  if (eng.elem_type == kElemMixed) {
    divblk_mixed_kernel<<<blocks, threads, 0, eng.stream>>>(d.n_nodes, eng.nen_max, d.inc_ptr, d.inc_idx, d.inc_tl,
                                                            d.inc_slot, d.conn, d.x, d.sidx, d.nbr_ptr, d.divblk);
    return cudaGetLastError();
  }
  return by_elem_type(eng.elem_type, [&](auto tag) {
    constexpr int TY = decltype(tag)::value;
    if constexpr (TY != B200FEM_ELEM_TET && !elem_ip_at_nodes(TY)) {
      return cudaErrorNotSupported;
    } else {
      if (eng.divblk_smem)
        divblk_smem_kernel<TY><<<(d.n_nodes + kDivSmemThreads - 1) / kDivSmemThreads, kDivSmemThreads, 0,
                                 eng.stream>>>(d.n_nodes, d.inc_ptr, d.inc_idx, d.inc_slot, d.conn, d.x, d.sidx,
                                               d.nbr_ptr, d.divblk);
      else
        divblk_kernel<TY><<<blocks, threads, 0, eng.stream>>>(
            d.n_nodes, d.inc_ptr, d.inc_idx, d.inc_slot, d.conn, d.x, d.sidx, d.nbr_ptr, d.divblk);
      return cudaGetLastError();
    }
  });
}

// ELEMENT soft incompressibility with one pressure value per element (tet
// and hex), computePressuresAndRinv (FemModel3d.java:2517-2591, npvals == 1):
// the current volume V (tet: det J / 6, TetElement.computeVolumes; hex: the
// sum of det J w over the points, FemElement3d.computeVolumes), J = V/V0,
// p = effectivePressure(kappa, J) and Rinv = effectiveModulus(kappa, J) / V0
// (IncompressibleMaterialBase.java:116-152), per element of the group.
template <int TYPE>
__global__ void element_pressure_kernel(int e0, int e1, const int* __restrict__ conn,
                                        const int* __restrict__ elem_mat, const double* __restrict__ x,
                                        const double* __restrict__ rest_vol, const double* __restrict__ mat,
                                        const double* __restrict__ detJ0, double* __restrict__ elem_p,
                                        double* __restrict__ elem_r) {
  constexpr int NEN = elem_nen(TYPE);
  constexpr int NIP = elem_nip(TYPE);
  constexpr int NPV = elem_npv(TYPE);
  const int e = e0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= e1) return;
  const int* nodes = conn + (size_t)e * NEN;
  if constexpr (NPV > 1) {
    // several pressure values (computePressuresAndRinv, FemModel3d.java:
    // 2538-2581): per point J_k = detJ/detJ0 and dV = detJ0 w;
    // pbuf = sum_k H p(K, J_k) dV, p = W pbuf / V0; Rinv = W K / V0 for the
    // quadratic potential, else Wt R Wt with Wt = W / V0 and
    // R = sum_k H H^T modulus(K, J_k) dV
    const double* mp = mat + (size_t)elem_mat[e] * kMatParams;
    const double K = mp[5], V0 = rest_vol[e];
    const bool quad = mp[7] == 0;
    double pbuf[NPV], R[NPV * NPV];
#pragma unroll
    for (int i = 0; i < NPV; i++) pbuf[i] = 0;
#pragma unroll
    for (int i = 0; i < NPV * NPV; i++) R[i] = 0;
    for (int k = 0; k < NIP; k++) {
      double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
      for (int n = 0; n < NEN; n++) {
        const double* pn = x + 3 * (size_t)nodes[n];
        const double g0 = gns<double, TYPE>(k, n, 0), g1 = gns<double, TYPE>(k, n, 1), g2 = gns<double, TYPE>(k, n, 2);
#pragma unroll
        for (int r = 0; r < 3; r++) {
          J[3 * r] += pn[r] * g0;
          J[3 * r + 1] += pn[r] * g1;
          J[3 * r + 2] += pn[r] * g2;
        }
      }
      const double dJ0 = detJ0[(size_t)e * NIP + k];
      const double Jk = det3(J) / dJ0;
      const double dV = dJ0 * ip_weight<double, TYPE>(k);
      const double pv = (quad ? K * (Jk - 1) : K * log(Jk) / Jk) * dV;
#pragma unroll
      for (int i = 0; i < NPV; i++) pbuf[i] += press_H<TYPE>(k, i) * pv;
      if (!quad) {
        const double mod = K * (1 - log(Jk)) / (Jk * Jk);
#pragma unroll
        for (int i = 0; i < NPV; i++)
#pragma unroll
          for (int j = 0; j < NPV; j++) R[i * NPV + j] += press_H<TYPE>(k, i) * press_H<TYPE>(k, j) * mod * dV;
      }
    }
#pragma unroll
    for (int i = 0; i < NPV; i++) {
      double pi = 0;
#pragma unroll
      for (int j = 0; j < NPV; j++) pi += press_W<TYPE>(i, j) * pbuf[j];
      elem_p[(size_t)e * NPV + i] = pi / V0;
    }
    double* Ro = elem_r + (size_t)e * NPV * NPV;
    if (quad) {
#pragma unroll
      for (int i = 0; i < NPV; i++)
#pragma unroll
        for (int j = 0; j < NPV; j++) Ro[i * NPV + j] = press_W<TYPE>(i, j) * (K / V0);
    } else {
      double RW[NPV * NPV];
#pragma unroll
      for (int i = 0; i < NPV; i++)
#pragma unroll
        for (int j = 0; j < NPV; j++) {
          double t = 0;
#pragma unroll
          for (int l = 0; l < NPV; l++) t += R[i * NPV + l] * (press_W<TYPE>(l, j) / V0);
          RW[i * NPV + j] = t;
        }
#pragma unroll
      for (int i = 0; i < NPV; i++)
#pragma unroll
        for (int j = 0; j < NPV; j++) {
          double t = 0;
#pragma unroll
          for (int l = 0; l < NPV; l++) t += (press_W<TYPE>(i, l) / V0) * RW[l * NPV + j];
          Ro[i * NPV + j] = t;
        }
    }
    return;
  }
  double V = 0;
#pragma unroll
  for (int q = 0; q < NIP; q++) {
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < NEN; k++) {
      const double* pk = x + 3 * (size_t)nodes[k];
      const double g0 = gns<double, TYPE>(q, k, 0), g1 = gns<double, TYPE>(q, k, 1), g2 = gns<double, TYPE>(q, k, 2);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        J[3 * r] += pk[r] * g0;
        J[3 * r + 1] += pk[r] * g1;
        J[3 * r + 2] += pk[r] * g2;
      }
    }
    V += TYPE == B200FEM_ELEM_TET ? det3(J) / 6 : det3(J) * ip_weight<double, TYPE>(q);
  }
  const double* mp = mat + (size_t)elem_mat[e] * kMatParams;
  const double K = mp[5], V0 = rest_vol[e], Jp = V / V0;
  double p, keff;
  if (mp[7] == 0) {
    p = K * (Jp - 1);
    keff = K;
  } else {
    p = K * log(Jp) / Jp;
    keff = K * (1 - log(Jp)) / (Jp * Jp);
  }
  elem_p[e] = p;
  elem_r[e] = keff / V0;
}

cudaError_t launch_element_pressure(Engine& eng) {
  DevPack& d = eng.d;
  for (const ElemGroup& g : eng.groups) {
    if (!g.elem_inc || g.e1 <= g.e0) continue;
    const int threads = 128, blocks = (g.e1 - g.e0 + threads - 1) / threads;
    cudaError_t e = by_elem_type(g.elem_type, [&](auto tag) {
      element_pressure_kernel<decltype(tag)::value><<<blocks, threads, 0, eng.stream>>>(
          0, g.e1 - g.e0, at(d.conn, g.c0), at(d.elem_mat, g.e0), d.x, at(d.elem_rest_vol, g.e0), d.mat,
          at(d.detJ0, g.ip0), at(d.elem_p, g.pv0), at(d.elem_r, g.pv20));
      return cudaGetLastError();
    });
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// One-time preparation before any stream capture: constant tables and the
// shared-memory opt-in of every element kernel this pack launches.
// ---------------------------------------------------------------------------
// Iterative refinement of the mixed form against the FP64 operator.  The
// mixed form solves with the FP32 matrix; a refinement sweep forms the FP64
// residual r = b - S64 v matrix-free -- S64 v = (1 + h alpha) M v +
// (h^2 + h beta) K v, with K v summed from the elements' FP64 tangents
// (recomputed per integration point: material part B_a^T D (B v), geometric
// part L sigma g_a with L = sum_b v_b g_b^T) -- solves S32 d = r loosely with
// the same PCG and updates v += d.
// ---------------------------------------------------------------------------
template <int TYPE, int MAT>
__global__ void __launch_bounds__(128) elem_kv_kernel(ElemArgs a, const double* __restrict__ v) {
  static_assert(TYPE == B200FEM_ELEM_TET || TYPE == B200FEM_ELEM_HEX, "refinement: tets and hexes");
  constexpr int NEN = elem_nen(TYPE);
  constexpr int NIP = elem_nip(TYPE);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int e = a.e0 + (int)(t / NIP);
  const int k = (int)(t % NIP);
  bool live = e < a.e1;
  if (live && a.active && !a.active[a.elem_model[e]]) live = false;
  if (NIP == 1 && !live) return;
  double fl[NEN][3];
#pragma unroll
  for (int n = 0; n < NEN; n++) fl[n][0] = fl[n][1] = fl[n][2] = 0;
  if (live) {
    const int* nodes = a.conn + (size_t)e * NEN;
    double J[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      const double* xn = a.x + 3 * (size_t)nodes[n];
      const double g0 = gns<double, TYPE>(k, n, 0), g1 = gns<double, TYPE>(k, n, 1), g2 = gns<double, TYPE>(k, n, 2);
#pragma unroll
      for (int r = 0; r < 3; r++) {
        J[3 * r] += xn[r] * g0;
        J[3 * r + 1] += xn[r] * g1;
        J[3 * r + 2] += xn[r] * g2;
      }
    }
    double iJ0[9], F[9], invJ[9];
#pragma unroll
    for (int i = 0; i < 9; i++) iJ0[i] = a.invJ0[((size_t)e * NIP + k) * 9 + i];
    matmul3(F, J, iJ0);
    const double detF = det3(F);
    const double detJ = invert3(invJ, J);
    const double dv = detJ * ip_weight<double, TYPE>(k);
    const double* mp = a.mat + (size_t)a.elem_mat[e] * kMatParams;
    double sig[6], D[36], ca = 0, cb = 0;
    if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) neohookean_point<double>(sig, &ca, &cb, mp[0], mp[1], F, detF);
    else material_point<MAT, double>(sig, D, mp, F, detF, 0.0);
    // L = sum_b v_b g_b^T (velocities of fixed nodes are zero)
    double g[NEN][3], L[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      const double g0 = gns<double, TYPE>(k, n, 0), g1 = gns<double, TYPE>(k, n, 1), g2 = gns<double, TYPE>(k, n, 2);
#pragma unroll
      for (int c = 0; c < 3; c++) g[n][c] = invJ[c] * g0 + invJ[3 + c] * g1 + invJ[6 + c] * g2;
      const int r = a.sidx[nodes[n]];
      if (r < 0) continue;
      const double* vn = v + 3 * (size_t)r;
#pragma unroll
      for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) L[3 * i + j] += vn[i] * g[n][j];
    }
    // engineering strain B v and tau = D (B v), Voigt xx yy zz xy yz xz
    const double eps[6] = {L[0], L[4], L[8], L[1] + L[3], L[5] + L[7], L[2] + L[6]};
    double tau[6];
    if constexpr (MAT == B200FEM_MAT_NEOHOOKEAN) {
      const double tr = eps[0] + eps[1] + eps[2];
#pragma unroll
      for (int i = 0; i < 3; i++) tau[i] = ca * tr + 2.0 * cb * eps[i];
#pragma unroll
      for (int i = 3; i < 6; i++) tau[i] = cb * eps[i];
    } else {
#pragma unroll
      for (int i = 0; i < 6; i++) {
        double s = 0;
#pragma unroll
        for (int j = 0; j < 6; j++) s += D[6 * i + j] * eps[j];
        tau[i] = s;
      }
    }
#pragma unroll
    for (int n = 0; n < NEN; n++) {
      add_stress_force(fl[n], g[n], tau, dv);
      // geometric part: L sigma g_a dv
      const double sg0 = sig[0] * g[n][0] + sig[3] * g[n][1] + sig[5] * g[n][2];
      const double sg1 = sig[3] * g[n][0] + sig[1] * g[n][1] + sig[4] * g[n][2];
      const double sg2 = sig[5] * g[n][0] + sig[4] * g[n][1] + sig[2] * g[n][2];
#pragma unroll
      for (int i = 0; i < 3; i++) fl[n][i] += dv * (L[3 * i] * sg0 + L[3 * i + 1] * sg1 + L[3 * i + 2] * sg2);
    }
  }
  if constexpr (NIP > 1) {
#pragma unroll
    for (int n = 0; n < NEN; n++)
#pragma unroll
      for (int c = 0; c < 3; c++)
#pragma unroll
        for (int off = 4; off > 0; off >>= 1) fl[n][c] += __shfl_xor_sync(0xffffffffu, fl[n][c], off);
    if (!live || k != 0) return;
  }
  double* out = (double*)a.elemF + (size_t)e * NEN * 3;
#pragma unroll
  for (int n = 0; n < NEN; n++)
#pragma unroll
    for (int c = 0; c < 3; c++) out[3 * n + c] = fl[n][c];
}

// r = b - (1 + h alpha) m v - (h^2 + h beta) (K v), per active row (K v
// summed from the element products in element order); the correction starts
// at zero
__global__ void refine_residual_kernel(int N, const int* __restrict__ inc_ptr, const int* __restrict__ inc_idx,
                                       const double* __restrict__ ekv, const int* __restrict__ sidx,
                                       const int* __restrict__ node_model, const double* __restrict__ mass,
                                       const double* __restrict__ step, const double* __restrict__ b,
                                       const double* __restrict__ v, double* __restrict__ r,
                                       double* __restrict__ dsol, const int* __restrict__ active) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  const int row = sidx[n];
  if (row < 0) return;
  double kv[3] = {0, 0, 0};
  const bool on = !active || active[node_model[n]];
  if (on)
    for (int i = inc_ptr[n]; i < inc_ptr[n + 1]; i++)
#pragma unroll
      for (int c = 0; c < 3; c++) kv[c] += ekv[(size_t)inc_idx[i] * 3 + c];
  const double* sp = step + (size_t)node_model[n] * 8;
  const double h = sp[0], al = sp[1], be = sp[2];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const size_t q = 3 * (size_t)row + c;
    r[q] = on ? b[q] - (1.0 + h * al) * mass[n] * v[q] - (h * h + h * be) * kv[c] : 0.0;
    dsol[q] = 0.0;
  }
}

__global__ void refine_add_kernel(int R, double* __restrict__ v, const double* __restrict__ dv) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q < 3LL * R) v[q] += dv[q];
}

// v_prev = v, v = v1, x += h v1 for the active rows (the PCG's own update,
// done here after the refinement sweeps)
__global__ void refine_state_kernel(int R, const int* __restrict__ act_node, const int* __restrict__ row_model,
                                    const double* __restrict__ step, const double* __restrict__ sol,
                                    double* __restrict__ x, double* __restrict__ vel, double* __restrict__ vprev,
                                    double* __restrict__ vprev2, double* __restrict__ vprev3,
                                    double* __restrict__ vprev4, const int* __restrict__ active) {
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= R) return;
  const int m = row_model[row];
  if (active && !active[m]) return;
  const int n = act_node[row];
  const double h = step[(size_t)m * 8];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double vn = sol[3 * (size_t)row + c];
    vprev4[3 * (size_t)n + c] = vprev3[3 * (size_t)n + c];
    vprev3[3 * (size_t)n + c] = vprev2[3 * (size_t)n + c];
    vprev2[3 * (size_t)n + c] = vprev[3 * (size_t)n + c];
    vprev[3 * (size_t)n + c] = vel[3 * (size_t)n + c];
    vel[3 * (size_t)n + c] = vn;
    x[3 * (size_t)n + c] += h * vn;
  }
}

// the solve phase of a BackwardEuler step: PCG, then the refinement sweeps
// of the mixed form (when asked for and supported) and the state update
cudaError_t launch_state_update(Engine& eng, const double* vsol) {
  DevPack& d = eng.d;
  const int* act = eng.any_inactive ? d.model_active : nullptr;
  refine_state_kernel<<<(d.n_rows + 127) / 128, 128, 0, eng.stream>>>(d.n_rows, d.act_node, d.row_model, d.step,
                                                                      vsol, d.x, d.v, d.vprev, d.vprev2, d.vprev3,
                                                                      d.vprev4, act);
  return cudaGetLastError();
}

cudaError_t launch_solve(Engine& eng, int max_iter) {
  if (eng.pcons.active() && eng.integrator == B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER)
    return launch_solve_points(eng, max_iter);
  DevPack& d = eng.d;
  const int sweeps = eng.refine_ok ? eng.opt_refine : 0;
  if (sweeps == 0) return launch_pcg(eng, max_iter, true, 0);
  cudaError_t e = launch_pcg(eng, max_iter, false, 0);
  const int* act = eng.any_inactive ? d.model_active : nullptr;
  const ElemGroup& g = eng.groups[0];
  ElemArgs a = elem_args(eng, g, true);
  const int ne = g.e1 - g.e0;
  constexpr int TET = B200FEM_ELEM_TET, HEX = B200FEM_ELEM_HEX, NH = B200FEM_MAT_NEOHOOKEAN,
                MR = B200FEM_MAT_MOONEYRIVLIN;
  const int nip = eng.elem_type == TET ? 1 : 8;
  const unsigned kb = (unsigned)(((long long)ne * nip + 127) / 128);
  for (int s = 0; s < sweeps && e == cudaSuccess; s++) {
    if (ne > 0) {
      if (eng.elem_type == TET) {
        if (g.mat_kind == NH) elem_kv_kernel<TET, NH><<<kb, 128, 0, eng.stream>>>(a, d.sol);
        else elem_kv_kernel<TET, MR><<<kb, 128, 0, eng.stream>>>(a, d.sol);
      } else {
        if (g.mat_kind == NH) elem_kv_kernel<HEX, NH><<<kb, 128, 0, eng.stream>>>(a, d.sol);
        else elem_kv_kernel<HEX, MR><<<kb, 128, 0, eng.stream>>>(a, d.sol);
      }
    }
    refine_residual_kernel<<<(d.n_nodes + 127) / 128, 128, 0, eng.stream>>>(
        d.n_nodes, d.inc_ptr, d.inc_idx, d.elemF, d.sidx, d.node_model, d.mass, d.step, d.b, d.sol, d.rref,
        d.dsol, act);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    e = launch_pcg_on(eng, max_iter, false, d.rref, d.dsol, eng.refine_tol, d.model_scal2);
    if (e != cudaSuccess) return e;
    refine_add_kernel<<<(unsigned)((3LL * d.n_rows + 255) / 256), 256, 0, eng.stream>>>(d.n_rows, d.sol, d.dsol);
  }
  refine_state_kernel<<<(d.n_rows + 127) / 128, 128, 0, eng.stream>>>(d.n_rows, d.act_node, d.row_model, d.step,
                                                                      d.sol, d.x, d.v, d.vprev, d.vprev2, d.vprev3,
                                                                      d.vprev4, act);
  return cudaGetLastError();
}

static cudaError_t launch_fused_blocks(Engine& eng, int chunks);

cudaError_t prepare_kernels(Engine& eng) {
  cudaError_t e = ensure_constants(eng.device);
  if (e != cudaSuccess) return e;
  if (eng.fused && (e = launch_fused_blocks(eng, -1)) != cudaSuccess) return e;
  if (eng.tet_rows && (e = launch_tet_rows(eng, true)) != cudaSuccess) return e;
  const bool fp32 = eng.precision == B200FEM_PREC_MIXED;
  for (ElemGroup g : eng.groups) {
    g.e1 = g.e0 - 1;  // ne = -1: set attributes only
    e = by_elem_type(g.elem_type, [&](auto tag) {
      constexpr int TY = decltype(tag)::value;
      return fp32 ? launch_group<TY, float>(eng, g, true) : launch_group<TY, double>(eng, g, false);
    });
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

size_t fused_elem_bytes(int elem_type, int mat_kind, bool fp32) {
  const bool tet = elem_type == B200FEM_ELEM_TET, nh = mat_kind == B200FEM_MAT_NEOHOOKEAN;
  if (tet) {
    if (nh) return fp32 ? FusedSmem<B200FEM_ELEM_TET, B200FEM_MAT_NEOHOOKEAN, float>::per_elem()
                        : FusedSmem<B200FEM_ELEM_TET, B200FEM_MAT_NEOHOOKEAN, double>::per_elem();
    return fp32 ? FusedSmem<B200FEM_ELEM_TET, B200FEM_MAT_MOONEYRIVLIN, float>::per_elem()
                : FusedSmem<B200FEM_ELEM_TET, B200FEM_MAT_MOONEYRIVLIN, double>::per_elem();
  }
  if (nh) return fp32 ? FusedSmem<B200FEM_ELEM_HEX, B200FEM_MAT_NEOHOOKEAN, float>::per_elem()
                      : FusedSmem<B200FEM_ELEM_HEX, B200FEM_MAT_NEOHOOKEAN, double>::per_elem();
  return fp32 ? FusedSmem<B200FEM_ELEM_HEX, B200FEM_MAT_MOONEYRIVLIN, float>::per_elem()
              : FusedSmem<B200FEM_ELEM_HEX, B200FEM_MAT_MOONEYRIVLIN, double>::per_elem();
}

// chunks < 0: set the kernel's shared-memory attribute only
static cudaError_t launch_fused_blocks(Engine& eng, int chunks) {
  DevPack& d = eng.d;
  FusedArgs fa;
  fa.chunk_row = d.chunk_row;
  fa.chunk_eptr = d.chunk_eptr;
  fa.chunk_elem = d.chunk_elem;
  fa.contrib_ptr = d.contrib_ptr;
  fa.contrib_loc = d.contrib_loc;
  fa.rowptr = d.blk_rowptr;
  fa.blk_row = d.blk_row;
  fa.blk_diag = d.blk_diag;
  fa.row_model = d.row_model;
  fa.act_node = d.act_node;
  fa.mass = d.mass;
  fa.step = d.step;
  fa.conn = d.conn;
  fa.elem_model = d.elem_model;
  fa.elem_mat = d.elem_mat;
  fa.active = eng.any_inactive ? d.model_active : nullptr;
  fa.x = d.x;
  fa.invJ0 = d.invJ0;
  fa.invJ0_f = d.invJ0_f;
  fa.mat = d.mat;
  const bool fp32 = eng.precision == B200FEM_PREC_MIXED;
  fa.out = fp32 ? (void*)d.S_f : (void*)d.S;
  const int em = eng.fused_emax;
  const bool tet = eng.elem_type == B200FEM_ELEM_TET;
  const bool nh = eng.groups[0].mat_kind == B200FEM_MAT_NEOHOOKEAN;
  constexpr int TET = B200FEM_ELEM_TET, HEX = B200FEM_ELEM_HEX, NH = B200FEM_MAT_NEOHOOKEAN,
                MR = B200FEM_MAT_MOONEYRIVLIN;
  cudaStream_t st = eng.stream;
  if (fp32) {
    if (tet) return nh ? launch_fused<TET, NH, float, float>(fa, chunks, em, st) : launch_fused<TET, MR, float, float>(fa, chunks, em, st);
    return nh ? launch_fused<HEX, NH, float, float>(fa, chunks, em, st) : launch_fused<HEX, MR, float, float>(fa, chunks, em, st);
  }
  if (tet) return nh ? launch_fused<TET, NH, double, double>(fa, chunks, em, st) : launch_fused<TET, MR, double, double>(fa, chunks, em, st);
  return nh ? launch_fused<HEX, NH, double, double>(fa, chunks, em, st) : launch_fused<HEX, MR, double, double>(fa, chunks, em, st);
}

// BackwardEuler assembly on the fused path: FP64 nodal forces (and the
// inverted-element statistics) per element, then the blocks of S per row chunk
static cudaError_t launch_assemble_fused(Engine& eng) {
  const ElemGroup& g = eng.groups[0];
  ElemArgs a = elem_args(eng, g, eng.precision == B200FEM_PREC_MIXED);
  a.det_stats = 1;
  const int ne = g.e1 - g.e0;
  cudaError_t e = cudaSuccess;
  constexpr int TET = B200FEM_ELEM_TET, HEX = B200FEM_ELEM_HEX, NH = B200FEM_MAT_NEOHOOKEAN,
                MR = B200FEM_MAT_MOONEYRIVLIN;
  if (ne > 0) {
    if (eng.elem_type == TET)
      e = g.mat_kind == NH ? launch_force<TET, NH, kIncOff>(a, ne, eng.stream) : launch_force<TET, MR, kIncOff>(a, ne, eng.stream);
    else
      e = g.mat_kind == NH ? launch_force<HEX, NH, kIncOff>(a, ne, eng.stream) : launch_force<HEX, MR, kIncOff>(a, ne, eng.stream);
  }
  if (e != cudaSuccess) return e;
  return launch_fused_blocks(eng, eng.fused_chunks);
}

cudaError_t launch_assemble(Engine& eng, double cK, double cM, bool want_K) {
  (void)cK;
  (void)cM;
  cudaError_t e = cudaSuccess;
  DevPack& d = eng.d;
  const bool fp32 = eng.precision == B200FEM_PREC_MIXED;
  if (!want_K && eng.fused) return launch_assemble_fused(eng);
  if ((e = launch_nodal_pressure(eng)) != cudaSuccess) return e;
  if ((e = launch_divblk(eng)) != cudaSuccess) return e;
  if ((e = launch_element_pressure(eng)) != cudaSuccess) return e;
  // the step on the node-row path: S, the nodal forces, b and the PCG's
  // initial guess in one launch per group (launch_rhs then has nothing left)
  if (!want_K && eng.tet_rows) return launch_tet_rows(eng, false);
  for (const ElemGroup& g : eng.groups) {
    e = by_elem_type(g.elem_type, [&](auto tag) {
      constexpr int TY = decltype(tag)::value;
      return fp32 ? launch_group<TY, float>(eng, g, true) : launch_group<TY, double>(eng, g, false);
    });
    if (e != cudaSuccess) return e;
  }
  const int* act = eng.any_inactive ? d.model_active : nullptr;
  if (d.n_up == 0) return cudaSuccess;
  if (!want_K && eng.factored) {
    // the step's factored solve matrix: the direct blocks into S1, without
    // the dilational triples (the PCG applies that term from divBlk)
    if (d.n_up1 == 0) return cudaSuccess;
    const unsigned blocks = (unsigned)((d.n_up1 + 255) / 256);
    if (fp32)
      gather_block_kernel<float, float><<<blocks, 256, 0, eng.stream>>>(
          d.n_up1, d.up1, d.contrib_ptr, d.contrib_idx, d.elemK_f, d.blk_row, d.blk_diag, d.row_model, d.act_node,
          d.mass, d.step, 1, d.S1_f, nullptr, nullptr, nullptr, nullptr, act, d.blk_mirror, d.up1_dst, d.up1_mdst);
    else
      gather_block_kernel<double, double><<<blocks, 256, 0, eng.stream>>>(
          d.n_up1, d.up1, d.contrib_ptr, d.contrib_idx, d.elemK, d.blk_row, d.blk_diag, d.row_model, d.act_node,
          d.mass, d.step, 1, d.S1, nullptr, nullptr, nullptr, nullptr, act, d.blk_mirror, d.up1_dst, d.up1_mdst);
    return cudaGetLastError();
  }
  // Matrices that stay in L2 (up to 64 MB of blocks): one thread per block
  // with warp-staged contiguous stores (the 40x10x10 hex beam: 13.1 us per
  // gather against 17.3 for the list form); larger ones stream from HBM and
  // take one thread per upper block from the list, so no lane idles (the
  // 256-beam pack: 378 -> 322 us; the 60x30x30 MooneyRivlin block: 490 -> 343)
  const double kbytes = 9.0 * (fp32 && !want_K ? 4 : 8) * (double)d.nnzb;
  if (kbytes <= 64e6) {
    const unsigned sb = (unsigned)((d.nnzb + 255) / 256);
    if (fp32) {
      if (want_K)
        gather_staged_kernel<float, double><<<sb, 256, 0, eng.stream>>>(
            d.nnzb, d.contrib_ptr, d.contrib_idx, d.elemK_f, d.blk_row, d.blk_diag, d.row_model, d.act_node, d.mass,
            d.step, 0, d.K, d.dil_ptr, d.dil_idx, d.divblk, d.node_kp, act, d.blk_mirror);
      else
        gather_staged_kernel<float, float><<<sb, 256, 0, eng.stream>>>(
            d.nnzb, d.contrib_ptr, d.contrib_idx, d.elemK_f, d.blk_row, d.blk_diag, d.row_model, d.act_node, d.mass,
            d.step, 1, d.S_f, d.dil_ptr, d.dil_idx, d.divblk, d.node_kp, act, d.blk_mirror);
    } else {
      gather_staged_kernel<double, double><<<sb, 256, 0, eng.stream>>>(
          d.nnzb, d.contrib_ptr, d.contrib_idx, d.elemK, d.blk_row, d.blk_diag, d.row_model, d.act_node, d.mass,
          d.step, want_K ? 0 : 1, want_K ? d.K : d.S, d.dil_ptr, d.dil_idx, d.divblk, d.node_kp, act, d.blk_mirror);
    }
    return cudaGetLastError();
  }
  // one thread per upper block
  const unsigned blocks = (unsigned)((d.n_up + 255) / 256);
  if (fp32) {
    if (want_K)
      gather_block_kernel<float, double><<<blocks, 256, 0, eng.stream>>>(
          d.n_up, d.up_blocks, d.contrib_ptr, d.contrib_idx, d.elemK_f, d.blk_row, d.blk_diag, d.row_model,
          d.act_node, d.mass, d.step, 0, d.K, d.dil_ptr, d.dil_idx, d.divblk, d.node_kp, act, d.blk_mirror, nullptr, nullptr);
    else
      gather_block_kernel<float, float><<<blocks, 256, 0, eng.stream>>>(
          d.n_up, d.up_blocks, d.contrib_ptr, d.contrib_idx, d.elemK_f, d.blk_row, d.blk_diag, d.row_model,
          d.act_node, d.mass, d.step, 1, d.S_f, d.dil_ptr, d.dil_idx, d.divblk, d.node_kp, act, d.blk_mirror, nullptr, nullptr);
  } else {
    gather_block_kernel<double, double><<<blocks, 256, 0, eng.stream>>>(
        d.n_up, d.up_blocks, d.contrib_ptr, d.contrib_idx, d.elemK, d.blk_row, d.blk_diag, d.row_model,
        d.act_node, d.mass, d.step, want_K ? 0 : 1, want_K ? d.K : d.S, d.dil_ptr, d.dil_idx, d.divblk,
        d.node_kp, act, d.blk_mirror, nullptr, nullptr);
  }
  return cudaGetLastError();
}

// per-call reset of the status words: error, inverted-element count, and
// the smallest detJ (ordered-bits image of DBL_MAX)
__global__ void reset_status_kernel(int* flags, long long* dmin) {
  if (threadIdx.x < 4) flags[threadIdx.x] = 0;
  if (threadIdx.x == 0) *dmin = 0x7fefffffffffffffll;
}

// one record of the step's status for the host: flags, smallest detJ (the
// ordered bits, moved as a double image) and the per-model results, written
// into mapped pinned memory so that a single synchronisation delivers it
__global__ void status_pack_kernel(const int* __restrict__ flags, const long long* __restrict__ dmin,
                                   const double* __restrict__ ms, int n, double* __restrict__ out) {
  if (threadIdx.x < 4) out[threadIdx.x] = (double)flags[threadIdx.x];
  if (threadIdx.x == 4) out[4] = __longlong_as_double(*dmin);
  for (int i = threadIdx.x; i < n; i += blockDim.x) out[5 + i] = ms[i];
}

cudaError_t launch_status_pack(Engine& eng) {
  status_pack_kernel<<<1, 256, 0, eng.stream>>>(eng.d.flags, (const long long*)eng.d.dmin, eng.d.model_scal,
                                                4 * eng.d.n_models, eng.d.status_dev);
  return cudaGetLastError();
}

cudaError_t launch_reset_status(Engine& eng) {
  reset_status_kernel<<<1, 32, 0, eng.stream>>>(eng.d.flags, (long long*)eng.d.dmin);
  return cudaGetLastError();
}

static cudaError_t launch_rows(Engine& eng, double* b, double* sol) {
  DevPack& d = eng.d;
  const int threads = 64;
  const int blocks = (d.n_nodes + threads - 1) / threads;
  const int* act = eng.any_inactive ? d.model_active : nullptr;
  const double* vp = eng.opt_warm_start >= 1 ? d.vprev : nullptr;
  const double* vp2 = eng.opt_warm_start >= 2 ? d.vprev2 : nullptr;
  const double* vp3 = eng.opt_warm_start >= 3 ? d.vprev3 : nullptr;
  const double* vp4 = eng.opt_warm_start == 4 ? d.vprev4 : nullptr;
  const double* nrm =
      (sol && eng.integrator == B200FEM_INTEGRATOR_CONSTRAINED_BACKWARD_EULER && d.row_nrm) ? d.row_nrm : nullptr;
  // nodal forces are FP64 in both forms
  rows_kernel<double><<<blocks, threads, 0, eng.stream>>>(d.n_nodes, d.inc_ptr, d.inc_idx, d.elemF, d.sidx,
                                                         d.node_model, d.mass, d.v, d.fext, d.step, d.fint, b, sol, act, vp,
                                                         vp2, vp3, vp4, nrm);
  return cudaGetLastError();
}

// follows launch_assemble(..., want_K = false) in the step; the node-row
// path has formed b and the initial guess already
cudaError_t launch_rhs(Engine& eng) { return eng.tet_rows ? cudaSuccess : launch_rows(eng, eng.d.b, eng.d.sol); }

cudaError_t launch_forces_only(Engine& eng) { return launch_rows(eng, nullptr, nullptr); }

cudaError_t launch_spmv(Engine& eng, const double* x, double* y) {
  DevPack& d = eng.d;
  int threads = 256;
  long long blocks = ((long long)d.n_rows * 32 + threads - 1) / threads;
  if (eng.factored) {
    if (eng.precision == B200FEM_PREC_MIXED)
      spmv_kernel<float><<<(unsigned)blocks, threads, 0, eng.stream>>>(d.n_rows, d.s1_rowptr, d.s1_col, d.S1_f, x, y);
    else
      spmv_kernel<double><<<(unsigned)blocks, threads, 0, eng.stream>>>(d.n_rows, d.s1_rowptr, d.s1_col, d.S1, x, y);
    if (d.n_dil_nodes > 0) {
      dil_t_kernel<<<(d.n_dil_nodes + 127) / 128, 128, 0, eng.stream>>>(
          d.n_dil_nodes, d.dil_nodes, d.nbr_ptr, d.nbr_row, d.divblk, d.node_kp, d.node_model, d.step, x, d.dil_t);
      dil_add_kernel<<<(d.n_rows + 127) / 128, 128, 0, eng.stream>>>(d.n_rows, d.dil_rptr, d.dil_node, d.dil_slot,
                                                                     d.divblk, d.dil_t, y);
    }
    return cudaGetLastError();
  }
  if (eng.precision == B200FEM_PREC_MIXED)
    spmv_kernel<float><<<(unsigned)blocks, threads, 0, eng.stream>>>(d.n_rows, d.blk_rowptr, d.blk_col, d.S_f, x, y);
  else
    spmv_kernel<double><<<(unsigned)blocks, threads, 0, eng.stream>>>(d.n_rows, d.blk_rowptr, d.blk_col, d.S, x, y);
  return cudaGetLastError();
}

void crs_export_kernel_launch(Engine& eng, long long nnzb, const int* blk_row, const int* rowptr, const double* vals,
                              double* crs) {
  const long long n9 = nnzb * 9;
  crs_export_kernel<<<(unsigned)((n9 + 255) / 256), 256, 0, eng.stream>>>(nnzb, blk_row, rowptr, vals, crs);
}

cudaError_t launch_crs_export(Engine& eng, const double* vals, double* crs) {
  DevPack& d = eng.d;
  long long n9 = d.nnzb * 9;
  int threads = 256;
  crs_export_kernel<<<(unsigned)((n9 + threads - 1) / threads), threads, 0, eng.stream>>>(d.nnzb, d.blk_row,
                                                                                         d.blk_rowptr, vals, crs);
  return cudaGetLastError();
}

}  // namespace b200fem
