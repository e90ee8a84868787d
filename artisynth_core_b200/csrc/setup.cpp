// setup.cpp -- host-side setup of the B200 FEM engine: grid factory, rest
// data, lumped masses, linear stiffness cache, block pattern, CRS slot map
// and the element-to-block scatter map.  Runs once per structure change
// (the reference rebuilds these only when the solve-matrix structure
// version changes, MechSystemSolver.updateSolveMatrixStructure,
// MechSystemSolver.java:2484-2493).
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <cstring>
#include <numeric>

#include "engine.h"

namespace b200fem {

namespace {

// Shape-function derivatives dN/ds for the reference elements.
// TetElement.getdNds (TetElement.java:204-215); one integration point, weight
// 1/6 (TetElement.java:31-33).
const double kTetGNs[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
// HexElement node natural coordinates (HexElement.java:119-129)
const double kHexNode[8][3] = {{-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
                               {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}};

void hex_grad(double* g, int i, double s0, double s1, double s2) {
  // HexElement.getdNds (HexElement.java:266-281)
  double a = kHexNode[i][0] < 0 ? -1 : 1, b = kHexNode[i][1] < 0 ? -1 : 1,
         c = kHexNode[i][2] < 0 ? -1 : 1;
  g[0] = 0.125 * a * (1 + b * s1) * (1 + c * s2);
  g[1] = 0.125 * (1 + a * s0) * b * (1 + c * s2);
  g[2] = 0.125 * (1 + a * s0) * (1 + b * s1) * c;
}

double det33(const double* m) {
  return m[0] * m[4] * m[8] + m[3] * m[7] * m[2] + m[6] * m[1] * m[5] - m[6] * m[4] * m[2] -
         m[0] * m[7] * m[5] - m[3] * m[1] * m[8];
}

// Matrix3dBase.fastInvert (Matrix3dBase.java:1615-1648)
double invert33(double* inv, const double* d) {
  double det = det33(d);
  if (det != 0) {
    double s = 1.0 / det;
    inv[0] = s * (d[4] * d[8] - d[5] * d[7]);
    inv[1] = s * (d[2] * d[7] - d[1] * d[8]);
    inv[2] = s * (d[1] * d[5] - d[4] * d[2]);
    inv[3] = s * (d[5] * d[6] - d[3] * d[8]);
    inv[4] = s * (d[0] * d[8] - d[2] * d[6]);
    inv[5] = s * (d[2] * d[3] - d[0] * d[5]);
    inv[6] = s * (d[3] * d[7] - d[4] * d[6]);
    inv[7] = s * (d[1] * d[6] - d[0] * d[7]);
    inv[8] = s * (d[0] * d[4] - d[1] * d[3]);
  }
  return det;
}

// WedgeElement.getdNds (WedgeElement.java:193-206): N_i = L_t(s1, s2) h_z(r)
// with the triangle coordinates L = (1 - s1 - s2, s1, s2) of node t = i % 3
// and the layer factor h = (1 -/+ r)/2 of z = i / 3
void wedge_grad(double* g, int i, double s1, double s2, double r) {
  const int t = i % 3;
  const double sgn = i < 3 ? -1.0 : 1.0, h = 0.5 * (1 + sgn * r);
  const double L = t == 0 ? 1 - s1 - s2 : (t == 1 ? s1 : s2);
  const double dL1 = t == 0 ? -1.0 : (t == 1 ? 1.0 : 0.0), dL2 = t == 0 ? -1.0 : (t == 2 ? 1.0 : 0.0);
  g[0] = dL1 * h;
  g[1] = dL2 * h;
  g[2] = L * 0.5 * sgn;
}

// PyramidElement.getdNds (PyramidElement.java:153-175): base nodes (a, b, -1)
// with N = (1 + a s0)(1 + b s1)(1 - s2)/8, apex N = (1 + s2)/2
const double kPyrBase[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
void pyramid_grad(double* g, int i, double s0, double s1, double s2) {
  if (i == 4) {
    g[0] = g[1] = 0;
    g[2] = 0.5;
    return;
  }
  const double a = kPyrBase[i][0], b = kPyrBase[i][1];
  g[0] = 0.125 * a * (1 + b * s1) * (1 - s2);
  g[1] = 0.125 * (1 + a * s0) * b * (1 - s2);
  g[2] = -0.125 * (1 + a * s0) * (1 + b * s1);
}

// QuadtetElement.getdNds (QuadtetElement.java:301-323) at (s1, s2, s3),
// s0 = 1 - s1 - s2 - s3: corner n has N = s_n (2 s_n - 1), the edge node
// between corners a and b N = 4 s_a s_b
const int kQtetEdge[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
void quadtet_grad(double* g, int i, const double* s /* s0..s3 */) {
  // ds_n/d(s1, s2, s3): s0 -> (-1, -1, -1), s_j -> unit j
  auto ds = [](int n, int c) { return n == 0 ? -1.0 : (n == c + 1 ? 1.0 : 0.0); };
  for (int c = 0; c < 3; c++) {
    if (i < 4) {
      g[c] = (4 * s[i] - 1) * ds(i, c);
    } else {
      const int a = kQtetEdge[i - 4][0], b = kQtetEdge[i - 4][1];
      g[c] = 4 * (ds(a, c) * s[b] + s[a] * ds(b, c));
    }
  }
}

// QuadhexElement node coordinates (QuadhexElement.java:117-142) and its
// serendipity shape gradients (getdNds, :482-560): a corner (a, b, c) has
// N = (1 + a s)(1 + b t)(1 + c r)(a s + b t + c r - 2)/8, an edge node with
// a zero coordinate, e.g. (0, b, c), N = (1 - s^2)(1 + b t)(1 + c r)/4
const double kQhexNode[20][3] = {{-1, -1, 1}, {1, -1, 1}, {1, 1, 1},  {-1, 1, 1},  {-1, -1, -1}, {1, -1, -1}, {1, 1, -1},
                                 {-1, 1, -1}, {0, -1, 1}, {1, 0, 1},  {0, 1, 1},   {-1, 0, 1},   {0, -1, -1}, {1, 0, -1},
                                 {0, 1, -1},  {-1, 0, -1}, {-1, -1, 0}, {1, -1, 0}, {1, 1, 0},   {-1, 1, 0}};
void quadhex_grad(double* g, int i, const double* x /* s, t, r */) {
  const double* c = kQhexNode[i];
  double f[3];  // 1 + c_j x_j
  for (int j = 0; j < 3; j++) f[j] = 1 + c[j] * x[j];
  if (c[0] != 0 && c[1] != 0 && c[2] != 0) {
    const double sum = c[0] * x[0] + c[1] * x[1] + c[2] * x[2];
    for (int j = 0; j < 3; j++) {
      const int a = (j + 1) % 3, b = (j + 2) % 3;
      g[j] = 0.125 * c[j] * f[a] * f[b] * (sum - 2 + f[j]);
    }
    return;
  }
  const int z = c[0] == 0 ? 0 : (c[1] == 0 ? 1 : 2);  // the edge's own direction
  for (int j = 0; j < 3; j++) {
    const int a = (j + 1) % 3, b = (j + 2) % 3;
    if (j == z) g[j] = -0.5 * x[z] * f[a] * f[b];
    else {
      const int o = (a == z) ? b : a;  // the other non-zero coordinate
      g[j] = 0.25 * (1 - x[z] * x[z]) * c[j] * f[o];
    }
  }
}

// QuadwedgeElement (QuadwedgeElement.java:129-148, getdNds :301-333) at
// (s1, s2, r), triangle coordinates L = (s0, s1, s2), layer z = -/+1:
// corners N = L_t (1 + z r)(2 L_t + z r - 2)/2, triangle mid-edges
// N = 2 L_a L_b (1 + z r), vertical mid-edges N = L_t (1 - r^2)
void quadwedge_grad(double* g, int i, double s1, double s2, double r) {
  const double L[3] = {1 - s1 - s2, s1, s2};
  auto dL = [](int t, int c) { return t == 0 ? -1.0 : (t == c + 1 ? 1.0 : 0.0); };  // dL_t/ds_c, c = 0, 1
  static const int tri[3][2] = {{0, 1}, {1, 2}, {2, 0}};
  if (i < 6) {
    const int t = i % 3;
    const double z = i < 3 ? -1.0 : 1.0, hz = 1 + z * r;
    for (int c = 0; c < 2; c++) g[c] = dL(t, c) * hz * (4 * L[t] + z * r - 2) / 2;
    g[2] = L[t] * z * (2 * L[t] + 2 * z * r - 1) / 2;
  } else if (i < 12) {
    const int a = tri[(i - 6) % 3][0], b = tri[(i - 6) % 3][1];
    const double z = i < 9 ? -1.0 : 1.0, hz = 1 + z * r;
    for (int c = 0; c < 2; c++) g[c] = 2 * (dL(a, c) * L[b] + L[a] * dL(b, c)) * hz;
    g[2] = 2 * L[a] * L[b] * z;
  } else {
    const int t = i - 12;
    for (int c = 0; c < 2; c++) g[c] = dL(t, c) * (1 - r * r);
    g[2] = -2 * r * L[t];
  }
}

// QuadpyramidElement.getdNds (QuadpyramidElement.java:260-319), the
// reference's per-node expressions with q = (1 - r)/2
void quadpyramid_grad(double* g, int i, double s, double t, double r) {
  const double q = (1 - r) / 2;
  double u;
  switch (i) {
    case 0: g[0] = q * (1 - t) * (1 + q * (2 * s + t - 1)) / 4; g[1] = q * (1 - s) * (1 + q * (2 * t + s - 1)) / 4;
            g[2] = (1 - s) * (1 - t) * (1 + 2 * q * (s + t)) / 8; break;
    case 1: g[0] = -q * (1 - t) * (1 + q * (-2 * s + t - 1)) / 4; g[1] = q * (1 + s) * (1 + q * (2 * t - s - 1)) / 4;
            g[2] = (1 + s) * (1 - t) * (1 + 2 * q * (t - s)) / 8; break;
    case 2: g[0] = -q * (1 + t) * (1 + q * (-2 * s - t - 1)) / 4; g[1] = -q * (1 + s) * (1 + q * (-2 * t - s - 1)) / 4;
            g[2] = (1 + s) * (1 + t) * (1 - 2 * q * (t + s)) / 8; break;
    case 3: g[0] = q * (1 + t) * (1 + q * (2 * s - t - 1)) / 4; g[1] = -q * (1 - s) * (1 + q * (-2 * t + s - 1)) / 4;
            g[2] = (1 - s) * (1 + t) * (1 + 2 * q * (s - t)) / 8; break;
    case 4: g[0] = 0; g[1] = 0; g[2] = 0.5 + r; break;
    case 5: g[0] = -s * q * q * (1 - t); g[1] = -q * q * (1 - s * s) / 2; g[2] = -q * (1 - t) * (1 - s * s) / 2; break;
    case 6: g[0] = q * q * (1 - t * t) / 2; g[1] = -t * q * q * (1 + s); g[2] = -q * (1 + s) * (1 - t * t) / 2; break;
    case 7: g[0] = -s * q * q * (1 + t); g[1] = q * q * (1 - s * s) / 2; g[2] = -q * (1 + t) * (1 - s * s) / 2; break;
    case 8: g[0] = -q * q * (1 - t * t) / 2; g[1] = -t * q * q * (1 - s); g[2] = -q * (1 - s) * (1 - t * t) / 2; break;
    case 9: u = q * (1 - q); g[0] = u * (t - 1); g[1] = u * (s - 1); g[2] = (2 * q - 1) * (1 - s - t + s * t) / 2; break;
    case 10: u = q * (1 - q); g[0] = u * (1 - t); g[1] = -u * (1 + s); g[2] = (2 * q - 1) * (1 + s - t - s * t) / 2; break;
    case 11: u = q * (1 - q); g[0] = u * (1 + t); g[1] = u * (1 + s); g[2] = (2 * q - 1) * (1 + s + t + s * t) / 2; break;
    default: u = q * (1 - q); g[0] = -u * (1 + t); g[1] = u * (1 - s); g[2] = (2 * q - 1) * (1 - s + t - s * t) / 2; break;
  }
}

}  // namespace

// Pressure weights of the multi-pressure elements at their integration
// points -- QuadhexElement.getH (1, s, t, r) (:451-470) and
// QuadwedgeElement.getH ((1 - r)/2, (1 + r)/2) (:275-291) -- and the
// weight matrix W = (sum_k H H^T)^-1 summed over the points without their
// weights, as FemElement3d.createPressureWeightMatrix does (:226-255).
void pressure_tables(int type, double* H, double* W) {
  const int npv = elem_npv(type), nip = elem_nip(type);
  for (int k = 0; k < nip; k++) {
    double* h = H + (size_t)k * npv;
    if (type == B200FEM_ELEM_QUADHEX) {
      // the 14-point rule's coordinates (shape_grads)
      const double q = 0.758686910639328, r = 0.795822425754222;
      double x[3] = {0, 0, 0};
      if (k < 8) {
        for (int j = 0; j < 3; j++) x[j] = kQhexNode[k][j] * q;
      } else {
        x[(k - 8) / 2] = (k % 2 == 0) ? -r : r;
      }
      h[0] = 1;
      h[1] = x[0];
      h[2] = x[1];
      h[3] = x[2];
    } else {
      const double q = std::sqrt(3 / 5.0), r = k < 3 ? -q : (k < 6 ? q : 0);
      h[0] = 0.5 * (1 - r);
      h[1] = 0.5 * (1 + r);
    }
  }
  // M = sum_k H H^T, then W = M^-1 by Gauss-Jordan with partial pivoting
  double M[16] = {0}, I[16] = {0};
  for (int k = 0; k < nip; k++)
    for (int i = 0; i < npv; i++)
      for (int j = 0; j < npv; j++) M[i * npv + j] += H[k * npv + i] * H[k * npv + j];
  for (int i = 0; i < npv; i++) I[i * npv + i] = 1;
  for (int c = 0; c < npv; c++) {
    int piv = c;
    for (int r = c + 1; r < npv; r++)
      if (std::fabs(M[r * npv + c]) > std::fabs(M[piv * npv + c])) piv = r;
    for (int j = 0; j < npv; j++) {
      std::swap(M[c * npv + j], M[piv * npv + j]);
      std::swap(I[c * npv + j], I[piv * npv + j]);
    }
    const double d = M[c * npv + c];
    for (int j = 0; j < npv; j++) {
      M[c * npv + j] /= d;
      I[c * npv + j] /= d;
    }
    for (int r = 0; r < npv; r++) {
      if (r == c) continue;
      const double f = M[r * npv + c];
      for (int j = 0; j < npv; j++) {
        M[r * npv + j] -= f * M[c * npv + j];
        I[r * npv + j] -= f * I[c * npv + j];
      }
    }
  }
  for (int i = 0; i < npv * npv; i++) W[i] = I[i];
}

// Shape gradients for integration point k (or the warping point, k = -1).
void shape_grads(int type, int k, double* g /* nen*3 */, double* w) {
  if (type == B200FEM_ELEM_QUADWEDGE) {
    if (k < 0) {
      // warping point (QuadwedgeElement.getWarpingPoint): the linear wedge's
      // gradients at (1/3, 1/3, 0) on the corners, zero elsewhere, weight 1
      std::memset(g, 0, 45 * sizeof(double));
      for (int i = 0; i < 6; i++) wedge_grad(g + 3 * i, i, 1.0 / 3.0, 1.0 / 3.0, 0);
      *w = 1;
      return;
    }
    // myIntegrationCoords (:151-170): the wedge's triangle points on the
    // layers r = -q, +q (weight 5/54) and 0 (weight 8/54), q = sqrt(3/5)
    const double a = 1.0 / 6.0, b = 2.0 / 3.0, q = std::sqrt(3 / 5.0);
    const int t = k % 3;
    const double s1 = t == 1 ? b : a, s2 = t == 2 ? b : a, r = k < 3 ? -q : (k < 6 ? q : 0);
    *w = k < 6 ? 5 / 54.0 : 8 / 54.0;
    for (int i = 0; i < 15; i++) quadwedge_grad(g + 3 * i, i, s1, s2, r);
    return;
  }
  if (type == B200FEM_ELEM_QUADPYRAMID) {
    if (k < 0) {
      // warping point (QuadpyramidElement.getWarpingPoint): the linear
      // pyramid's gradients at (0, 0, -1/2) on the corners, weight 1
      std::memset(g, 0, 39 * sizeof(double));
      for (int i = 0; i < 5; i++) pyramid_grad(g + 3 * i, i, 0, 0, -0.5);
      *w = 1;
      return;
    }
    // the pyramid's five points (:151-165)
    double s0 = 0, s1 = 0, s2 = 2.0 / 5.0;
    *w = 125 / 27.0;
    if (k < 4) {
      const double a = (8 / 5.0) * std::sqrt(2 / 15.0);
      s0 = kPyrBase[k][0] * a;
      s1 = kPyrBase[k][1] * a;
      s2 = -2.0 / 3.0;
      *w = 81 / 100.0;
    }
    for (int i = 0; i < 13; i++) quadpyramid_grad(g + 3 * i, i, s0, s1, s2);
    return;
  }
  if (type == B200FEM_ELEM_QUADHEX) {
    if (k < 0) {
      // warping point (QuadhexElement.getWarpingPoint, :37-75): the linear
      // hex's gradients at the centre on the corners, zero elsewhere, weight 1
      std::memset(g, 0, 60 * sizeof(double));
      for (int i = 0; i < 8; i++) hex_grad(g + 3 * i, i, 0, 0, 0);
      *w = 1;
      return;
    }
    // 14-point rule (myIntegrationCoords14, :159-182): the eight corners at
    // +-q in node order with weight wc, then -+r on s, t, r with weight wf
    const double q = 0.758686910639328, wc = 0.335180055401662;
    const double r = 0.795822425754222, wf = 0.886426592797784;
    double x[3] = {0, 0, 0};
    if (k < 8) {
      for (int j = 0; j < 3; j++) x[j] = kQhexNode[k][j] * q;
      *w = wc;
    } else {
      x[(k - 8) / 2] = (k % 2 == 0) ? -r : r;
      *w = wf;
    }
    for (int i = 0; i < 20; i++) quadhex_grad(g + 3 * i, i, x);
    return;
  }
  if (type == B200FEM_ELEM_QUADTET) {
    if (k < 0) {
      // warping point (QuadtetElement.getWarpingPoint, :45-85): the linear
      // tet's gradients on the corners, zero on the edge nodes, weight 1
      std::memset(g, 0, 30 * sizeof(double));
      std::memcpy(g, kTetGNs, sizeof(kTetGNs));
      *w = 1;
      return;
    }
    // myIntegrationCoords (QuadtetElement.java:22-23, 255-262): the
    // reference's rounded alpha, beta; weight 0.25/6
    const double alpha = 0.58541020, beta = 0.13819660;
    const double c[3] = {k == 1 ? alpha : beta, k == 2 ? alpha : beta, k == 3 ? alpha : beta};
    const double sv[4] = {1 - c[0] - c[1] - c[2], c[0], c[1], c[2]};
    for (int i = 0; i < 10; i++) quadtet_grad(g + 3 * i, i, sv);
    *w = 0.25 / 6.0;
    return;
  }
  if (type == B200FEM_ELEM_WEDGE) {
    // integration points (WedgeElement.java:36-49): (1/6, 1/6), (2/3, 1/6),
    // (1/6, 2/3) on the layers r = -/+ 1/sqrt(3), weight 1/6; warping point
    // (1/3, 1/3, 0), weight 1 (:128-133)
    double s1 = 1.0 / 3.0, s2 = 1.0 / 3.0, r = 0;
    *w = 1;
    if (k >= 0) {
      const double a = 1.0 / 6.0, b = 2.0 / 3.0, q = 1 / std::sqrt(3.0);
      const int t = k % 3;
      s1 = t == 1 ? b : a;
      s2 = t == 2 ? b : a;
      r = k < 3 ? -q : q;
      *w = 1.0 / 6.0;
    }
    for (int i = 0; i < 6; i++) wedge_grad(g + 3 * i, i, s1, s2, r);
    return;
  }
  if (type == B200FEM_ELEM_PYRAMID) {
    // integration points (PyramidElement.java:69-83): (-/+a, -/+a, -2/3) in
    // base-node order, weight 81/100, and (0, 0, 2/5), weight 125/27, with
    // a = (8/5) sqrt(2/15); warping point (0, 0, -1/2), weight 128/27 (:38-44)
    double s0 = 0, s1 = 0, s2 = -0.5;
    *w = 128 / 27.0;
    if (k >= 0 && k < 4) {
      const double a = (8 / 5.0) * std::sqrt(2 / 15.0);
      s0 = kPyrBase[k][0] * a;
      s1 = kPyrBase[k][1] * a;
      s2 = -2.0 / 3.0;
      *w = 81 / 100.0;
    } else if (k == 4) {
      s2 = 2.0 / 5.0;
      *w = 125 / 27.0;
    }
    for (int i = 0; i < 5; i++) pyramid_grad(g + 3 * i, i, s0, s1, s2);
    return;
  }
  if (type == B200FEM_ELEM_TET) {
    std::memcpy(g, kTetGNs, sizeof(kTetGNs));
    *w = 1.0 / 6.0;
  } else if (k < 0) {
    // warping point: centre, weight 8 (HexElement.java:84-90)
    for (int i = 0; i < 8; i++) hex_grad(g + 3 * i, i, 0, 0, 0);
    *w = 8;
  } else {
    // INTEGRATION_COORDS_GAUSS_8 (HexElement.java:159-170): point k sits at
    // the node-k corner scaled by 1/sqrt(3), weight 1
    double q = 1 / std::sqrt(3.0);
    for (int i = 0; i < 8; i++)
      hex_grad(g + 3 * i, i, kHexNode[k][0] * q, kHexNode[k][1] * q, kHexNode[k][2] * q);
    *w = 1;
  }
}

namespace {

// J = sum_n x_n (outer) dN_n/ds  (IntegrationPoint3d.computeJacobian,
// IntegrationPoint3d.java:190-201)
void jacobian(double* J, const double* g, int nen, const double* xyz, const int* nodes) {
  for (int i = 0; i < 9; i++) J[i] = 0;
  for (int n = 0; n < nen; n++) {
    const double* p = xyz + 3 * (size_t)nodes[n];
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) J[3 * r + c] += p[r] * g[3 * n + c];
  }
}

// LinearMaterial.getC (LinearMaterial.java:148-159), Voigt (xx,yy,zz,xy,yz,xz)
void linear_tangent(double* C, double E, double nu) {
  double a = E / (1 + nu);
  double dia = (1 - nu) / (1 - 2 * nu) * a, mu = 0.5 * a, off = nu / (1 - 2 * nu) * a;
  std::fill(C, C + 36, 0.0);
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) C[6 * i + j] = i == j ? dia : off;
  C[21] = C[28] = C[35] = mu;
}

// K += B_i^T D B_j dv  (FemUtilities.addMaterialStiffness, FemUtilities.java:78-129)
void add_bdb(double* K, const double* gi, const double* D, const double* gj, double dv) {
  double x = gj[0] * dv, y = gj[1] * dv, z = gj[2] * dv;
  double t[6][3];
  for (int r = 0; r < 6; r++) {
    const double* d = D + 6 * r;
    t[r][0] = d[0] * x + d[3] * y + d[5] * z;
    t[r][1] = d[1] * y + d[3] * x + d[4] * z;
    t[r][2] = d[2] * z + d[4] * y + d[5] * x;
  }
  for (int c = 0; c < 3; c++) {
    K[c] += gi[0] * t[0][c] + gi[1] * t[3][c] + gi[2] * t[5][c];
    K[3 + c] += gi[1] * t[1][c] + gi[0] * t[3][c] + gi[2] * t[4][c];
    K[6 + c] += gi[2] * t[2][c] + gi[1] * t[4][c] + gi[0] * t[5][c];
  }
}

}  // namespace

int grid_dims(int type, int nx, int ny, int nz, int* nn, int* ne) {
  if (nx < 1 || ny < 1 || nz < 1) return B200FEM_ERR_INVALID_ARG;
  if (elem_nen(type) == 0) return B200FEM_ERR_INVALID_ARG;
  *nn = (nx + 1) * (ny + 1) * (nz + 1);
  const int per_cell[8] = {5, 1, 2, 3, 5, 1, 2, 3};  // tet, hex, wedge, pyramid and quadratic forms
  *ne = per_cell[type] * nx * ny * nz;
  if (elem_linear_base(type) >= 0) {
    // the linear grid plus its edge nodes
    const int lt = elem_linear_base(type);
    std::vector<double> xyz(3 * (size_t)*nn);
    std::vector<int> conn(elem_nen(lt) * (size_t)*ne);
    create_grid(lt, 1, 1, 1, nx, ny, nz, xyz.data(), conn.data());
    std::vector<double> qx;
    std::vector<int> qc;
    quadratic_mesh(lt, *nn, xyz.data(), *ne, conn.data(), qx, qc);
    *nn = (int)(qx.size() / 3);
  }
  return B200FEM_OK;
}

// FemFactory.createQuadraticModel (FemFactory.java:5641-5710): the linear
// nodes keep their indices; each element in order adds the midpoints
// (a + b) * 0.5 of its edges (FemElement3dBase.createEdgeNode, :1591-1596)
// unless a node already sits at exactly that position -- tets: edges 01, 12,
// 02, 03, 13, 23 (QuadtetElement.getQuadraticNodes :130-175); hexes: 01 12 23
// 30, 45 56 67 74, 04 15 26 37 (QuadhexElement.getQuadraticNodes :237-260)
void quadratic_mesh(int lin_type, int nn, const double* xyz, int ne, const int* conn, std::vector<double>& out_xyz,
                    std::vector<int>& out_conn) {
  // wedges: 01 12 20, 34 45 53, 03 14 25 (QuadwedgeElement.getQuadraticNodes);
  // pyramids: 01 12 23 30, 04 14 24 34 (QuadpyramidElement.getQuadraticNodes)
  static const int kQhexEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                       {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  static const int kQwedEdge[9][2] = {{0, 1}, {1, 2}, {2, 0}, {3, 4}, {4, 5}, {5, 3}, {0, 3}, {1, 4}, {2, 5}};
  static const int kQpyrEdge[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 4}, {2, 4}, {3, 4}};
  const int nl = elem_nen(lin_type);
  const int nedge = lin_type == B200FEM_ELEM_HEX ? 12 : lin_type == B200FEM_ELEM_WEDGE ? 9
                    : lin_type == B200FEM_ELEM_PYRAMID ? 8 : 6;
  const int nq = nl + nedge;
  const int(*edge)[2] = lin_type == B200FEM_ELEM_HEX ? kQhexEdge : lin_type == B200FEM_ELEM_WEDGE ? kQwedEdge
                        : lin_type == B200FEM_ELEM_PYRAMID ? kQpyrEdge : kQtetEdge;
  std::map<std::array<double, 3>, int> at;
  out_xyz.assign(xyz, xyz + 3 * (size_t)nn);
  for (int n = 0; n < nn; n++) at.emplace(std::array<double, 3>{xyz[3 * n], xyz[3 * n + 1], xyz[3 * n + 2]}, n);
  out_conn.assign(nq * (size_t)ne, 0);
  for (int e = 0; e < ne; e++) {
    const int* c = conn + nl * (size_t)e;
    int* q = &out_conn[nq * (size_t)e];
    for (int a = 0; a < nl; a++) q[a] = c[a];
    for (int j = 0; j < nedge; j++) {
      const double* pa = xyz + 3 * (size_t)c[edge[j][0]];
      const double* pb = xyz + 3 * (size_t)c[edge[j][1]];
      const std::array<double, 3> p{(pa[0] + pb[0]) * 0.5, (pa[1] + pb[1]) * 0.5, (pa[2] + pb[2]) * 0.5};
      auto it = at.find(p);
      if (it == at.end()) {
        it = at.emplace(p, (int)(out_xyz.size() / 3)).first;
        out_xyz.insert(out_xyz.end(), p.begin(), p.end());
      }
      q[nl + j] = it->second;
    }
  }
}

// FemFactory.createGridNodes (FemFactory.java:53-78); createTetGrid
// (:86-126) splits each cell with Tetrahedralizer.subdivideHex(allOnX =
// (i+j+k) odd) (Tetrahedralizer.java:135-141), whose parseCode /
// getTetIndicesForHex (:203-300) reduce to the two 5-tet tables below;
// createHexGrid (:203-255); createWedgeGrid (:266-310): two wedges per cell;
// createPyramidGrid (:137-195): three pyramids per cell sharing the apex
// corner that the cell's (i, j, k) parities select (apexNodeTable, :128-129),
// the bases being the three faces through the opposite corner in the order
// and orientation of PyramidElement.createCubeTesselation
// (PyramidElement.java:216-270).
void create_grid(int type, double wx, double wy, double wz, int nx, int ny, int nz, double* xyz,
                 int* conn) {
  if (elem_linear_base(type) >= 0) {
    // createQuadtetGrid / createQuadhexGrid / createQuadwedgeGrid /
    // createQuadpyramidGrid (FemFactory.java:316-376): the linear grid made
    // quadratic
    const int lt = elem_linear_base(type);
    int nl, ne;
    grid_dims(lt, nx, ny, nz, &nl, &ne);
    std::vector<double> lx(3 * (size_t)nl);
    std::vector<int> lc(elem_nen(lt) * (size_t)ne);
    create_grid(lt, wx, wy, wz, nx, ny, nz, lx.data(), lc.data());
    std::vector<double> qx;
    std::vector<int> qc;
    quadratic_mesh(lt, nl, lx.data(), ne, lc.data(), qx, qc);
    std::copy(qx.begin(), qx.end(), xyz);
    std::copy(qc.begin(), qc.end(), conn);
    return;
  }
  const double sx = 1.0 / nx, sy = 1.0 / ny, sz = 1.0 / nz;
  size_t n = 0;
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++, n++) {
        xyz[3 * n + 0] = wx * (-0.5 + i * sx);
        xyz[3 * n + 1] = wy * (-0.5 + j * sy);
        xyz[3 * n + 2] = wz * (-0.5 + k * sz);
      }
  // central tetrahedron {0,2,5,7} when allOnX, {1,6,4,3} otherwise
  static const int kOdd[5][4] = {{1, 0, 2, 5}, {3, 0, 7, 2}, {4, 0, 5, 7}, {6, 2, 7, 5}, {0, 2, 5, 7}};
  static const int kEven[5][4] = {{0, 1, 4, 3}, {2, 3, 6, 1}, {5, 4, 1, 6}, {7, 6, 3, 4}, {1, 6, 4, 3}};
  const int wk = (nx + 1) * (ny + 1), wj = nx + 1;
  size_t e = 0;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        const int c[8] = {(k + 1) * wk + j * wj + i,       (k + 1) * wk + j * wj + i + 1,
                          (k + 1) * wk + (j + 1) * wj + i + 1, (k + 1) * wk + (j + 1) * wj + i,
                          k * wk + j * wj + i,             k * wk + j * wj + i + 1,
                          k * wk + (j + 1) * wj + i + 1,   k * wk + (j + 1) * wj + i};
        if (type == B200FEM_ELEM_HEX) {
          std::memcpy(conn + 8 * e, c, sizeof(c));
          e++;
        } else if (type == B200FEM_ELEM_WEDGE) {
          static const int kWedge[2][6] = {{0, 1, 4, 3, 2, 7}, {1, 5, 4, 2, 6, 7}};
          for (int q = 0; q < 2; q++, e++)
            for (int a = 0; a < 6; a++) conn[6 * e + a] = c[kWedge[q][a]];
        } else if (type == B200FEM_ELEM_PYRAMID) {
          static const int kApex[8] = {2, 3, 1, 0, 6, 7, 5, 4};
          static const int kBase[8][3][4] = {
              {{6, 2, 3, 7}, {6, 5, 1, 2}, {6, 7, 4, 5}}, {{7, 6, 2, 3}, {7, 3, 0, 4}, {7, 4, 5, 6}},
              {{4, 5, 6, 7}, {4, 0, 1, 5}, {4, 7, 3, 0}}, {{5, 1, 2, 6}, {5, 4, 0, 1}, {5, 6, 7, 4}},
              {{2, 3, 7, 6}, {2, 1, 0, 3}, {2, 6, 5, 1}}, {{3, 2, 1, 0}, {3, 0, 4, 7}, {3, 7, 6, 2}},
              {{0, 3, 2, 1}, {0, 1, 5, 4}, {0, 4, 7, 3}}, {{1, 0, 3, 2}, {1, 2, 6, 5}, {1, 5, 4, 0}}};
          const int code = (i % 2 == 0 ? 1 : 0) | (j % 2 == 0 ? 2 : 0) | (k % 2 == 0 ? 4 : 0);
          const int apex = kApex[code];
          for (int q = 0; q < 3; q++, e++) {
            for (int a = 0; a < 4; a++) conn[5 * e + a] = c[kBase[apex][q][a]];
            conn[5 * e + 4] = c[apex];
          }
        } else {
          const int(*t)[4] = ((i + j + k) % 2 != 0) ? kOdd : kEven;
          for (int q = 0; q < 5; q++, e++)
            for (int a = 0; a < 4; a++) conn[4 * e + a] = c[t[q][a]];
        }
      }
}

void jitter_grid(int nx, int ny, int nz, double wx, double wy, double wz, double frac,
                 unsigned long long seed, double* xyz) {
  unsigned long long s = seed;
  auto next = [&s]() {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  };
  const double sp[3] = {wx / nx, wy / ny, wz / nz};
  size_t n = 0;
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++, n++) {
        if (i == 0 || i == nx || j == 0 || j == ny || k == 0 || k == nz) continue;
        for (int a = 0; a < 3; a++) xyz[3 * n + a] += (2 * next() - 1) * frac * sp[a];
      }
}

int setup_model_host(const ModelDesc& m, ModelHost& h, std::string& err) {
  const int N = m.n_nodes, E = m.n_elems;
  // element types in the caller's order, and the storage order: stable by
  // type, so that every type is one contiguous section
  std::vector<int> otype(E);
  for (int e = 0; e < E; e++) {
    otype[e] = m.elem_type == kElemMixed ? m.etypes[e] : m.elem_type;
    if (elem_nen(otype[e]) == 0) {
      err = "element " + std::to_string(e) + " has an unknown type";
      return B200FEM_ERR_INVALID_ARG;
    }
  }
  std::vector<long long> ooff(E + 1, 0);  // caller's node offsets
  for (int e = 0; e < E; e++) ooff[e + 1] = ooff[e] + elem_nen(otype[e]);
  if ((long long)m.conn.size() != ooff[E]) {
    err = "connectivity size does not match the element types";
    return B200FEM_ERR_INVALID_ARG;
  }
  for (long long q = 0; q < ooff[E]; q++)
    if (m.conn[q] < 0 || m.conn[q] >= N) {
      err = "connectivity index out of range";
      return B200FEM_ERR_INVALID_ARG;
    }
  // each element's material: its own, else the model's
  // (FemModel3d.getElementMaterial, FemModel3d.java:608-614)
  const bool own = !m.emat.empty();
  if (own && (int)m.emat.size() != E) {
    err = "element materials do not match the element count";
    return B200FEM_ERR_INVALID_ARG;
  }
  auto kind_of = [&](int o) { return own && m.emat[o] >= 0 ? m.emat_kind[m.emat[o]] : m.mat_kind; };
  auto params_of = [&](int o) {
    return own && m.emat[o] >= 0 ? &m.emat_params[(size_t)m.emat[o] * kMatParams] : m.mat_params;
  };
  auto corot_of = [&](int o) { return kind_of(o) == B200FEM_MAT_LINEAR && params_of(o)[2] != 0; };
  auto class_of = [&](int o) { return (otype[o] * 8 + kind_of(o)) * 2 + (corot_of(o) ? 1 : 0); };
  h.perm.resize(E);
  for (int e = 0; e < E; e++) h.perm[e] = e;
  std::stable_sort(h.perm.begin(), h.perm.end(), [&](int a, int b) { return class_of(a) < class_of(b); });
  h.iperm.assign(E, 0);
  h.stype.assign(E, 0);
  h.smat.assign(E, 0);
  h.skind.assign(E, 0);
  h.scorot.assign(E, 0);
  h.sec.assign(1, 0);
  h.coff.assign(E + 1, 0);
  h.ipoff.assign(E + 1, 0);
  h.sqoff.assign(E + 1, 0);
  for (int s = 0; s < E; s++) {
    const int o = h.perm[s], t = otype[o], nen = elem_nen(t);
    h.iperm[o] = s;
    h.stype[s] = t;
    h.smat[s] = own && m.emat[o] >= 0 ? m.emat[o] + 1 : 0;
    h.skind[s] = kind_of(o);
    h.scorot[s] = corot_of(o) ? 1 : 0;
    if (s > 0 && class_of(o) != class_of(h.perm[s - 1])) h.sec.push_back(s);
    h.coff[s + 1] = h.coff[s] + nen;
    h.ipoff[s + 1] = h.ipoff[s] + elem_nip(t);
    h.sqoff[s + 1] = h.sqoff[s] + (long long)nen * nen;
  }
  h.sec.push_back(E);
  h.sconn.resize(h.coff[E]);
  for (int s = 0; s < E; s++) {
    const int o = h.perm[s];
    std::copy(m.conn.begin() + ooff[o], m.conn.begin() + ooff[o + 1], h.sconn.begin() + h.coff[s]);
  }
  // solve indices in node order (MechSystemBase.updateDynamicComponentLists,
  // MechSystemBase.java:689-760: active components numbered in tree order)
  h.sidx.assign(N, -1);
  h.act_node.clear();
  for (int n = 0; n < N; n++)
    if (!m.fixed[n]) {
      h.sidx[n] = (int)h.act_node.size();
      h.act_node.push_back(n);
    }
  h.n_active = (int)h.act_node.size();
  // soft incompressibility.  NODAL needs the model's material to be
  // incompressible and every element to be a tet or to have its integration
  // points at its nodes (softNodalIncompressAllowed, FemModel3d.java:400-405);
  // otherwise NODAL and AUTO resolve to ELEMENT (QuadhexElement's four and
  // QuadwedgeElement's two pressure values), and AUTO -> NODAL if #elements >
  // #active nodes, else ELEMENT (getAllowedSoftIncompMethod, :462-481).  An
  // element of a compressible material runs with OFF (:3346-3348), so a model
  // none of whose elements is incompressible resolves to OFF.
  bool nodal_ok = true, any_incomp = false, all_incomp = true;
  for (int s = 0; s < E; s++) {
    nodal_ok &= h.stype[s] == B200FEM_ELEM_TET || elem_ip_at_nodes(h.stype[s]);
    any_incomp |= h.skind[s] == B200FEM_MAT_MOONEYRIVLIN;
    all_incomp &= h.skind[s] == B200FEM_MAT_MOONEYRIVLIN;
  }
  int method = m.incomp_request;
  if (!any_incomp) method = B200FEM_INCOMP_OFF;
  else if ((m.mat_kind != B200FEM_MAT_MOONEYRIVLIN || !nodal_ok) &&
           (method == B200FEM_INCOMP_NODAL || method == B200FEM_INCOMP_AUTO))
    method = B200FEM_INCOMP_ELEMENT;
  else if (method == B200FEM_INCOMP_AUTO)
    method = (E > h.n_active) ? B200FEM_INCOMP_NODAL : B200FEM_INCOMP_ELEMENT;
  if (method == B200FEM_INCOMP_NODAL && !all_incomp) {
    // the reference sums nodal volumes over the incompressible elements only
    // (updateNodalPressures, :2471-2503) and divides by a zero rest volume at a
    // node that only compressible elements touch
    err = "NODAL soft incompressibility with elements of compressible materials";
    return B200FEM_ERR_UNSUPPORTED;
  }
  h.incomp = method;

  // rest data: IntegrationData3d.myInvJ0/myDetJ0 (IntegrationData3d.java:108-111)
  h.invJ0.assign((size_t)h.ipoff[E] * 9, 0);
  h.detJ0.assign((size_t)h.ipoff[E], 0);
  h.winvJ0.assign((size_t)E * 9, 0);
  h.rest_vol.assign(E, 0);
  double g[kMaxNen * 3], wgt, J[9];
  for (int s = 0; s < E; s++) {
    const int t = h.stype[s], nen = elem_nen(t), nip = elem_nip(t);
    const int* nodes = &h.sconn[h.coff[s]];
    double vol = 0;
    for (int k = 0; k < nip; k++) {
      shape_grads(t, k, g, &wgt);
      jacobian(J, g, nen, m.rest.data(), nodes);
      double d = invert33(&h.invJ0[(size_t)(h.ipoff[s] + k) * 9], J);
      if (!(d > 0)) {
        err = "element " + std::to_string(h.perm[s]) + " has non-positive rest volume";
        return B200FEM_ERR_INVERTED;
      }
      h.detJ0[h.ipoff[s] + k] = d;
      vol += d * wgt;
    }
    if (t == B200FEM_ELEM_TET) {
      // TetElement.computeRestVolumes = detJ0/6 (TetElement.java:247-254)
      vol = h.detJ0[h.ipoff[s]] / 6;
      std::memcpy(&h.winvJ0[(size_t)s * 9], &h.invJ0[(size_t)h.ipoff[s] * 9], 9 * sizeof(double));
    } else {
      shape_grads(t, -1, g, &wgt);
      jacobian(J, g, nen, m.rest.data(), nodes);
      invert33(&h.winvJ0[(size_t)s * 9], J);
    }
    h.rest_vol[s] = vol;
  }
  // lumped masses (FemNode3d.computeMassFromDensity, FemNode3d.java:1030-1045),
  // summed in the caller's element order
  h.mass.assign(N, 0);
  for (int o = 0; o < E; o++) {
    const int s = h.iperm[o], nen = elem_nen(h.stype[s]);
    double share = h.rest_vol[s] * m.density / nen;
    for (int a = 0; a < nen; a++) h.mass[h.sconn[h.coff[s] + a]] += share;
  }
  // linear materials: rest stiffness K0 and f0 = K0 x_rest
  // (LinearMaterialCache.addInitialStiffness, LinearMaterialCache.java:115-160)
  // (each linear element with its own E and nu)
  h.K0.clear();
  h.f0.clear();
  bool any_linear = false;
  for (int s = 0; s < E; s++) any_linear |= h.skind[s] == B200FEM_MAT_LINEAR;
  if (any_linear) {
    double C[36];
    h.K0.assign((size_t)h.sqoff[E] * 9, 0);
    h.f0.assign((size_t)h.coff[E] * 3, 0);
    double gx[kMaxNen * 3];
    for (int s = 0; s < E; s++) {
      if (h.skind[s] != B200FEM_MAT_LINEAR) continue;
      const double* prm = params_of(h.perm[s]);
      linear_tangent(C, prm[0], prm[1]);
      const int t = h.stype[s], nen = elem_nen(t), nip = elem_nip(t);
      double* K0 = &h.K0[(size_t)h.sqoff[s] * 9];
      for (int k = 0; k < nip; k++) {
        shape_grads(t, k, g, &wgt);
        const double* iJ = &h.invJ0[(size_t)(h.ipoff[s] + k) * 9];
        double dv0 = h.detJ0[h.ipoff[s] + k] * wgt;
        for (int n = 0; n < nen; n++)
          for (int c = 0; c < 3; c++)
            gx[3 * n + c] = iJ[c] * g[3 * n] + iJ[3 + c] * g[3 * n + 1] + iJ[6 + c] * g[3 * n + 2];
        for (int i = 0; i < nen; i++)
          for (int j = 0; j < nen; j++) add_bdb(&K0[(i * nen + j) * 9], &gx[3 * i], C, &gx[3 * j], dv0);
      }
      const int* nodes = &h.sconn[h.coff[s]];
      for (int i = 0; i < nen; i++)
        for (int j = 0; j < nen; j++) {
          const double* Kij = &K0[(i * nen + j) * 9];
          const double* p = &m.rest[3 * (size_t)nodes[j]];
          for (int r = 0; r < 3; r++)
            h.f0[(size_t)(h.coff[s] + i) * 3 + r] +=
                Kij[3 * r] * p[0] + Kij[3 * r + 1] * p[1] + Kij[3 * r + 2] * p[2];
        }
    }
  }
  // node neighbours: nodes sharing an element, self included
  // (FemNodeNeighbor lists; FemModel3d.addSolveBlocks, FemModel3d.java:4099-4112)
  std::vector<int> inc_ptr(N + 1, 0);
  for (int n : h.sconn) inc_ptr[n + 1]++;
  for (int n = 0; n < N; n++) inc_ptr[n + 1] += inc_ptr[n];
  std::vector<int> inc(h.sconn.size()), fill(inc_ptr.begin(), inc_ptr.end() - 1);
  for (int s = 0; s < E; s++)
    for (long long q = h.coff[s]; q < h.coff[s + 1]; q++) inc[fill[h.sconn[q]]++] = s;
  h.nbr.assign(N, {});
  for (int n = 0; n < N; n++) {
    auto& v = h.nbr[n];
    for (int q = inc_ptr[n]; q < inc_ptr[n + 1]; q++) {
      const int s = inc[q];
      v.insert(v.end(), h.sconn.begin() + h.coff[s], h.sconn.begin() + h.coff[s + 1]);
    }
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  // block rows over active nodes; NODAL adds every pair of nodes that share
  // a neighbour (indirect neighbours, FemModel3d.java:5397-5416)
  h.rowptr.assign(h.n_active + 1, 0);
  h.col.clear();
  std::vector<int> cols;
  for (int r = 0; r < h.n_active; r++) {
    int n = h.act_node[r];
    cols.clear();
    if (h.incomp == B200FEM_INCOMP_NODAL) {
      for (int a : h.nbr[n])
        for (int b : h.nbr[a])
          if (h.sidx[b] >= 0) cols.push_back(h.sidx[b]);
    } else {
      for (int b : h.nbr[n])
        if (h.sidx[b] >= 0) cols.push_back(h.sidx[b]);
    }
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    h.col.insert(h.col.end(), cols.begin(), cols.end());
    h.rowptr[r + 1] = (int)h.col.size();
  }
  if (h.incomp == B200FEM_INCOMP_NODAL) {
    // nodal rest volumes (updateNodalRestVolumes, FemModel3d.java:2594-2628),
    // summed in the caller's element order
    h.node_rest_vol.assign(N, 0);
    double wts[kMaxNen];
    for (int o = 0; o < E; o++) {
      const int s = h.iperm[o], t = h.stype[s], nen = elem_nen(t);
      const int* nodes = &h.sconn[h.coff[s]];
      if (t == B200FEM_ELEM_TET) {
        for (int a = 0; a < 4; a++) h.node_rest_vol[nodes[a]] += h.rest_vol[s] / 4;
      } else {
        // integration point a maps to node a: its rest dv = w_a detJ0_a
        for (int a = 0; a < nen; a++) {
          shape_grads(t, a, g, &wts[a]);
          h.node_rest_vol[nodes[a]] += wts[a] * h.detJ0[h.ipoff[s] + a];
        }
      }
    }
  }
  return B200FEM_OK;
}

}  // namespace b200fem
