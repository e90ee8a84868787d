// fem_oracle.cpp -- CPU FP64 restatement of ArtiSynth's FEM force/stiffness
// assembly (FemModel3d.updateStressAndStiffness) and of the BackwardEuler
// step (MechSystemSolver.backwardEuler).
//
// TEST INFRASTRUCTURE ONLY.  This file is the correctness oracle: it may be
// loaded by tests/, by __graft_entry__.smoke() and by the CPU-baseline leg of
// bench.py, and only as the checker.  The product (artisynth_core_b200) never
// links, loads or calls it.
//
// Every routine cites the reference file:line it restates (paths relative to
// the artisynth_core source tree).  Arithmetic follows the reference
// formulas; summation order follows the reference loops where practical.
// The element loop runs over OpenMP threads but writes per-element buffers
// that are reduced in a fixed order, so the result does not depend on the
// thread count.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

enum { ELEM_TET = 0, ELEM_HEX = 1, ELEM_WEDGE = 2, ELEM_PYRAMID = 3, ELEM_QUADTET = 4, ELEM_QUADHEX = 5,
       ELEM_QUADWEDGE = 6, ELEM_QUADPYRAMID = 7 };
enum { MAT_LINEAR = 0, MAT_NEOHOOKEAN = 1, MAT_MOONEYRIVLIN = 2, MAT_STVK = 3 };
enum { INCOMP_OFF = 0, INCOMP_NODAL = 1, INCOMP_AUTO = 2, INCOMP_ELEMENT = 3 };

// ---------------------------------------------------------------------------
// small dense helpers (row-major 3x3)
// ---------------------------------------------------------------------------

static inline double det3(const double* m) {
  // Matrix3dBase.determinant / fastInvert ordering (Matrix3dBase.java:1629)
  return m[0] * m[4] * m[8] + m[3] * m[7] * m[2] + m[6] * m[1] * m[5] -
         m[6] * m[4] * m[2] - m[0] * m[7] * m[5] - m[3] * m[1] * m[8];
}

// Matrix3dBase.fastInvert (Matrix3dBase.java:1615-1648): returns det, fills
// inv only when det != 0.
static double fast_invert(double* inv, const double* d) {
  double det = det3(d);
  if (det != 0) {
    double deti = 1.0 / det;
    inv[0] = deti * (d[4] * d[8] - d[5] * d[7]);
    inv[3] = deti * (d[5] * d[6] - d[3] * d[8]);
    inv[6] = deti * (d[3] * d[7] - d[4] * d[6]);
    inv[1] = deti * (d[2] * d[7] - d[1] * d[8]);
    inv[4] = deti * (d[0] * d[8] - d[2] * d[6]);
    inv[7] = deti * (d[1] * d[6] - d[0] * d[7]);
    inv[2] = deti * (d[1] * d[5] - d[4] * d[2]);
    inv[5] = deti * (d[2] * d[3] - d[0] * d[5]);
    inv[8] = deti * (d[0] * d[4] - d[1] * d[3]);
  }
  return det;
}

static inline void mul3(double* c, const double* a, const double* b) {
  double t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      t[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
  std::memcpy(c, t, sizeof(t));
}

// ---------------------------------------------------------------------------
// polar decomposition: R of F = R P with det(R) = +1
// SVDecomposition3d.polarDecomposition (SVDecomposition3d.java:1418-1541):
// R = U V^T, and when det(U) det(V) < 0 the column of U belonging to the
// smallest singular value is negated.  Restated with a one-sided Jacobi
// (Hestenes) SVD; the third column of U is formed as det(V) * (u1 x u2),
// which is the same rotation for non-degenerate F and stays defined when the
// smallest singular value vanishes.
// ---------------------------------------------------------------------------
static void polar_rotation(double* R, const double* F) {
  double A[9], V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  std::memcpy(A, F, sizeof(A));
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0;
    for (int p = 0; p < 2; p++) {
      for (int q = p + 1; q < 3; q++) {
        double al = 0, be = 0, ga = 0;
        for (int r = 0; r < 3; r++) {
          al += A[3 * r + p] * A[3 * r + p];
          be += A[3 * r + q] * A[3 * r + q];
          ga += A[3 * r + p] * A[3 * r + q];
        }
        if (ga == 0 || std::fabs(ga) <= 1e-300) continue;
        double rel = std::fabs(ga) / std::sqrt(al * be);
        off = std::max(off, rel);
        if (rel < 1e-17) continue;
        double zeta = (be - al) / (2 * ga);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
        double c = 1.0 / std::sqrt(1 + t * t), s = c * t;
        for (int r = 0; r < 3; r++) {
          double ap = A[3 * r + p], aq = A[3 * r + q];
          A[3 * r + p] = c * ap - s * aq;
          A[3 * r + q] = s * ap + c * aq;
          double vp = V[3 * r + p], vq = V[3 * r + q];
          V[3 * r + p] = c * vp - s * vq;
          V[3 * r + q] = s * vp + c * vq;
        }
      }
    }
    if (off < 1e-16) break;
  }
  double sig[3];
  int ord[3] = {0, 1, 2};
  for (int k = 0; k < 3; k++)
    sig[k] = std::sqrt(A[k] * A[k] + A[3 + k] * A[3 + k] + A[6 + k] * A[6 + k]);
  std::sort(ord, ord + 3, [&](int a, int b) { return sig[a] > sig[b]; });
  double U[9], Vs[9];
  for (int kk = 0; kk < 3; kk++) {
    int k = ord[kk];
    for (int r = 0; r < 3; r++) {
      Vs[3 * r + kk] = V[3 * r + k];
      U[3 * r + kk] = sig[k] > 0 ? A[3 * r + k] / sig[k] : 0.0;
    }
  }
  if (sig[ord[0]] == 0) {  // F == 0: reference falls back to identity
    for (int i = 0; i < 9; i++) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return;
  }
  // re-orthonormalise u2 against u1 (protects rank-deficient F)
  double d = U[0] * U[1] + U[3] * U[4] + U[6] * U[7];
  for (int r = 0; r < 3; r++) U[3 * r + 1] -= d * U[3 * r];
  double n2 = std::sqrt(U[1] * U[1] + U[4] * U[4] + U[7] * U[7]);
  if (n2 < 1e-300) {
    // pick any unit vector orthogonal to u1
    double ax = std::fabs(U[0]), ay = std::fabs(U[3]), az = std::fabs(U[6]);
    double e[3] = {0, 0, 0};
    e[(ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2)] = 1;
    double dd = e[0] * U[0] + e[1] * U[3] + e[2] * U[6];
    for (int r = 0; r < 3; r++) U[3 * r + 1] = e[r] - dd * U[3 * r];
    n2 = std::sqrt(U[1] * U[1] + U[4] * U[4] + U[7] * U[7]);
  }
  for (int r = 0; r < 3; r++) U[3 * r + 1] /= n2;
  double detV = det3(Vs) >= 0 ? 1.0 : -1.0;
  U[2] = detV * (U[3] * U[7] - U[6] * U[4]);
  U[5] = detV * (U[6] * U[1] - U[0] * U[7]);
  U[8] = detV * (U[0] * U[4] - U[3] * U[1]);
  // R = U Vs^T
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      R[3 * i + j] = U[3 * i] * Vs[3 * j] + U[3 * i + 1] * Vs[3 * j + 1] + U[3 * i + 2] * Vs[3 * j + 2];
}

// ---------------------------------------------------------------------------
// element shape data
// ---------------------------------------------------------------------------

// TetElement.getdNds (TetElement.java:204-215), one integration point at
// (1/4,1/4,1/4) with weight 1/6 (TetElement.java:31-33).
static const double TET_GNS[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
static const double TET_W = 1.0 / 6.0;

// HexElement node coordinates (HexElement.java:119-129)
static const double HEX_NODE[8][3] = {{-1, -1, 1}, {1, -1, 1}, {1, 1, 1}, {-1, 1, 1},
                                      {-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1}};

// HexElement.getdNds (HexElement.java:266-281)
static void hex_dNds(double* out, int i, double s0, double s1, double s2) {
  double g0 = HEX_NODE[i][0] < 0 ? -1 : 1, g1 = HEX_NODE[i][1] < 0 ? -1 : 1,
         g2 = HEX_NODE[i][2] < 0 ? -1 : 1;
  out[0] = 0.125 * (g0) * (1 + g1 * s1) * (1 + g2 * s2);
  out[1] = 0.125 * (1 + g0 * s0) * (g1) * (1 + g2 * s2);
  out[2] = 0.125 * (1 + g0 * s0) * (1 + g1 * s1) * (g2);
}

// WedgeElement.getdNds (WedgeElement.java:193-206), node by node, at
// (s1, s2, r)
static void wedge_dNds(double* out, int i, double s1, double s2, double r) {
  const double lo = 1 - r, hi = 1 + r, t = 1 - s1 - s2;
  const double v[6][3] = {{-0.5 * lo, -0.5 * lo, -0.5 * t}, {0.5 * lo, 0, -0.5 * s1}, {0, 0.5 * lo, -0.5 * s2},
                          {-0.5 * hi, -0.5 * hi, 0.5 * t},  {0.5 * hi, 0, 0.5 * s1},  {0, 0.5 * hi, 0.5 * s2}};
  for (int c = 0; c < 3; c++) out[c] = v[i][c];
}

// PyramidElement.getdNds (PyramidElement.java:153-175), node by node
static void pyramid_dNds(double* out, int i, double s0, double s1, double s2) {
  const double v[5][3] = {
      {-0.125 * (1 - s1) * (1 - s2), -0.125 * (1 - s0) * (1 - s2), -0.125 * (1 - s0) * (1 - s1)},
      {+0.125 * (1 - s1) * (1 - s2), -0.125 * (1 + s0) * (1 - s2), -0.125 * (1 + s0) * (1 - s1)},
      {+0.125 * (1 + s1) * (1 - s2), +0.125 * (1 + s0) * (1 - s2), -0.125 * (1 + s0) * (1 + s1)},
      {-0.125 * (1 + s1) * (1 - s2), +0.125 * (1 - s0) * (1 - s2), -0.125 * (1 - s0) * (1 + s1)},
      {0, 0, 0.5}};
  for (int c = 0; c < 3; c++) out[c] = v[i][c];
}

// QuadtetElement.getdNds (QuadtetElement.java:301-323), case by case
static void quadtet_dNds(double* out, int i, double s1, double s2, double s3) {
  const double s0 = 1 - s1 - s2 - s3;
  const double v[10][3] = {{-4 * s0 + 1, -4 * s0 + 1, -4 * s0 + 1},
                           {4 * s1 - 1, 0, 0},
                           {0, 4 * s2 - 1, 0},
                           {0, 0, 4 * s3 - 1},
                           {4 * (s0 - s1), -4 * s1, -4 * s1},
                           {4 * s2, 4 * s1, 0},
                           {-4 * s2, 4 * (s0 - s2), -4 * s2},
                           {-4 * s3, -4 * s3, 4 * (s0 - s3)},
                           {4 * s3, 0, 4 * s1},
                           {0, 4 * s3, 4 * s2}};
  for (int c = 0; c < 3; c++) out[c] = v[i][c];
}

// QuadhexElement.getdNds (QuadhexElement.java:482-560), case by case at
// (s, t, r)
static void quadhex_dNds(double* out, int i, double s, double t, double r) {
  double u, a, b, c;
  switch (i) {
    case 0: u = (s + t - r + 1); a = (1 - t) * (1 + r) * (s + u); b = (1 - s) * (1 + r) * (t + u); c = (1 - s) * (1 - t) * (r - u); break;
    case 1: u = (s - t + r - 1); a = (1 - t) * (1 + r) * (s + u); b = (1 + s) * (1 + r) * (t - u); c = (1 + s) * (1 - t) * (r + u); break;
    case 2: u = (s + t + r - 1); a = (1 + t) * (1 + r) * (s + u); b = (1 + s) * (1 + r) * (t + u); c = (1 + s) * (1 + t) * (r + u); break;
    case 3: u = (s - t - r + 1); a = (1 + t) * (1 + r) * (s + u); b = (1 - s) * (1 + r) * (t - u); c = (1 - s) * (1 + t) * (r - u); break;
    case 4: u = (s + t + r + 1); a = (1 - t) * (1 - r) * (s + u); b = (1 - s) * (1 - r) * (t + u); c = (1 - s) * (1 - t) * (r + u); break;
    case 5: u = (s - t - r - 1); a = (1 - t) * (1 - r) * (s + u); b = (1 + s) * (1 - r) * (t - u); c = (1 + s) * (1 - t) * (r - u); break;
    case 6: u = (s + t - r - 1); a = (1 + t) * (1 - r) * (s + u); b = (1 + s) * (1 - r) * (t + u); c = (1 + s) * (1 + t) * (r - u); break;
    case 7: u = (s - t + r + 1); a = (1 + t) * (1 - r) * (s + u); b = (1 - s) * (1 - r) * (t - u); c = (1 - s) * (1 + t) * (r + u); break;
    case 8: out[0] = -.5 * s * (1 - t) * (1 + r); out[1] = -.25 * (1 - s * s) * (1 + r); out[2] = .25 * (1 - s * s) * (1 - t); return;
    case 9: out[0] = .25 * (1 - t * t) * (1 + r); out[1] = -.5 * t * (1 + s) * (1 + r); out[2] = .25 * (1 + s) * (1 - t * t); return;
    case 10: out[0] = -.5 * s * (1 + t) * (1 + r); out[1] = .25 * (1 - s * s) * (1 + r); out[2] = .25 * (1 - s * s) * (1 + t); return;
    case 11: out[0] = -.25 * (1 - t * t) * (1 + r); out[1] = -.5 * t * (1 - s) * (1 + r); out[2] = .25 * (1 - s) * (1 - t * t); return;
    case 12: out[0] = -.5 * s * (1 - t) * (1 - r); out[1] = -.25 * (1 - s * s) * (1 - r); out[2] = -.25 * (1 - s * s) * (1 - t); return;
    case 13: out[0] = .25 * (1 - t * t) * (1 - r); out[1] = -.5 * t * (1 + s) * (1 - r); out[2] = -.25 * (1 + s) * (1 - t * t); return;
    case 14: out[0] = -.5 * s * (1 + t) * (1 - r); out[1] = .25 * (1 - s * s) * (1 - r); out[2] = -.25 * (1 - s * s) * (1 + t); return;
    case 15: out[0] = -.25 * (1 - t * t) * (1 - r); out[1] = -.5 * t * (1 - s) * (1 - r); out[2] = -.25 * (1 - s) * (1 - t * t); return;
    case 16: out[0] = -.25 * (1 - t) * (1 - r * r); out[1] = -.25 * (1 - s) * (1 - r * r); out[2] = -.5 * r * (1 - s) * (1 - t); return;
    case 17: out[0] = .25 * (1 - t) * (1 - r * r); out[1] = -.25 * (1 + s) * (1 - r * r); out[2] = -.5 * r * (1 + s) * (1 - t); return;
    case 18: out[0] = .25 * (1 + t) * (1 - r * r); out[1] = .25 * (1 + s) * (1 - r * r); out[2] = -.5 * r * (1 + s) * (1 + t); return;
    default: out[0] = -.25 * (1 + t) * (1 - r * r); out[1] = .25 * (1 - s) * (1 - r * r); out[2] = -.5 * r * (1 - s) * (1 + t); return;
  }
  out[0] = a * 0.125;  // Vector3d.scale(0.125)
  out[1] = b * 0.125;
  out[2] = c * 0.125;
}

// QuadwedgeElement.getdNds (QuadwedgeElement.java:301-333), case by case
static void quadwedge_dNds(double* o, int i, double s1, double s2, double r) {
  const double s0 = 1 - s1 - s2;
  const double v[15][3] = {
      {(1 - r) * (4 * s1 + 4 * s2 + r - 2) / 2, (1 - r) * (4 * s1 + 4 * s2 + r - 2) / 2, s0 * (2 * s1 + 2 * s2 + 2 * r - 1) / 2},
      {(1 - r) * (4 * s1 - r - 2) / 2, 0, -s1 * (2 * s1 - 2 * r - 1) / 2},
      {0, (1 - r) * (4 * s2 - r - 2) / 2, -s2 * (2 * s2 - 2 * r - 1) / 2},
      {(1 + r) * (4 * s1 + 4 * s2 - r - 2) / 2, (1 + r) * (4 * s1 + 4 * s2 - r - 2) / 2, s0 * (1 - 2 * s1 - 2 * s2 + 2 * r) / 2},
      {(1 + r) * (4 * s1 + r - 2) / 2, 0, s1 * (2 * s1 + 2 * r - 1) / 2},
      {0, (1 + r) * (4 * s2 + r - 2) / 2, s2 * (2 * s2 + 2 * r - 1) / 2},
      {2 * (s0 - s1) * (1 - r), -2 * s1 * (1 - r), -2 * s1 * s0},
      {2 * s2 * (1 - r), 2 * s1 * (1 - r), -2 * s1 * s2},
      {-2 * s2 * (1 - r), 2 * (s0 - s2) * (1 - r), -2 * s2 * s0},
      {2 * (s0 - s1) * (1 + r), -2 * s1 * (1 + r), 2 * s1 * s0},
      {2 * s2 * (1 + r), 2 * s1 * (1 + r), 2 * s1 * s2},
      {-2 * s2 * (1 + r), 2 * (s0 - s2) * (1 + r), 2 * s2 * s0},
      {r * r - 1, r * r - 1, -2 * r * s0},
      {1 - r * r, 0, -2 * r * s1},
      {0, 1 - r * r, -2 * r * s2}};
  for (int c = 0; c < 3; c++) o[c] = v[i][c];
}

// QuadpyramidElement.getdNds (QuadpyramidElement.java:260-319), q = (1 - r)/2
static void quadpyramid_dNds(double* o, int i, double s, double t, double r) {
  const double q = (1 - r) / 2, u = q * (1 - q);
  const double v[13][3] = {
      {q * (1 - t) * (1 + q * (2 * s + t - 1)) / 4, q * (1 - s) * (1 + q * (2 * t + s - 1)) / 4, (1 - s) * (1 - t) * (1 + 2 * q * (s + t)) / 8},
      {-q * (1 - t) * (1 + q * (-2 * s + t - 1)) / 4, q * (1 + s) * (1 + q * (2 * t - s - 1)) / 4, (1 + s) * (1 - t) * (1 + 2 * q * (t - s)) / 8},
      {-q * (1 + t) * (1 + q * (-2 * s - t - 1)) / 4, -q * (1 + s) * (1 + q * (-2 * t - s - 1)) / 4, (1 + s) * (1 + t) * (1 - 2 * q * (t + s)) / 8},
      {q * (1 + t) * (1 + q * (2 * s - t - 1)) / 4, -q * (1 - s) * (1 + q * (-2 * t + s - 1)) / 4, (1 - s) * (1 + t) * (1 + 2 * q * (s - t)) / 8},
      {0, 0, 0.5 + r},
      {-s * q * q * (1 - t), -q * q * (1 - s * s) / 2, -q * (1 - t) * (1 - s * s) / 2},
      {q * q * (1 - t * t) / 2, -t * q * q * (1 + s), -q * (1 + s) * (1 - t * t) / 2},
      {-s * q * q * (1 + t), q * q * (1 - s * s) / 2, -q * (1 + t) * (1 - s * s) / 2},
      {-q * q * (1 - t * t) / 2, -t * q * q * (1 - s), -q * (1 - s) * (1 - t * t) / 2},
      {u * (t - 1), u * (s - 1), (2 * q - 1) * (1 - s - t + s * t) / 2},
      {u * (1 - t), -u * (1 + s), (2 * q - 1) * (1 + s - t - s * t) / 2},
      {u * (1 + t), u * (1 + s), (2 * q - 1) * (1 + s + t + s * t) / 2},
      {-u * (1 + t), u * (1 - s), (2 * q - 1) * (1 - s + t - s * t) / 2}};
  for (int c = 0; c < 3; c++) o[c] = v[i][c];
}

struct ShapeTable {
  int nen, nip;
  std::vector<double> GNs;  // nip * nen * 3
  std::vector<double> w;    // nip
  std::vector<double> wGNs; // warping point: nen * 3
  double ww;
  // ELEMENT soft incompressibility: pressure values per element
  // (FemElement3d.numPressureVals), the pressure weights H of every point
  // (IntegrationPoint3d.getPressureWeights: nip * npv) and the pressure
  // weight matrix W = (sum_k H H^T)^-1 (FemElement3d.createPressureWeightMatrix,
  // FemElement3d.java:226-255)
  int npv = 1;
  std::vector<double> H;
  std::vector<double> W;
};

// in-place Gauss-Jordan inverse of an n x n matrix (partial pivoting)
static void invert_small(std::vector<double>& A, int n) {
  std::vector<double> I((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) I[(size_t)i * n + i] = 1;
  for (int c = 0; c < n; c++) {
    int piv = c;
    for (int r = c + 1; r < n; r++)
      if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)piv * n + c])) piv = r;
    for (int k = 0; k < n; k++) {
      std::swap(A[(size_t)c * n + k], A[(size_t)piv * n + k]);
      std::swap(I[(size_t)c * n + k], I[(size_t)piv * n + k]);
    }
    const double d = A[(size_t)c * n + c];
    for (int k = 0; k < n; k++) {
      A[(size_t)c * n + k] /= d;
      I[(size_t)c * n + k] /= d;
    }
    for (int r = 0; r < n; r++) {
      if (r == c) continue;
      const double f = A[(size_t)r * n + c];
      for (int k = 0; k < n; k++) {
        A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
        I[(size_t)r * n + k] -= f * I[(size_t)c * n + k];
      }
    }
  }
  A = I;
}

// pressure weights and weight matrix of a multi-pressure element from its
// integration-point coordinates: QuadhexElement.getH (1, s, t, r),
// QuadwedgeElement.getH ((1 - r)/2, (1 + r)/2)
static void set_pressure_weights(ShapeTable& s, int npv, const double (*ip)[3]) {
  s.npv = npv;
  s.H.assign((size_t)s.nip * npv, 0.0);
  for (int k = 0; k < s.nip; k++) {
    double* h = &s.H[(size_t)k * npv];
    if (npv == 4) {
      h[0] = 1;
      h[1] = ip[k][0];
      h[2] = ip[k][1];
      h[3] = ip[k][2];
    } else {
      h[0] = 0.5 * (1 - ip[k][2]);
      h[1] = 0.5 * (1 + ip[k][2]);
    }
  }
  s.W.assign((size_t)npv * npv, 0.0);
  for (int k = 0; k < s.nip; k++)
    for (int i = 0; i < npv; i++)
      for (int j = 0; j < npv; j++) s.W[(size_t)i * npv + j] += s.H[(size_t)k * npv + i] * s.H[(size_t)k * npv + j];
  invert_small(s.W, npv);
}

static ShapeTable make_shape(int type) {
  ShapeTable s;
  if (type == ELEM_TET) {
    s.nen = 4; s.nip = 1;
    s.GNs.assign(&TET_GNS[0][0], &TET_GNS[0][0] + 12);
    s.w = {TET_W};
    s.wGNs = s.GNs;  // TetElement.getWarpingPoint == integration point 0
    s.ww = TET_W;
  } else if (type == ELEM_QUADWEDGE) {
    s.nen = 15; s.nip = 9;
    // myIntegrationCoords (QuadwedgeElement.java:151-170)
    const double a = 1.0 / 6.0, b = 2.0 / 3.0, q = std::sqrt(3 / 5.0), w1 = 5 / 54.0, w2 = 8 / 54.0;
    const double ip[9][3] = {{a, a, -q}, {b, a, -q}, {a, b, -q}, {a, a, q}, {b, a, q},
                             {a, b, q},  {a, a, 0},  {b, a, 0},  {a, b, 0}};
    s.GNs.resize(9 * 15 * 3);
    s.w = {w1, w1, w1, w1, w1, w1, w2, w2, w2};
    for (int k = 0; k < 9; k++)
      for (int i = 0; i < 15; i++) quadwedge_dNds(&s.GNs[(k * 15 + i) * 3], i, ip[k][0], ip[k][1], ip[k][2]);
    // warping point: the linear wedge at (1/3, 1/3, 0) on the corners
    s.wGNs.assign(45, 0.0);
    for (int i = 0; i < 6; i++) wedge_dNds(&s.wGNs[i * 3], i, 1 / 3.0, 1 / 3.0, 0);
    s.ww = 1;
    set_pressure_weights(s, 2, ip);  // QuadwedgeElement.numPressureVals (:267-269)
  } else if (type == ELEM_QUADPYRAMID) {
    s.nen = 13; s.nip = 5;
    // the pyramid's five points (QuadpyramidElement.java:151-165)
    const double a = (8 / 5.0) * std::sqrt(2 / 15.0), b = -2.0 / 3.0, c = 2.0 / 5.0;
    const double ip[5][3] = {{-a, -a, b}, {a, -a, b}, {a, a, b}, {-a, a, b}, {0, 0, c}};
    s.GNs.resize(5 * 13 * 3);
    s.w = {81 / 100.0, 81 / 100.0, 81 / 100.0, 81 / 100.0, 125 / 27.0};
    for (int k = 0; k < 5; k++)
      for (int i = 0; i < 13; i++) quadpyramid_dNds(&s.GNs[(k * 13 + i) * 3], i, ip[k][0], ip[k][1], ip[k][2]);
    // warping point: the linear pyramid at (0, 0, -1/2) on the corners
    s.wGNs.assign(39, 0.0);
    for (int i = 0; i < 5; i++) pyramid_dNds(&s.wGNs[i * 3], i, 0, 0, -0.5);
    s.ww = 1;
  } else if (type == ELEM_QUADHEX) {
    s.nen = 20; s.nip = 14;
    // myIntegrationCoords14 (QuadhexElement.java:159-182)
    const double q = 0.758686910639328, wc = 0.335180055401662;
    const double r = 0.795822425754222, wf = 0.886426592797784;
    const double ip[14][3] = {{-q, -q, q}, {q, -q, q}, {q, q, q}, {-q, q, q}, {-q, -q, -q}, {q, -q, -q}, {q, q, -q},
                              {-q, q, -q}, {-r, 0, 0}, {r, 0, 0}, {0, -r, 0}, {0, r, 0},  {0, 0, -r},  {0, 0, r}};
    s.GNs.resize(14 * 20 * 3);
    s.w.assign(14, wf);
    for (int k = 0; k < 8; k++) s.w[k] = wc;
    for (int k = 0; k < 14; k++)
      for (int i = 0; i < 20; i++) quadhex_dNds(&s.GNs[(k * 20 + i) * 3], i, ip[k][0], ip[k][1], ip[k][2]);
    // getWarpingPoint (:37-75): the linear hex's gradients at the centre on
    // the corners, zero on the edge nodes, weight 1
    s.wGNs.assign(60, 0.0);
    for (int i = 0; i < 8; i++) hex_dNds(&s.wGNs[i * 3], i, 0, 0, 0);
    s.ww = 1;
    set_pressure_weights(s, 4, ip);  // QuadhexElement.numPressureVals (:443-445)
  } else if (type == ELEM_QUADTET) {
    s.nen = 10; s.nip = 4;
    // myIntegrationCoords with the reference's rounded constants
    // (QuadtetElement.java:22-23, 255-262), weight 0.25/6
    const double alpha = 0.58541020, beta = 0.13819660;
    const double ip[4][3] = {{beta, beta, beta}, {alpha, beta, beta}, {beta, alpha, beta}, {beta, beta, alpha}};
    s.GNs.resize(4 * 10 * 3);
    s.w.assign(4, 0.25 / 6.0);
    for (int k = 0; k < 4; k++)
      for (int i = 0; i < 10; i++) quadtet_dNds(&s.GNs[(k * 10 + i) * 3], i, ip[k][0], ip[k][1], ip[k][2]);
    // getWarpingPoint (QuadtetElement.java:45-85): linear-tet gradients on the
    // corner nodes, zero on the edge nodes, weight 1
    s.wGNs.assign(30, 0.0);
    for (int i = 0; i < 4; i++)
      for (int c = 0; c < 3; c++) s.wGNs[i * 3 + c] = TET_GNS[i][c];
    s.ww = 1;
  } else if (type == ELEM_WEDGE) {
    s.nen = 6; s.nip = 6;
    // myIntegrationCoords (WedgeElement.java:34-49)
    const double a = 1.0 / 6.0, b = 2.0 / 3.0, q = 1 / std::sqrt(3.0);
    const double ip[6][3] = {{a, a, -q}, {b, a, -q}, {a, b, -q}, {a, a, q}, {b, a, q}, {a, b, q}};
    s.GNs.resize(6 * 6 * 3);
    s.w.assign(6, 1.0 / 6.0);
    for (int k = 0; k < 6; k++)
      for (int i = 0; i < 6; i++) wedge_dNds(&s.GNs[(k * 6 + i) * 3], i, ip[k][0], ip[k][1], ip[k][2]);
    // getWarpingPoint (WedgeElement.java:128-133): (1/3, 1/3, 0), weight 1
    s.wGNs.resize(18);
    for (int i = 0; i < 6; i++) wedge_dNds(&s.wGNs[i * 3], i, 1 / 3.0, 1 / 3.0, 0);
    s.ww = 1;
  } else if (type == ELEM_PYRAMID) {
    s.nen = 5; s.nip = 5;
    // myIntegrationCoords (PyramidElement.java:69-83)
    const double a = (8 / 5.0) * std::sqrt(2 / 15.0), b = -2.0 / 3.0, c = 2.0 / 5.0;
    const double ip[5][3] = {{-a, -a, b}, {a, -a, b}, {a, a, b}, {-a, a, b}, {0, 0, c}};
    s.GNs.resize(5 * 5 * 3);
    s.w = {81 / 100.0, 81 / 100.0, 81 / 100.0, 81 / 100.0, 125 / 27.0};
    for (int k = 0; k < 5; k++)
      for (int i = 0; i < 5; i++) pyramid_dNds(&s.GNs[(k * 5 + i) * 3], i, ip[k][0], ip[k][1], ip[k][2]);
    // getWarpingPoint (PyramidElement.java:38-44): (0, 0, -1/2), weight 128/27
    s.wGNs.resize(15);
    for (int i = 0; i < 5; i++) pyramid_dNds(&s.wGNs[i * 3], i, 0, 0, -0.5);
    s.ww = 128 / 27.0;
  } else {
    s.nen = 8; s.nip = 8;
    // INTEGRATION_COORDS_GAUSS_8 (HexElement.java:159-170)
    double q = 1 / std::sqrt(3.0);
    s.GNs.resize(8 * 8 * 3);
    s.w.assign(8, 1.0);
    for (int k = 0; k < 8; k++) {
      double c0 = HEX_NODE[k][0] * q, c1 = HEX_NODE[k][1] * q, c2 = HEX_NODE[k][2] * q;
      for (int i = 0; i < 8; i++) hex_dNds(&s.GNs[(k * 8 + i) * 3], i, c0, c1, c2);
    }
    // warping point at the centre with weight 8 (HexElement.java:84-90)
    s.wGNs.resize(24);
    for (int i = 0; i < 8; i++) hex_dNds(&s.wGNs[i * 3], i, 0, 0, 0);
    s.ww = 8;
  }
  return s;
}

// IntegrationPoint3d.computeJacobian (IntegrationPoint3d.java:190-201):
// J += pos (outer) dNds
static void compute_jacobian(double* J, const double* GNs, int nen, const double* xyz,
                             const int* nodes) {
  for (int i = 0; i < 9; i++) J[i] = 0;
  for (int n = 0; n < nen; n++) {
    const double* p = xyz + 3 * nodes[n];
    const double* g = GNs + 3 * n;
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) J[3 * r + c] += p[r] * g[c];
  }
}

// ---------------------------------------------------------------------------
// materials
// ---------------------------------------------------------------------------

struct Material {
  int kind = MAT_LINEAR;
  double E = 0, nu = 0;
  int corotated = 1;
  double c10 = 0, c01 = 0, c11 = 0, c20 = 0, c02 = 0, kappa = 0, jlimit = 0;
  int bulk_potential = 0;  // 0 QUADRATIC, 1 LOGARITHMIC
  bool incompressible() const { return kind == MAT_MOONEYRIVLIN; }
  bool linear() const { return kind == MAT_LINEAR; }
};

// D is a 6x6 row-major Voigt matrix, order (xx, yy, zz, xy, yz, xz);
// sigma is (s00, s11, s22, s01, s12, s02).

// LinearMaterial.getC (LinearMaterial.java:148-159)
static void linear_C(double* D, double E, double nu) {
  double a = E / (1 + nu);
  double dia = (1 - nu) / (1 - 2 * nu) * a;
  double mu = 0.5 * a;
  double off = nu / (1 - 2 * nu) * a;
  for (int i = 0; i < 36; i++) D[i] = 0;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[6 * i + j] = (i == j) ? dia : off;
  D[21] = mu; D[28] = mu; D[35] = mu;
}

// TensorUtils.addScaledIdentityProduct (TensorUtils.java:474-486)
static void add_scaled_identity_product(double* D, double s) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[6 * i + j] += s;
}
// TensorUtils.addScaledIdentity (TensorUtils.java:496-507)
static void add_scaled_identity(double* D, double s) {
  D[0] += s; D[7] += s; D[14] += s;
  D[21] += 0.5 * s; D[28] += 0.5 * s; D[35] += 0.5 * s;
}
// Matrix6d.setLowerToUpper (Matrix6d.java:532-538): lower := upper
static void set_lower_to_upper(double* D) {
  for (int i = 0; i < 6; i++)
    for (int j = 0; j < i; j++) D[6 * i + j] = D[6 * j + i];
}
// sym 3x3 stored as (00,11,22,01,12,02) -> accessor
static inline void sym_from6(double* m, const double* s) {
  m[0] = s[0]; m[4] = s[1]; m[8] = s[2];
  m[1] = m[3] = s[3]; m[5] = m[7] = s[4]; m[2] = m[6] = s[5];
}
// TensorUtils.addSymmetricTensorProduct(D, s, A, B) (TensorUtils.java:220-268):
// upper part only
static void add_sym_tensor_product(double* D, double s, const double* A6, const double* B6) {
  double a00 = s * A6[0], a11 = s * A6[1], a22 = s * A6[2], a01 = s * A6[3], a12 = s * A6[4], a02 = s * A6[5];
  double b00 = B6[0], b11 = B6[1], b22 = B6[2], b01 = B6[3], b12 = B6[4], b02 = B6[5];
  D[0] += 2 * a00 * b00; D[1] += a00 * b11 + b00 * a11; D[2] += a00 * b22 + b00 * a22;
  D[3] += a00 * b01 + b00 * a01; D[4] += a00 * b12 + b00 * a12; D[5] += a00 * b02 + b00 * a02;
  D[7] += 2 * a11 * b11; D[8] += a11 * b22 + b11 * a22; D[9] += a11 * b01 + b11 * a01;
  D[10] += a11 * b12 + b11 * a12; D[11] += a11 * b02 + b11 * a02;
  D[14] += 2 * a22 * b22; D[15] += a22 * b01 + b22 * a01; D[16] += a22 * b12 + b22 * a12;
  D[17] += a22 * b02 + b22 * a02;
  D[21] += 2 * a01 * b01; D[22] += a01 * b12 + b01 * a12; D[23] += a01 * b02 + b01 * a02;
  D[28] += 2 * a12 * b12; D[29] += a12 * b02 + b12 * a02;
  D[35] += 2 * a02 * b02;
}
// TensorUtils.addTensorProduct(D, s, A) (TensorUtils.java:340-380): upper part
static void add_tensor_product(double* D, double s, const double* A6) {
  double a[6] = {A6[0], A6[1], A6[2], A6[3], A6[4], A6[5]};
  for (int i = 0; i < 6; i++)
    for (int j = i; j < 6; j++) D[6 * i + j] += (s * a[i]) * a[j];
}
// TensorUtils.addTensorProduct4 (TensorUtils.java:608-645): upper part
static void add_tensor_product4(double* D, double s, const double* A6) {
  double a00 = A6[0], a11 = A6[1], a22 = A6[2], a01 = A6[3], a12 = A6[4], a02 = A6[5];
  double s00 = s * a00, s11 = s * a11, s22 = s * a22, s01 = s * a01, s02 = s * a02, s12 = s * a12;
  D[0] += s00 * a00; D[1] += s01 * a01; D[2] += s02 * a02; D[3] += s00 * a01;
  D[4] += s01 * a02; D[5] += s00 * a02;
  D[7] += s11 * a11; D[8] += s12 * a12; D[9] += s01 * a11; D[10] += s11 * a12; D[11] += s01 * a12;
  D[14] += s22 * a22; D[15] += s02 * a12; D[16] += s12 * a22; D[17] += s02 * a22;
  D[21] += (s00 * a11 + s01 * a01) * 0.5; D[22] += (s01 * a12 + s02 * a11) * 0.5;
  D[23] += (s00 * a12 + s02 * a01) * 0.5;
  D[28] += (s11 * a22 + s12 * a12) * 0.5; D[29] += (s01 * a22 + s02 * a12) * 0.5;
  D[35] += (s00 * a22 + s02 * a02) * 0.5;
}

// B = F F^T as (00,11,22,01,12,02)  (FemMaterial.computeLeftCauchyGreen,
// FemMaterial.java:199-202)
static void left_cauchy_green(double* B6, const double* F) {
  double B[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      B[3 * i + j] = F[3 * i] * F[3 * j] + F[3 * i + 1] * F[3 * j + 1] + F[3 * i + 2] * F[3 * j + 2];
  B6[0] = B[0]; B6[1] = B[4]; B6[2] = B[8]; B6[3] = B[1]; B6[4] = B[5]; B6[5] = B[2];
}

// NeoHookeanMaterial.computeStressAndTangent (NeoHookeanMaterial.java:113-139)
static void neohookean(double* sig, double* D, const Material& m, const double* F, double J) {
  double E = m.E, nu = m.nu;
  double G = E / (2 * (1 + nu));
  double lam = (E * nu) / ((1 - 2 * nu) * (1 + nu));
  double mu = G;
  double B6[6];
  left_cauchy_green(B6, F);
  for (int i = 0; i < 6; i++) sig[i] = (mu / J) * B6[i];
  double diagTerm = (lam * std::log(J) - mu) / J;
  sig[0] += diagTerm; sig[1] += diagTerm; sig[2] += diagTerm;
  if (D) {
    for (int i = 0; i < 36; i++) D[i] = 0;
    add_scaled_identity_product(D, lam / J);
    add_scaled_identity(D, 2 * (mu - lam * std::log(J)) / J);
    set_lower_to_upper(D);
  }
}

// MooneyRivlinMaterial.computePhiVals (MooneyRivlinMaterial.java:314-331)
static void mr_phi(double* vals, const Material& m, double J) {
  if (m.jlimit > 0 && J < m.jlimit) {
    double phi0 = 1 / std::pow(m.jlimit, 2.0 / 3.0);
    double dphi0 = -(2.0 / 3.0) * phi0 / m.jlimit;
    double ddphi0 = -(5.0 / 3.0) * dphi0 / m.jlimit;
    double delJ = J - m.jlimit;
    vals[0] = (0.5 * ddphi0 * delJ + dphi0) * delJ + phi0;
    vals[1] = ddphi0 * delJ + dphi0;
    vals[2] = ddphi0;
  } else {
    double phi = 1 / std::pow(J, 2.0 / 3.0);
    double dphi = -(2.0 / 3.0) * phi / J;
    vals[0] = phi;
    vals[1] = dphi;
    vals[2] = -(5.0 / 3.0) * dphi / J;
  }
}

// MooneyRivlinMaterial.computeDevStressAndTangent (MooneyRivlinMaterial.java:344-431)
// followed by IncompressibleMaterialBase.computeStressAndTangent
// (IncompressibleMaterialBase.java:249-260): add pressure stress/tangent.
static void mooneyrivlin(double* sig, double* D, const Material& m, const double* F, double J,
                         double p) {
  double pv[3];
  mr_phi(pv, m, J);
  double phi = pv[0], dphi = pv[1];
  double B6[6], B[9], B2[9], B26[6];
  left_cauchy_green(B6, F);
  for (int i = 0; i < 6; i++) B6[i] *= phi;
  sym_from6(B, B6);
  mul3(B2, B, B);  // myB2.mulTransposeLeft(myB) = B^T B = B B
  B26[0] = B2[0]; B26[1] = B2[4]; B26[2] = B2[8]; B26[3] = B2[1]; B26[4] = B2[5]; B26[5] = B2[2];
  double c10 = m.c10, c01 = m.c01, c11 = m.c11, c20 = m.c20, c02 = m.c02;
  double I1 = B6[0] + B6[1] + B6[2];
  double I2 = 0.5 * (I1 * I1 - (B26[0] + B26[1] + B26[2]));
  double W1 = c10 + c11 * (I2 - 3) + c20 * 2 * (I1 - 3);
  double W2 = c01 + c11 * (I1 - 3) + c02 * 2 * (I2 - 3);
  for (int i = 0; i < 6; i++) sig[i] = (W1 + W2 * I1) * B6[i];
  for (int i = 0; i < 6; i++) sig[i] += -W2 * B26[i];
  double dev = (dphi / phi) * (sig[0] + sig[1] + sig[2]);
  for (int i = 0; i < 6; i++) sig[i] *= 2.0 / J;
  sig[0] += dev; sig[1] += dev; sig[2] += dev;
  if (D) {
    double Ji = 1.0 / J;
    double ddphi = pv[2];
    double W11 = 2 * c20, W12 = c11, W22 = 2 * c02;
    double w1 = -W2;
    double w2 = W11 + 2 * W12 * I1 + W2 + W22 * I2 * I2;
    double w3 = W12 + W22 * I1;
    double w4 = W22;
    double wc1 = (w2 - W12 + W22 * I1) * I1;
    double wc2 = -(W12 + W22 * I1 - W22 * I1 * I1 + 2 * W22 * I2 + W2);
    double wcc = wc1 * I1 + wc2 * (I1 * I1 - 2 * I2);
    double w0 = W1 * I1 + 2 * W2 * I2;
    for (int i = 0; i < 36; i++) D[i] = 0;
    double zeta = ((dphi + J * ddphi) * w0 + J * dphi * dphi / phi * (wcc - 2 * w0)) / phi;
    double r = dphi / phi;
    add_scaled_identity_product(D, zeta);
    add_scaled_identity(D, -2 * r * w0);
    static const double I6[6] = {1, 1, 1, 0, 0, 0};
    add_sym_tensor_product(D, J * r, sig, I6);
    add_tensor_product4(D, w1 * 4.0 * Ji, B6);
    add_tensor_product(D, w2 * 4.0 * Ji, B6);
    add_sym_tensor_product(D, w3 * 4.0 * Ji, B6, B26);
    add_tensor_product(D, w4 * 4.0 * Ji, B26);
    double T6[6];
    for (int i = 0; i < 6; i++) T6[i] = wc1 * B6[i] + wc2 * B26[i];
    add_sym_tensor_product(D, 2 * r, T6, I6);
    set_lower_to_upper(D);
    // IncompressibleMaterialBase.addPressureTangent (:218-224)
    add_scaled_identity_product(D, p);
    add_scaled_identity(D, -2 * p);
  }
  // IncompressibleMaterialBase.addPressureStress (:209-213)
  sig[0] += p; sig[1] += p; sig[2] += p;
}

// TensorUtils.addSymmetricTensorProduct4 (TensorUtils.java:674-716): upper part
static void add_sym_tensor_product4(double* D, double s, const double* A6, const double* B6) {
  const double a00 = s * A6[0], a11 = s * A6[1], a22 = s * A6[2], a01 = s * A6[3], a12 = s * A6[4],
               a02 = s * A6[5];
  const double b00 = B6[0], b11 = B6[1], b22 = B6[2], b01 = B6[3], b12 = B6[4], b02 = B6[5];
  D[0] += 2 * a00 * b00;
  D[1] += 2 * a01 * b01;
  D[2] += 2 * a02 * b02;
  D[3] += a01 * b00 + a00 * b01;
  D[4] += a02 * b01 + a01 * b02;
  D[5] += a02 * b00 + a00 * b02;
  D[7] += 2 * a11 * b11;
  D[8] += 2 * a12 * b12;
  D[9] += a11 * b01 + a01 * b11;
  D[10] += a12 * b11 + a11 * b12;
  D[11] += a12 * b01 + a01 * b12;
  D[14] += 2 * a22 * b22;
  D[15] += a12 * b02 + a02 * b12;
  D[16] += a22 * b12 + a12 * b22;
  D[17] += a22 * b02 + a02 * b22;
  D[21] += 0.5 * (a11 * b00 + 2 * a01 * b01 + a00 * b11);
  D[22] += 0.5 * (a12 * b01 + a11 * b02 + a02 * b11 + a01 * b12);
  D[23] += 0.5 * (a12 * b00 + a02 * b01 + a01 * b02 + a00 * b12);
  D[28] += 0.5 * (a22 * b11 + 2 * a12 * b12 + a11 * b22);
  D[29] += 0.5 * (a22 * b01 + a12 * b02 + a02 * b12 + a01 * b22);
  D[35] += 0.5 * (a22 * b00 + 2 * a02 * b02 + a00 * b22);
}

// StVenantKirchoffMaterial.computeStressAndTangent
// (StVenantKirchoffMaterial.java:136-164): FEBio's form
// sigma = ((lam trE - mu)/J) B + (mu/J) B^2, trE = (tr B - 3)/2;
// D = (lam/J) B(x)B (TensorUtils.addTensorProduct(D, s, B, B), :401-456) +
// (mu/J) addSymmetricTensorProduct4(B, B), then setLowerToUpper.
static void stvk(double* sig, double* D, const Material& m, const double* F, double J) {
  const double G = m.E / (2 * (1 + m.nu));
  const double lam = (m.E * m.nu) / ((1 - 2 * m.nu) * (1 + m.nu));
  const double mu = G;
  double B6[6];
  left_cauchy_green(B6, F);
  const double tr = 0.5 * (B6[0] + B6[1] + B6[2] - 3);
  // myB2.mulTransposeLeft(myB): B^T B = B B for symmetric B
  double Bf[9];
  sym_from6(Bf, B6);
  double B2f[9];
  mul3(B2f, Bf, Bf);
  const double B26[6] = {B2f[0], B2f[4], B2f[8], B2f[1], B2f[5], B2f[2]};
  for (int i = 0; i < 6; i++) sig[i] = ((lam * tr - mu) / J) * B6[i];
  for (int i = 0; i < 6; i++) sig[i] += (mu / J) * B26[i];
  if (D) {
    for (int i = 0; i < 36; i++) D[i] = 0;
    add_tensor_product(D, lam / J, B6);
    add_sym_tensor_product4(D, mu / J, B6, B6);
    set_lower_to_upper(D);
  }
}

static void material_stress_tangent(double* sig, double* D, const Material& m, const double* F,
                                    double J, double p) {
  if (m.kind == MAT_NEOHOOKEAN) neohookean(sig, D, m, F, J);
  else if (m.kind == MAT_MOONEYRIVLIN) mooneyrivlin(sig, D, m, F, J, p);
  else if (m.kind == MAT_STVK) stvk(sig, D, m, F, J);
  else {
    // linear small-strain (non-corotated) stress, used only by point tests:
    // LinearMaterialBase.computeStressAndTangent with R = null, corotated off
    double eps[6] = {F[0] - 1, F[4] - 1, F[8] - 1, 0.5 * (F[1] + F[3]), 0.5 * (F[5] + F[7]),
                     0.5 * (F[2] + F[6])};
    double lam = m.E * m.nu / ((1 + m.nu) * (1 - 2 * m.nu));
    double mu = m.E / (2 * (1 + m.nu));
    double tr = lam * (eps[0] + eps[1] + eps[2]);
    sig[0] = 2 * mu * eps[0] + tr; sig[1] = 2 * mu * eps[1] + tr; sig[2] = 2 * mu * eps[2] + tr;
    sig[3] = 2 * mu * eps[3]; sig[4] = 2 * mu * eps[4]; sig[5] = 2 * mu * eps[5];
    if (D) linear_C(D, m.E, m.nu);
  }
}

// FemUtilities.addStressForce (FemUtilities.java:40-49)
static inline void add_stress_force(double* f, const double* g, const double* s, double dv) {
  double gx = g[0] * dv, gy = g[1] * dv, gz = g[2] * dv;
  f[0] += gx * s[0] + gy * s[3] + gz * s[5];
  f[1] += gy * s[1] + gx * s[3] + gz * s[4];
  f[2] += gz * s[2] + gy * s[4] + gx * s[5];
}

// FemUtilities.addMaterialStiffness(K, gi, D, gj, dv) (FemUtilities.java:78-129)
static void add_material_stiffness(double* K, const double* gi, const double* D, const double* gj,
                                   double dv) {
  double gjx = gj[0] * dv, gjy = gj[1] * dv, gjz = gj[2] * dv;
#define DM(r, c) D[6 * (r) + (c)]
  double dm[6][3];
  for (int r = 0; r < 6; r++) {
    dm[r][0] = DM(r, 0) * gjx + DM(r, 3) * gjy + DM(r, 5) * gjz;
    dm[r][1] = DM(r, 1) * gjy + DM(r, 3) * gjx + DM(r, 4) * gjz;
    dm[r][2] = DM(r, 2) * gjz + DM(r, 4) * gjy + DM(r, 5) * gjx;
  }
#undef DM
  double gix = gi[0], giy = gi[1], giz = gi[2];
  for (int c = 0; c < 3; c++) {
    K[c] += gix * dm[0][c] + giy * dm[3][c] + giz * dm[5][c];
    K[3 + c] += giy * dm[1][c] + gix * dm[3][c] + giz * dm[4][c];
    K[6 + c] += giz * dm[2][c] + giy * dm[4][c] + gix * dm[5][c];
  }
}

// FemUtilities.addGeometricStiffness (FemUtilities.java:131-144)
static void add_geometric_stiffness(double* K, const double* gi, const double* s, const double* gj,
                                    double dv) {
  double Kg = gi[0] * (s[0] * gj[0] + s[3] * gj[1] + s[5] * gj[2]) +
              gi[1] * (s[3] * gj[0] + s[1] * gj[1] + s[4] * gj[2]) +
              gi[2] * (s[5] * gj[0] + s[4] * gj[1] + s[2] * gj[2]);
  Kg = Kg * dv;
  K[0] += Kg; K[4] += Kg; K[8] += Kg;
}

// ---------------------------------------------------------------------------
// model
// ---------------------------------------------------------------------------

struct Model {
  int type = ELEM_TET, N = 0, E = 0, nen = 4;  // type and nen of the first element
  ShapeTable sh;                               // its shape table
  // per element (a mesh may mix element types): type, first connectivity
  // entry, first integration point, first linear-cache block; one shape
  // table per element type present
  std::vector<int> etype, eoff, ipoff, k0off;
  std::vector<ShapeTable> shapes;
  const ShapeTable& shp(int e) const { return shapes[etype[e]]; }
  int nen_of(int e) const { return shapes[etype[e]].nen; }
  const int* nodes_of(int e) const { return &conn[eoff[e]]; }
  std::vector<double> rest;
  std::vector<int> conn;
  std::vector<int> sidx;  // solve index (block row) per node, -1 when fixed
  int nact = 0;
  Material mat;
  // per-element materials, one per element when any element has its own
  // (FemModel3d.getElementMaterial, FemModel3d.java:608-614)
  std::vector<Material> emats;
  const Material& mat_of(int e) const { return emats.empty() ? mat : emats[e]; }
  double density = 1000;
  int incomp_request = INCOMP_AUTO;
  int incomp = INCOMP_OFF;  // resolved method
  // an element of a compressible material runs with OFF (FemModel3d.java:3346-3348)
  int incomp_of(int e) const { return mat_of(e).incompressible() ? incomp : INCOMP_OFF; }
  // rest data
  std::vector<double> invJ0, detJ0;  // per element per IP
  std::vector<double> winvJ0;        // warping-point invJ0 per element
  std::vector<double> restVol;       // per element
  std::vector<double> mass;          // per node
  std::vector<double> K0, f0;        // linear cache: E*nen*nen*9, E*nen*3
  // node neighbours (direct: share an element), sorted by node index
  std::vector<std::vector<int>> nbr;
  std::vector<std::vector<int>> ind;  // indirect (NODAL 2-ring minus direct)
  // BSR over active nodes
  std::vector<int> rowptr, col;
  // NODAL data
  std::vector<double> nodeRestVol, nodeVol, nodePressure;
  // of the last update: per node kp = effective modulus / rest volume (0 for
  // fixed nodes) and its divBlk row, one 3-vector per direct neighbour
  std::vector<double> nodeKp;
  std::vector<std::vector<double>> divBlk;
  // results of the last update
  std::vector<double> K;     // nnzb * 9
  std::vector<double> fint;  // 3N
  int numInverted = 0;
  double minDetJ = 0;
  std::string err;

  int block_index(int bi, int bj) const {
    auto b = col.begin() + rowptr[bi], e = col.begin() + rowptr[bi + 1];
    auto it = std::lower_bound(b, e, bj);
    if (it == e || *it != bj) return -1;
    return (int)(it - col.begin());
  }
};

static bool contains_sorted(const std::vector<int>& v, int x) {
  return std::binary_search(v.begin(), v.end(), x);
}

static void build_rest_data(Model& m) {
  const size_t nips = (size_t)m.ipoff[m.E];
  m.invJ0.assign(nips * 9, 0);
  m.detJ0.assign(nips, 0);
  m.winvJ0.assign((size_t)m.E * 9, 0);
  m.restVol.assign(m.E, 0);
  for (int e = 0; e < m.E; e++) {
    const ShapeTable& s = m.shp(e);
    const int nen = s.nen;
    const int* nodes = m.nodes_of(e);
    double J0[9];
    double vol = 0;
    for (int k = 0; k < s.nip; k++) {
      compute_jacobian(J0, &s.GNs[k * nen * 3], nen, m.rest.data(), nodes);
      // IntegrationData3d.setRestJacobian (IntegrationData3d.java:108-111)
      double d = fast_invert(&m.invJ0[((size_t)m.ipoff[e] + k) * 9], J0);
      m.detJ0[(size_t)m.ipoff[e] + k] = d;
      vol += d * s.w[k];
    }
    if (m.etype[e] == ELEM_TET) {
      // TetElement.computeRestVolumes (TetElement.java:247-254): signed
      // volume of the rest tetrahedron
      const double *p0 = &m.rest[3 * nodes[0]], *p1 = &m.rest[3 * nodes[1]],
                   *p2 = &m.rest[3 * nodes[2]], *p3 = &m.rest[3 * nodes[3]];
      double a[9] = {p1[0] - p0[0], p2[0] - p0[0], p3[0] - p0[0], p1[1] - p0[1], p2[1] - p0[1],
                     p3[1] - p0[1], p1[2] - p0[2], p2[2] - p0[2], p3[2] - p0[2]};
      vol = det3(a) / 6;
      std::memcpy(&m.winvJ0[(size_t)e * 9], &m.invJ0[(size_t)m.ipoff[e] * 9], 9 * sizeof(double));
    } else {
      // FemElement3d.computeVolumes(rest) (FemElement3d.java:95-130)
      compute_jacobian(J0, s.wGNs.data(), nen, m.rest.data(), nodes);
      fast_invert(&m.winvJ0[(size_t)e * 9], J0);
    }
    m.restVol[e] = vol;
  }
  // lumped masses: FemNode3d.computeMassFromDensity (FemNode3d.java:1030-1045)
  m.mass.assign(m.N, 0);
  for (int e = 0; e < m.E; e++) {
    double rm = m.restVol[e] * m.density;
    const int nen = m.nen_of(e);
    for (int a = 0; a < nen; a++) m.mass[m.nodes_of(e)[a]] += rm / nen;
  }
}

// LinearMaterialCache.addInitialStiffness (LinearMaterialCache.java:115-160)
static void build_linear_cache(Model& m) {
  m.K0.assign((size_t)m.k0off[m.E] * 9, 0);
  m.f0.assign((size_t)m.eoff[m.E] * 3, 0);
  double C[36];
  for (int e = 0; e < m.E; e++) {
    const Material& mat = m.mat_of(e);
    if (!mat.linear()) continue;
    linear_C(C, mat.E, mat.nu);
    const ShapeTable& s = m.shp(e);
    const int nen = s.nen;
    const int* nodes = m.nodes_of(e);
    double* K0 = &m.K0[(size_t)m.k0off[e] * 9];
    for (int k = 0; k < s.nip; k++) {
      const double* invJ0 = &m.invJ0[((size_t)m.ipoff[e] + k) * 9];
      double dv0 = m.detJ0[(size_t)m.ipoff[e] + k] * 1.0 * s.w[k];
      std::vector<double> GNx0(nen * 3);
      for (int n = 0; n < nen; n++) {
        const double* g = &s.GNs[(k * nen + n) * 3];
        for (int c = 0; c < 3; c++)
          GNx0[3 * n + c] = invJ0[c] * g[0] + invJ0[3 + c] * g[1] + invJ0[6 + c] * g[2];
      }
      for (int i = 0; i < nen; i++)
        for (int j = 0; j < nen; j++)
          add_material_stiffness(&K0[(i * nen + j) * 9], &GNx0[3 * i], C, &GNx0[3 * j], dv0);
    }
    for (int i = 0; i < nen; i++) {
      double tmp[3] = {0, 0, 0};
      for (int j = 0; j < nen; j++) {
        const double* Kij = &K0[(i * nen + j) * 9];
        const double* p = &m.rest[3 * nodes[j]];
        for (int r = 0; r < 3; r++) tmp[r] += Kij[3 * r] * p[0] + Kij[3 * r + 1] * p[1] + Kij[3 * r + 2] * p[2];
      }
      for (int r = 0; r < 3; r++) m.f0[((size_t)m.eoff[e] + i) * 3 + r] = tmp[r];
    }
  }
}

static void build_pattern(Model& m) {
  // FemNodeNeighbor lists: every pair of nodes sharing an element (self
  // included); FemModel3d.addSolveBlocks (FemModel3d.java:4099-4112) makes a
  // block for each pair with both solve indices != -1.
  m.nbr.assign(m.N, {});
  for (int e = 0; e < m.E; e++) {
    const int* nodes = m.nodes_of(e);
    const int nen = m.nen_of(e);
    for (int a = 0; a < nen; a++)
      for (int b = 0; b < nen; b++) m.nbr[nodes[a]].push_back(nodes[b]);
  }
  for (auto& v : m.nbr) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }
  m.ind.assign(m.N, {});
  if (m.incomp == INCOMP_NODAL) {
    // FemModel3d.setNodalIncompBlocksAllocated (FemModel3d.java:5397-5416)
    for (int n = 0; n < m.N; n++) {
      const auto& nb = m.nbr[n];
      for (int a : nb)
        for (int b : nb)
          if (!contains_sorted(m.nbr[a], b)) m.ind[a].push_back(b);
    }
    for (auto& v : m.ind) {
      std::sort(v.begin(), v.end());
      v.erase(std::unique(v.begin(), v.end()), v.end());
    }
  }
  m.rowptr.assign(m.nact + 1, 0);
  std::vector<int> act_nodes(m.nact);
  for (int n = 0; n < m.N; n++)
    if (m.sidx[n] >= 0) act_nodes[m.sidx[n]] = n;
  m.col.clear();
  for (int bi = 0; bi < m.nact; bi++) {
    int n = act_nodes[bi];
    std::vector<int> cols;
    for (int j : m.nbr[n])
      if (m.sidx[j] >= 0) cols.push_back(m.sidx[j]);
    for (int j : m.ind[n])
      if (m.sidx[j] >= 0) cols.push_back(m.sidx[j]);
    std::sort(cols.begin(), cols.end());
    cols.erase(std::unique(cols.begin(), cols.end()), cols.end());
    m.col.insert(m.col.end(), cols.begin(), cols.end());
    m.rowptr[bi + 1] = (int)m.col.size();
  }
}

// ---------------------------------------------------------------------------
// FemModel3d.updateStressAndStiffness (FemModel3d.java:2894-3051) with
// computeStressAndStiffness (:3333-3666) and the NODAL soft-incompressibility
// terms (:2471-2515, :2594-2669).
// ---------------------------------------------------------------------------

struct ElemOut {
  std::vector<double> f;     // nen*3
  std::vector<double> K;     // nen*nen*9 (only (i,j) with bj >= bi valid)
  std::vector<double> div;   // NODAL divBlk contributions: nen*nen*3, [i][j]
  int inverted = 0;
  double minDetJ = 1e300;
};

static double current_volume(const Model& m, int e, const double* x);

// ELEMENT soft incompressibility with several pressure values per element
// (computePressuresAndRinv, FemModel3d.java:2538-2581): per point the
// Jacobian ratio detJ/detJ0, dV = detJ0 w, pbuf_i = sum_k H_i p(K, J_k) dV,
// p = W pbuf / V0; Rinv = W K / V0 for the quadratic potential, else
// Wt R Wt with Wt = W / V0 and R_ij = sum_k H_i H_j modulus(K, J_k) dV
static void multi_pressures(const Model& m, int e, const double* x, std::vector<double>& pvals,
                            std::vector<double>& Rinv) {
  const ShapeTable& s = m.shp(e);
  const int nen = s.nen, npv = s.npv;
  const int* nodes = m.nodes_of(e);
  const Material& mat = m.mat_of(e);
  const double V0 = m.restVol[e], K = mat.kappa;
  const bool quad = mat.bulk_potential == 0;
  std::vector<double> pbuf(npv, 0.0), R((size_t)npv * npv, 0.0);
  for (int k = 0; k < s.nip; k++) {
    double J[9];
    compute_jacobian(J, &s.GNs[k * nen * 3], nen, x, nodes);
    const double detJ0 = m.detJ0[(size_t)m.ipoff[e] + k];
    const double Jk = det3(J) / detJ0;
    const double dV = detJ0 * s.w[k];
    const double* H = &s.H[(size_t)k * npv];
    const double pv = (quad ? K * (Jk - 1) : K * std::log(Jk) / Jk) * dV;
    for (int i = 0; i < npv; i++) pbuf[i] += H[i] * pv;
    if (!quad) {
      const double mod = K * (1 - std::log(Jk)) / (Jk * Jk);
      for (int i = 0; i < npv; i++)
        for (int j = 0; j < npv; j++) R[(size_t)i * npv + j] += H[i] * H[j] * mod * dV;
    }
  }
  pvals.assign(npv, 0.0);
  for (int i = 0; i < npv; i++) {
    for (int j = 0; j < npv; j++) pvals[i] += s.W[(size_t)i * npv + j] * pbuf[j];
    pvals[i] /= V0;
  }
  Rinv.assign((size_t)npv * npv, 0.0);
  if (quad) {
    for (int q = 0; q < npv * npv; q++) Rinv[q] = s.W[q] * (K / V0);
  } else {
    std::vector<double> Wt(s.W), RW((size_t)npv * npv, 0.0);
    for (double& v : Wt) v /= V0;
    for (int i = 0; i < npv; i++)
      for (int j = 0; j < npv; j++)
        for (int l = 0; l < npv; l++) RW[(size_t)i * npv + j] += R[(size_t)i * npv + l] * Wt[(size_t)l * npv + j];
    for (int i = 0; i < npv; i++)
      for (int j = 0; j < npv; j++)
        for (int l = 0; l < npv; l++) Rinv[(size_t)i * npv + j] += Wt[(size_t)i * npv + l] * RW[(size_t)l * npv + j];
  }
}


static void element_update(const Model& m, int e, const double* x, ElemOut& out) {
  // the element's own material, else the model's (FemModel3d.java:2950-2951)
  const Material& mat = m.mat_of(e);
  const int incomp = m.incomp_of(e);
  const ShapeTable& s = m.shp(e);
  int nen = s.nen;
  const int* nodes = m.nodes_of(e);
  out.f.assign(nen * 3, 0);
  out.K.assign(nen * nen * 9, 0);
  out.div.assign(incomp == INCOMP_NODAL ? nen * nen * 3 : 0, 0);
  out.inverted = 0;
  out.minDetJ = 1e300;
  if (mat.linear()) {
    // linear cached path (FemModel3d.java:3359-3390)
    const double* K0 = &m.K0[(size_t)m.k0off[e] * 9];
    const double* f0 = &m.f0[(size_t)m.eoff[e] * 3];
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (mat.corotated) {
      // StiffnessWarper3d.computeWarpingRotation (StiffnessWarper3d.java:154-159)
      double J[9], F[9];
      compute_jacobian(J, s.wGNs.data(), nen, x, nodes);
      mul3(F, J, &m.winvJ0[(size_t)e * 9]);
      polar_rotation(R, F);
    }
    for (int i = 0; i < nen; i++) {
      int bi = m.sidx[nodes[i]];
      if (bi == -1) continue;
      for (int j = 0; j < nen; j++) {
        int bj = m.sidx[nodes[j]];
        if (bj >= bi) {
          const double* Kij = &K0[(i * nen + j) * 9];
          double* Ko = &out.K[(i * nen + j) * 9];
          if (mat.corotated) {
            // StiffnessWarper3d.rotateStiffness: R K R^T (:219-222)
            double T[9];
            for (int a = 0; a < 3; a++)
              for (int b = 0; b < 3; b++)
                T[3 * a + b] = Kij[3 * a] * R[3 * b] + Kij[3 * a + 1] * R[3 * b + 1] + Kij[3 * a + 2] * R[3 * b + 2];
            double U[9];
            mul3(U, R, T);
            for (int q = 0; q < 9; q++) Ko[q] += U[q];
          } else {
            for (int q = 0; q < 9; q++) Ko[q] += Kij[q];
          }
        }
      }
      // StiffnessWarper3d.addNodeForce (:278-307)
      double tmp[3] = {0, 0, 0};
      for (int j = 0; j < nen; j++) {
        const double* p = &x[3 * nodes[j]];
        double pos[3];
        if (mat.corotated) {
          for (int r = 0; r < 3; r++) pos[r] = R[r] * p[0] + R[3 + r] * p[1] + R[6 + r] * p[2];
        } else {
          pos[0] = p[0]; pos[1] = p[1]; pos[2] = p[2];
        }
        const double* Kij = &K0[(i * nen + j) * 9];
        for (int r = 0; r < 3; r++) tmp[r] += Kij[3 * r] * pos[0] + Kij[3 * r + 1] * pos[1] + Kij[3 * r + 2] * pos[2];
      }
      for (int r = 0; r < 3; r++) tmp[r] -= f0[3 * i + r];
      if (mat.corotated) {
        double t2[3];
        for (int r = 0; r < 3; r++) t2[r] = R[3 * r] * tmp[0] + R[3 * r + 1] * tmp[1] + R[3 * r + 2] * tmp[2];
        for (int r = 0; r < 3; r++) out.f[3 * i + r] += t2[r];
      } else {
        for (int r = 0; r < 3; r++) out.f[3 * i + r] += tmp[r];
      }
    }
    return;
  }
  // non-linear path (FemModel3d.java:3443-3631)
  std::vector<double> GNx(nen * 3);
  // ELEMENT soft incompressibility, one pressure value per element (tet and
  // hex): computePressuresAndRinv (FemModel3d.java:2517-2591, npvals == 1):
  // J = V/V0, p = effectivePressure(K, J), Rinv = effectiveModulus(K, J)/V0
  // (IncompressibleMaterialBase.java:116-152); the constraint vectors
  // c_i = sum_k GNx_i dv (FemUtilities.addToIncompressConstraints) and the
  // dilational stiffness Rinv c_i c_j^T (:3650-3663)
  const bool elem_inc = incomp == INCOMP_ELEMENT;
  const int npv = s.npv;
  double elem_p = 0, elem_rinv = 0;
  std::vector<double> cst, pvals, Rinv;
  if (elem_inc && npv == 1) {
    const double V0 = m.restVol[e];
    const double Jp = current_volume(m, e, x) / V0;
    const double K = mat.kappa;
    elem_p = (mat.bulk_potential == 0) ? K * (Jp - 1) : K * std::log(Jp) / Jp;
    const double keff = (mat.bulk_potential == 0) ? K : K * (1 - std::log(Jp)) / (Jp * Jp);
    elem_rinv = keff / V0;
    cst.assign(nen * 3, 0);
  } else if (elem_inc) {
    multi_pressures(m, e, x, pvals, Rinv);
    cst.assign((size_t)nen * 3 * npv, 0);  // node i, row r, pressure value l
  }
  for (int k = 0; k < s.nip; k++) {
    const double* GNs = &s.GNs[k * nen * 3];
    double J[9], invJ[9], F[9];
    compute_jacobian(J, GNs, nen, x, nodes);
    mul3(F, J, &m.invJ0[((size_t)m.ipoff[e] + k) * 9]);
    double detF = det3(F);
    double detJ = fast_invert(invJ, J);
    out.minDetJ = std::min(out.minDetJ, detJ);
    if (detJ <= 0) out.inverted = 1;
    double dv = detJ * s.w[k];
    for (int n = 0; n < nen; n++) {
      const double* g = GNs + 3 * n;
      for (int c = 0; c < 3; c++)
        GNx[3 * n + c] = invJ[c] * g[0] + invJ[3 + c] * g[1] + invJ[6 + c] * g[2];
    }
    double pressure = 0;
    if (incomp == INCOMP_NODAL) {
      if (m.etype[e] == ELEM_TET) {
        for (int i = 0; i < nen; i++) pressure += m.nodePressure[nodes[i]];
        pressure /= nen;
      } else {
        pressure = m.nodePressure[nodes[k]];
      }
    } else if (elem_inc && npv == 1) {
      pressure = elem_p;
      for (int n = 0; n < nen; n++)
        for (int c = 0; c < 3; c++) cst[3 * n + c] += GNx[3 * n + c] * dv;
    } else if (elem_inc) {
      // pressure = sum_l H_l p_l at the point (FemModel3d.java:3465-3471);
      // constraints += H dv GNx (FemUtilities.addToIncompressConstraints)
      const double* H = &s.H[(size_t)k * npv];
      for (int l = 0; l < npv; l++) pressure += H[l] * pvals[l];
      for (int n = 0; n < nen; n++)
        for (int l = 0; l < npv; l++) {
          const double hd = H[l] * dv;
          for (int c = 0; c < 3; c++) cst[((size_t)n * 3 + c) * npv + l] += hd * GNx[3 * n + c];
        }
    }
    double sig[6], D[36];
    material_stress_tangent(sig, D, mat, F, detF, pressure);
    for (int i = 0; i < nen; i++) {
      add_stress_force(&out.f[3 * i], &GNx[3 * i], sig, dv);
      int bi = m.sidx[nodes[i]];
      if (bi != -1) {
        for (int j = 0; j < nen; j++) {
          int bj = m.sidx[nodes[j]];
          if (bj >= bi) {
            double* Ko = &out.K[(i * nen + j) * 9];
            add_material_stiffness(Ko, &GNx[3 * i], D, &GNx[3 * j], dv);
            add_geometric_stiffness(Ko, &GNx[3 * i], sig, &GNx[3 * j], dv);
            // FemNodeNeighbor.addPressureStiffness is a no-op unless
            // noIncompressStiffnessDamping (FemNodeNeighbor.java:541-551)
          }
        }
      }
    }
    if (incomp == INCOMP_NODAL && m.etype[e] != ELEM_TET) {
      // integration points map to nodes (FemModel3d.java:3604-3614):
      // divBlk(node_k, node_j) += dv * GNx_j
      for (int j = 0; j < nen; j++)
        for (int c = 0; c < 3; c++) out.div[(k * nen + j) * 3 + c] += dv * GNx[3 * j + c];
    }
  }
  if (elem_inc) {
    for (int i = 0; i < nen; i++) {
      int bi = m.sidx[nodes[i]];
      if (bi == -1) continue;
      for (int j = 0; j < nen; j++) {
        int bj = m.sidx[nodes[j]];
        if (bj < bi) continue;
        double* Ko = &out.K[(i * nen + j) * 9];
        if (npv == 1) {
          for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) Ko[3 * r + q] += elem_rinv * cst[3 * i + r] * cst[3 * j + q];
        } else {
          // FemUtilities.addDilationalStiffness (FemUtilities.java:317-342):
          // X = Rinv GT_j^T, K_ij += GT_i X
          for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) {
              double acc = 0;
              for (int l = 0; l < npv; l++) {
                double xq = 0;
                for (int mm = 0; mm < npv; mm++)
                  xq += Rinv[(size_t)l * npv + mm] * cst[((size_t)j * 3 + q) * npv + mm];
                acc += cst[((size_t)i * 3 + r) * npv + l] * xq;
              }
              Ko[3 * r + q] += acc;
            }
        }
      }
    }
  }
  if (incomp == INCOMP_NODAL && m.etype[e] == ELEM_TET) {
    // TetElement.getAreaWeightedNormals (TetElement.java:333-362) * (-1/12)
    const double *p0 = &x[3 * nodes[0]], *p1 = &x[3 * nodes[1]], *p2 = &x[3 * nodes[2]],
                 *p3 = &x[3 * nodes[3]];
    const double* tri[4][3] = {{p1, p2, p3}, {p0, p3, p2}, {p0, p1, p3}, {p0, p2, p1}};
    double c[4][3];
    for (int a = 0; a < 4; a++) {
      const double *q0 = tri[a][0], *q1 = tri[a][1], *q2 = tri[a][2];
      double ux = q1[0] - q0[0], uy = q1[1] - q0[1], uz = q1[2] - q0[2];
      double vx = q2[0] - q0[0], vy = q2[1] - q0[1], vz = q2[2] - q0[2];
      c[a][0] = 0.5 * (uy * vz - uz * vy) * (-1 / 12.0);
      c[a][1] = 0.5 * (uz * vx - ux * vz) * (-1 / 12.0);
      c[a][2] = 0.5 * (ux * vy - uy * vx) * (-1 / 12.0);
    }
    // divBlk(node_i, node_j) += c_j for every element node i (:3632-3643)
    for (int i = 0; i < 4; i++)
      for (int j = 0; j < 4; j++)
        for (int q = 0; q < 3; q++) out.div[(i * 4 + j) * 3 + q] += c[j][q];
  }
}

static double current_volume(const Model& m, int e, const double* x) {
  const int* nodes = m.nodes_of(e);
  const ShapeTable& s = m.shp(e);
  if (m.etype[e] == ELEM_TET) {
    const double *p0 = &x[3 * nodes[0]], *p1 = &x[3 * nodes[1]], *p2 = &x[3 * nodes[2]],
                 *p3 = &x[3 * nodes[3]];
    double a[9] = {p1[0] - p0[0], p2[0] - p0[0], p3[0] - p0[0], p1[1] - p0[1], p2[1] - p0[1],
                   p3[1] - p0[1], p1[2] - p0[2], p2[2] - p0[2], p3[2] - p0[2]};
    return det3(a) / 6;
  }
  double vol = 0, J[9];
  for (int k = 0; k < s.nip; k++) {
    compute_jacobian(J, &s.GNs[k * s.nen * 3], s.nen, x, nodes);
    vol += det3(J) * s.w[k];
  }
  return vol;
}

static int update_stress_stiffness(Model& m, const double* x) {
  size_t nnzb = m.col.size();
  m.K.assign(nnzb * 9, 0);
  m.fint.assign((size_t)3 * m.N, 0);
  bool nodal = (m.incomp == INCOMP_NODAL);
  if (nodal) {
    // updateNodalRestVolumes (FemModel3d.java:2594-2628) -- rest volumes are
    // constant; computed once in orc_create.
    // updateNodalPressures (FemModel3d.java:2471-2515)
    m.nodeVol.assign(m.N, 0);
    for (int e = 0; e < m.E; e++) {
      const int* nodes = m.nodes_of(e);
      const ShapeTable& s = m.shp(e);
      const int nen = s.nen;
      if (m.etype[e] == ELEM_TET) {
        double vol = current_volume(m, e, x);
        for (int i = 0; i < nen; i++) m.nodeVol[nodes[i]] += vol / 4;
      } else {
        double J[9];
        for (int k = 0; k < s.nip; k++) {
          compute_jacobian(J, &s.GNs[k * nen * 3], nen, x, nodes);
          m.nodeVol[nodes[k]] += det3(J) * s.w[k];
        }
      }
    }
    m.nodePressure.assign(m.N, 0);
    for (int n = 0; n < m.N; n++) {
      if (m.sidx[n] >= 0) {
        double Jn = m.nodeVol[n] / m.nodeRestVol[n];
        double K = m.mat.kappa;
        m.nodePressure[n] = (m.mat.bulk_potential == 0) ? K * (Jn - 1) : K * std::log(Jn) / Jn;
      }
    }
  }
  std::vector<ElemOut> outs(m.E);
#pragma omp parallel for schedule(static)
  for (int e = 0; e < m.E; e++) element_update(m, e, x, outs[e]);

  m.numInverted = 0;
  m.minDetJ = 1e300;
  // divBlk storage: per node n, one 3-vector per direct neighbour (sorted)
  std::vector<std::vector<double>> div;
  if (nodal) {
    div.resize(m.N);
    for (int n = 0; n < m.N; n++) div[n].assign(m.nbr[n].size() * 3, 0);
  }
  for (int e = 0; e < m.E; e++) {
    const ElemOut& o = outs[e];
    const int* nodes = m.nodes_of(e);
    const int nen = m.nen_of(e);
    m.numInverted += o.inverted;
    m.minDetJ = std::min(m.minDetJ, o.minDetJ);
    for (int i = 0; i < nen; i++) {
      for (int r = 0; r < 3; r++) m.fint[3 * nodes[i] + r] += o.f[3 * i + r];
      int bi = m.sidx[nodes[i]];
      if (bi == -1) continue;
      for (int j = 0; j < nen; j++) {
        int bj = m.sidx[nodes[j]];
        if (bj >= bi) {
          int b = m.block_index(bi, bj);
          for (int q = 0; q < 9; q++) m.K[(size_t)b * 9 + q] += o.K[(i * nen + j) * 9 + q];
        }
      }
    }
    if (nodal && !o.div.empty()) {
      for (int i = 0; i < nen; i++) {
        int n = nodes[i];
        for (int j = 0; j < nen; j++) {
          auto it = std::lower_bound(m.nbr[n].begin(), m.nbr[n].end(), nodes[j]);
          size_t idx = it - m.nbr[n].begin();
          for (int q = 0; q < 3; q++) div[n][idx * 3 + q] += o.div[(i * nen + j) * 3 + q];
        }
      }
    }
  }
  if (nodal) {
    // computeNodalIncompressibility (FemModel3d.java:2632-2669)
    m.nodeKp.assign(m.N, 0.0);
    for (int n = 0; n < m.N; n++) {
      if (m.sidx[n] < 0) continue;
      double restVol = m.nodeRestVol[n];
      double Jn = m.nodeVol[n] / restVol;
      double K = m.mat.kappa;
      double keff = (m.mat.bulk_potential == 0) ? K : K * (1 - std::log(Jn)) / (Jn * Jn);
      double kp = keff / restVol;
      m.nodeKp[n] = kp;
      if (kp == 0) continue;
      const auto& nb = m.nbr[n];
      for (size_t a = 0; a < nb.size(); a++) {
        int bi = m.sidx[nb[a]];
        if (bi < 0) continue;
        for (size_t c = 0; c < nb.size(); c++) {
          int bj = m.sidx[nb[c]];
          if (bj < bi) continue;
          int b = m.block_index(bi, bj);
          const double* gi = &div[n][a * 3];
          const double* gj = &div[n][c * 3];
          // FemUtilities.addDilationalStiffness: K += kp * gi gj^T
          for (int r = 0; r < 3; r++)
            for (int q = 0; q < 3; q++) m.K[(size_t)b * 9 + 3 * r + q] += kp * gi[r] * gj[q];
        }
      }
    }
  }
  if (nodal) m.divBlk = std::move(div);
  // symmetrise: lower block := transpose of upper (FemModel3d.java:3003-3026)
  for (int bi = 0; bi < m.nact; bi++) {
    for (int p = m.rowptr[bi]; p < m.rowptr[bi + 1]; p++) {
      int bj = m.col[p];
      if (bj >= bi) continue;
      int bu = m.block_index(bj, bi);
      for (int r = 0; r < 3; r++)
        for (int q = 0; q < 3; q++) m.K[(size_t)p * 9 + 3 * r + q] = m.K[(size_t)bu * 9 + 3 * q + r];
    }
  }
  return 0;
}

// y = K x over active blocks (x, y indexed by block row / solve index)
static void bsr_mul(const Model& m, const std::vector<double>& vals, const double* x, double* y) {
#pragma omp parallel for schedule(static)
  for (int bi = 0; bi < m.nact; bi++) {
    double a0 = 0, a1 = 0, a2 = 0;
    for (int p = m.rowptr[bi]; p < m.rowptr[bi + 1]; p++) {
      const double* B = &vals[(size_t)p * 9];
      const double* v = &x[3 * m.col[p]];
      a0 += B[0] * v[0] + B[1] * v[1] + B[2] * v[2];
      a1 += B[3] * v[0] + B[4] * v[1] + B[5] * v[2];
      a2 += B[6] * v[0] + B[7] * v[1] + B[8] * v[2];
    }
    y[3 * bi] = a0; y[3 * bi + 1] = a1; y[3 * bi + 2] = a2;
  }
}

static double dot(const std::vector<double>& a, const std::vector<double>& b) {
  double s = 0;
  for (size_t i = 0; i < a.size(); i++) s += a[i] * b[i];
  return s;
}

// Jacobi-preconditioned CG to a relative residual ||b - A x|| / ||b|| <= tol
// (CGSolver.solve, CGSolver.java:42-134, with a diagonal preconditioner).
static int cg_solve(const Model& m, const std::vector<double>& S, const std::vector<double>& b,
                    std::vector<double>& x, double tol, int maxit, int* iters, double* relres) {
  size_t n = b.size();
  std::vector<double> r(n), z(n), p(n), q(n), dinv(n);
  for (int bi = 0; bi < m.nact; bi++) {
    int d = m.block_index(bi, bi);
    for (int c = 0; c < 3; c++) dinv[3 * bi + c] = 1.0 / S[(size_t)d * 9 + 4 * c];
  }
  bsr_mul(m, S, x.data(), q.data());
  for (size_t i = 0; i < n; i++) r[i] = b[i] - q[i];
  double bn = std::sqrt(dot(b, b));
  if (bn == 0) bn = 1;
  for (size_t i = 0; i < n; i++) z[i] = dinv[i] * r[i];
  p = z;
  double rho = dot(r, z);
  int it = 0;
  double rr = std::sqrt(dot(r, r));
  while (rr / bn > tol && it < maxit) {
    bsr_mul(m, S, p.data(), q.data());
    double alpha = rho / dot(p, q);
    for (size_t i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * q[i]; }
    for (size_t i = 0; i < n; i++) z[i] = dinv[i] * r[i];
    double rho1 = dot(r, z);
    double beta = rho1 / rho;
    rho = rho1;
    for (size_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    rr = std::sqrt(dot(r, r));
    it++;
  }
  if (iters) *iters = it;
  if (relres) *relres = rr / bn;
  return (rr / bn <= tol) ? 0 : 1;
}

// dense Cholesky for small systems (stands in for the reference's direct
// PARDISO solve, MechSystemSolver.doDirectSolve, MechSystemSolver.java:2113)
static int dense_solve(const Model& m, const std::vector<double>& S, const std::vector<double>& b,
                       std::vector<double>& x) {
  int n = 3 * m.nact;
  std::vector<double> A((size_t)n * n, 0);
  for (int bi = 0; bi < m.nact; bi++)
    for (int p = m.rowptr[bi]; p < m.rowptr[bi + 1]; p++) {
      int bj = m.col[p];
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) A[(size_t)(3 * bi + r) * n + 3 * bj + c] = S[(size_t)p * 9 + 3 * r + c];
    }
  for (int j = 0; j < n; j++) {
    double d = A[(size_t)j * n + j];
    for (int k = 0; k < j; k++) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
    if (d <= 0) return 2;
    d = std::sqrt(d);
    A[(size_t)j * n + j] = d;
    for (int i = j + 1; i < n; i++) {
      double s = A[(size_t)i * n + j];
      for (int k = 0; k < j; k++) s -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
      A[(size_t)i * n + j] = s / d;
    }
  }
  x.assign(n, 0);
  std::vector<double> y(n);
  for (int i = 0; i < n; i++) {
    double s = b[i];
    for (int k = 0; k < i; k++) s -= A[(size_t)i * n + k] * y[k];
    y[i] = s / A[(size_t)i * n + i];
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = y[i];
    for (int k = i + 1; k < n; k++) s -= A[(size_t)k * n + i] * x[k];
    x[i] = s / A[(size_t)i * n + i];
  }
  return 0;
}

static uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

}  // namespace

// ---------------------------------------------------------------------------
// C API (ctypes)
// ---------------------------------------------------------------------------
extern "C" {

int orc_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
#else
  (void)n;
  return 1;
#endif
}

void orc_create_grid(int type, double wx, double wy, double wz, int nx, int ny, int nz, double* xyz, int* conn);

// FemFactory.createQuadraticModel (FemFactory.java:5641-5710) for tets, as
// the reference does it: for each element in order, the edge midpoints of
// QuadtetElement.getQuadraticNodes (:130-175) are compared with every node so
// far (exact position equality) and appended when new.  *nout = node count;
// oxyz / oconn may be null.
static void quadratic_model(int lin, int nn, const double* xyz, int ne, const int* conn, int* nout, double* oxyz,
                            int* oconn) {
  std::vector<double> P(xyz, xyz + 3 * (size_t)nn);
  // getQuadraticNodes of QuadtetElement (:130-175), QuadhexElement
  // (:237-260), QuadwedgeElement (:343-360), QuadpyramidElement (:336-350)
  const int tedges[6][2] = {{0, 1}, {1, 2}, {0, 2}, {0, 3}, {1, 3}, {2, 3}};
  const int hedges[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6}, {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
  const int wedges[9][2] = {{0, 1}, {1, 2}, {2, 0}, {3, 4}, {4, 5}, {5, 3}, {0, 3}, {1, 4}, {2, 5}};
  const int pedges[8][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {0, 4}, {1, 4}, {2, 4}, {3, 4}};
  const int nls[4] = {4, 8, 6, 5}, nes[4] = {6, 12, 9, 8};
  const int nl = nls[lin], nedge = nes[lin], nq = nl + nedge;
  const int(*edges)[2] = lin == ELEM_HEX ? hedges : lin == ELEM_WEDGE ? wedges : lin == ELEM_PYRAMID ? pedges : tedges;
  std::vector<int> Q(nq * (size_t)ne);
  for (int e = 0; e < ne; e++) {
    const int* c = conn + nl * (size_t)e;
    for (int a = 0; a < nl; a++) Q[nq * (size_t)e + a] = c[a];
    for (int j = 0; j < nedge; j++) {
      const double* pa = xyz + 3 * (size_t)c[edges[j][0]];
      const double* pb = xyz + 3 * (size_t)c[edges[j][1]];
      double p[3];
      for (int r = 0; r < 3; r++) p[r] = (pa[r] + pb[r]) * 0.5;  // Point3d.add, scale(0.5)
      int found = -1;
      const int cur = (int)(P.size() / 3);
      for (int n = 0; n < cur && found < 0; n++)
        if (P[3 * n] == p[0] && P[3 * n + 1] == p[1] && P[3 * n + 2] == p[2]) found = n;
      if (found < 0) {
        found = cur;
        P.insert(P.end(), p, p + 3);
      }
      Q[nq * (size_t)e + nl + j] = found;
    }
  }
  *nout = (int)(P.size() / 3);
  if (oxyz) std::copy(P.begin(), P.end(), oxyz);
  if (oconn) std::copy(Q.begin(), Q.end(), oconn);
}

void orc_quadratic_tets(int nn, const double* xyz, int ne, const int* conn, int* nout, double* oxyz,
                        int* oconn) {
  quadratic_model(ELEM_TET, nn, xyz, ne, conn, nout, oxyz, oconn);
}

void orc_quadratic_hexes(int nn, const double* xyz, int ne, const int* conn, int* nout, double* oxyz,
                         int* oconn) {
  quadratic_model(ELEM_HEX, nn, xyz, ne, conn, nout, oxyz, oconn);
}

void orc_grid_dims(int type, int nx, int ny, int nz, int* nnodes, int* nelems) {
  *nnodes = (nx + 1) * (ny + 1) * (nz + 1);
  const int per_cell[8] = {5, 1, 2, 3, 5, 1, 2, 3};
  *nelems = per_cell[type] * nx * ny * nz;
  if (type >= ELEM_QUADTET) {
    const int lin = type - ELEM_QUADTET;  // tet, hex, wedge, pyramid
    const int nls[4] = {4, 8, 6, 5};
    std::vector<double> x(3 * (size_t)*nnodes);
    std::vector<int> c(nls[lin] * (size_t)*nelems);
    orc_create_grid(lin, 1, 1, 1, nx, ny, nz, x.data(), c.data());
    quadratic_model(lin, *nnodes, x.data(), *nelems, c.data(), nnodes, nullptr, nullptr);
  }
}

// FemFactory.createGridNodes (FemFactory.java:53-78), createTetGrid (:86-126)
// with Tetrahedralizer.subdivideHex(..., allOnX) (Tetrahedralizer.java:135-141,
// parseCode :203-263, getTetIndicesForHex :265-300), createHexGrid (:203-255).
void orc_create_grid(int type, double wx, double wy, double wz, int nx, int ny, int nz,
                     double* xyz, int* conn) {
  if (type >= ELEM_QUADTET) {
    // createQuadtetGrid / createQuadhexGrid / createQuadwedgeGrid /
    // createQuadpyramidGrid (FemFactory.java:316-376)
    const int lin = type - ELEM_QUADTET;
    const int nls[4] = {4, 8, 6, 5}, per[4] = {5, 1, 2, 3};
    const int nl = (nx + 1) * (ny + 1) * (nz + 1), ne = per[lin] * nx * ny * nz;
    std::vector<double> x(3 * (size_t)nl);
    std::vector<int> c(nls[lin] * (size_t)ne);
    orc_create_grid(lin, wx, wy, wz, nx, ny, nz, x.data(), c.data());
    int nout;
    quadratic_model(lin, nl, x.data(), ne, c.data(), &nout, xyz, conn);
    return;
  }
  double dx = 1.0 / nx, dy = 1.0 / ny, dz = 1.0 / nz;
  int idx = 0;
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++) {
        xyz[3 * idx] = wx * (-0.5 + i * dx);
        xyz[3 * idx + 1] = wy * (-0.5 + j * dy);
        xyz[3 * idx + 2] = wz * (-0.5 + k * dz);
        idx++;
      }
  int wk = (nx + 1) * (ny + 1), wj = nx + 1;
  static const int tetsA[5][4] = {{1, 0, 2, 5}, {3, 0, 7, 2}, {4, 0, 5, 7}, {6, 2, 7, 5}, {0, 2, 5, 7}};
  static const int tetsB[5][4] = {{0, 1, 4, 3}, {2, 3, 6, 1}, {5, 4, 1, 6}, {7, 6, 3, 4}, {1, 6, 4, 3}};
  int e = 0;
  for (int i = 0; i < nx; i++)
    for (int j = 0; j < ny; j++)
      for (int k = 0; k < nz; k++) {
        int h[8] = {(k + 1) * wk + j * wj + i,     (k + 1) * wk + j * wj + i + 1,
                    (k + 1) * wk + (j + 1) * wj + i + 1, (k + 1) * wk + (j + 1) * wj + i,
                    k * wk + j * wj + i,           k * wk + j * wj + i + 1,
                    k * wk + (j + 1) * wj + i + 1, k * wk + (j + 1) * wj + i};
        if (type == ELEM_HEX) {
          for (int a = 0; a < 8; a++) conn[8 * e + a] = h[a];
          e++;
        } else if (type == ELEM_WEDGE) {
          // createWedgeGrid (FemFactory.java:266-310)
          const int w[2][6] = {{h[0], h[1], h[4], h[3], h[2], h[7]}, {h[1], h[5], h[4], h[2], h[6], h[7]}};
          for (int q = 0; q < 2; q++, e++)
            for (int a = 0; a < 6; a++) conn[6 * e + a] = w[q][a];
        } else if (type == ELEM_PYRAMID) {
          // createPyramidGrid (FemFactory.java:137-195): apexNodeTable
          // (:128-129) indexed by the parity code, then
          // PyramidElement.createCubeTesselation (PyramidElement.java:216-270)
          static const int apexTable[8] = {2, 3, 1, 0, 6, 7, 5, 4};
          static const int tess[8][3][5] = {
              {{6, 2, 3, 7, 0}, {6, 5, 1, 2, 0}, {6, 7, 4, 5, 0}},
              {{7, 6, 2, 3, 1}, {7, 3, 0, 4, 1}, {7, 4, 5, 6, 1}},
              {{4, 5, 6, 7, 2}, {4, 0, 1, 5, 2}, {4, 7, 3, 0, 2}},
              {{5, 1, 2, 6, 3}, {5, 4, 0, 1, 3}, {5, 6, 7, 4, 3}},
              {{2, 3, 7, 6, 4}, {2, 1, 0, 3, 4}, {2, 6, 5, 1, 4}},
              {{3, 2, 1, 0, 5}, {3, 0, 4, 7, 5}, {3, 7, 6, 2, 5}},
              {{0, 3, 2, 1, 6}, {0, 1, 5, 4, 6}, {0, 4, 7, 3, 6}},
              {{1, 0, 3, 2, 7}, {1, 2, 6, 5, 7}, {1, 5, 4, 0, 7}}};
          int code = 0;
          if (i % 2 == 0) code |= 1;
          if (j % 2 == 0) code |= 2;
          if (k % 2 == 0) code |= 4;
          const int apex = apexTable[code];
          for (int q = 0; q < 3; q++, e++)
            for (int a = 0; a < 5; a++) conn[5 * e + a] = h[tess[apex][q][a]];
        } else {
          bool allOnX = ((i + j + k) % 2) != 0;
          const int(*t)[4] = allOnX ? tetsA : tetsB;
          for (int q = 0; q < 5; q++) {
            for (int a = 0; a < 4; a++) conn[4 * e + a] = h[t[q][a]];
            e++;
          }
        }
      }
}

// Seeded interior-node jitter: every node strictly inside the box moves by
// (2u-1)*frac*spacing along each axis, u from splitmix64 in node order.
void orc_jitter(int nx, int ny, int nz, double wx, double wy, double wz, double frac,
                uint64_t seed, double* xyz) {
  uint64_t s = seed;
  double sp[3] = {wx / nx, wy / ny, wz / nz};
  int idx = 0;
  for (int k = 0; k <= nz; k++)
    for (int j = 0; j <= ny; j++)
      for (int i = 0; i <= nx; i++, idx++) {
        if (i == 0 || i == nx || j == 0 || j == ny || k == 0 || k == nz) continue;
        for (int a = 0; a < 3; a++) {
          double u = (double)(splitmix64(s) >> 11) * (1.0 / 9007199254740992.0);
          xyz[3 * idx + a] += (2 * u - 1) * frac * sp[a];
        }
      }
}

// mat_params: LINEAR {E, nu, corotated}; NEOHOOKEAN {E, nu};
// MOONEYRIVLIN {c10, c01, c11, c20, c02, kappa, jlimit, bulk_potential}
static Material make_material(int kind, const double* p) {
  Material mat;
  mat.kind = kind;
  if (kind == MAT_LINEAR) {
    mat.E = p[0]; mat.nu = p[1]; mat.corotated = (int)p[2];
  } else if (kind == MAT_NEOHOOKEAN || kind == MAT_STVK) {
    mat.E = p[0]; mat.nu = p[1];
  } else {
    mat.c10 = p[0]; mat.c01 = p[1]; mat.c11 = p[2];
    mat.c20 = p[3]; mat.c02 = p[4]; mat.kappa = p[5];
    mat.jlimit = p[6]; mat.bulk_potential = (int)p[7];
  }
  return mat;
}

// Soft incompressibility and the data that depend on the materials.  NODAL
// needs the model's material to be incompressible and every element to be a
// tet or to have its points at its nodes (softNodalIncompressAllowed,
// FemModel3d.java:400-405); otherwise NODAL and AUTO resolve to ELEMENT
// (getAllowedSoftIncompMethod, :462-481), and AUTO -> NODAL when #elements >
// #active nodes, else ELEMENT.  An element of a compressible material runs
// with OFF (computeStressAndStiffness, :3346-3348), so a model without an
// incompressible element resolves to OFF.
static int finalize_model(Model& m) {
  bool nodal_ok = true, any_incomp = false, all_incomp = true;
  for (int e = 0; e < m.E; e++) {
    const int t = m.etype[e];
    nodal_ok &= (t == ELEM_TET || t == ELEM_HEX || t == ELEM_WEDGE || t == ELEM_PYRAMID);
    any_incomp |= m.mat_of(e).incompressible();
    all_incomp &= m.mat_of(e).incompressible();
  }
  int method = m.incomp_request;
  if (!any_incomp) method = INCOMP_OFF;
  else if ((!m.mat.incompressible() || !nodal_ok) && (method == INCOMP_NODAL || method == INCOMP_AUTO))
    method = INCOMP_ELEMENT;
  else if (method == INCOMP_AUTO) method = (m.E > m.nact) ? INCOMP_NODAL : INCOMP_ELEMENT;
  m.incomp = method;
  bool any_linear = false;
  for (int e = 0; e < m.E; e++) any_linear |= m.mat_of(e).linear();
  m.K0.clear();
  m.f0.clear();
  if (any_linear) build_linear_cache(m);
  build_pattern(m);
  m.nodeRestVol.clear();
  m.nodePressure.clear();
  if (m.incomp == INCOMP_NODAL) {
    // updateNodalRestVolumes (FemModel3d.java:2594-2628)
    m.nodeRestVol.assign(m.N, 0);
    for (int e = 0; e < m.E; e++) {
      const int* nodes = m.nodes_of(e);
      const ShapeTable& st = m.shp(e);
      if (m.etype[e] == ELEM_TET) {
        for (int i = 0; i < 4; i++) m.nodeRestVol[nodes[i]] += m.restVol[e] / 4;
      } else {
        // integration points map to nodes (FemModel3d.java:2608-2614)
        for (int i = 0; i < st.nen; i++)
          m.nodeRestVol[nodes[i]] += st.w[i] * m.detJ0[(size_t)m.ipoff[e] + i];
      }
    }
    if (!all_incomp) return -2;
  }
  return 0;
}
// A mesh of one element type per element (FemModel3d holds any mix of
// FemElement3d types, FemModel3d.java:3333): types[e], and conn the
// concatenation of every element's nodes in its type's local order.
void* orc_create_mixed(int nnodes, const double* rest, int nelems, const int* types, const int* conn,
                       const int* fixed, int mat_kind, const double* mat_params, double density,
                       int incomp_method) {
  Model* m = new Model();
  m->shapes.resize(8);
  std::vector<char> have(8, 0);
  m->etype.assign(types, types + nelems);
  m->eoff.assign(nelems + 1, 0);
  m->ipoff.assign(nelems + 1, 0);
  m->k0off.assign(nelems + 1, 0);
  for (int e = 0; e < nelems; e++) {
    const int t = types[e];
    if (t < 0 || t > 7) {
      delete m;
      return nullptr;
    }
    if (!have[t]) {
      m->shapes[t] = make_shape(t);
      have[t] = 1;
    }
    const ShapeTable& st = m->shapes[t];
    m->eoff[e + 1] = m->eoff[e] + st.nen;
    m->ipoff[e + 1] = m->ipoff[e] + st.nip;
    m->k0off[e + 1] = m->k0off[e] + st.nen * st.nen;
  }
  m->type = nelems > 0 ? types[0] : ELEM_TET;
  m->sh = m->shapes[m->type];
  m->nen = m->sh.nen;
  m->N = nnodes;
  m->E = nelems;
  m->rest.assign(rest, rest + 3 * (size_t)nnodes);
  m->conn.assign(conn, conn + (size_t)m->eoff[nelems]);
  m->sidx.assign(nnodes, -1);
  m->nact = 0;
  for (int n = 0; n < nnodes; n++)
    if (!fixed[n]) m->sidx[n] = m->nact++;
  m->mat = make_material(mat_kind, mat_params);
  m->density = density;
  m->incomp_request = incomp_method;
  build_rest_data(*m);
  finalize_model(*m);
  return m;
}

// Per-element materials (FemElement.setMaterial): kinds[e] < 0 keeps the
// model's material, else element e gets kinds[e] with params[8e .. 8e+7].
// kinds == NULL gives every element the model's material again.  Returns 0,
// or -2 when soft incompressibility resolves to NODAL while some element's
// material is compressible (updateNodalPressures, FemModel3d.java:2471-2503,
// sums nodal volumes over incompressible elements only; a node that only
// compressible elements touch has a zero rest volume).
int orc_set_element_materials(void* h, const int* kinds, const double* params) {
  Model& m = *(Model*)h;
  m.emats.clear();
  if (kinds) {
    m.emats.assign(m.E, m.mat);
    for (int e = 0; e < m.E; e++)
      if (kinds[e] >= 0) m.emats[e] = make_material(kinds[e], params + 8 * (size_t)e);
  }
  return finalize_model(m);
}

void* orc_create(int type, int nnodes, const double* rest, int nelems, const int* conn,
                 const int* fixed, int mat_kind, const double* mat_params, double density,
                 int incomp_method) {
  std::vector<int> types(nelems, type);
  return orc_create_mixed(nnodes, rest, nelems, types.data(), conn, fixed, mat_kind, mat_params, density,
                          incomp_method);
}

void orc_destroy(void* h) { delete (Model*)h; }

// The NODAL terms of the last orc_update_stress_stiffness: per node its
// direct neighbours (sorted: ptr[N+1], idx), kp (0 for fixed nodes) and its
// divBlk row (3 values per neighbour, in idx order).  Any output may be
// NULL; returns the neighbour count, or -1 when the model is not NODAL or
// has not been updated.
int orc_nodal_factors(void* h, int* ptr, int* idx, double* kp, double* div) {
  const Model& m = *(const Model*)h;
  if (m.incomp != INCOMP_NODAL || (int)m.divBlk.size() != m.N || (int)m.nodeKp.size() != m.N) return -1;
  int q = 0;
  for (int n = 0; n < m.N; n++) {
    if (ptr) ptr[n] = q;
    for (size_t a = 0; a < m.nbr[n].size(); a++, q++) {
      if (idx) idx[q] = m.nbr[n][a];
      if (div)
        for (int c = 0; c < 3; c++) div[3 * (size_t)q + c] = m.divBlk[n][3 * a + c];
    }
    if (kp) kp[n] = m.nodeKp[n];
  }
  if (ptr) ptr[m.N] = q;
  return q;
}
int orc_incomp_method(void* h) { return ((Model*)h)->incomp; }
int orc_num_active(void* h) { return ((Model*)h)->nact; }
int orc_nnzb(void* h) { return (int)((Model*)h)->col.size(); }
void orc_solve_index(void* h, int* out) {
  Model* m = (Model*)h;
  std::copy(m->sidx.begin(), m->sidx.end(), out);
}
void orc_pattern(void* h, int* rowptr, int* col) {
  Model* m = (Model*)h;
  std::copy(m->rowptr.begin(), m->rowptr.end(), rowptr);
  std::copy(m->col.begin(), m->col.end(), col);
}
void orc_masses(void* h, double* mass) {
  Model* m = (Model*)h;
  std::copy(m->mass.begin(), m->mass.end(), mass);
}
void orc_rest_volumes(void* h, double* vol) {
  Model* m = (Model*)h;
  std::copy(m->restVol.begin(), m->restVol.end(), vol);
}

// Scalar CRS view of the block pattern (SparseBlockMatrix.getCRSIndices,
// SparseBlockMatrix.java:1511-1532, made 0-based as in
// SparseNumberedBlockMatrix.createCrsBlockSlotMap :396-398).
// partition 0 = Full, 1 = UpperTriangular.  Returns nnz.
int orc_crs(void* h, int partition, int* row_offs, int* col_idx, int* slots) {
  Model* m = (Model*)h;
  int nnz = 0;
  int nrows = 3 * m->nact;
  std::vector<int> slot((size_t)m->col.size() * 9, -1);
  for (int bi = 0; bi < m->nact; bi++) {
    for (int r = 0; r < 3; r++) {
      int row = 3 * bi + r;
      if (row_offs) row_offs[row] = nnz;
      for (int p = m->rowptr[bi]; p < m->rowptr[bi + 1]; p++) {
        int bj = m->col[p];
        for (int c = 0; c < 3; c++) {
          int colg = 3 * bj + c;
          if (partition == 1 && colg < row) continue;
          if (col_idx) col_idx[nnz] = colg;
          slot[(size_t)p * 9 + 3 * r + c] = nnz;
          nnz++;
        }
      }
    }
  }
  if (row_offs) row_offs[nrows] = nnz;
  if (slots) std::copy(slot.begin(), slot.end(), slots);
  return nnz;
}

// FemModel3d.updateStressAndStiffness at positions x (3N): returns the
// internal force per node (3N) and the assembled stiffness blocks (9*nnzb,
// BSR order, both triangles).  Returns the number of inverted elements.
int orc_update_stress_stiffness(void* h, const double* x, double* fint, double* K) {
  Model* m = (Model*)h;
  update_stress_stiffness(*m, x);
  if (fint) std::copy(m->fint.begin(), m->fint.end(), fint);
  if (K) std::copy(m->K.begin(), m->K.end(), K);
  return m->numInverted;
}

void orc_nodal_pressures(void* h, double* p) {
  Model* m = (Model*)h;
  if (m->nodePressure.empty()) std::fill(p, p + m->N, 0.0);
  else std::copy(m->nodePressure.begin(), m->nodePressure.end(), p);
}

// One MechSystemSolver.backwardEuler step (MechSystemSolver.java:2171-2476).
// prm = {alpha_m (massDamping), beta_k (stiffnessDamping), gx, gy, gz}.
// fext: 3N external nodal forces (may be null).  x, v (3N) updated in place.
// solver 0 = Jacobi-PCG to tol, 1 = dense Cholesky.
// Returns 0, or 1 when CG did not converge, 2 when the dense solve failed.
// The BackwardEuler velocity system S v = b of MechSystemSolver.backwardEuler
// (MechSystemSolver.java:2171-2476) at positions x and velocities v (3N):
// S in BSR order (9*nnzb), b and the active velocities vact (3*nact).
// ConstrainedBackwardEuler (MechSystemSolver.java:4804-4923) forms the same
// M block and right-hand side (KKTFactorAndSolve with a0 = -h, a1 = -h^2,
// a2 = -h, a3 = 0: the velocity-Jacobian term times v0, as here).
static void be_system(Model* m, double hstep, const double* prm, const double* fext, const double* x,
                      const double* v, std::vector<double>& S, std::vector<double>& b,
                      std::vector<double>& vact) {
  double am = prm[0], bk = prm[1];
  const double* g = prm + 2;
  update_stress_stiffness(*m, x);
  int nv = 3 * m->nact;
  // FemModel3d.updateNodeForces (FemModel3d.java:2740-2847): for each node
  // f = fext + m g - f_int - (beta_k sum_j K_ij v_j + alpha_m m v)
  std::vector<double> f((size_t)3 * m->N, 0);
  vact.assign(nv, 0);
  std::vector<double> xact(nv);
  for (int n = 0; n < m->N; n++)
    if (m->sidx[n] >= 0)
      for (int c = 0; c < 3; c++) {
        vact[3 * m->sidx[n] + c] = v[3 * n + c];
        xact[3 * m->sidx[n] + c] = x[3 * n + c];
      }
  std::vector<double> Kv(nv, 0);
  if (bk != 0) bsr_mul(*m, m->K, vact.data(), Kv.data());
  for (int n = 0; n < m->N; n++) {
    for (int c = 0; c < 3; c++) {
      double fi = fext ? fext[3 * n + c] : 0.0;
      fi += m->mass[n] * g[c];
      double fk = m->fint[3 * n + c];
      double fd = 0;
      int bi = m->sidx[n];
      if (bi >= 0) fd = bk * Kv[3 * bi + c];
      fd += am * m->mass[n] * v[3 * n + c];
      fi -= fk;
      fi -= fd;
      f[3 * n + c] = fi;
    }
  }
  // b = M v + h f   (:2194-2200)
  b.assign(nv, 0);
  for (int n = 0; n < m->N; n++) {
    int bi = m->sidx[n];
    if (bi < 0) continue;
    for (int c = 0; c < 3; c++) b[3 * bi + c] = m->mass[n] * v[3 * n + c] + hstep * f[3 * n + c];
  }
  // S = h(alpha_m M + beta_k K)  (addVelJacobian, s = -h)
  size_t nnzb = m->col.size();
  S.assign(nnzb * 9, 0);
  for (size_t q = 0; q < nnzb * 9; q++) S[q] = (hstep * bk) * m->K[q];
  for (int n = 0; n < m->N; n++) {
    int bi = m->sidx[n];
    if (bi < 0) continue;
    int d = m->block_index(bi, bi);
    for (int c = 0; c < 3; c++) S[(size_t)d * 9 + 4 * c] += hstep * am * m->mass[n];
  }
  // b += S v   (:2299-2301)
  std::vector<double> Sv(nv);
  bsr_mul(*m, S, vact.data(), Sv.data());
  for (int i = 0; i < nv; i++) b[i] += Sv[i];
  // S += h^2 K  (addPosJacobian, s = -h^2), then S += M (:2312, :2334)
  for (size_t q = 0; q < nnzb * 9; q++) S[q] += (hstep * hstep) * m->K[q];
  for (int n = 0; n < m->N; n++) {
    int bi = m->sidx[n];
    if (bi < 0) continue;
    int d = m->block_index(bi, bi);
    for (int c = 0; c < 3; c++) S[(size_t)d * 9 + 4 * c] += m->mass[n];
  }
}

int orc_be_step(void* h, double hstep, const double* prm, const double* fext, double* x,
                double* v, int solver, double tol, int maxit, int* iters, double* relres) {
  Model* m = (Model*)h;
  int nv = 3 * m->nact;
  std::vector<double> S, b, vact;
  be_system(m, hstep, prm, fext, x, v, S, b, vact);
  std::vector<double> vn = vact;
  int status = 0;
  if (solver == 1) {
    status = dense_solve(*m, S, b, vn);
    if (iters) *iters = 0;
    if (relres) {
      std::vector<double> r(nv);
      bsr_mul(*m, S, vn.data(), r.data());
      double rn = 0, bn = 0;
      for (int i = 0; i < nv; i++) { rn += (b[i] - r[i]) * (b[i] - r[i]); bn += b[i] * b[i]; }
      *relres = std::sqrt(rn / (bn > 0 ? bn : 1));
    }
  } else {
    status = cg_solve(*m, S, b, vn, tol, maxit, iters, relres);
  }
  // setActiveVelState, x1 = x0 + h v1 (:2465-2475)
  for (int n = 0; n < m->N; n++) {
    int bi = m->sidx[n];
    if (bi < 0) continue;
    for (int c = 0; c < 3; c++) {
      v[3 * n + c] = vn[3 * bi + c];
      x[3 * n + c] = x[3 * n + c] + hstep * vn[3 * bi + c];
    }
  }
  return status;
}

// One MechSystemSolver.constrainedBackwardEuler step (MechSystemSolver.java:
// 4804-4923) with bilateral particle-plane constraints
// (ParticlePlaneConstraint.java:144-160, ParticleConstraintBase.java:163-200):
// constraint i holds node nodes[i] on the plane nrm_i . x = off_i (nrm_i unit,
// one constraint per node, nodes not fixed).  The velocity solve is the KKT
// system [S G^T; G 0][v; lam] = [b; 0] with G_i = nrm_i^T on the node (a fixed
// plane has no velocity offset: setBilateralOffsets, :2697-2721, with zero
// compliance and gdot), solved densely (Gaussian elimination, partial
// pivoting); then x1 = x0 + h v1 and the GlobalMass position correction,
// which for one single-particle constraint moves the node onto its plane
// along nrm_i (x -= nrm_i (nrm_i . x - off_i)).  Returns 0, or 2 when the
// KKT matrix is singular.
int orc_cbe_step(void* h, double hstep, const double* prm, const double* fext, double* x, double* v,
                 int ncons, const int* nodes, const double* nrm, const double* off) {
  Model* m = (Model*)h;
  const int nv = 3 * m->nact;
  std::vector<double> S, b, vact;
  be_system(m, hstep, prm, fext, x, v, S, b, vact);
  const int n = nv + ncons;
  std::vector<double> A((size_t)n * n, 0), rhs(n, 0);
  for (int bi = 0; bi < m->nact; bi++)
    for (int p = m->rowptr[bi]; p < m->rowptr[bi + 1]; p++) {
      int bj = m->col[p];
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) A[(size_t)(3 * bi + r) * n + 3 * bj + c] = S[(size_t)p * 9 + 3 * r + c];
    }
  for (int i = 0; i < nv; i++) rhs[i] = b[i];
  for (int k = 0; k < ncons; k++) {
    const int bi = m->sidx[nodes[k]];
    if (bi < 0) return 2;
    for (int c = 0; c < 3; c++) {
      A[(size_t)(nv + k) * n + 3 * bi + c] = nrm[3 * k + c];
      A[(size_t)(3 * bi + c) * n + nv + k] = nrm[3 * k + c];
    }
  }
  // Gaussian elimination with partial pivoting
  std::vector<int> piv(n);
  for (int i = 0; i < n; i++) piv[i] = i;
  for (int j = 0; j < n; j++) {
    int best = j;
    for (int i = j + 1; i < n; i++)
      if (std::fabs(A[(size_t)i * n + j]) > std::fabs(A[(size_t)best * n + j])) best = i;
    if (A[(size_t)best * n + j] == 0) return 2;
    if (best != j) {
      for (int c = 0; c < n; c++) std::swap(A[(size_t)j * n + c], A[(size_t)best * n + c]);
      std::swap(rhs[j], rhs[best]);
    }
    const double d = A[(size_t)j * n + j];
    for (int i = j + 1; i < n; i++) {
      const double f = A[(size_t)i * n + j] / d;
      if (f == 0) continue;
      for (int c = j; c < n; c++) A[(size_t)i * n + c] -= f * A[(size_t)j * n + c];
      rhs[i] -= f * rhs[j];
    }
  }
  std::vector<double> sol(n);
  for (int i = n - 1; i >= 0; i--) {
    double t = rhs[i];
    for (int c = i + 1; c < n; c++) t -= A[(size_t)i * n + c] * sol[c];
    sol[i] = t / A[(size_t)i * n + i];
  }
  for (int nd = 0; nd < m->N; nd++) {
    const int bi = m->sidx[nd];
    if (bi < 0) continue;
    for (int c = 0; c < 3; c++) {
      v[3 * nd + c] = sol[3 * bi + c];
      x[3 * nd + c] += hstep * sol[3 * bi + c];
    }
  }
  for (int k = 0; k < ncons; k++) {
    double* p = &x[3 * nodes[k]];
    const double* q = &nrm[3 * k];
    const double d = q[0] * p[0] + q[1] * p[1] + q[2] * p[2] - off[k];
    for (int c = 0; c < 3; c++) p[c] -= q[c] * d;
  }
  return 0;
}

// dense Gaussian elimination with partial pivoting: solves A x = rhs (n x n,
// row-major, destroyed); returns false for a singular matrix
static bool dense_gauss(std::vector<double>& A, std::vector<double>& rhs, int n, std::vector<double>& sol) {
  for (int j = 0; j < n; j++) {
    int best = j;
    for (int i = j + 1; i < n; i++)
      if (std::fabs(A[(size_t)i * n + j]) > std::fabs(A[(size_t)best * n + j])) best = i;
    if (A[(size_t)best * n + j] == 0) return false;
    if (best != j) {
      for (int c = 0; c < n; c++) std::swap(A[(size_t)j * n + c], A[(size_t)best * n + c]);
      std::swap(rhs[j], rhs[best]);
    }
    const double d = A[(size_t)j * n + j];
    for (int i = j + 1; i < n; i++) {
      const double f = A[(size_t)i * n + j] / d;
      if (f == 0) continue;
      for (int c = j; c < n; c++) A[(size_t)i * n + c] -= f * A[(size_t)j * n + c];
      rhs[i] -= f * rhs[j];
    }
  }
  sol.assign(n, 0.0);
  for (int i = n - 1; i >= 0; i--) {
    double t = rhs[i];
    for (int c = i + 1; c < n; c++) t -= A[(size_t)i * n + c] * sol[c];
    sol[i] = t / A[(size_t)i * n + i];
  }
  return true;
}

// One ConstrainedBackwardEuler step (MechSystemSolver.java:4804-4923) with
// LinearPointConstraints (LinearPointConstraint.java): constraint c holds
// sum_i w_i x_i = target_c, three rows (x, y, z); the row of axis d carries
// w_i on the d component of every point with a solve index
// (addBilateralConstraints).  Velocity: the KKT system [S G^T; G 0][v; lam]
// = [b; 0] (zero compliance and gdot, setBilateralOffsets :2697-2721),
// solved densely; x1 = x0 + h v1; then the GlobalMass position correction
// (applyPosCorrection): with dist = sum_i w_i x_i - target over all points
// of each constraint (getBilateralInfo), dx = M^-1 G^T mu with
// (G M^-1 G^T) mu = -dist, on the active nodes.  ptr (ncons + 1) indexes the
// constraints' points in nodes / w; targets holds 3 values per constraint.
// Returns 0, or 2 when a system is singular.
int orc_cbe_step_points(void* h, double hstep, const double* prm, const double* fext, double* x, double* v,
                        int ncons, const int* ptr, const int* nodes, const double* w, const double* targets) {
  Model* m = (Model*)h;
  const int nv = 3 * m->nact;
  std::vector<double> S, b, vact;
  be_system(m, hstep, prm, fext, x, v, S, b, vact);
  const int mc = 3 * ncons, n = nv + mc;
  std::vector<double> A((size_t)n * n, 0), rhs(n, 0);
  for (int bi = 0; bi < m->nact; bi++)
    for (int p = m->rowptr[bi]; p < m->rowptr[bi + 1]; p++) {
      const int bj = m->col[p];
      for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) A[(size_t)(3 * bi + r) * n + 3 * bj + c] = S[(size_t)p * 9 + 3 * r + c];
    }
  for (int i = 0; i < nv; i++) rhs[i] = b[i];
  for (int c = 0; c < ncons; c++)
    for (int q = ptr[c]; q < ptr[c + 1]; q++) {
      const int bi = m->sidx[nodes[q]];
      if (bi < 0) continue;
      for (int d = 0; d < 3; d++) {
        A[(size_t)(nv + 3 * c + d) * n + 3 * bi + d] += w[q];
        A[(size_t)(3 * bi + d) * n + nv + 3 * c + d] += w[q];
      }
    }
  std::vector<double> sol;
  if (!dense_gauss(A, rhs, n, sol)) return 2;
  for (int nd = 0; nd < m->N; nd++) {
    const int bi = m->sidx[nd];
    if (bi < 0) continue;
    for (int c = 0; c < 3; c++) {
      v[3 * nd + c] = sol[3 * bi + c];
      x[3 * nd + c] += hstep * sol[3 * bi + c];
    }
  }
  // GlobalMass position correction
  std::vector<double> P((size_t)mc * mc, 0), g(mc, 0);
  for (int c = 0; c < ncons; c++)
    for (int d = 0; d < 3; d++) {
      double dist = -targets[3 * c + d];
      for (int q = ptr[c]; q < ptr[c + 1]; q++) dist += w[q] * x[3 * nodes[q] + d];
      g[3 * c + d] = -dist;
    }
  for (int c = 0; c < ncons; c++)
    for (int c2 = 0; c2 < ncons; c2++)
      for (int q = ptr[c]; q < ptr[c + 1]; q++) {
        if (m->sidx[nodes[q]] < 0) continue;
        for (int q2 = ptr[c2]; q2 < ptr[c2 + 1]; q2++) {
          if (nodes[q2] != nodes[q]) continue;
          const double s = w[q] * w[q2] / m->mass[nodes[q]];
          for (int d = 0; d < 3; d++) P[(size_t)(3 * c + d) * mc + 3 * c2 + d] += s;
        }
      }
  std::vector<double> mu;
  if (!dense_gauss(P, g, mc, mu)) return 2;
  for (int c = 0; c < ncons; c++)
    for (int q = ptr[c]; q < ptr[c + 1]; q++) {
      const int nd = nodes[q];
      if (m->sidx[nd] < 0) continue;
      for (int d = 0; d < 3; d++) x[3 * nd + d] += w[q] * mu[3 * c + d] / m->mass[nd];
    }
  return 0;
}

int orc_num_ip(void* h) { return ((Model*)h)->sh.nip; }
int orc_elem_num_ip(void* h, int e) { return ((Model*)h)->shp(e).nip; }

// Integration point k of element e at positions x (3N), as the non-linear
// element loop forms it (FemModel3d.java:3443-3470): shape gradients in the
// current configuration GNx (nen x 3), dv = det J * w, and the material's
// Cauchy stress sig (xx, yy, zz, xy, yz, xz) and tangent D (6x6 row-major,
// same order), with the NODAL pressure of the last update_stress_stiffness
// call where the model uses it.  These are the per-block descriptor inputs
// of the reference's device assembly (FemModel3d.java:4613-4936).  Returns
// nen, or -1 for linear materials (whose blocks come from the rest
// stiffness) and out-of-range e or k.
int orc_ip_data(void* h, const double* x, int e, int k, double* GNx, double* dv, double* sig, double* D) {
  const Model& m = *(const Model*)h;
  if (e < 0 || e >= m.E || m.mat_of(e).linear()) return -1;
  const Material& mat = m.mat_of(e);
  const int incomp = m.incomp_of(e);
  const ShapeTable& s = m.shp(e);
  if (k < 0 || k >= s.nip) return -1;
  const int nen = s.nen;
  const int* nodes = m.nodes_of(e);
  const double* GNs = &s.GNs[k * nen * 3];
  double J[9], invJ[9], F[9];
  compute_jacobian(J, GNs, nen, x, nodes);
  mul3(F, J, &m.invJ0[((size_t)m.ipoff[e] + k) * 9]);
  const double detF = det3(F);
  const double detJ = fast_invert(invJ, J);
  *dv = detJ * s.w[k];
  for (int n = 0; n < nen; n++) {
    const double* g = GNs + 3 * n;
    for (int c = 0; c < 3; c++) GNx[3 * n + c] = invJ[c] * g[0] + invJ[3 + c] * g[1] + invJ[6 + c] * g[2];
  }
  double pressure = 0;
  if (incomp == INCOMP_NODAL && !m.nodePressure.empty()) {
    if (m.etype[e] == ELEM_TET) {
      for (int i = 0; i < nen; i++) pressure += m.nodePressure[nodes[i]];
      pressure /= nen;
    } else {
      pressure = m.nodePressure[nodes[k]];
    }
  } else if (incomp == INCOMP_ELEMENT && s.npv == 1) {
    const double Jp = current_volume(m, e, x) / m.restVol[e];
    const double K = mat.kappa;
    pressure = (mat.bulk_potential == 0) ? K * (Jp - 1) : K * std::log(Jp) / Jp;
  } else if (incomp == INCOMP_ELEMENT) {
    std::vector<double> pvals, Rinv;
    multi_pressures(m, e, x, pvals, Rinv);
    for (int l = 0; l < s.npv; l++) pressure += s.H[(size_t)k * s.npv + l] * pvals[l];
  }
  material_stress_tangent(sig, D, mat, F, detF, pressure);
  return nen;
}

// point-level material evaluation for known-answer and finite-difference tests
void orc_material_eval(int mat_kind, const double* mat_params, const double* F, double pressure,
                       double* sig6, double* D36) {
  Material mt;
  mt.kind = mat_kind;
  if (mat_kind == MAT_LINEAR) { mt.E = mat_params[0]; mt.nu = mat_params[1]; }
  else if (mat_kind == MAT_NEOHOOKEAN || mat_kind == MAT_STVK) { mt.E = mat_params[0]; mt.nu = mat_params[1]; }
  else {
    mt.c10 = mat_params[0]; mt.c01 = mat_params[1]; mt.c11 = mat_params[2]; mt.c20 = mat_params[3];
    mt.c02 = mat_params[4]; mt.kappa = mat_params[5]; mt.jlimit = mat_params[6];
  }
  material_stress_tangent(sig6, D36, mt, F, det3(F), pressure);
}

void orc_material_stiffness_block(const double* gi, const double* D36, const double* sig6,
                                  const double* gj, double dv, double* K9) {
  for (int i = 0; i < 9; i++) K9[i] = 0;
  add_material_stiffness(K9, gi, D36, gj, dv);
  if (sig6) add_geometric_stiffness(K9, gi, sig6, gj, dv);
}

void orc_linear_C(double E, double nu, double* D36) { linear_C(D36, E, nu); }

void orc_polar(const double* F, double* R) { polar_rotation(R, F); }

}  // extern "C"
