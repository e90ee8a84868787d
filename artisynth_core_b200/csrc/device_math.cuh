// device_math.cuh -- per-point FEM arithmetic shared by the element kernels:
// Jacobian inverse, polar rotation, constitutive laws and the B^T D B block
// formula.  Templated on the value type so the FP64 drop-in and the FP32
// element pass of the mixed form share one implementation.
#pragma once

#include <cuda_runtime.h>

#include "../../include/b200fem.h"

namespace b200fem {

template <typename T>
__device__ __forceinline__ T det3(const T* m) {
  return m[0] * m[4] * m[8] + m[3] * m[7] * m[2] + m[6] * m[1] * m[5] - m[6] * m[4] * m[2] -
         m[0] * m[7] * m[5] - m[3] * m[1] * m[8];
}

// Matrix3dBase.fastInvert (Matrix3dBase.java:1615-1648): inverse by
// cofactors, returns the determinant; inv is left untouched when det == 0.
template <typename T>
__device__ __forceinline__ T invert3(T* inv, const T* d) {
  T det = det3(d);
  if (det != T(0)) {
    T s = T(1) / det;
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

template <typename T>
__device__ __forceinline__ void matmul3(T* c, const T* a, const T* b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++)
      c[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

// Rotation R of the polar decomposition F = R P with det(R) = +1, the
// factor SVDecomposition3d.polarDecomposition returns
// (SVDecomposition3d.java:1418-1541: R = U V^T, the U column of the smallest
// singular value negated when det(U) det(V) < 0).  Computed from the
// symmetric eigen-decomposition of C = F^T F by cyclic Jacobi rotations:
// V = eigenvectors (descending eigenvalues), u_k = F v_k / sigma_k for the
// two largest, u_3 = det(V) (u_1 x u_2), R = U V^T.
__device__ inline void polar_rotation(const double* F, double* R) {
  double A[9], V[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) A[3 * i + j] = F[i] * F[j] + F[3 + i] * F[3 + j] + F[6 + i] * F[6 + j];
  const double scale = A[0] + A[4] + A[8];
  for (int sweep = 0; sweep < 16; sweep++) {
    double off = A[1] * A[1] + A[2] * A[2] + A[5] * A[5];
    if (off <= 1e-34 * scale * scale) break;
#pragma unroll
    for (int pq = 0; pq < 3; pq++) {
      const int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
      double apq = A[3 * p + q];
      if (apq == 0.0) continue;
      double theta = (A[3 * q + q] - A[3 * p + p]) / (2.0 * apq);
      double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
      // A <- J^T A J with J the (p,q) rotation
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double akp = A[3 * k + p], akq = A[3 * k + q];
        A[3 * k + p] = c * akp - s * akq;
        A[3 * k + q] = s * akp + c * akq;
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double apk = A[3 * p + k], aqk = A[3 * q + k];
        A[3 * p + k] = c * apk - s * aqk;
        A[3 * q + k] = s * apk + c * aqk;
      }
#pragma unroll
      for (int k = 0; k < 3; k++) {
        double vkp = V[3 * k + p], vkq = V[3 * k + q];
        V[3 * k + p] = c * vkp - s * vkq;
        V[3 * k + q] = s * vkp + c * vkq;
      }
    }
  }
  // order eigenpairs by descending eigenvalue
  int o0 = 0, o1 = 1, o2 = 2;
  double l0 = A[0], l1 = A[4], l2 = A[8];
  if (l0 < l1) { double t = l0; l0 = l1; l1 = t; int u = o0; o0 = o1; o1 = u; }
  if (l1 < l2) { double t = l1; l1 = l2; l2 = t; int u = o1; o1 = o2; o2 = u; }
  if (l0 < l1) { double t = l0; l0 = l1; l1 = t; int u = o0; o0 = o1; o1 = u; }
  double v0[3] = {V[o0], V[3 + o0], V[6 + o0]};
  double v1[3] = {V[o1], V[3 + o1], V[6 + o1]};
  double v2[3] = {V[o2], V[3 + o2], V[6 + o2]};
  if (!(l0 > 0)) {
#pragma unroll
    for (int i = 0; i < 9; i++) R[i] = (i % 4 == 0) ? 1.0 : 0.0;
    return;
  }
  double u0[3], u1[3], u2[3];
#pragma unroll
  for (int r = 0; r < 3; r++) {
    u0[r] = F[3 * r] * v0[0] + F[3 * r + 1] * v0[1] + F[3 * r + 2] * v0[2];
    u1[r] = F[3 * r] * v1[0] + F[3 * r + 1] * v1[1] + F[3 * r + 2] * v1[2];
  }
  double n0 = sqrt(u0[0] * u0[0] + u0[1] * u0[1] + u0[2] * u0[2]);
#pragma unroll
  for (int r = 0; r < 3; r++) u0[r] /= n0;
  double d = u0[0] * u1[0] + u0[1] * u1[1] + u0[2] * u1[2];
#pragma unroll
  for (int r = 0; r < 3; r++) u1[r] -= d * u0[r];
  double n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  if (!(n1 > 1e-300)) {
    // rank-one F: any unit vector orthogonal to u0
    double ax = fabs(u0[0]), ay = fabs(u0[1]), az = fabs(u0[2]);
    double e[3] = {0, 0, 0};
    e[(ax <= ay && ax <= az) ? 0 : (ay <= az ? 1 : 2)] = 1;
    double dd = e[0] * u0[0] + e[1] * u0[1] + e[2] * u0[2];
#pragma unroll
    for (int r = 0; r < 3; r++) u1[r] = e[r] - dd * u0[r];
    n1 = sqrt(u1[0] * u1[0] + u1[1] * u1[1] + u1[2] * u1[2]);
  }
#pragma unroll
  for (int r = 0; r < 3; r++) u1[r] /= n1;
  double Vm[9] = {v0[0], v1[0], v2[0], v0[1], v1[1], v2[1], v0[2], v1[2], v2[2]};
  double sgn = det3(Vm) >= 0 ? 1.0 : -1.0;
  u2[0] = sgn * (u0[1] * u1[2] - u0[2] * u1[1]);
  u2[1] = sgn * (u0[2] * u1[0] - u0[0] * u1[2]);
  u2[2] = sgn * (u0[0] * u1[1] - u0[1] * u1[0]);
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) R[3 * i + j] = u0[i] * v0[j] + u1[i] * v1[j] + u2[i] * v2[j];
}

// Symmetric 3x3 tensors are stored as (00, 11, 22, 01, 12, 02); 4th-order
// tangents as a full 6x6 row-major Voigt matrix in (xx, yy, zz, xy, yz, xz)
// order, the layout of the reference's Matrix6d.

template <typename T>
__device__ __forceinline__ void left_cauchy_green(T* B6, const T* F) {
  B6[0] = F[0] * F[0] + F[1] * F[1] + F[2] * F[2];
  B6[1] = F[3] * F[3] + F[4] * F[4] + F[5] * F[5];
  B6[2] = F[6] * F[6] + F[7] * F[7] + F[8] * F[8];
  B6[3] = F[0] * F[3] + F[1] * F[4] + F[2] * F[5];
  B6[4] = F[3] * F[6] + F[4] * F[7] + F[5] * F[8];
  B6[5] = F[0] * F[6] + F[1] * F[7] + F[2] * F[8];
}

// NeoHookeanMaterial.computeStressAndTangent (NeoHookeanMaterial.java:113-139):
// sigma = (mu/J) B + ((lam ln J - mu)/J) I;
// D = (lam/J) I(x)I + (2 (mu - lam ln J)/J) II.  The tangent is isotropic, so
// only its two coefficients are returned: D = a I(x)I + 2 b II with
// a = lam/J, b = (mu - lam ln J)/J.
template <typename T>
__device__ __forceinline__ void neohookean_point(T* sig, T* a, T* b, T E, T nu, const T* F, T J) {
  T G = E / (T(2) * (T(1) + nu));
  T lam = (E * nu) / ((T(1) - T(2) * nu) * (T(1) + nu));
  T mu = G;
  T B6[6];
  left_cauchy_green(B6, F);
  T lnJ = log(J);
#pragma unroll
  for (int i = 0; i < 6; i++) sig[i] = (mu / J) * B6[i];
  T diag = (lam * lnJ - mu) / J;
  sig[0] += diag;
  sig[1] += diag;
  sig[2] += diag;
  *a = lam / J;
  *b = (mu - lam * lnJ) / J;
}

// upper-part tensor products of TensorUtils (TensorUtils.java:153-268,
// 340-380, 608-645); the caller mirrors the upper part afterwards.
template <typename T>
__device__ __forceinline__ void d_add_sym_product(T* D, T s, const T* A, const T* B) {
  T a00 = s * A[0], a11 = s * A[1], a22 = s * A[2], a01 = s * A[3], a12 = s * A[4], a02 = s * A[5];
  T b00 = B[0], b11 = B[1], b22 = B[2], b01 = B[3], b12 = B[4], b02 = B[5];
  D[0] += T(2) * a00 * b00; D[1] += a00 * b11 + b00 * a11; D[2] += a00 * b22 + b00 * a22;
  D[3] += a00 * b01 + b00 * a01; D[4] += a00 * b12 + b00 * a12; D[5] += a00 * b02 + b00 * a02;
  D[7] += T(2) * a11 * b11; D[8] += a11 * b22 + b11 * a22; D[9] += a11 * b01 + b11 * a01;
  D[10] += a11 * b12 + b11 * a12; D[11] += a11 * b02 + b11 * a02;
  D[14] += T(2) * a22 * b22; D[15] += a22 * b01 + b22 * a01; D[16] += a22 * b12 + b22 * a12;
  D[17] += a22 * b02 + b22 * a02;
  D[21] += T(2) * a01 * b01; D[22] += a01 * b12 + b01 * a12; D[23] += a01 * b02 + b01 * a02;
  D[28] += T(2) * a12 * b12; D[29] += a12 * b02 + b12 * a02;
  D[35] += T(2) * a02 * b02;
}
template <typename T>
__device__ __forceinline__ void d_add_product(T* D, T s, const T* A) {
  const int idx[21] = {0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11, 14, 15, 16, 17, 21, 22, 23, 28, 29, 35};
  const int ri[21] = {0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 2, 2, 2, 2, 3, 3, 3, 4, 4, 5};
  const int ci[21] = {0, 1, 2, 3, 4, 5, 1, 2, 3, 4, 5, 2, 3, 4, 5, 3, 4, 5, 4, 5, 5};
#pragma unroll
  for (int k = 0; k < 21; k++) D[idx[k]] += (s * A[ri[k]]) * A[ci[k]];
}
template <typename T>
__device__ __forceinline__ void d_add_product4(T* D, T s, const T* A) {
  T a00 = A[0], a11 = A[1], a22 = A[2], a01 = A[3], a12 = A[4], a02 = A[5];
  T s00 = s * a00, s11 = s * a11, s22 = s * a22, s01 = s * a01, s02 = s * a02, s12 = s * a12;
  D[0] += s00 * a00; D[1] += s01 * a01; D[2] += s02 * a02; D[3] += s00 * a01;
  D[4] += s01 * a02; D[5] += s00 * a02;
  D[7] += s11 * a11; D[8] += s12 * a12; D[9] += s01 * a11; D[10] += s11 * a12; D[11] += s01 * a12;
  D[14] += s22 * a22; D[15] += s02 * a12; D[16] += s12 * a22; D[17] += s02 * a22;
  D[21] += (s00 * a11 + s01 * a01) * T(0.5); D[22] += (s01 * a12 + s02 * a11) * T(0.5);
  D[23] += (s00 * a12 + s02 * a01) * T(0.5);
  D[28] += (s11 * a22 + s12 * a12) * T(0.5); D[29] += (s01 * a22 + s02 * a12) * T(0.5);
  D[35] += (s00 * a22 + s02 * a02) * T(0.5);
}

// TensorUtils.addSymmetricTensorProduct4 (TensorUtils.java:674-716): upper
// part; the caller mirrors it afterwards.
template <typename T>
__device__ __forceinline__ void d_add_sym_product4(T* D, T s, const T* A, const T* B) {
  T a00 = s * A[0], a11 = s * A[1], a22 = s * A[2], a01 = s * A[3], a12 = s * A[4], a02 = s * A[5];
  T b00 = B[0], b11 = B[1], b22 = B[2], b01 = B[3], b12 = B[4], b02 = B[5];
  D[0] += T(2) * a00 * b00; D[1] += T(2) * a01 * b01; D[2] += T(2) * a02 * b02;
  D[3] += a01 * b00 + a00 * b01; D[4] += a02 * b01 + a01 * b02; D[5] += a02 * b00 + a00 * b02;
  D[7] += T(2) * a11 * b11; D[8] += T(2) * a12 * b12;
  D[9] += a11 * b01 + a01 * b11; D[10] += a12 * b11 + a11 * b12; D[11] += a12 * b01 + a01 * b12;
  D[14] += T(2) * a22 * b22;
  D[15] += a12 * b02 + a02 * b12; D[16] += a22 * b12 + a12 * b22; D[17] += a22 * b02 + a02 * b22;
  D[21] += T(0.5) * (a11 * b00 + T(2) * a01 * b01 + a00 * b11);
  D[22] += T(0.5) * (a12 * b01 + a11 * b02 + a02 * b11 + a01 * b12);
  D[23] += T(0.5) * (a12 * b00 + a02 * b01 + a01 * b02 + a00 * b12);
  D[28] += T(0.5) * (a22 * b11 + T(2) * a12 * b12 + a11 * b22);
  D[29] += T(0.5) * (a22 * b01 + a12 * b02 + a02 * b12 + a01 * b22);
  D[35] += T(0.5) * (a22 * b00 + T(2) * a02 * b02 + a00 * b22);
}

// StVenantKirchoffMaterial.computeStressAndTangent
// (StVenantKirchoffMaterial.java:136-164), the FEBio form:
// sigma = ((lam tr E - mu)/J) B + (mu/J) B^2 with tr E = (tr B - 3)/2;
// D = (lam/J) B(x)B + (mu/J) symmetric4(B, B).  D may be null.
template <typename T>
__device__ inline void stvk_point(T* sig, T* D, T E, T nu, const T* F, T J) {
  const T mu = E / (T(2) * (T(1) + nu));
  const T lam = (E * nu) / ((T(1) - T(2) * nu) * (T(1) + nu));
  T B[6], B2[6];
  left_cauchy_green(B, F);
  const T tr = T(0.5) * (B[0] + B[1] + B[2] - T(3));
  B2[0] = B[0] * B[0] + B[3] * B[3] + B[5] * B[5];
  B2[1] = B[3] * B[3] + B[1] * B[1] + B[4] * B[4];
  B2[2] = B[5] * B[5] + B[4] * B[4] + B[2] * B[2];
  B2[3] = B[0] * B[3] + B[3] * B[1] + B[5] * B[4];
  B2[4] = B[3] * B[5] + B[1] * B[4] + B[4] * B[2];
  B2[5] = B[0] * B[5] + B[3] * B[4] + B[5] * B[2];
  const T cb = (lam * tr - mu) / J, cb2 = mu / J;
#pragma unroll
  for (int i = 0; i < 6; i++) sig[i] = cb * B[i] + cb2 * B2[i];
  if (D) {
#pragma unroll
    for (int i = 0; i < 36; i++) D[i] = T(0);
    d_add_product(D, lam / J, B);
    d_add_sym_product4(D, mu / J, B, B);
#pragma unroll
    for (int i = 1; i < 6; i++)
#pragma unroll
      for (int j = 0; j < i; j++) D[6 * i + j] = D[6 * j + i];
  }
}

// MooneyRivlinMaterial.computeDevStressAndTangent (MooneyRivlinMaterial.java:344-431)
// plus the pressure terms of IncompressibleMaterialBase.computeStressAndTangent
// (IncompressibleMaterialBase.java:249-260).  mp = {c10, c01, c11, c20, c02,
// kappa, jlimit, potential}.  D receives the full symmetric 6x6 tangent.
template <typename T>
__device__ inline void mooneyrivlin_point(T* sig, T* D, const T* mp, const T* F, T J, T p) {
  const T jl = mp[6];
  T phi, dphi, ddphi;
  if (jl > T(0) && J < jl) {
    // MooneyRivlinMaterial.computePhiVals, J below JLimit (:314-325)
    T phi0 = T(1) / pow(jl, T(2.0 / 3.0));
    T dphi0 = -(T(2.0 / 3.0)) * phi0 / jl;
    T ddphi0 = -(T(5.0 / 3.0)) * dphi0 / jl;
    T delJ = J - jl;
    phi = (T(0.5) * ddphi0 * delJ + dphi0) * delJ + phi0;
    dphi = ddphi0 * delJ + dphi0;
    ddphi = ddphi0;
  } else {
    phi = T(1) / pow(J, T(2.0 / 3.0));
    dphi = -(T(2.0 / 3.0)) * phi / J;
    ddphi = -(T(5.0 / 3.0)) * dphi / J;
  }
  T B[6], B2[6];
  left_cauchy_green(B, F);
#pragma unroll
  for (int i = 0; i < 6; i++) B[i] *= phi;
  // B2 = B B for symmetric B
  B2[0] = B[0] * B[0] + B[3] * B[3] + B[5] * B[5];
  B2[1] = B[3] * B[3] + B[1] * B[1] + B[4] * B[4];
  B2[2] = B[5] * B[5] + B[4] * B[4] + B[2] * B[2];
  B2[3] = B[0] * B[3] + B[3] * B[1] + B[5] * B[4];
  B2[4] = B[3] * B[5] + B[1] * B[4] + B[4] * B[2];
  B2[5] = B[0] * B[5] + B[3] * B[4] + B[5] * B[2];
  const T c10 = mp[0], c01 = mp[1], c11 = mp[2], c20 = mp[3], c02 = mp[4];
  T I1 = B[0] + B[1] + B[2];
  T I2 = T(0.5) * (I1 * I1 - (B2[0] + B2[1] + B2[2]));
  T W1 = c10 + c11 * (I2 - T(3)) + c20 * T(2) * (I1 - T(3));
  T W2 = c01 + c11 * (I1 - T(3)) + c02 * T(2) * (I2 - T(3));
#pragma unroll
  for (int i = 0; i < 6; i++) sig[i] = (W1 + W2 * I1) * B[i] - W2 * B2[i];
  T dev = (dphi / phi) * (sig[0] + sig[1] + sig[2]);
#pragma unroll
  for (int i = 0; i < 6; i++) sig[i] *= T(2) / J;
  sig[0] += dev;
  sig[1] += dev;
  sig[2] += dev;
  if (D) {
    T Ji = T(1) / J;
    T W11 = T(2) * c20, W12 = c11, W22 = T(2) * c02;
    T w1 = -W2;
    T w2 = W11 + T(2) * W12 * I1 + W2 + W22 * I2 * I2;
    T w3 = W12 + W22 * I1;
    T w4 = W22;
    T wc1 = (w2 - W12 + W22 * I1) * I1;
    T wc2 = -(W12 + W22 * I1 - W22 * I1 * I1 + T(2) * W22 * I2 + W2);
    T wcc = wc1 * I1 + wc2 * (I1 * I1 - T(2) * I2);
    T w0 = W1 * I1 + T(2) * W2 * I2;
#pragma unroll
    for (int i = 0; i < 36; i++) D[i] = T(0);
    T zeta = ((dphi + J * ddphi) * w0 + J * dphi * dphi / phi * (wcc - T(2) * w0)) / phi;
    T r = dphi / phi;
    // addScaledIdentityProduct(zeta), addScaledIdentity(-2 r w0)
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) D[6 * i + j] += zeta;
    T s = T(-2) * r * w0;
    D[0] += s; D[7] += s; D[14] += s;
    D[21] += T(0.5) * s; D[28] += T(0.5) * s; D[35] += T(0.5) * s;
    const T I6[6] = {1, 1, 1, 0, 0, 0};
    d_add_sym_product(D, J * r, sig, I6);
    d_add_product4(D, w1 * T(4) * Ji, B);
    d_add_product(D, w2 * T(4) * Ji, B);
    d_add_sym_product(D, w3 * T(4) * Ji, B, B2);
    d_add_product(D, w4 * T(4) * Ji, B2);
    T Tm[6];
#pragma unroll
    for (int i = 0; i < 6; i++) Tm[i] = wc1 * B[i] + wc2 * B2[i];
    d_add_sym_product(D, T(2) * r, Tm, I6);
    // setLowerToUpper (Matrix6d.java:532-538)
#pragma unroll
    for (int i = 1; i < 6; i++)
#pragma unroll
      for (int j = 0; j < i; j++) D[6 * i + j] = D[6 * j + i];
    // addPressureTangent (IncompressibleMaterialBase.java:218-224)
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
      for (int j = 0; j < 3; j++) D[6 * i + j] += p;
    T s2 = T(-2) * p;
    D[0] += s2; D[7] += s2; D[14] += s2;
    D[21] += T(0.5) * s2; D[28] += T(0.5) * s2; D[35] += T(0.5) * s2;
  }
  sig[0] += p;
  sig[1] += p;
  sig[2] += p;
}

// K += B_i^T D B_j dv for a full 6x6 D (FemUtilities.addMaterialStiffness,
// FemUtilities.java:78-129); gi, gj already scaled as needed.
template <typename T>
__device__ __forceinline__ void add_bdb(T* K, const T* gi, const T* D, const T* gj, T dv) {
  T x = gj[0] * dv, y = gj[1] * dv, z = gj[2] * dv;
  T t[6][3];
#pragma unroll
  for (int r = 0; r < 6; r++) {
    const T* d = D + 6 * r;
    t[r][0] = d[0] * x + d[3] * y + d[5] * z;
    t[r][1] = d[1] * y + d[3] * x + d[4] * z;
    t[r][2] = d[2] * z + d[4] * y + d[5] * x;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    K[c] += gi[0] * t[0][c] + gi[1] * t[3][c] + gi[2] * t[5][c];
    K[3 + c] += gi[1] * t[1][c] + gi[0] * t[3][c] + gi[2] * t[4][c];
    K[6 + c] += gi[2] * t[2][c] + gi[1] * t[4][c] + gi[0] * t[5][c];
  }
}

// K += B_i^T D B_j dv for the isotropic D = a I(x)I + 2 b II of NeoHookean:
// a gi gj^T + b (gi.gj I + gj gi^T)   (same value as add_bdb on that D)
template <typename T>
__device__ __forceinline__ void add_bdb_iso(T* K, const T* gi, T a, T b, const T* gj, T dv) {
  T ad = a * dv, bd = b * dv;
  T gg = (gi[0] * gj[0] + gi[1] * gj[1] + gi[2] * gj[2]) * bd;
#pragma unroll
  for (int r = 0; r < 3; r++)
#pragma unroll
    for (int c = 0; c < 3; c++) K[3 * r + c] += ad * gi[r] * gj[c] + bd * gj[r] * gi[c];
  K[0] += gg;
  K[4] += gg;
  K[8] += gg;
}

// (gi^T sigma gj) dv on the diagonal (FemUtilities.addGeometricStiffness,
// FemUtilities.java:131-144)
template <typename T>
__device__ __forceinline__ void add_geometric(T* K, const T* gi, const T* s, const T* gj, T dv) {
  T kg = gi[0] * (s[0] * gj[0] + s[3] * gj[1] + s[5] * gj[2]) +
         gi[1] * (s[3] * gj[0] + s[1] * gj[1] + s[4] * gj[2]) +
         gi[2] * (s[5] * gj[0] + s[4] * gj[1] + s[2] * gj[2]);
  kg *= dv;
  K[0] += kg;
  K[4] += kg;
  K[8] += kg;
}

// f += B^T sigma dv  (FemUtilities.addStressForce, FemUtilities.java:40-49)
template <typename T>
__device__ __forceinline__ void add_stress_force(T* f, const T* g, const T* s, T dv) {
  T gx = g[0] * dv, gy = g[1] * dv, gz = g[2] * dv;
  f[0] += gx * s[0] + gy * s[3] + gz * s[5];
  f[1] += gy * s[1] + gx * s[3] + gz * s[4];
  f[2] += gz * s[2] + gy * s[4] + gx * s[5];
}

// Stress and full tangent of the general-tangent materials (MooneyRivlin
// with its pressure p, StVenantKirchhoff) at one point; mp holds the model's
// material parameters.
template <int MAT, typename T>
__device__ __forceinline__ void material_point(T* sig, T* D, const T* mp, const T* F, T J, T p) {
  if constexpr (MAT == B200FEM_MAT_STVK) stvk_point<T>(sig, D, mp[0], mp[1], F, J);
  else mooneyrivlin_point<T>(sig, D, mp, F, J, p);
}

}  // namespace b200fem
