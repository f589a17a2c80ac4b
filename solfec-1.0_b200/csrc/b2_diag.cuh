// b2_diag.cuh -- per-contact Signorini-Coulomb diagonal solvers in FP64.
//
// Device forms of the reference's CONTACT + SIGNORINI_COULOMB diagonal block
// solvers (dbs.c:35-326) and of the smoothed contact formulation they use
// (scf.c:28-174). One thread solves one contact; every function works on
// register arrays. The 3x3 linear solve is LU with partial pivoting in the
// LAPACK dgetf2/dgetrs arithmetic (pivot = first largest |a(i,j)|, column
// scaled by the pivot reciprocal, unit-lower forward and upper back solves).
#pragma once

#include <cmath>
#include "b2_common.cuh"

namespace b2 {

// Parameters of one contact row, gathered once per solve.
struct ContactParams {
  double friction, restitution, cohesion, gap, step;
  int dynamic;
};

// LU factorisation with partial pivoting of a 3x3 A (column-major, in place)
// in the arithmetic of LAPACK dgetf2. Returns 0, or k > 0 when U(k,k) is
// exactly zero.
__device__ __forceinline__ int lu3_factor(double* a, int* ipiv) {
  int info = 0;
#pragma unroll
  for (int j = 0; j < 3; j++) {
    int p = j;
    double apiv = a[j + 3 * j];  // a[p + 3 j], tracked so that no index is a runtime value
    double amax = fabs(apiv);
#pragma unroll
    for (int i = j + 1; i < 3; i++) {
      double v = fabs(a[i + 3 * j]);
      if (v > amax) { amax = v; p = i; apiv = a[i + 3 * j]; }
    }
    ipiv[j] = p;
    if (apiv != 0.0) {
      if (p != j) {
#pragma unroll
        for (int c = 0; c < 3; c++) {
          // p is a runtime index; select-based swap keeps the array in registers
          double tj = a[j + 3 * c];
          double tp = (p == 1) ? a[1 + 3 * c] : a[2 + 3 * c];
          a[j + 3 * c] = tp;
          if (p == 1) a[1 + 3 * c] = tj; else a[2 + 3 * c] = tj;
        }
      }
      double piv = a[j + 3 * j];
      if (fabs(piv) >= 2.2250738585072014e-308) {
        double r = 1.0 / piv;
#pragma unroll
        for (int i = j + 1; i < 3; i++) a[i + 3 * j] *= r;
      } else {
#pragma unroll
        for (int i = j + 1; i < 3; i++) a[i + 3 * j] /= piv;
      }
    } else if (info == 0) {
      info = j + 1;
    }
#pragma unroll
    for (int c = j + 1; c < 3; c++) {
      double u = a[j + 3 * c];
      if (u != 0.0) {
        double t = -u;
#pragma unroll
        for (int i = j + 1; i < 3; i++) a[i + 3 * c] += a[i + 3 * j] * t;
      }
    }
  }
  return info;
}

// x = A^-1 b from lu3_factor's factors (dgetrs, one right-hand side, in place).
__device__ __forceinline__ void lu3_apply(const double* a, const int* ipiv, double* b) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    int p = ipiv[i];
    if (p != i) {
      double t = b[i];
      double bp = (p == 1) ? b[1] : b[2];
      b[i] = bp;
      if (p == 1) b[1] = t; else b[2] = t;
    }
  }
#pragma unroll
  for (int k = 0; k < 3; k++) {
    if (b[k] != 0.0) {
#pragma unroll
      for (int i = k + 1; i < 3; i++) b[i] -= b[k] * a[i + 3 * k];
    }
  }
#pragma unroll
  for (int k = 2; k >= 0; k--) {
    if (b[k] != 0.0) {
      b[k] /= a[k + 3 * k];
#pragma unroll
      for (int i = 0; i < k; i++) b[i] -= b[k] * a[i + 3 * k];
    }
  }
}

// Solve A x = b (3x3, column-major, one right-hand side). Returns 0, or k > 0
// when U(k,k) is exactly zero (b untouched), as LAPACK dgesv reports.
__device__ __forceinline__ int lu3_solve(double* a, double* b) {
  int ipiv[3];
  const int info = lu3_factor(a, ipiv);
  if (info) return info;
  lu3_apply(a, ipiv, b);
  return 0;
}

// A x = b for a 3x3 A (column-major) by the adjugate and one reciprocal of
// the determinant (Cramer's rule): a shorter dependent chain than the pivoted
// LU, for the FP32 sweeps' Newton steps only (not the reference's
// arithmetic). Returns 0, or 1 for a zero or non-finite determinant.
__device__ __forceinline__ int cramer3_solve(const double* a, double* b) {
  const double c00 = a[4] * a[8] - a[7] * a[5], c01 = a[7] * a[2] - a[1] * a[8], c02 = a[1] * a[5] - a[4] * a[2];
  const double det = a[0] * c00 + a[3] * c01 + a[6] * c02;
  if (det == 0.0 || !isfinite(det)) return 1;
  const double c10 = a[6] * a[5] - a[3] * a[8], c11 = a[0] * a[8] - a[6] * a[2], c12 = a[3] * a[2] - a[0] * a[5];
  const double c20 = a[3] * a[7] - a[6] * a[4], c21 = a[6] * a[1] - a[0] * a[7], c22 = a[0] * a[4] - a[3] * a[1];
  const double r = 1.0 / det;
  const double x0 = (c00 * b[0] + c10 * b[1] + c20 * b[2]) * r;
  const double x1 = (c01 * b[0] + c11 * b[1] + c21 * b[2]) * r;
  const double x2 = (c02 * b[0] + c12 * b[1] + c22 * b[2]) * r;
  b[0] = x0; b[1] = x1; b[2] = x2;
  return 0;
}

// dashed normal velocity (dbs.c:52-53; scf.c:43-44)
__device__ __forceinline__ double dashed_un(const ContactParams& cp, const double* U, const double* V) {
  if (cp.dynamic) return U[2] + cp.restitution * B2_MIN(V[2], 0);
  return (B2_MAX(cp.gap, 0) / cp.step) + U[2];
}

// SCF_Project (scf.c:136-174); S is read-only here (the reference adds and
// removes the cohesion in place, which leaves it unchanged up to rounding of
// (S2 + c) - c; that rounding is reproduced).
__device__ __forceinline__ void scf_project(double fri, double coh, double* S, double* R) {
  S[2] += coh;
  double fri2 = fri * fri;
  double slen = sqrt(S[0] * S[0] + S[1] * S[1]);
  double l1 = -(S[2] + fri * slen) / (1.0 + fri2);
  double l2 = (slen - fri * S[2]) / (1.0 + fri2);
  double u1[3], u2[3];
  if (slen != 0.0) {
    u2[0] = S[0] / slen; u2[1] = S[1] / slen; u2[2] = -fri;
    u1[0] = -fri * u2[0]; u1[1] = -fri * u2[1]; u1[2] = -1.0;
  } else {
    u2[0] = 1.0; u2[1] = 0.0; u2[2] = -fri;
    u1[0] = -fri; u1[1] = 0.0; u1[2] = -1.0;
  }
  double g1 = B2_MAX(l1, 0.0), g2 = B2_MAX(l2, 0.0);
  double m0 = g1 * u1[0] + g2 * u2[0];
  double m1 = g1 * u1[1] + g2 * u2[1];
  double m2 = g1 * u1[2] + g2 * u2[2];
  S[2] -= coh;
  R[0] = S[0] - m0; R[1] = S[1] - m1; R[2] = S[2] - m2;
}

// SCF_Linearize (scf.c:28-133) with UT = -1 and zero smoothing, the values
// every caller on the path passes. X, Y (Jacobians) only when WITHXY. FAST
// (the merit terms of the FP32 sweeps of mixed precision, which are not
// bitwise the reference's anyway): one reciprocal per shared divisor and
// |l| for sqrt(l l).
template <bool WITHXY, bool FAST = false>
__device__ __forceinline__ void scf_linearize(const ContactParams& cp, const double* V, const double* U,
                                              const double* R, double* C, double* X, double* Y) {
  const double fri = cp.friction;
  double fri2 = fri * fri, onefri2 = 1.0 + fri2;
  double udash = dashed_un(cp, U, V);
  double ulen = sqrt(U[0] * U[0] + U[1] * U[1]);
  double F0 = U[0], F1 = U[1], F2 = udash + fri * ulen;
  double S[3] = {R[0] - F0, R[1] - F1, R[2] - F2};
  S[2] += cp.cohesion;
  double sdot = S[0] * S[0] + S[1] * S[1];
  double slen = sqrt(sdot);
  double l1, l2;
  if constexpr (FAST) {
    const double r = 1.0 / onefri2;
    l1 = -(S[2] + fri * slen) * r;
    l2 = (slen - fri * S[2]) * r;
  } else {
    l1 = -(S[2] + fri * slen) / onefri2;
    l2 = (slen - fri * S[2]) / onefri2;
  }
  double u1[3], u2[3];
  if (slen != 0.0) {
    if constexpr (FAST) {
      const double r = 1.0 / slen;
      u2[0] = S[0] * r; u2[1] = S[1] * r;
    } else {
      u2[0] = S[0] / slen; u2[1] = S[1] / slen;
    }
    u2[2] = -fri;
    u1[0] = -fri * u2[0]; u1[1] = -fri * u2[1]; u1[2] = -1.0;
  } else {
    u2[0] = 1.0; u2[1] = 0.0; u2[2] = -fri;
    u1[0] = -fri; u1[1] = 0.0; u1[2] = -1.0;
  }
  double sq1 = FAST ? fabs(l1) : sqrt(l1 * l1), sq2 = FAST ? fabs(l2) : sqrt(l2 * l2);
  double g1 = 0.5 * (sq1 + l1), g2 = 0.5 * (sq2 + l2);
  C[0] = F0 + (g1 * u1[0] + g2 * u2[0]);
  C[1] = F1 + (g1 * u1[1] + g2 * u2[1]);
  C[2] = F2 + (g1 * u1[2] + g2 * u2[2]);
  if constexpr (WITHXY) {
    double dF[9] = {1.0, 0.0, fri * U[0] / ulen, 0.0, 1.0, fri * U[1] / ulen, 0.0, 0.0, 1.0};
    double dg1 = 0.5 * (1.0 + l1 / sq1);
    if (slen != 0.0) {
      double dg2 = 0.5 * (1.0 + l2 / sq2);
      double a = 0.5 * (1.0 + (l2 + fri * l1) / (sq2 + fri * sq1));
      double b = (fri2 * dg1 + dg2) / onefri2;
      double c = (fri * (dg1 - dg2)) / onefri2;
      double d = (dg1 + fri2 * dg2) / onefri2;
      Y[0] = a + (b - a) * S[0] * S[0] / sdot;
      Y[1] = (b - a) * S[1] * S[0] / sdot;
      Y[2] = c * S[0] / slen;
      Y[3] = Y[1];
      Y[4] = a + (b - a) * S[1] * S[1] / sdot;
      Y[5] = c * S[1] / slen;
      Y[6] = Y[2];
      Y[7] = Y[5];
      Y[8] = d;
    } else {
      Y[1] = Y[2] = Y[3] = Y[5] = Y[6] = Y[7] = 0.0;
      Y[0] = Y[4] = Y[8] = dg1;
    }
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++)
        X[3 * j + i] = dF[3 * j + i] - (Y[i] * dF[3 * j] + Y[3 + i] * dF[3 * j + 1] + Y[6 + i] * dF[3 * j + 2]);
  }
}

// projected_gradient (dbs.c:35-94)
static __device__ __noinline__ int projected_gradient(const ContactParams& cp, double epsilon, int maxiter, double rho,
                                               const double* W, const double* B, const double* V, double* U,
                                               double* R) {
  if (cp.dynamic && cp.gap > 0) {
    R[0] = R[1] = R[2] = 0.0;
    U[0] = B[0]; U[1] = B[1]; U[2] = B[2];
    return 0;
  }
  int iter = 0;
  double scalar;
  do {
    double v0 = R[0], v1 = R[1], v2 = R[2];
    nvaddmul(B, W, R, U);
    double UN = dashed_un(cp, U, V);
    R[0] -= rho * U[0];
    R[1] -= rho * U[1];
    R[2] -= rho * UN - cp.cohesion;
    R[2] = B2_MAX(0, R[2]);
    scalar = sqrt(R[0] * R[0] + R[1] * R[1]);
    if (scalar >= cp.friction * R[2]) {
      if (scalar > 0.0) scalar = cp.friction * R[2] / scalar;
      R[0] *= scalar;
      R[1] *= scalar;
    }
    R[2] -= cp.cohesion;
    double d[3] = {R[0] - v0, R[1] - v1, R[2] - v2};
    scalar = dot3(R, R);
    scalar = sqrt(dot3(d, d) / B2_MAX(scalar, 1.0));
  } while (++iter < maxiter && scalar > epsilon);
  return iter;
}

// de_saxce_feng (dbs.c:96-140)
static __device__ __noinline__ int de_saxce_feng(const ContactParams& cp, double epsilon, int maxiter, double rho,
                                          const double* W, const double* B, const double* V, double* U, double* R) {
  if (cp.dynamic && cp.gap > 0) {
    R[0] = R[1] = R[2] = 0.0;
    U[0] = B[0]; U[1] = B[1]; U[2] = B[2];
    return 0;
  }
  int iter = 0;
  double scalar;
  do {
    double v0 = R[0], v1 = R[1], v2 = R[2];
    nvaddmul(B, W, R, U);
    double UN = dashed_un(cp, U, V);
    double tau[3];
    tau[0] = R[0] - rho * U[0];
    tau[1] = R[1] - rho * U[1];
    tau[2] = R[2] - rho * (UN + cp.friction * sqrt(U[0] * U[0] + U[1] * U[1]));
    scf_project(cp.friction, cp.cohesion, tau, R);
    double d[3] = {R[0] - v0, R[1] - v1, R[2] - v2};
    scalar = dot3(R, R);
    scalar = sqrt(dot3(d, d) / B2_MAX(scalar, 1.0));
  } while (++iter < maxiter && scalar > epsilon);
  return iter;
}

// semismooth_newton (dbs.c:142-303): the default diagonal solver. RECIP (the
// FP32 sweeps of mixed precision only, which are not bitwise the reference's
// anyway) shortens the solve's dependent chain of divisions: one reciprocal
// where the reference divides several values by the same divisor (the slip
// branch's norm and den, the stick branch's d2), the slip branch's alfa delta
// as (R.d)/den (the same quantity), the Newton step by Cramer's rule instead
// of the pivoted LU, and the error test squared; the results then differ from
// the reference's in the last bits.
template <bool RECIP = false>
__device__ __forceinline__ int semismooth_newton(const ContactParams& cp, double epsilon, int maxiter, double rho,
                                                 const double* W, const double* B, const double* V, double* U,
                                                 double* R) {
  if (cp.dynamic && cp.gap > 0) {
    R[0] = R[1] = R[2] = 0.0;
    U[0] = B[0]; U[1] = B[1]; U[2] = B[2];
    return 0;
  }
  const double friction = cp.friction, cohesion = cp.cohesion;
  const int divi = maxiter / 10;
  int until = divi;  // iterations left until rho grows (iter % divi == 0 without an integer division)
  int iter = 0;
  double error;
  do {
    double R00 = R[0], R01 = R[1], R02 = R[2];
    double UN = dashed_un(cp, U, V);
    double d0 = R[0] - rho * U[0];
    double d1 = R[1] - rho * U[1];
    double d2 = (R[2] + cohesion) - rho * UN;
    double RES[3];
    nvaddmul(B, W, R, RES);
    RES[0] -= U[0]; RES[1] -= U[1]; RES[2] -= U[2];
    double a[9], b[3];
    if (d2 >= 0) {
      double norm = sqrt(d0 * d0 + d1 * d1);
      double lim = friction * B2_MAX(0, d2);
      if (norm >= lim) {  // slip
        if (lim > 0.0) {
          double len = sqrt(R[0] * R[0] + R[1] * R[1]);
          double den = B2_MAX(lim, len) * norm;
          double rnorm = 0.0, rden = 0.0;
          if constexpr (RECIP) { rnorm = 1.0 / norm; rden = 1.0 / den; }
          double e = RECIP ? lim * rnorm : lim / norm;
          double beta;
          if constexpr (RECIP) {
            // alfa delta = (R.d) / (len norm) min(len / lim, 1) = (R.d) / (max(lim, len) norm) = (R.d) / den,
            // and alfa has the sign of R.d (0 when len = 0, where beta = 1)
            const double rd = R[0] * d0 + R[1] * d1;
            beta = (len != 0.0 && rd < 0.0) ? 1.0 / (1.0 - rd * rden) : 1.0;
          } else if (len == 0.0) {
            beta = 1.0;
          } else {
            double alfa = (R[0] * d0 + R[1] * d1) / (len * norm);
            double delta = B2_MIN(len / lim, 1.0);
            beta = (alfa < 0.0 ? 1.0 / (1.0 - alfa * delta) : 1.0);
          }
          double F0, F1, F2, F3;
          if constexpr (RECIP) {
            F0 = (R[0] * d0) * rden; F1 = (R[1] * d0) * rden; F2 = (R[0] * d1) * rden; F3 = (R[1] * d1) * rden;
          } else {
            F0 = (R[0] * d0) / den; F1 = (R[1] * d0) / den; F2 = (R[0] * d1) / den; F3 = (R[1] * d1) / den;
          }
          const double n0 = RECIP ? d0 * rnorm : d0 / norm, n1 = RECIP ? d1 * rnorm : d1 / norm;
          double M0 = e * (1.0 - F0), M1 = -e * F1, M2 = -e * F2, M3 = e * (1.0 - F3);
          double H0 = 1.0 - beta * M0, H1 = -beta * M1, H2 = -beta * M2, H3 = 1.0 - beta * M3;
          a[0] = H0 + rho * (M0 * W[0] + M2 * W[1]);
          a[1] = H1 + rho * (M1 * W[0] + M3 * W[1]);
          a[2] = W[2];
          a[3] = H2 + rho * (M0 * W[3] + M2 * W[4]);
          a[4] = H3 + rho * (M1 * W[3] + M3 * W[4]);
          a[5] = W[5];
          a[6] = rho * (M0 * W[6] + M2 * W[7]) - friction * n0;
          a[7] = rho * (M1 * W[6] + M3 * W[7]) - friction * n1;
          a[8] = W[8];
          b[0] = friction * n0 * (R[2] + cohesion) - R[0] - rho * (M0 * RES[0] + M2 * RES[1]);
          b[1] = friction * n1 * (R[2] + cohesion) - R[1] - rho * (M1 * RES[0] + M3 * RES[1]);
          b[2] = -UN - RES[2];
        } else {  // degenerate: homogeneous tangential tractions
          a[0] = 1.0; a[1] = 0.0; a[2] = W[2];
          a[3] = 0.0; a[4] = 1.0; a[5] = W[5];
          a[6] = 0.0; a[7] = 0.0; a[8] = W[8];
          b[0] = -R[0] - RES[0];
          b[1] = -R[1] - RES[1];
          b[2] = -UN - RES[2];
        }
      } else {  // stick
        a[0] = W[0]; a[1] = W[1]; a[2] = W[2];
        a[3] = W[3]; a[4] = W[4]; a[5] = W[5];
        a[8] = W[8];
        if constexpr (RECIP) {
          const double rd2 = 1.0 / d2;
          a[6] = W[6] + U[0] * rd2;
          a[7] = W[7] + U[1] * rd2;
          const double f = 1.0 + (rho * U[2]) * rd2;
          b[0] = -f * U[0] - RES[0];
          b[1] = -f * U[1] - RES[1];
        } else {
          a[6] = W[6] + U[0] / d2;
          a[7] = W[7] + U[1] / d2;
          b[0] = -(1.0 + rho * U[2] / d2) * U[0] - RES[0];
          b[1] = -(1.0 + rho * U[2] / d2) * U[1] - RES[1];
        }
        b[2] = -UN - RES[2];
      }
    } else {  // separation
      a[0] = 1.0; a[1] = 0.0; a[2] = 0.0;
      a[3] = 0.0; a[4] = 1.0; a[5] = 0.0;
      a[6] = 0.0; a[7] = 0.0; a[8] = 1.0;
      b[0] = -R[0]; b[1] = -R[1]; b[2] = -R[2];
    }
    if (RECIP ? cramer3_solve(a, b) : lu3_solve(a, b)) return -1;
    if (!isfinite(b[0] + b[1] + b[2])) return -1;
    double c[3];
    nvaddmul(RES, W, b, c);
    R[0] += b[0]; R[1] += b[1]; R[2] += b[2];
    U[0] += c[0]; U[1] += c[1]; U[2] += c[2];
    double e0 = R[0] - R00, e1 = R[1] - R01, e2 = R[2] - R02;
    error = dot3(R, R);
    if (RECIP && epsilon * epsilon > 0.0) {  // error > epsilon compared squared: no division or root
      const double d = e0 * e0 + e1 * e1 + e2 * e2, q = epsilon * epsilon * B2_MAX(error, 1.0);
      error = d > q ? 2.0 * epsilon : 0.0;
    } else {
      error = sqrt((e0 * e0 + e1 * e1 + e2 * e2) / B2_MAX(error, 1.0));
    }
    iter++;
    if (--until == 0) {
      until = divi;
      rho *= 10.0;
      if (isinf(rho)) return -1;
    }
  } while (iter < maxiter && error > epsilon);
  return iter;
}

// projected_newton (dbs.c:305-326)
static __device__ __noinline__ int projected_newton(const ContactParams& cp, double epsilon, int maxiter, const double* W,
                                             const double* B, const double* V, double* U, double* R) {
  double T[9], X[9], Y[9], Cv[3];
  int iter = 0;
  double merit;
  nvaddmul(B, W, R, U);
  scf_linearize<true>(cp, V, U, R, Cv, X, Y);
  do {
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
      for (int i = 0; i < 3; i++)
        T[3 * j + i] = (X[i] * W[3 * j] + X[3 + i] * W[3 * j + 1] + X[6 + i] * W[3 * j + 2]) + Y[3 * j + i];
    if (lu3_solve(T, Cv)) return -1;
    R[0] -= Cv[0]; R[1] -= Cv[1]; R[2] -= Cv[2];
    scf_project(cp.friction, cp.cohesion, R, R);
    nvaddmul(B, W, R, U);
    scf_linearize<true>(cp, V, U, R, Cv, X, Y);
    merit = sqrt(dot3(Cv, Cv));
  } while (merit > epsilon && ++iter < maxiter);
  return iter;
}

__device__ __forceinline__ int diagonal_solve(int solver, const ContactParams& cp, double epsilon, int maxiter,
                                              double rho, const double* W, const double* B, const double* V,
                                              double* U, double* R) {
  switch (solver) {  // dbs.c:507-521
    case DS_PROJECTED_GRADIENT: return projected_gradient(cp, epsilon, maxiter, rho, W, B, V, U, R);
    case DS_DE_SAXCE_FENG: return de_saxce_feng(cp, epsilon, maxiter, rho, W, B, V, U, R);
    case DS_SEMISMOOTH_NEWTON: return semismooth_newton(cp, epsilon, maxiter, rho, W, B, V, U, R);
    case DS_PROJECTED_NEWTON: return projected_newton(cp, epsilon, maxiter, W, B, V, U, R);
  }
  return 0;
}

// State of one row handed to the out-of-line path (rare: a failed first
// attempt or a solver other than SSN). Only this copy has its address taken,
// so the common path keeps the row's parameters and arrays in registers.
struct RowState {
  ContactParams cp;
  double W[9], B[3], V[3], U[3], R[3], R0[3];
};

// Everything after a failed SSN attempt (it = its return value), or the whole
// solve for the other solvers (bgs.c:969-1013). FAILURE_CONTINUE runs the
// fallback chain (bgs.c:976-1003): the other solvers in the order SSN, PG, DSF,
// PN, each from the previous reaction R0; if all fail the previous reaction is
// kept (U keeps the last attempt's value). Returns the failure kind of the
// first attempt: 0 none, 1 diverged (iterations >= maxiter), 2 failed (< 0).
static __device__ __noinline__ int diagonal_solve_row_slow(int solver, int failure, double epsilon, int maxiter, double rho,
                                                    int it, RowState& st) {
  if (solver != DS_SEMISMOOTH_NEWTON) {
    it = diagonal_solve(solver, st.cp, epsilon, maxiter, rho, st.W, st.B, st.V, st.U, st.R);
    if (it < maxiter && it >= 0) return 0;
  }
  const int kind = it < 0 ? 2 : 1;
  if (failure == FAIL_CONTINUE) {
    const int chain[4] = {DS_SEMISMOOTH_NEWTON, DS_PROJECTED_GRADIENT, DS_DE_SAXCE_FENG, DS_PROJECTED_NEWTON};
    it = maxiter;
    for (int t = 0; t < 4; t++) {
      if (chain[t] != solver) {
        st.R[0] = st.R0[0]; st.R[1] = st.R0[1]; st.R[2] = st.R0[2];
        it = diagonal_solve(chain[t], st.cp, epsilon, maxiter, rho, st.W, st.B, st.V, st.U, st.R);
        if (it < maxiter && it >= 0) break;
      }
    }
    if (it >= maxiter || it < 0) { st.R[0] = st.R0[0]; st.R[1] = st.R0[1]; st.R[2] = st.R0[2]; }
  }
  return kind;
}

// Diagonal solve of one row with the reference's failure handling
// (bgs.c:969-1013). Returns the failure kind of the first attempt: 0 none,
// 1 diverged (iterations >= maxiter), 2 failed (< 0).
template <bool RECIP = false>
__device__ __forceinline__ int diagonal_solve_row(int solver, int failure, const ContactParams& cp, double epsilon,
                                                  int maxiter, double rho, const double* W, const double* B,
                                                  const double* V, double* U, double* R) {
  const double r0 = R[0], r1 = R[1], r2 = R[2];
  int it = -1;
  if (solver == DS_SEMISMOOTH_NEWTON) {
    it = semismooth_newton<RECIP>(cp, epsilon, maxiter, rho, W, B, V, U, R);
    if (it < maxiter && it >= 0) return 0;
  }
  RowState st;
  st.cp = cp;
#pragma unroll
  for (int q = 0; q < 9; q++) st.W[q] = W[q];
#pragma unroll
  for (int q = 0; q < 3; q++) { st.B[q] = B[q]; st.V[q] = V[q]; st.U[q] = U[q]; st.R[q] = R[q]; }
  st.R0[0] = r0; st.R0[1] = r1; st.R0[2] = r2;
  const int kind = diagonal_solve_row_slow(solver, failure, epsilon, maxiter, rho, it, st);
#pragma unroll
  for (int q = 0; q < 3; q++) { U[q] = st.U[q]; R[q] = st.R[q]; }
  return kind;
}

// Merit numerator of one CONTACT row (mrf.c:81-87): C = SCF_Linearize(U, R),
// up = <A C, C>.
template <bool FAST = false>
__device__ __forceinline__ double merit_row(const ContactParams& cp, const double* A, const double* V,
                                            const double* U, const double* R) {
  double P[3];
  scf_linearize<false, FAST>(cp, V, U, R, P, nullptr, nullptr);
  double Q0 = A[0] * P[0] + A[3] * P[1] + A[6] * P[2];
  double Q1 = A[1] * P[0] + A[4] * P[1] + A[7] * P[2];
  double Q2 = A[2] * P[0] + A[5] * P[1] + A[8] * P[2];
  return Q0 * P[0] + Q1 * P[1] + Q2 * P[2];
}

// ---- bilateral constraints (dbs.c:328-450, mrf.c:88-137) ----
//
// Constraint kinds as dom.h:98 numbers them. A row of a kind other than
// CONTACT carries Z[4]: VELODIR the prescribed normal velocity Z[0]; VELODIR3
// the prescribed velocity Z[0..2]; RIGLNK the link vector in the row's local
// frame (base^T Z of riglnk, dbs.c:412) in Z[0..2] and the link length Z[3].
enum { CON_CONTACT = 0, CON_FIXPNT = 1, CON_FIXDIR = 2, CON_VELODIR = 3, CON_VELODIR3 = 4, CON_RIGLNK = 5 };

// A x = b for a symmetric positive definite 3x3 A (column-major, upper
// triangle read), Cholesky A = U^T U in the order of the 3x3 dposv the
// reference is linked with here (oracle/lu_small.c): 0, or j + 1 for a
// non-positive or NaN pivot
__device__ __forceinline__ int chol3_solve(double* a, double* b) {
#pragma unroll
  for (int j = 0; j < 3; j++) {
    double s = a[j + 3 * j];
    for (int k = 0; k < j; k++) s -= a[k + 3 * j] * a[k + 3 * j];
    if (s <= 0.0 || isnan(s)) return j + 1;
    s = sqrt(s);
    a[j + 3 * j] = s;
    for (int c = j + 1; c < 3; c++) {
      double t = a[j + 3 * c];
      for (int k = 0; k < j; k++) t -= a[k + 3 * j] * a[k + 3 * c];
      a[j + 3 * c] = t / s;
    }
  }
#pragma unroll
  for (int i = 0; i < 3; i++) {  // U^T y = b
    double t = b[i];
    for (int k = 0; k < i; k++) t -= a[k + 3 * i] * b[k];
    b[i] = t / a[i + 3 * i];
  }
#pragma unroll
  for (int i = 2; i >= 0; i--) {  // U x = y
    double t = b[i];
    for (int k = i + 1; k < 3; k++) t -= a[i + 3 * k] * b[k];
    b[i] = t / a[i + 3 * i];
  }
  return 0;
}

// A x = b for a 2x2 A (column-major) by LU with partial pivoting in the
// arithmetic of LAPACK dgetf2 / dgetrs; 0, or k > 0 for an exactly zero U(k,k)
__device__ __forceinline__ int lu2_solve(double* a, double* b) {
  int p = fabs(a[1]) > fabs(a[0]) ? 1 : 0;
  if (a[p] == 0.0) return 1;
  if (p) {
    double t = a[0]; a[0] = a[1]; a[1] = t;
    t = a[2]; a[2] = a[3]; a[3] = t;
  }
  const double piv = a[0];
  if (fabs(piv) >= 2.2250738585072014e-308) a[1] *= 1.0 / piv;
  else a[1] /= piv;
  const double u = a[2];
  if (u != 0.0) a[3] += a[1] * -u;
  if (a[3] == 0.0) return 2;
  if (p) { const double t = b[0]; b[0] = b[1]; b[1] = t; }
  if (b[0] != 0.0) b[1] -= b[0] * a[1];
  if (b[1] != 0.0) { b[1] /= a[3]; b[0] -= b[1] * a[2]; }
  if (b[0] != 0.0) b[0] /= a[0];
  return 0;
}

// DIAGONAL_BLOCK_Solver (dbs.c:492-550) for the bilateral kinds: fixpnt,
// fixdir, velodir, velodir3, riglnk (dbs.c:328-450). Returns the iterations
// (riglnk) or 0, and -1 when a factorisation fails.
static __device__ __noinline__ int bilateral_solve(int kind, const double* Z, double step, int dynamic, double epsilon,
                                                   int maxiter, const double* W, const double* B, const double* V,
                                                   double* U, double* R) {
  switch (kind) {
    case CON_FIXPNT: {  // W R = -V - B (dynamic) or -B, U = -V or 0
      double A[9];
      for (int q = 0; q < 9; q++) A[q] = W[q];
      if (dynamic) { U[0] = -V[0]; U[1] = -V[1]; U[2] = -V[2]; }
      else { U[0] = U[1] = U[2] = 0.0; }
      R[0] = U[0] - B[0]; R[1] = U[1] - B[1]; R[2] = U[2] - B[2];
      return chol3_solve(A, R) ? -1 : 0;
    }
    case CON_FIXDIR:
    case CON_VELODIR: {
      R[0] = 0.0;
      R[1] = 0.0;
      if (kind == CON_VELODIR) R[2] = (Z[0] - B[2]) / W[8];
      else R[2] = dynamic ? -(V[2] + B[2]) / W[8] : -B[2] / W[8];
      U[0] = B[0] + R[2] * W[6]; U[1] = B[1] + R[2] * W[7]; U[2] = B[2] + R[2] * W[8];
      return 0;
    }
    case CON_VELODIR3: {  // W R = Z - B, U = Z
      double A[9];
      for (int q = 0; q < 9; q++) A[q] = W[q];
      U[0] = Z[0]; U[1] = Z[1]; U[2] = Z[2];
      R[0] = U[0] - B[0]; R[1] = U[1] - B[1]; R[2] = U[2] - B[2];
      return chol3_solve(A, R) ? -1 : 0;
    }
    case CON_RIGLNK: {  // min 0.5 W_NN R_N^2 subject to |Z + h (W_.N R_N + B)|^2 = d^2 (dbs.c:396-450)
      const double h = dynamic ? step * 0.5 : step;
      const double len = Z[3];
      double l = 0.0, error;
      int iter = 0;
      R[0] = R[1] = 0.0;
      do {
        double C[3], D[4], X[2], L[4];
        C[0] = B[0] + R[2] * W[6]; C[1] = B[1] + R[2] * W[7]; C[2] = B[2] + R[2] * W[8];
        D[0] = Z[0] + h * C[0]; D[1] = Z[1] + h * C[1]; D[2] = Z[2] + h * C[2];
        X[1] = (D[0] * D[0] + D[1] * D[1] + D[2] * D[2]) - len * len;
        D[3] = (W[6] * D[0] + W[7] * D[1] + W[8] * D[2]) * 2.0 * h;
        X[0] = W[8] * R[2] + l * D[3];
        L[0] = W[8]; L[2] = D[3];
        L[1] = D[3]; L[3] = 0.0;
        if (lu2_solve(L, X)) return -1;
        R[2] -= X[0];
        l -= X[1];
        error = sqrt((X[0] * X[0] + X[1] * X[1]) / (R[2] * R[2] + l * l));
      } while (error > epsilon && ++iter < maxiter);
      if (dynamic && iter >= maxiter) {  // the velocity zeroing formula
        R[2] = -B[2] / W[8];
        iter = 0;
      }
      U[0] = B[0] + R[2] * W[6]; U[1] = B[1] + R[2] * W[7]; U[2] = B[2] + R[2] * W[8];
      return iter;
    }
  }
  return -1;
}

// a bilateral row with the reference's failure handling (bgs.c:969-1013): no
// fallback chain outside contacts; under CONTINUE a failed or diverged row
// keeps its previous reaction. Returns 0, 1 diverged, 2 failed.
__device__ __forceinline__ int bilateral_solve_row(int kind, const double* Z, double step, int dynamic, int failure,
                                                   double epsilon, int maxiter, const double* W, const double* B,
                                                   const double* V, double* U, double* R) {
  const double r0 = R[0], r1 = R[1], r2 = R[2];
  const int it = bilateral_solve(kind, Z, step, dynamic, epsilon, maxiter, W, B, V, U, R);
  if (it < maxiter && it >= 0) return 0;
  if (failure == FAIL_CONTINUE) { R[0] = r0; R[1] = r1; R[2] = r2; }
  return it < 0 ? 2 : 1;
}

// merit numerator of a bilateral row (mrf.c:88-137, the GAUSS_SEIDEL_SOLVER
// form for RIGLNK)
__device__ __forceinline__ double merit_row_bilateral(int kind, const double* Z, double gap, double step, int dynamic,
                                                      const double* A, const double* V, const double* U) {
  switch (kind) {
    case CON_FIXPNT:
    case CON_VELODIR3: {
      double P[3];
      if (kind == CON_FIXPNT) {
        if (dynamic) { P[0] = U[0] + V[0]; P[1] = U[1] + V[1]; P[2] = U[2] + V[2]; }
        else { P[0] = U[0]; P[1] = U[1]; P[2] = U[2]; }
      } else {
        P[0] = Z[0] - U[0]; P[1] = Z[1] - U[1]; P[2] = Z[2] - U[2];
      }
      const double Q0 = A[0] * P[0] + A[3] * P[1] + A[6] * P[2];
      const double Q1 = A[1] * P[0] + A[4] * P[1] + A[7] * P[2];
      const double Q2 = A[2] * P[0] + A[5] * P[1] + A[8] * P[2];
      return Q0 * P[0] + Q1 * P[1] + Q2 * P[2];
    }
    case CON_FIXDIR:
    case CON_VELODIR:
    case CON_RIGLNK: {
      double P2;
      if (kind == CON_FIXDIR) P2 = dynamic ? U[2] + V[2] : U[2];
      else if (kind == CON_VELODIR) P2 = Z[0] - U[2];
      else P2 = gap / (step * (dynamic ? 0.5 : 1.0)) + U[2];
      const double Q2 = A[8] * P2;
      return Q2 * P2;
    }
  }
  return 0.0;
}

}  // namespace b2
