// b2_rigid.cuh -- rigid-body time integration on the device, on either side of
// the contact solve: BODY_Dynamic_Step_Begin / BODY_Dynamic_Step_End for RIG
// and OBS bodies (bod.c:1313-1374, 1425-1493) with the reference's default
// scheme NEW2 (SCH_RIG_NEG) and NEW1 (SCH_RIG_POS), the loads of rig_force
// (bod.c:327-352: the point loads summed on the host, gravity here) and the
// constraint reactions of rig_constraints_force (bod.c:390-439).
//
// One thread per body. The body arrays are the ones the assembly reads
// (rotation, velocities), updated in place, so a time step runs
// begin -> assemble -> solve -> end without returning to the host.
//
// Arithmetic follows the reference's operation order (the algebra macros of
// alg.h and the netlib order of the BLAS calls: dgemv 'N' adds the columns in
// turn, dgemv 'T' forms each dot product in row order), built without
// multiply-add contraction, so results are bitwise those of the CPU
// restatement in oracle/rigid_oracle.py when the exponential map takes its
// small-angle branch; the large-angle branch calls sin and cos.
#pragma once

#include <cuda_runtime.h>
#include "b2_common.cuh"
#include "b2_assemble.cuh"
#include "b2_diag.cuh"

namespace b2 {

enum { SCH_RIG_POS = 0, SCH_RIG_NEG = 1, SCH_RIG_IMP = 2 };  // bod.h:80-91

// Rotation matrix (column-major) of the rotation vector w: Rodrigues' formula
// I + s [w]x + c [w]x^2 with s = sin|w|/|w| and c = (1-cos|w|)/|w|^2. Below ten
// degrees s and c are the Taylor polynomials in |w|^2 that alg.h:1138-1200
// evaluates (same coefficients, same Horner order), so small rotations are
// bitwise reproducible on any IEEE machine.
__device__ __forceinline__ void expmap(const double* w, double* R) {
  const double a2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  double s, c;
  if (a2 < 3.0461741978671E-02) {  // (10 degrees)^2
    s = 1.0 + (-1.666666666666667E-1 +
               (8.333333333333333E-3 +
                (-1.984126984126984E-4 + (2.755731922398589E-6 + (-2.505210838544172E-8 + 1.605904383682161E-10 * a2) * a2) * a2) *
                    a2) *
                   a2) *
                  a2;
    c = 0.5 + (-4.166666666666667E-2 +
               (1.388888888888889E-3 +
                (-2.480158730158730E-5 + (2.755731922398589E-7 + (-2.087675698786810E-9 + 1.147074559772972E-11 * a2) * a2) * a2) *
                    a2) *
                   a2) *
                  a2;
  } else {
    const double a = sqrt(a2);
    s = sin(a) / a;
    c = (1.0 - cos(a)) / a2;
  }
  const double q0 = w[0] * w[0], q1 = w[1] * w[1], q2 = w[2] * w[2];
  const double p01 = w[0] * w[1], p02 = w[0] * w[2], p12 = w[1] * w[2];
  const double s0 = s * w[0], s1 = s * w[1], s2 = s * w[2];
  const double c01 = c * p01, c02 = c * p02, c12 = c * p12;
  R[0] = -c * (q2 + q1) + 1.0;
  R[4] = -c * (q2 + q0) + 1.0;
  R[8] = -c * (q1 + q0) + 1.0;
  R[1] = c01 + s2;
  R[3] = c01 - s2;
  R[2] = c02 - s1;
  R[6] = c02 + s1;
  R[5] = c12 + s0;
  R[7] = c12 - s0;
}

__device__ __forceinline__ void mat_mul(const double* A, const double* B, double* C) {  // C = A B
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int i = 0; i < 3; i++) C[3 * j + i] = A[i] * B[3 * j] + A[3 + i] * B[3 * j + 1] + A[6 + i] * B[3 * j + 2];
}
__device__ __forceinline__ void mat_vec(const double* A, const double* x, double* y) {  // y = A x
#pragma unroll
  for (int i = 0; i < 3; i++) y[i] = A[i] * x[0] + A[3 + i] * x[1] + A[6 + i] * x[2];
}
__device__ __forceinline__ void matt_vec(const double* A, const double* x, double* y) {  // y = A^T x
#pragma unroll
  for (int i = 0; i < 3; i++) y[i] = A[3 * i] * x[0] + A[3 * i + 1] * x[1] + A[3 * i + 2] * x[2];
}

// u += step * blockdiag(J^-1, (1/m) I) f: the two 3x3 blocks of
// MX_Matvec (mtx.c:2297-2307) as netlib dgemv 'N' with beta = 1 (column by
// column, alpha folded into the column's x entry). The zero off-diagonal
// entries of the mass block add nothing.
__device__ __forceinline__ void add_minv_force(const double* jinv, double minv, double step, const double* f, double* u) {
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const double t = step * f[j];
    u[0] = u[0] + t * jinv[3 * j];
    u[1] = u[1] + t * jinv[3 * j + 1];
    u[2] = u[2] + t * jinv[3 * j + 2];
  }
#pragma unroll
  for (int i = 0; i < 3; i++) u[3 + i] = u[3 + i] + (step * f[3 + i]) * minv;
}

// EXPMAP123, alg.h:1280-1382: the derivatives R0, R1, R2 of exp[w] with
// respect to w[0], w[1], w[2] (column-major); below ten degrees the Taylor
// polynomials of EXPMAP, above them sin and cos
__device__ __noinline__ void expmap123(const double* w, double* R0, double* R1, double* R2) {
  double x = w[0] * w[0] + w[1] * w[1] + w[2] * w[2];
  if (x < 1E-16 * 3.0461741978671E-02) {
    for (int q = 0; q < 9; q++) R0[q] = R1[q] = R2[q] = 0.0;
    R0[5] = 1.0; R0[7] = -1.0;
    R1[2] = -1.0; R1[6] = 1.0;
    R2[1] = 1.0; R2[3] = -1.0;
    return;
  }
  const double c = 1.0 / x;
  double a, b;
  if (x < 3.0461741978671E-02) {
    a = 1.0 + (-1.666666666666667E-1 +
               (8.333333333333333E-3 +
                (-1.984126984126984E-4 + (2.755731922398589E-6 + (-2.505210838544172E-8 + 1.605904383682161E-10 * x) * x) * x) *
                    x) *
                   x) *
                  x;
    b = c - 0.5 +
        (4.166666666666667E-2 +
         (-1.388888888888889E-3 +
          (2.480158730158730E-5 + (-2.755731922398589E-7 + (2.087675698786810E-9 - 1.147074559772972E-11 * x) * x) * x) * x) *
             x) *
            x;
  } else {
    x = sqrt(x);
    a = sin(x) / x;
    b = c * cos(x);
  }
  const double b_ac = b - a * c;
  const double ac_2cc_2bc = (a - 2.0 * (c - b)) * c;
  const double c_b = c - b;
  double aux[9];
  for (int j = 0; j < 3; j++)
    for (int i = 0; i < 3; i++) aux[3 * j + i] = w[i] * w[j];
  for (int q = 0; q < 9; q++) aux[q] *= ac_2cc_2bc;
  double t[3] = {w[0] * b_ac, w[1] * b_ac, w[2] * b_ac};
  aux[0] -= a; aux[1] += t[2]; aux[2] -= t[1];
  aux[3] -= t[2]; aux[4] -= a; aux[5] += t[0];
  aux[6] += t[1]; aux[7] -= t[0]; aux[8] -= a;
  t[0] = w[0] * c_b; t[1] = w[1] * c_b; t[2] = w[2] * c_b;
  R0[0] = aux[0] * w[0] + 2.0 * t[0]; R0[1] = aux[1] * w[0] + t[1]; R0[2] = aux[2] * w[0] + t[2];
  R0[3] = aux[3] * w[0] + t[1]; R0[4] = aux[4] * w[0]; R0[5] = aux[5] * w[0] + a;
  R0[6] = aux[6] * w[0] + t[2]; R0[7] = aux[7] * w[0] - a; R0[8] = aux[8] * w[0];
  R1[0] = aux[0] * w[1]; R1[1] = aux[1] * w[1] + t[0]; R1[2] = aux[2] * w[1] - a;
  R1[3] = aux[3] * w[1] + t[0]; R1[4] = aux[4] * w[1] + 2.0 * t[1]; R1[5] = aux[5] * w[1] + t[2];
  R1[6] = aux[6] * w[1] + a; R1[7] = aux[7] * w[1] + t[2]; R1[8] = aux[8] * w[1];
  R2[0] = aux[0] * w[2]; R2[1] = aux[1] * w[2] + a; R2[2] = aux[2] * w[2] + t[0];
  R2[3] = aux[3] * w[2] - a; R2[4] = aux[4] * w[2]; R2[5] = aux[5] * w[2] + t[1];
  R2[6] = aux[6] * w[2] + t[0]; R2[7] = aux[7] * w[2] + t[1]; R2[8] = aux[8] * w[2] + 2.0 * t[2];
}

__device__ __forceinline__ double maxabs3(const double* r) {  // MAXABS, alg.h:434-442
  double m = r[0] > 0 ? r[0] : -r[0];
  const double a1 = r[1] > 0 ? r[1] : -r[1], a2 = r[2] > 0 ? r[2] : -r[2];
  if (m < a1) m = a1;
  if (m < a2) m = a2;
  return m;
}

// SOLVE, bod.c:163-209 (NEW3): W with exp[hW] J W = G by Newton's method from
// the given W, A = exp[hW]; the Jacobian dexp[hW] h J W + exp[hW] J is solved
// by LU as LAPACK dgesv does. Returns 0, 1 for a singular Jacobian
// (ERR_BOD_NEW3_SINGULAR_JACOBIAN) or 2 after 50 Newton steps
// (ERR_BOD_NEW3_NEWTON_DIVERGENCE); the reference stops the program there.
__device__ __noinline__ int rig_new3_solve(double h, const double* J, double* W, const double* G, double* A) {
  double O[3], B[9], R[3];
  int i = 0;
  O[0] = W[0] * h; O[1] = W[1] * h; O[2] = W[2] * h;
  expmap(O, A);
  mat_mul(A, J, B);
  mat_vec(B, W, R);
  R[0] = R[0] - G[0]; R[1] = R[1] - G[1]; R[2] = R[2] - G[2];
  const double level = 1E-12 * h;
  double error = maxabs3(R);
  while (error > level) {
    double JW[3], Z0[9], Z1[9], Z2[9], Z[9];
    mat_vec(J, W, JW);
    expmap123(O, Z0, Z1, Z2);
    mat_vec(Z0, JW, Z);
    mat_vec(Z1, JW, Z + 3);
    mat_vec(Z2, JW, Z + 6);
    for (int q = 0; q < 9; q++) Z[q] *= h;
    for (int q = 0; q < 9; q++) Z[q] = Z[q] + B[q];
    if (lu3_solve(Z, R)) return 1;
    W[0] = W[0] - R[0]; W[1] = W[1] - R[1]; W[2] = W[2] - R[2];
    O[0] = W[0] * h; O[1] = W[1] * h; O[2] = W[2] * h;
    expmap(O, A);
    mat_mul(A, J, B);
    mat_vec(B, W, R);
    R[0] = R[0] - G[0]; R[1] = R[1] - G[1]; R[2] = R[2] - G[2];
    error = maxabs3(R);
    if (!(++i < 50)) return 2;
  }
  return 0;
}

struct RigidDev {
  int nbod;
  double* rot;          // [nbod][9] R, column-major (in place)
  double* x;            // [nbod][3] mass centre (in place)
  double* velo;         // [nbod][6] [Omega; v] (in place)
  double* velo0;        // [nbod][6] the same at the start of the step (written by begin)
  double* fext;         // [nbod][6] external force of the step (written by begin)
  double* aux;          // [nbod][3] the NEW2 auxiliary vector (RIG_AUXILIARY)
  const double* J;      // [nbod][9] referential inertia
  const double* jinv;   // [nbod][9] its inverse
  const double* mass;   // [nbod]
  const double* minv;   // [nbod]
  const int* scheme;    // [nbod]
  const int* obstacle;  // [nbod]
  const int* flags;     // [nbod] BODY_* flags (BODY_DISABLE_ROTATION = 4 honoured), or null
  int* fail;            // NEW3 failures (bit or of rig_new3_solve's codes)
};

constexpr int kBodyDisableRotation = 0x0004;  // BODY_DISABLE_ROTATION, bod.h:144

// BODY_Dynamic_Step_Begin (bod.c:1316-1370) for every body. loads[9 b ..]:
// linear force, spatial torque, referential torque of the body's point loads
// at time + step/2 (may be null: none); gravity g: m g is added to the linear
// force of every non-obstacle body.
__global__ void k_rigid_begin(RigidDev d, double step, double g0, double g1, double g2, const double* loads) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nbod) return;
  const double half = 0.5 * step;
  double* u = d.velo + 6 * (size_t)b;
  double* u0 = d.velo0 + 6 * (size_t)b;
  double* R = d.rot + 9 * (size_t)b;
  double* x = d.x + 3 * (size_t)b;
  double J[9], I[9], W[3], DR[9], O[3], Rold[9], f[6];
#pragma unroll
  for (int q = 0; q < 9; q++) { J[q] = d.J[9 * (size_t)b + q]; I[q] = d.jinv[9 * (size_t)b + q]; Rold[q] = R[q]; }
  if (d.flags && (d.flags[b] & kBodyDisableRotation)) u[0] = u[1] = u[2] = 0.0;
#pragma unroll
  for (int q = 0; q < 6; q++) u0[q] = u[q];
  W[0] = u[0]; W[1] = u[1]; W[2] = u[2];
  O[0] = W[0] * half; O[1] = W[1] * half; O[2] = W[2] * half;
  expmap(O, DR);
  double Rn[9];
  mat_mul(Rold, DR, Rn);  // R(t+h/2) = R(t) exp[(h/2) W(t)]
#pragma unroll
  for (int q = 0; q < 9; q++) R[q] = Rn[q];
#pragma unroll
  for (int i = 0; i < 3; i++) x[i] = x[i] + half * u[3 + i];  // x(t+h/2) = x(t) + (h/2) v(t)

  // rig_force at t + h/2: point loads, then gravity (none for obstacles)
  double lin[3] = {0.0, 0.0, 0.0}, spat[3] = {0.0, 0.0, 0.0}, ref[3] = {0.0, 0.0, 0.0};
  if (!d.obstacle[b]) {
    if (loads) {
      const double* L = loads + 9 * (size_t)b;
#pragma unroll
      for (int i = 0; i < 3; i++) { lin[i] = L[i] + lin[i]; spat[i] = L[3 + i] + spat[i]; ref[i] = L[6 + i] + ref[i]; }
    }
    const double m = d.mass[b];
    lin[0] = lin[0] + m * g0; lin[1] = lin[1] + m * g1; lin[2] = lin[2] + m * g2;
  }
  f[3] = lin[0]; f[4] = lin[1]; f[5] = lin[2];
  {
    double t[3];
    matt_vec(Rn, spat, t);
    f[0] = ref[0] + t[0]; f[1] = ref[1] + t[1]; f[2] = ref[2] + t[2];  // T = reftorq + R^T spatorq
  }
  const int sch = d.scheme[b];
  if (sch > SCH_RIG_POS) {  // A = exp[-(h/2)W(t)] J W(t) + h T(t+h/2)
    double JW[3], A[3];
    mat_vec(J, W, JW);
    matt_vec(DR, JW, A);
    double* aux = d.aux + 3 * (size_t)b;
#pragma unroll
    for (int i = 0; i < 3; i++) aux[i] = A[i] + step * f[i];
  }
  double W05[3], P[3];
  P[0] = f[0] * half; P[1] = f[1] * half; P[2] = f[2] * half;
  mat_vec(J, W, W05);
  {
    double t[3];
    matt_vec(DR, W05, t);
    P[0] = P[0] + t[0]; P[1] = P[1] + t[1]; P[2] = P[2] + t[2];
  }
  mat_vec(I, P, W05);  // W05 = I [exp[-(h/2)W(t)] J W(t) + (h/2) T(t+h/2)]
  mat_vec(J, W05, P);
  f[0] -= W05[1] * P[2] - W05[2] * P[1];  // T - W05 x J W05
  f[1] -= W05[2] * P[0] - W05[0] * P[2];
  f[2] -= W05[0] * P[1] - W05[1] * P[0];
  double* fe = d.fext + 6 * (size_t)b;
#pragma unroll
  for (int q = 0; q < 6; q++) fe[q] = f[q];
  add_minv_force(I, d.minv[b], step, f, u);  // u(t+h) = u(t) + h M^-1 f(t+h/2)
}

// BODY_Dynamic_Step_End (bod.c:1428-1485) for every body: the constraint
// reactions of the last solve (rig_constraints_force, bod.c:419-439: the
// body's contacts in ascending order, obstacles skipped), the velocity
// update, the second half step of the position and the rotation update of the
// body's scheme. R64/iperm: the solve's reactions in sorted row order and the
// sorted position of each contact (all contact arrays may be null when the
// scene has no contacts, with bptr null).
__global__ void k_rigid_end(RigidDev d, double step, const double* x0, const int* master, const double* mpnt,
                            const double* spnt, const double* cbase, const int* bptr, const int* brow,
                            const double4* R64, const int* iperm) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= d.nbod) return;
  const double half = 0.5 * step;
  double* u = d.velo + 6 * (size_t)b;
  double* R = d.rot + 9 * (size_t)b;
  double* x = d.x + 3 * (size_t)b;
  double Rb[9], X0[3], f[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int q = 0; q < 9; q++) Rb[q] = R[q];
  X0[0] = x0[3 * (size_t)b]; X0[1] = x0[3 * (size_t)b + 1]; X0[2] = x0[3 * (size_t)b + 2];
  if (bptr && !d.obstacle[b]) {  // obstacles do not react to contact forces
    for (int k = bptr[b]; k < bptr[b + 1]; k++) {
      const int i = brow[k];
      const bool isma = master[i] == b;
      const double* X = (isma ? mpnt : spnt) + 3 * (size_t)i;
      double H[18];
      rig_H(Rb, X0, cbase + 9 * (size_t)i, X, H);
      const double4 rc = R64[iperm[i]];
      double r[6];
#pragma unroll
      for (int j = 0; j < 6; j++) r[j] = H[3 * j] * rc.x + H[3 * j + 1] * rc.y + H[3 * j + 2] * rc.z;  // H^T R
      if (isma) {
#pragma unroll
        for (int j = 0; j < 6; j++) f[j] += r[j];
      } else {
#pragma unroll
        for (int j = 0; j < 6; j++) f[j] -= r[j];
      }
    }
  }
  double I[9];
#pragma unroll
  for (int q = 0; q < 9; q++) I[q] = d.jinv[9 * (size_t)b + q];
  add_minv_force(I, d.minv[b], step, f, u);                   // u(t+h) += h M^-1 r
#pragma unroll
  for (int i = 0; i < 3; i++) x[i] = x[i] + half * u[3 + i];  // x(t+h) = x(t+h/2) + (h/2) v(t+h)
  if (d.flags && (d.flags[b] & kBodyDisableRotation)) u[0] = u[1] = u[2] = 0.0;
  const int sch = d.scheme[b];
  double DR[9];
  if (sch <= SCH_RIG_NEG) {  // R(t+h) = R(t+h/2) exp[(h/2) W(t+h)]
    const double O[3] = {u[0] * half, u[1] * half, u[2] * half};
    expmap(O, DR);
    double Rn[9];
    mat_mul(Rb, DR, Rn);
#pragma unroll
    for (int q = 0; q < 9; q++) R[q] = Rn[q];
  }
  if (sch > SCH_RIG_POS) {
    double* aux = d.aux + 3 * (size_t)b;
    double A[3];
#pragma unroll
    for (int i = 0; i < 3; i++) A[i] = aux[i] + step * f[i];
#pragma unroll
    for (int i = 0; i < 3; i++) aux[i] = A[i];
    if (sch == SCH_RIG_NEG) {  // W(t+h) = I exp[-(h/2)W1(t+h)] A
      double O[3];
      matt_vec(DR, A, O);
      mat_vec(I, O, u);
    } else {  // NEW3: exp[(h/2)W(t+h)] J W(t+h) = A, then R(t+h) = R(t+h/2) exp[(h/2)W(t+h)]
      double J[9], W[3] = {u[0], u[1], u[2]};
#pragma unroll
      for (int q = 0; q < 9; q++) J[q] = d.J[9 * (size_t)b + q];
      const int e = rig_new3_solve(half, J, W, A, DR);
      if (e) atomicOr(d.fail, e);
      u[0] = W[0]; u[1] = W[1]; u[2] = W[2];
      double Rn[9];
      mat_mul(Rb, DR, Rn);
#pragma unroll
      for (int q = 0; q < 9; q++) R[q] = Rn[q];
    }
  }
}

}  // namespace b2
