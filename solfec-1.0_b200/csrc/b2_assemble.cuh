// b2_assemble.cuh -- local dynamics assembly on the device for rigid bodies.
//
// Device form of update_V_and_B (ldy.c:364-474) and LOCDYN_Update_Begin
// (ldy.c:626-876) on top of the rigid operators rig_operator_H (bod.c:216-229),
// rig_dynamic_inverse (bod.c:232-258), BODY_Local_Velo (bod.c:1817-1844) and
// BODY_Gen_To_Loc_Operator (bod.c:1846-1871, an obstacle contributes H = 0 to
// contacts). The contact graph is that of LOCDYN_Insert (ldy.c:492-568): rows
// are adjacent through every non-obstacle body they share, one block per
// shared body.
#pragma once

#include <cuda_runtime.h>
#include "b2_common.cuh"

namespace b2 {

// Per-row factors kept for the off-diagonal pass: for the master and the slave
// side the operator H (3x6, slave negated as ldy.c:685 does) and
// P = M^-1 H^T (6x3). Zero for an obstacle side.
constexpr int kFactorStride = 72;  // Hm[18] Pm[18] Hs[18] Ps[18]

// 16-byte store and load of two doubles (p 16-byte aligned: a row's factors
// start at a multiple of 72 doubles and each part at an even offset)
__device__ __forceinline__ void st2(double* p, double a, double b) {
  *reinterpret_cast<double2*>(p) = make_double2(a, b);
}
__device__ __forceinline__ double2 ld2(const double* p) { return __ldg(reinterpret_cast<const double2*>(p)); }
// the six velocity components of a body (6 doubles a body: 16-byte aligned)
__device__ __forceinline__ void ld6(const double* p, double* u) {
  const double2 a = ld2(p), b = ld2(p + 2), c = ld2(p + 4);
  u[0] = a.x; u[1] = a.y; u[2] = b.x; u[3] = b.y; u[4] = c.x; u[5] = c.y;
}

struct SceneDev {
  int nbod, ncon;
  const double* rot;    // [nbod][9]
  const double* x0;     // [nbod][3]
  const double* jinv;   // [nbod][9]
  const double* minv;   // [nbod]
  const double* velo;   // [nbod][6]
  const double* velo0;  // [nbod][6]
  const int* obstacle;  // [nbod]
  const int* master;    // [ncon]
  const int* slave;     // [ncon]
  const double* mpnt;   // [ncon][3]
  const double* spnt;   // [ncon][3]
  const double* base;   // [ncon][9]
};

__device__ __forceinline__ void rig_H(const double* R, const double* X0, const double* base, const double* X,
                                      double* H) {
  const double A0 = X[0] - X0[0], A1 = X[1] - X0[1], A2 = X[2] - X0[2];
  const double S[9] = {0.0, A2, -A1, -A2, 0.0, A0, A1, -A0, 0.0};  // skew(A), column-major
  double T[9];
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int i = 0; i < 3; i++) T[3 * j + i] = R[i] * S[j] + R[3 + i] * S[3 + j] + R[6 + i] * S[6 + j];
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int i = 0; i < 3; i++)
      H[3 * j + i] = base[3 * i] * T[3 * j] + base[3 * i + 1] * T[3 * j + 1] + base[3 * i + 2] * T[3 * j + 2];
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int i = 0; i < 3; i++) H[9 + 3 * j + i] = base[3 * i + j];
}

__device__ __forceinline__ void h_times(const double* H, const double* x, double* y) {
  y[0] = y[1] = y[2] = 0.0;
#pragma unroll
  for (int j = 0; j < 6; j++) {
    const double t = x[j];
    y[0] += t * H[3 * j];
    y[1] += t * H[3 * j + 1];
    y[2] += t * H[3 * j + 2];
  }
}

__device__ __forceinline__ void minv_ht(const double* J, double minv, const double* H, double* P) {
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const double h0 = H[c], h1 = H[3 + c], h2 = H[6 + c];
    P[6 * c + 0] = J[0] * h0 + J[3] * h1 + J[6] * h2;
    P[6 * c + 1] = J[1] * h0 + J[4] * h1 + J[7] * h2;
    P[6 * c + 2] = J[2] * h0 + J[5] * h1 + J[8] * h2;
    P[6 * c + 3] = minv * H[9 + c];
    P[6 * c + 4] = minv * H[12 + c];
    P[6 * c + 5] = minv * H[15 + c];
  }
}

// C += L (3x6) * P (6x3)
__device__ __forceinline__ void hp_add(const double* L, const double* P, double* C) {
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 6; k++) s += L[3 * k + i] * P[6 * j + k];
      C[3 * j + i] += s;
    }
}

// Largest eigenvalue of a symmetric 3x3 matrix by cyclic Jacobi rotations
// (Golub & Van Loan, symmetric Schur decomposition); rho = 1/lambda_max
// replaces LAPACK dsyev in ldy.c:719-724.
__device__ __forceinline__ double sym3_max_eig(const double* W) {
  double a[3][3];
#pragma unroll
  for (int j = 0; j < 3; j++)
#pragma unroll
    for (int i = 0; i < 3; i++) a[i][j] = 0.5 * (W[3 * j + i] + W[3 * i + j]);
  for (int sweep = 0; sweep < 32; sweep++) {
    const double off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
    const double dia = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
    if (off <= 1e-36 * dia || off == 0.0) break;
#pragma unroll
    for (int p = 0; p < 2; p++)
#pragma unroll
      for (int q = p + 1; q < 3; q++) {
        if (a[p][q] == 0.0) continue;
        const double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
        a[p][q] = a[q][p] = 0.0;
      }
  }
  double m = a[0][0];
  if (a[1][1] > m) m = a[1][1];
  if (a[2][2] > m) m = a[2][2];
  return m;
}

// A = W^-1 by three LU solves (replaces MX_Inverse, mtx.c:1599-1626).
__device__ __forceinline__ void inv3(const double* W, double* A);

// Row pass (thread per contact, caller order): H/P factors, W_ii, rho, A, B, V
// and the per-block partial of the free energy sum_i B_i^T A_i B_i.
__global__ void k_row_factors(SceneDev sc, double step, double* factors, double* Wii, double* Aii, double* rho,
                              double* Bo, double* Vo, double* fe_part, int* bad, int write_factors) {
  __shared__ double red[256 / kWarp];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double fe = 0.0;
  if (i < sc.ncon) {
    const int m = sc.master[i], s = sc.slave[i];
    double base[9], X[3], H[18], y[3];
    double* F = factors + (size_t)i * kFactorStride;
#pragma unroll
    for (int q = 0; q < 9; q++) base[q] = sc.base[(size_t)9 * i + q];
    double V[3] = {0, 0, 0}, B[3] = {0, 0, 0}, W[9];
#pragma unroll
    for (int q = 0; q < 9; q++) W[q] = 0.0;
    if (m == s || m < 0 || m >= sc.nbod || s >= sc.nbod) {
      atomicExch(bad, 1);  // self-contact or invalid body index
    } else {
      // master side (ldy.c:376-381, bod.c:1825-1829)
#pragma unroll
      for (int q = 0; q < 3; q++) X[q] = sc.mpnt[(size_t)3 * i + q];
      rig_H(sc.rot + (size_t)9 * m, sc.x0 + (size_t)3 * m, base, X, H);
      double u[6];
      ld6(sc.velo0 + (size_t)6 * m, u);
      h_times(H, u, y); V[0] += y[0]; V[1] += y[1]; V[2] += y[2];
      ld6(sc.velo + (size_t)6 * m, u);
      h_times(H, u, y); B[0] += y[0]; B[1] += y[1]; B[2] += y[2];
      if (!sc.obstacle[m]) {
        double P[18];
        minv_ht(sc.jinv + (size_t)9 * m, sc.minv[m], H, P);
#pragma unroll
        if (write_factors)
          for (int q = 0; q < 18; q += 2) { st2(F + q, H[q], H[q + 1]); st2(F + 18 + q, P[q], P[q + 1]); }
        hp_add(H, P, W);
      } else {
#pragma unroll
        if (write_factors)
          for (int q = 0; q < 36; q += 2) st2(F + q, 0.0, 0.0);
      }
      // slave side, subtracted (ldy.c:383-393), H negated for W (ldy.c:685)
      if (s >= 0) {
#pragma unroll
        for (int q = 0; q < 3; q++) X[q] = sc.spnt[(size_t)3 * i + q];
        rig_H(sc.rot + (size_t)9 * s, sc.x0 + (size_t)3 * s, base, X, H);
        double u[6];
        ld6(sc.velo0 + (size_t)6 * s, u);
        h_times(H, u, y); V[0] -= y[0]; V[1] -= y[1]; V[2] -= y[2];
        ld6(sc.velo + (size_t)6 * s, u);
        h_times(H, u, y); B[0] -= y[0]; B[1] -= y[1]; B[2] -= y[2];
      }
      if (s >= 0 && !sc.obstacle[s]) {
        double P[18];
#pragma unroll
        for (int q = 0; q < 18; q++) H[q] = -H[q];
        minv_ht(sc.jinv + (size_t)9 * s, sc.minv[s], H, P);
#pragma unroll
        if (write_factors)
          for (int q = 0; q < 18; q += 2) { st2(F + 36 + q, H[q], H[q + 1]); st2(F + 54 + q, P[q], P[q + 1]); }
        hp_add(H, P, W);
      } else {
#pragma unroll
        if (write_factors)
          for (int q = 0; q < 36; q += 2) st2(F + 36 + q, 0.0, 0.0);
      }
    }
#pragma unroll
    for (int q = 0; q < 9; q++) W[q] *= step;
    double A[9];
    inv3(W, A);
    const double r = 1.0 / sym3_max_eig(W);
#pragma unroll
    for (int q = 0; q < 9; q++) { Wii[(size_t)9 * i + q] = W[q]; Aii[(size_t)9 * i + q] = A[q]; }
#pragma unroll
    for (int q = 0; q < 3; q++) { Bo[(size_t)3 * i + q] = B[q]; Vo[(size_t)3 * i + q] = V[q]; }
    rho[i] = r;
    const double Q0 = A[0] * B[0] + A[3] * B[1] + A[6] * B[2];
    const double Q1 = A[1] * B[0] + A[4] * B[1] + A[7] * B[2];
    const double Q2 = A[2] * B[0] + A[5] * B[1] + A[8] * B[2];
    fe = Q0 * B[0] + Q1 * B[1] + Q2 * B[2];
  }
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) fe += __shfl_down_sync(0xffffffffu, fe, d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = fe;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    fe_part[blockIdx.x] = t;
  }
}

}  // namespace b2

#include "b2_diag.cuh"

namespace b2 {
// (one factorisation applied to the three unit vectors: the same arithmetic
// as three dgesv calls, which factorise the same matrix identically; a
// singular W leaves the unit vectors in A, as the three calls do)
__device__ __forceinline__ void inv3(const double* W, double* A) {
  double a[9];
  int ipiv[3];
#pragma unroll
  for (int q = 0; q < 9; q++) a[q] = W[q];
  const int info = lu3_factor(a, ipiv);
#pragma unroll
  for (int j = 0; j < 3; j++) {
    double b[3] = {0.0, 0.0, 0.0};
    b[j] = 1.0;
    if (!info) lu3_apply(a, ipiv, b);
    A[3 * j] = b[0]; A[3 * j + 1] = b[1]; A[3 * j + 2] = b[2];
  }
}

// deterministic sum of the free-energy partials (one block)
__global__ void k_sum_partials(const double* part, int n, double* out) {
  __shared__ double red[32];
  double t = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) t += part[i];
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) t += __shfl_down_sync(0xffffffffu, t, d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    *out = 0.5 * s;  // ldy.c:739
  }
}

// Free energy of each problem of a batch (ldy.c:739 per problem): block k
// sums 1/2 B^T A B over the caller rows off[k] .. off[k+1]-1.
__global__ void k_problem_free_energy(const int* __restrict__ off, const double* __restrict__ Aii,
                                      const double* __restrict__ Bc, double* __restrict__ out) {
  __shared__ double red[32];
  const int k = blockIdx.x;
  double t = 0.0;
  for (int i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x) {
    const double* A = Aii + (size_t)9 * i;
    const double* B = Bc + (size_t)3 * i;
    const double Q0 = A[0] * B[0] + A[3] * B[1] + A[6] * B[2];
    const double Q1 = A[1] * B[0] + A[4] * B[1] + A[7] * B[2];
    const double Q2 = A[2] * B[0] + A[5] * B[1] + A[8] * B[2];
    t += Q0 * B[0] + Q1 * B[1] + Q2 * B[2];
  }
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) t += __shfl_down_sync(0xffffffffu, t, d);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
    out[k] = 0.5 * s;
  }
}

// ---- contact graph (LOCDYN_Insert adjacency) ----

__device__ __forceinline__ bool graph_body(const int* obstacle, int b) { return b >= 0 && !obstacle[b]; }

__global__ void k_body_count(int ncon, const int* master, const int* slave, const int* obstacle, int* bdeg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncon) return;
  const int m = master[i], s = slave[i];
  if (graph_body(obstacle, m)) atomicAdd(bdeg + m, 1);
  if (graph_body(obstacle, s)) atomicAdd(bdeg + s, 1);
}

__global__ void k_body_fill(int ncon, const int* master, const int* slave, const int* obstacle, const int* bptr,
                            int* cursor, int* brow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncon) return;
  const int m = master[i], s = slave[i];
  if (graph_body(obstacle, m)) brow[bptr[m] + atomicAdd(cursor + m, 1)] = i;
  if (graph_body(obstacle, s)) brow[bptr[s] + atomicAdd(cursor + s, 1)] = i;
}

// rows of each body in ascending order (makes the graph independent of the
// order the atomics above landed in)
__global__ void k_body_sort(int nbod, const int* bptr, int* brow) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nbod) return;
  const int lo = bptr[b], hi = bptr[b + 1];
  for (int x = lo + 1; x < hi; x++) {
    const int v = brow[x];
    int y = x - 1;
    while (y >= lo && brow[y] > v) { brow[y + 1] = brow[y]; y--; }
    brow[y + 1] = v;
  }
}

__global__ void k_row_degree(int ncon, const int* master, const int* slave, const int* obstacle, const int* bptr,
                             int* deg) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncon) return;
  const int m = master[i], s = slave[i];
  int d = 0;
  if (graph_body(obstacle, m)) d += bptr[m + 1] - bptr[m] - 1;
  if (graph_body(obstacle, s)) d += bptr[s + 1] - bptr[s] - 1;
  deg[i] = d;
}

// adjacency of row i: neighbours through the master body, then through the
// slave body, each ascending; adjbod holds the shared body
__global__ void k_adj_fill(int ncon, const int* master, const int* slave, const int* obstacle, const int* bptr,
                           const int* brow, const int* adjptr, int* adjcol, int* adjbod) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncon) return;
  int k = adjptr[i];
  const int bods[2] = {master[i], slave[i]};
  for (int t = 0; t < 2; t++) {
    const int b = bods[t];
    if (!graph_body(obstacle, b)) continue;
    for (int q = bptr[b]; q < bptr[b + 1]; q++) {
      const int j = brow[q];
      if (j != i) { adjcol[k] = j; adjbod[k] = b; k++; }
    }
  }
}

}  // namespace b2
