/*
 * oracle_bgs.c -- TEST INFRASTRUCTURE. Not part of the product.
 *
 * CPU restatement of the reference block Gauss-Seidel contact solver:
 *   diagonal block solvers   dbs.c:35-326 (CONTACT + SIGNORINI_COULOMB)
 *   smoothed contact formula scf.c:28-174
 *   merit function           mrf.c:35-185 (CONTACT rows)
 *   serial Gauss-Seidel loop bgs.c:913-1069
 * The 3x3 linear solves use lu_small.c (LAPACK dgetf2/dgetrs arithmetic), the
 * same routine the compiled reference links in oracle/_ref.
 */
#include <math.h>
#include <float.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "lu_small.h"

#define OMIN(v, w) ((v) < (w) ? (v) : (w)) /* alg.h:44 */
#define OMAX(v, w) ((v) > (w) ? (v) : (w)) /* alg.h:48 */

enum { DS_PG = 0, DS_DSF = 1, DS_SSN = 2, DS_PN = 3 };        /* dbs.h:27-33 */
enum { GS_OK = 0, GS_DIVERGED, GS_DIAGONAL_DIVERGED, GS_DIAGONAL_FAILED }; /* bgs.h:31-37 */
enum { FAIL_CONTINUE = 0, FAIL_EXIT, FAIL_CALLBACK };                     /* bgs.h:39-44 */

/* D = C + A*b with A column-major (alg.h:948 NVADDMUL) */
static void nvaddmul (const double *C, const double *A, const double *b, double *D)
{
  double d0 = C[0] + (A[0]*b[0] + A[3]*b[1] + A[6]*b[2]);
  double d1 = C[1] + (A[1]*b[0] + A[4]*b[1] + A[7]*b[2]);
  double d2 = C[2] + (A[2]*b[0] + A[5]*b[1] + A[8]*b[2]);
  D[0] = d0; D[1] = d1; D[2] = d2;
}

static double dot3 (const double *a, const double *b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }

/* dashed normal velocity (dbs.c:52-53, 164-165; scf.c:43-44) */
static double dashed_un (int dynamic, double step, double restitution, double gap, const double *U, const double *V)
{
  if (dynamic) return U[2] + restitution * OMIN (V[2], 0);
  else return (OMAX (gap, 0) / step) + U[2];
}

/* SCF_Project (scf.c:136-174): projection onto the friction cone; S is
 * restored on return exactly as the reference does (S[2] += c ... S[2] -= c). */
static void scf_project (double fri, double cohesion, double *S, double *R)
{
  double m[3], slen, l1, l2, u1[3], u2[3], g1, g2, fri2;

  S[2] += cohesion;
  fri2 = fri*fri;
  slen = sqrt (S[0]*S[0] + S[1]*S[1]);
  l1 = -(S[2] + fri*slen) / (1.0 + fri2);
  l2 =  (slen - fri*S[2]) / (1.0 + fri2);
  if (slen != 0.0)
  {
    u2[0] = S[0]/slen; u2[1] = S[1]/slen; u2[2] = -fri;
    u1[0] = -fri*u2[0]; u1[1] = -fri*u2[1]; u1[2] = -1.0;
  }
  else
  {
    u2[0] = 1.0; u2[1] = 0.0; u2[2] = -fri;
    u1[0] = -fri; u1[1] = 0.0; u1[2] = -1.0;
  }
  g1 = OMAX (l1, 0.0);
  g2 = OMAX (l2, 0.0);
  m[0] = g1*u1[0] + g2*u2[0];
  m[1] = g1*u1[1] + g2*u2[1];
  m[2] = g1*u1[2] + g2*u2[2];
  S[2] -= cohesion;
  R[0] = S[0] - m[0];
  R[1] = S[1] - m[1];
  R[2] = S[2] - m[2];
}

/* SCF_Linearize (scf.c:28-133) with UT = -1 and smoothing 0 as every caller on
 * the path passes (dbs.c:316,324; mrf.c:84); X, Y may be NULL. */
static void scf_linearize (int dynamic, double step, double fri, double res, double coh, double gap,
                           const double *V, const double *U, const double *R, double *C, double *X, double *Y)
{
  const double eps = 0.0, UT = -1.0;
  double dF[9], S[3], F[3], m[3];
  double udash, ulen, sdot, slen, l1, l2, u1[3], u2[3], eps2, fri2, onefri2, sq1, sq2, g1, g2, dg1, dg2, a, b, c, d;

  eps2 = eps*eps;
  fri2 = fri*fri;
  onefri2 = 1.0 + fri2;
  udash = dashed_un (dynamic, step, res, gap, U, V);
  ulen = sqrt (U[0]*U[0] + U[1]*U[1] + eps2);

  F[0] = U[0];
  F[1] = U[1];
  if (UT >= 0.0) F[2] = (udash + fri * UT);
  else F[2] = (udash + fri * (ulen - eps));

  S[0] = R[0] - F[0];
  S[1] = R[1] - F[1];
  S[2] = R[2] - F[2];
  S[2] += coh;

  sdot = S[0]*S[0] + S[1]*S[1];
  slen = sqrt (sdot);
  l1 = -(S[2] + fri*slen) / onefri2;
  l2 =  (slen - fri*S[2]) / onefri2;
  if (slen != 0.0)
  {
    u2[0] = S[0]/slen; u2[1] = S[1]/slen; u2[2] = -fri;
    u1[0] = -fri*u2[0]; u1[1] = -fri*u2[1]; u1[2] = -1.0;
  }
  else
  {
    u2[0] = 1.0; u2[1] = 0.0; u2[2] = -fri;
    u1[0] = -fri; u1[1] = 0.0; u1[2] = -1.0;
  }
  sq1 = sqrt (l1*l1 + 4.0*eps2);
  sq2 = sqrt (l2*l2 + 4.0*eps2*fri2);
  g1 = 0.5 * (sq1 + l1);
  g2 = 0.5 * (sq2 + l2);

  m[0] = g1*u1[0] + g2*u2[0];
  m[1] = g1*u1[1] + g2*u2[1];
  m[2] = g1*u1[2] + g2*u2[2];

  C[0] = F[0] + m[0];
  C[1] = F[1] + m[1];
  C[2] = F[2] + m[2];

  if (X)
  {
    double T[9];
    dF[1] = dF[3] = dF[6] = dF[7] = 0.0;
    dF[0] = dF[4] = dF[8] = 1.0;
    dF[2] = fri * U[0] / ulen;
    dF[5] = fri * U[1] / ulen;

    dg1 = 0.5*(1.0+l1/sq1);
    if (slen != 0.0)
    {
      dg2 = 0.5*(1.0+l2/sq2);
      a = 0.5*(1.0+(l2 + fri*l1)/(sq2 + fri*sq1));
      b = (fri2 * dg1 + dg2) / onefri2;
      c = (fri * (dg1 - dg2)) / onefri2;
      d = (dg1 + fri2 * dg2) / onefri2;
      Y[0] = a + (b - a) * S[0]*S[0] / sdot;
      Y[1] = (b - a) * S[1]*S[0] / sdot;
      Y[2] = c * S[0] / slen;
      Y[3] = Y[1];
      Y[4] = a + (b - a) * S[1]*S[1] / sdot;
      Y[5] = c * S[1] / slen;
      Y[6] = Y[2];
      Y[7] = Y[5];
      Y[8] = d;
    }
    else
    {
      Y[1] = Y[2] = Y[3] = Y[5] = Y[6] = Y[7] = 0.0;
      Y[0] = Y[4] = Y[8] = dg1;
    }
    /* X = dF - Y*dF (scf.c:128-129, NNMUL then NNSUB) */
    for (int j = 0; j < 3; j ++)
      for (int i = 0; i < 3; i ++)
        T[3*j+i] = Y[i]*dF[3*j] + Y[3+i]*dF[3*j+1] + Y[6+i]*dF[3*j+2];
    for (int k = 0; k < 9; k ++) X[k] = dF[k] - T[k];
  }
}

/* projected_gradient (dbs.c:35-94) */
static int projected_gradient (int dynamic, double epsilon, int maxiter, double step, double friction,
  double restitution, double cohesion, double gap, double rho, const double *W, const double *B,
  const double *V, double *U, double *R)
{
  double vector[3], scalar, UN;
  int iter = 0;

  if (dynamic && gap > 0)
  {
    R[0] = R[1] = R[2] = 0.0;
    U[0] = B[0]; U[1] = B[1]; U[2] = B[2];
    return 0;
  }

  do
  {
    vector[0] = R[0]; vector[1] = R[1]; vector[2] = R[2];
    nvaddmul (B, W, R, U);
    UN = dashed_un (dynamic, step, restitution, gap, U, V);
    R[0] -= rho * U[0];
    R[1] -= rho * U[1];
    R[2] -= rho * UN - cohesion;
    R[2] = OMAX (0, R[2]);
    scalar = sqrt (R[0]*R[0] + R[1]*R[1]);
    if (scalar >= friction * R[2])
    {
      if (scalar > 0.0) scalar = friction * R[2] / scalar;
      R[0] *= scalar;
      R[1] *= scalar;
    }
    R[2] -= cohesion;
    vector[0] = R[0] - vector[0]; vector[1] = R[1] - vector[1]; vector[2] = R[2] - vector[2];
    scalar = dot3 (R, R);
    scalar = sqrt (dot3 (vector, vector) / OMAX (scalar, 1.0));
  }
  while (++ iter < maxiter && scalar > epsilon);

  return iter;
}

/* de_saxce_feng (dbs.c:96-140) */
static int de_saxce_feng (int dynamic, double epsilon, int maxiter, double step, double friction,
  double restitution, double cohesion, double gap, double rho, const double *W, const double *B,
  const double *V, double *U, double *R)
{
  double vector[3], scalar, tau[3], UN;
  int iter = 0;

  if (dynamic && gap > 0)
  {
    R[0] = R[1] = R[2] = 0.0;
    U[0] = B[0]; U[1] = B[1]; U[2] = B[2];
    return 0;
  }

  do
  {
    vector[0] = R[0]; vector[1] = R[1]; vector[2] = R[2];
    nvaddmul (B, W, R, U);
    UN = dashed_un (dynamic, step, restitution, gap, U, V);
    tau[0] = R[0] - rho * U[0];
    tau[1] = R[1] - rho * U[1];
    tau[2] = R[2] - rho * (UN + friction * sqrt (U[0]*U[0] + U[1]*U[1]));
    scf_project (friction, cohesion, tau, R);
    vector[0] = R[0] - vector[0]; vector[1] = R[1] - vector[1]; vector[2] = R[2] - vector[2];
    scalar = dot3 (R, R);
    scalar = sqrt (dot3 (vector, vector) / OMAX (scalar, 1.0));
  }
  while (++ iter < maxiter && scalar > epsilon);

  return iter;
}

/* semismooth_newton (dbs.c:142-303) */
static int semismooth_newton (int dynamic, double epsilon, int maxiter, double step, double friction,
  double restitution, double cohesion, double gap, double rho, const double *W, const double *B,
  const double *V, double *U, double *R)
{
  double RES[3], UN, norm, lim, a[9], b[3], c[3], d[3], R0[3], error;
  int divi, ipiv[3], iter;

  if (dynamic && gap > 0)
  {
    R[0] = R[1] = R[2] = 0.0;
    U[0] = B[0]; U[1] = B[1]; U[2] = B[2];
    return 0;
  }

  divi = maxiter / 10;
  iter = 0;
  do
  {
    R0[0] = R[0]; R0[1] = R[1]; R0[2] = R[2];
    UN = dashed_un (dynamic, step, restitution, gap, U, V);

    d[0] = R[0] - rho * U[0];
    d[1] = R[1] - rho * U[1];
    d[2] = (R[2]+cohesion) - rho * UN;

    nvaddmul (B, W, R, RES); /* RES = W*R + B - U */
    RES[0] -= U[0]; RES[1] -= U[1]; RES[2] -= U[2];

    if (d[2] >= 0)
    {
      norm = sqrt (d[0]*d[0]+d[1]*d[1]);
      lim = friction * OMAX (0, d[2]);

      if (norm >= lim) /* slip */
      {
        if (lim > 0.0)
        {
          double F[4], M[4], H[4], delta, alfa, beta, den, len, e;
          len = sqrt (R[0]*R[0]+R[1]*R[1]);
          den = OMAX (lim, len) * norm;
          e = lim / norm;
          if (len == 0.0) beta = 1.0;
          else
          {
            alfa = (R[0]*d[0]+R[1]*d[1]) / (len*norm);
            delta = OMIN (len/lim, 1.0);
            beta = (alfa < 0.0 ? 1.0 / (1.0 - alfa*delta) : 1.0);
          }
          F[0] = (R[0]*d[0])/den;
          F[1] = (R[1]*d[0])/den;
          F[2] = (R[0]*d[1])/den;
          F[3] = (R[1]*d[1])/den;
          M[0] = e * (1.0 - F[0]);
          M[1] = - e * F[1];
          M[2] = - e * F[2];
          M[3] = e * (1.0 - F[3]);
          H[0] = 1.0 - beta * M[0];
          H[1] = - beta * M[1];
          H[2] = - beta * M[2];
          H[3] = 1.0 - beta * M[3];
          a[0] = H[0] + rho*(M[0]*W[0] + M[2]*W[1]);
          a[1] = H[1] + rho*(M[1]*W[0] + M[3]*W[1]);
          a[2] = W[2];
          a[3] = H[2] + rho*(M[0]*W[3] + M[2]*W[4]);
          a[4] = H[3] + rho*(M[1]*W[3] + M[3]*W[4]);
          a[5] = W[5];
          a[6] = rho*(M[0]*W[6] + M[2]*W[7]) - friction*(d[0]/norm);
          a[7] = rho*(M[1]*W[6] + M[3]*W[7]) - friction*(d[1]/norm);
          a[8] = W[8];
          b[0] = friction*(d[0]/norm)*(R[2]+cohesion) - R[0] - rho*(M[0]*RES[0] + M[2]*RES[1]);
          b[1] = friction*(d[1]/norm)*(R[2]+cohesion) - R[1] - rho*(M[1]*RES[0] + M[3]*RES[1]);
          b[2] = -UN - RES[2];
        }
        else /* degenerate: homogeneous tangential tractions */
        {
          a[0] = 1.0; a[1] = 0.0; a[2] = W[2];
          a[3] = 0.0; a[4] = 1.0; a[5] = W[5];
          a[6] = 0.0; a[7] = 0.0; a[8] = W[8];
          b[0] = -R[0] - RES[0];
          b[1] = -R[1] - RES[1];
          b[2] = -UN - RES[2];
        }
      }
      else /* stick */
      {
        a[0] = W[0]; a[1] = W[1]; a[2] = W[2];
        a[3] = W[3]; a[4] = W[4]; a[5] = W[5];
        a[6] = W[6]+U[0]/d[2];
        a[7] = W[7]+U[1]/d[2];
        a[8] = W[8];
        b[0] = -(1.0 + rho*U[2]/d[2])*U[0] - RES[0];
        b[1] = -(1.0 + rho*U[2]/d[2])*U[1] - RES[1];
        b[2] = -UN - RES[2];
      }
    }
    else /* separation */
    {
      a[0] = 1.0; a[1] = 0.0; a[2] = 0.0;
      a[3] = 0.0; a[4] = 1.0; a[5] = 0.0;
      a[6] = 0.0; a[7] = 0.0; a[8] = 1.0;
      b[0] = -R[0];
      b[1] = -R[1];
      b[2] = -R[2];
    }

    if (orc_dgesv (3, a, ipiv, b)) return -1;
    if (!isfinite (b[0]+b[1]+b[2])) return -1;

    nvaddmul (RES, W, b, c);
    R[0] += b[0]; R[1] += b[1]; R[2] += b[2];
    U[0] += c[0]; U[1] += c[1]; U[2] += c[2];

    R0[0] = R[0] - R0[0]; R0[1] = R[1] - R0[1]; R0[2] = R[2] - R0[2];
    error = dot3 (R, R);
    error = sqrt (dot3 (R0, R0) / OMAX (error, 1.0));
    iter ++;

    if ((iter % divi) == 0)
    {
      rho *= 10.0;
      if (isinf (rho)) return -1;
    }
  }
  while (iter < maxiter && error > epsilon);

  return iter;
}

/* projected_newton (dbs.c:305-326) */
static int projected_newton (double epsilon, int maxiter, int dynamic, double step, double friction,
  double restitution, double cohesion, double gap, const double *W, const double *B, const double *V,
  double *U, double *R)
{
  double T[9], X[9], Y[9], C[3], merit;
  int ipiv[3], iter = 0;

  nvaddmul (B, W, R, U);
  scf_linearize (dynamic, step, friction, restitution, cohesion, gap, V, U, R, C, X, Y);
  do
  {
    for (int j = 0; j < 3; j ++) /* T = X*W + Y (NNMUL, NNADD) */
      for (int i = 0; i < 3; i ++)
        T[3*j+i] = X[i]*W[3*j] + X[3+i]*W[3*j+1] + X[6+i]*W[3*j+2];
    for (int k = 0; k < 9; k ++) T[k] = T[k] + Y[k];
    if (orc_dgesv (3, T, ipiv, C)) return -1;
    R[0] -= C[0]; R[1] -= C[1]; R[2] -= C[2];
    scf_project (friction, cohesion, R, R);
    nvaddmul (B, W, R, U);
    scf_linearize (dynamic, step, friction, restitution, cohesion, gap, V, U, R, C, X, Y);
    merit = sqrt (dot3 (C, C));
  } while (merit > epsilon && ++iter < maxiter);

  return iter;
}

/* ---- bilateral constraints (dbs.c:328-450, mrf.c:88-137), kinds as dom.h:98:
 * 1 FIXPNT, 2 FIXDIR, 3 VELODIR, 4 VELODIR3, 5 RIGLNK; Z[4] per row: VELODIR
 * Z[0], VELODIR3 Z[0..2], RIGLNK the local link vector (base^T Z) and length */
static const int *g_kind = NULL;
static const double *g_Z = NULL;

void orc_gs_set_kinds (const int *kind, const double *Z)
{
  g_kind = kind;
  g_Z = Z;
}

static int orc_bilateral (int kind, const double *Z, int dynamic, double step, double epsilon, int maxiter,
                          const double *W, const double *B, const double *V, double *U, double *R)
{
  double A[9];
  switch (kind)
  {
  case 1: /* fixpnt, dbs.c:328-350 */
    for (int q = 0; q < 9; q ++) A[q] = W[q];
    for (int q = 0; q < 3; q ++) U[q] = dynamic ? V[q] * -1.0 : 0.0;
    for (int q = 0; q < 3; q ++) R[q] = U[q] - B[q];
    return orc_dposv (3, A, R) ? -1 : 0;
  case 2: /* fixdir, dbs.c:352-369 */
  case 3: /* velodir, dbs.c:371-379 */
    R[0] = 0.0;
    R[1] = 0.0;
    if (kind == 3) R[2] = (Z[0] - B[2]) / W[8];
    else R[2] = dynamic ? -(V[2] + B[2]) / W[8] : -B[2] / W[8];
    for (int q = 0; q < 3; q ++) U[q] = B[q] + R[2] * W[6+q];
    return 0;
  case 4: /* velodir3, dbs.c:381-394 */
    for (int q = 0; q < 9; q ++) A[q] = W[q];
    for (int q = 0; q < 3; q ++) U[q] = Z[q];
    for (int q = 0; q < 3; q ++) R[q] = U[q] - B[q];
    return orc_dposv (3, A, R) ? -1 : 0;
  case 5: /* riglnk, dbs.c:396-450 */
  {
    double h = dynamic ? 0.5 * step : step, len = Z[3], l = 0.0, error, X[2], C[3], D[4], L[4];
    int ipiv[2], iter = 0;
    R[0] = R[1] = 0.0;
    do
    {
      for (int q = 0; q < 3; q ++) C[q] = B[q] + R[2] * W[6+q];
      for (int q = 0; q < 3; q ++) D[q] = Z[q] + h * C[q];
      X[1] = dot3 (D, D) - len*len;
      D[3] = dot3 (W+6, D) * 2.0 * h;
      X[0] = W[8]*R[2] + l*D[3];
      L[0] = W[8]; L[2] = D[3];
      L[1] = D[3]; L[3] = 0.0;
      if (orc_dgesv (2, L, ipiv, X)) return -1;
      R[2] -= X[0];
      l -= X[1];
      error = sqrt ((X[0]*X[0] + X[1]*X[1])/(R[2]*R[2] + l*l));
    } while (error > epsilon && ++iter < maxiter);
    if (dynamic && iter >= maxiter) { R[2] = -B[2] / W[8]; iter = 0; }
    for (int q = 0; q < 3; q ++) U[q] = B[q] + R[2] * W[6+q];
    return iter;
  }
  }
  return -1;
}

static double orc_bilateral_merit (int kind, const double *Z, double gap, int dynamic, double step,
                                   const double *A, const double *V, const double *U)
{
  double P[3], Q[3];
  switch (kind)
  {
  case 1: case 4: /* FIXPNT, VELODIR3 */
    for (int q = 0; q < 3; q ++) P[q] = kind == 1 ? (dynamic ? U[q] + V[q] : U[q]) : Z[q] - U[q];
    Q[0] = A[0]*P[0] + A[3]*P[1] + A[6]*P[2];
    Q[1] = A[1]*P[0] + A[4]*P[1] + A[7]*P[2];
    Q[2] = A[2]*P[0] + A[5]*P[1] + A[8]*P[2];
    return dot3 (Q, P);
  case 2: P[2] = dynamic ? U[2] + V[2] : U[2]; break;
  case 3: P[2] = Z[0] - U[2]; break;
  case 5: P[2] = gap/(step * (dynamic ? 0.5 : 1.0)) + U[2]; break;
  default: return 0.0;
  }
  Q[2] = A[8] * P[2];
  return Q[2] * P[2];
}

int orc_diagonal_solve (int diagsolver, double diagepsilon, int diagmaxiter, int dynamic, double step,
                        double friction, double restitution, double cohesion, double gap, double rho,
                        const double *W, const double *B, const double *V, double *U, double *R)
{
  switch (diagsolver) /* dbs.c:507-521 */
  {
  case DS_PG: return projected_gradient (dynamic, diagepsilon, diagmaxiter, step, friction, restitution, cohesion, gap, rho, W, B, V, U, R);
  case DS_DSF: return de_saxce_feng (dynamic, diagepsilon, diagmaxiter, step, friction, restitution, cohesion, gap, rho, W, B, V, U, R);
  case DS_SSN: return semismooth_newton (dynamic, diagepsilon, diagmaxiter, step, friction, restitution, cohesion, gap, rho, W, B, V, U, R);
  case DS_PN: return projected_newton (diagepsilon, diagmaxiter, dynamic, step, friction, restitution, cohesion, gap, W, B, V, U, R);
  }
  return 0;
}

double orc_merit (int n, const int *adjptr, const int *adjcol, const double *Woff,
                  const double *W, const double *A, const double *B, const double *V,
                  const double *gap, const double *friction, const double *restitution, const double *cohesion,
                  const double *R, double *U, double *conmerit, double free_energy, int dynamic, double step)
{
  double up, lo, P[3], Q[3], sum = 0.0;

  lo = free_energy < DBL_EPSILON ? 1.0 : free_energy; /* mrf.c:45 */
  for (int i = 0; i < n; i ++) /* mrf.c:51-169 */
  {
    double *Ui = U + 3*i;
    nvaddmul (B + 3*i, W + 9*i, R + 3*i, Ui);
    for (int k = adjptr[i]; k < adjptr[i+1]; k ++)
      nvaddmul (Ui, Woff + 9*(size_t)k, R + 3*adjcol[k], Ui);
    if (g_kind && g_kind[i])
      up = orc_bilateral_merit (g_kind[i], g_Z + 4*i, gap[i], dynamic, step, A + 9*i, V + 3*i, Ui);
    else
    {
      scf_linearize (dynamic, step, friction[i], restitution[i], cohesion[i], gap[i], V + 3*i, Ui, R + 3*i, P, NULL, NULL);
      const double *Ai = A + 9*i; /* NVMUL (A, P, Q) */
      Q[0] = Ai[0]*P[0] + Ai[3]*P[1] + Ai[6]*P[2];
      Q[1] = Ai[1]*P[0] + Ai[4]*P[1] + Ai[7]*P[2];
      Q[2] = Ai[2]*P[0] + Ai[5]*P[1] + Ai[8]*P[2];
      up = dot3 (Q, P);
    }
    if (conmerit) conmerit[i] = up;
    sum += up;
  }
  sum *= 0.5; /* mrf.c:176 */
  lo = (lo == 0 ? 1 : lo);
  if (conmerit) for (int i = 0; i < n; i ++) conmerit[i] /= lo; /* mrf.c:179-182 */
  return sum / lo;
}

int orc_gs_solve (int n, const int *adjptr, const int *adjcol, const double *Woff,
                  const double *W, const double *A, const double *rho, const double *B, const double *V,
                  const double *gap, const double *friction, const double *restitution, const double *cohesion,
                  double *R, double *U, double *conmerit,
                  double free_energy, int dynamic, double step,
                  double epsilon, int maxiter, double meritval, int failure,
                  double diagepsilon, int diagmaxiter, int diagsolver, int reverse,
                  int *out_iters, int *out_error, double *out_merit,
                  double *rerhist, double *merhist, int *out_ncallbacks)
{
  double error = 0.0, merit = 0.0;
  int iters = 0, gserror = GS_OK, ncallbacks = 0, thrown = 0;
  int nomerit = meritval >= 1.0 ? 1 : 0; /* bgs.c:927 */
  int backward = reverse && n > 0;

  do
  {
    double errup = 0.0, errlo = 0.0;
    int odd = backward && (iters % 2);

    for (int s = 0; s < n; s ++) /* bgs.c:950: forward and backward alternately */
    {
      int i = odd ? n - 1 - s : s;
      double R0[3], Bp[3];
      double *Ri = R + 3*i, *Ui = U + 3*i;
      int diagiters;

      Bp[0] = B[3*i]; Bp[1] = B[3*i+1]; Bp[2] = B[3*i+2];
      for (int k = adjptr[i]; k < adjptr[i+1]; k ++) /* bgs.c:957-963 */
        nvaddmul (Bp, Woff + 9*(size_t)k, R + 3*adjcol[k], Bp);

      R0[0] = Ri[0]; R0[1] = Ri[1]; R0[2] = Ri[2];

      int kind = g_kind ? g_kind[i] : 0;
      if (kind)
        diagiters = orc_bilateral (kind, g_Z + 4*i, dynamic, step, diagepsilon, diagmaxiter, W + 9*i, Bp, V + 3*i,
                                   Ui, Ri);
      else
        diagiters = orc_diagonal_solve (diagsolver, diagepsilon, diagmaxiter, dynamic, step, friction[i],
                      restitution[i], cohesion[i], gap[i], rho[i], W + 9*i, Bp, V + 3*i, Ui, Ri);

      if (diagiters >= diagmaxiter || diagiters < 0) /* bgs.c:971-1013 */
      {
        gserror = diagiters < 0 ? GS_DIAGONAL_FAILED : GS_DIAGONAL_DIVERGED;
        if (failure == FAIL_CONTINUE && kind) /* no fallback chain outside contacts */
        {
          Ri[0] = R0[0]; Ri[1] = R0[1]; Ri[2] = R0[2];
        }
        else if (failure == FAIL_CONTINUE)
        {
          static const int chain[4] = {DS_SSN, DS_PG, DS_DSF, DS_PN};
          for (int t = 0; t < 4; t ++)
          {
            if (chain[t] != diagsolver)
            {
              Ri[0] = R0[0]; Ri[1] = R0[1]; Ri[2] = R0[2];
              diagiters = orc_diagonal_solve (chain[t], diagepsilon, diagmaxiter, dynamic, step, friction[i],
                            restitution[i], cohesion[i], gap[i], rho[i], W + 9*i, Bp, V + 3*i, Ui, Ri);
              if (diagiters < diagmaxiter && diagiters >= 0) break;
            }
          }
          if (diagiters >= diagmaxiter || diagiters < 0)
          {
            Ri[0] = R0[0]; Ri[1] = R0[1]; Ri[2] = R0[2];
          }
        }
        else if (failure == FAIL_EXIT)
        {
          thrown = ORC_ERR_GAUSS_SEIDEL_DIAGONAL_DIVERGED;
          goto out;
        }
        else ncallbacks ++;
      }

      R0[0] = Ri[0] - R0[0]; R0[1] = Ri[1] - R0[1]; R0[2] = Ri[2] - R0[2];
      errup += dot3 (R0, R0);
      errlo += dot3 (Ri, Ri);
    }

    if (!nomerit) merit = orc_merit (n, adjptr, adjcol, Woff, W, A, B, V, gap, friction, restitution, cohesion,
                                     R, U, conmerit, free_energy, dynamic, step);

    error = sqrt (errup) / sqrt (errlo == 0.0 ? 1.0 : errlo);
    if (rerhist) rerhist[iters] = error;
    if (merhist) merhist[iters] = merit;
  }
  while (++ iters < maxiter && (error > epsilon || merit > meritval));

  if (iters >= maxiter) /* bgs.c:1053-1068 */
  {
    gserror = GS_DIVERGED;
    if (failure == FAIL_EXIT) thrown = ORC_ERR_GAUSS_SEIDEL_DIVERGED;
    else if (failure == FAIL_CALLBACK) ncallbacks ++;
  }

out:
  *out_iters = iters;
  *out_error = gserror;
  *out_merit = merit;
  if (out_ncallbacks) *out_ncallbacks = ncallbacks;
  return thrown;
}
