/*
 * oracle_ldy.c -- TEST INFRASTRUCTURE. Not part of the product.
 *
 * CPU restatement of the local-dynamics assembly for rigid bodies:
 *   rig_operator_H         bod.c:216-229
 *   BODY_Local_Velo        bod.c:1817-1844 (RIG and OBS)
 *   BODY_Gen_To_Loc_Op.    bod.c:1846-1871 (OBS contributes H = 0 to contacts)
 *   update_V_and_B         ldy.c:364-474
 *   LOCDYN_Insert          ldy.c:492-568 (adjacency through non-obstacle bodies)
 *   LOCDYN_Update_Begin    ldy.c:626-876 (W_ii, rho, A, free energy, W_ij,
 *                          lower triangle as the transposed upper block)
 * and the host colouring that the device Jones-Plassmann kernel must match.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "oracle.h"
#include "lu_small.h"

/* H (3x6, column-major) of a rigid body at referential point X in frame base
 * (bod.c:216-229): A = X - X0, S = skew(A), T = R*S^T, H = [base^T*T | base^T]. */
static void rig_H (const double *R, const double *X0, const double *base, const double *X, double *H)
{
  double A[3], S[9], T[9];

  A[0] = X[0] - X0[0]; A[1] = X[1] - X0[1]; A[2] = X[2] - X0[2];
  S[0] = 0; S[1] = A[2]; S[2] = -A[1];          /* VECSKEW alg.h:1060 */
  S[3] = -A[2]; S[4] = 0; S[5] = A[0];
  S[6] = A[1]; S[7] = -A[0]; S[8] = 0;
  for (int j = 0; j < 3; j ++)                  /* T = R S^T (NTMUL) */
    for (int i = 0; i < 3; i ++)
      T[3*j+i] = R[i]*S[j] + R[3+i]*S[3+j] + R[6+i]*S[6+j];
  for (int j = 0; j < 3; j ++)                  /* H[0..8] = base^T T (TNMUL) */
    for (int i = 0; i < 3; i ++)
      H[3*j+i] = base[3*i]*T[3*j] + base[3*i+1]*T[3*j+1] + base[3*i+2]*T[3*j+2];
  for (int j = 0; j < 3; j ++)                  /* H[9..17] = base^T (TNCOPY) */
    for (int i = 0; i < 3; i ++)
      H[9 + 3*j+i] = base[3*i+j];
}

/* y = H x for a 3x6 H, accumulated column by column (BLAS dgemv 'N'). */
static void h_times (const double *H, const double *x, double *y)
{
  y[0] = y[1] = y[2] = 0.0;
  for (int j = 0; j < 6; j ++)
  {
    double t = x[j];
    y[0] += t * H[3*j];
    y[1] += t * H[3*j+1];
    y[2] += t * H[3*j+2];
  }
}

/* P (6x3) = Minv * H^T with Minv = blockdiag(jinv, (1/m) I) (bod.c:232-258). */
static void minv_ht (const double *jinv, double minv, const double *H, double *P)
{
  for (int c = 0; c < 3; c ++)
  {
    double h0 = H[c], h1 = H[3+c], h2 = H[6+c];          /* row c of H, angular part */
    P[6*c+0] = jinv[0]*h0 + jinv[3]*h1 + jinv[6]*h2;
    P[6*c+1] = jinv[1]*h0 + jinv[4]*h1 + jinv[7]*h2;
    P[6*c+2] = jinv[2]*h0 + jinv[5]*h1 + jinv[8]*h2;
    P[6*c+3] = minv * H[9+c];
    P[6*c+4] = minv * H[12+c];
    P[6*c+5] = minv * H[15+c];
  }
}

/* C (3x3) += L (3x6) * P (6x3), P stored column-major with leading dim 6. */
static void hp_add (const double *L, const double *P, double *C)
{
  for (int j = 0; j < 3; j ++)
    for (int i = 0; i < 3; i ++)
    {
      double s = 0.0;
      for (int k = 0; k < 6; k ++) s += L[3*k+i] * P[6*j+k];
      C[3*j+i] += s;
    }
}

/* Largest eigenvalue of a symmetric 3x3 matrix by cyclic Jacobi rotations
 * (Golub & Van Loan, Alg. 8.5.3); stands in for LAPACK dsyev (ldy.c:719-724). */
static double sym3_max_eig (const double *W)
{
  double a[3][3];
  for (int j = 0; j < 3; j ++) for (int i = 0; i < 3; i ++) a[i][j] = 0.5 * (W[3*j+i] + W[3*i+j]);
  for (int sweep = 0; sweep < 32; sweep ++)
  {
    double off = a[0][1]*a[0][1] + a[0][2]*a[0][2] + a[1][2]*a[1][2];
    double dia = a[0][0]*a[0][0] + a[1][1]*a[1][1] + a[2][2]*a[2][2];
    if (off <= 1e-36 * dia || off == 0.0) break;
    for (int p = 0; p < 2; p ++)
      for (int q = p + 1; q < 3; q ++)
      {
        if (a[p][q] == 0.0) continue;
        double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs (theta) + sqrt (theta*theta + 1.0));
        double c = 1.0 / sqrt (t*t + 1.0), s = t * c;
        for (int k = 0; k < 3; k ++) /* A = J^T A J, columns then rows */
        {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c*akp - s*akq;
          a[k][q] = s*akp + c*akq;
        }
        for (int k = 0; k < 3; k ++)
        {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c*apk - s*aqk;
          a[q][k] = s*apk + c*aqk;
        }
        a[p][q] = a[q][p] = 0.0;
      }
  }
  double m = a[0][0];
  if (a[1][1] > m) m = a[1][1];
  if (a[2][2] > m) m = a[2][2];
  return m;
}

/* A = W^-1 by three LU solves (stands in for MX_Inverse, mtx.c:1599-1626). */
static void inv3 (const double *W, double *A)
{
  for (int j = 0; j < 3; j ++)
  {
    double a[9], b[3] = {0, 0, 0};
    int ipiv[3];
    memcpy (a, W, sizeof a);
    b[j] = 1.0;
    orc_dgesv (3, a, ipiv, b);
    A[3*j] = b[0]; A[3*j+1] = b[1]; A[3*j+2] = b[2];
  }
}

/* rows of every non-obstacle body, ascending; returns CSR over bodies */
static void body_rows (int nbod, const int *obstacle, int ncon, const int *master, const int *slave, int **pptr, int **prow)
{
  int *ptr = calloc ((size_t) nbod + 1, sizeof (int));
  for (int i = 0; i < ncon; i ++)
  {
    if (master[i] >= 0 && !obstacle[master[i]]) ptr[master[i]+1] ++;
    if (slave[i] >= 0 && !obstacle[slave[i]]) ptr[slave[i]+1] ++;
  }
  for (int b = 0; b < nbod; b ++) ptr[b+1] += ptr[b];
  int *fill = malloc (((size_t) nbod + 1) * sizeof (int));
  memcpy (fill, ptr, ((size_t) nbod + 1) * sizeof (int));
  int *row = malloc (((size_t) ptr[nbod] + 1) * sizeof (int));
  for (int i = 0; i < ncon; i ++) /* ascending i => ascending rows per body */
  {
    if (master[i] >= 0 && !obstacle[master[i]]) row[fill[master[i]] ++] = i;
    if (slave[i] >= 0 && !obstacle[slave[i]]) row[fill[slave[i]] ++] = i;
  }
  free (fill);
  *pptr = ptr;
  *prow = row;
}

int64_t orc_count_blocks (int nbod, const int *obstacle, int ncon, const int *master, const int *slave, int *adjptr)
{
  int *bptr, *brow;
  body_rows (nbod, obstacle, ncon, master, slave, &bptr, &brow);
  int64_t total = 0;
  adjptr[0] = 0;
  for (int i = 0; i < ncon; i ++)
  {
    int64_t d = 0;
    if (master[i] >= 0 && !obstacle[master[i]]) d += bptr[master[i]+1] - bptr[master[i]] - 1;
    if (slave[i] >= 0 && !obstacle[slave[i]]) d += bptr[slave[i]+1] - bptr[slave[i]] - 1;
    total += d;
    adjptr[i+1] = (int) total;
  }
  free (bptr);
  free (brow);
  return total;
}

int orc_assemble (int nbod, const double *rot, const double *x0, const double *jinv, const double *minv,
                  const double *velo, const double *velo0, const int *obstacle,
                  int ncon, const int *master, const int *slave, const double *mpnt, const double *spnt,
                  const double *base, double step,
                  double *W, double *A, double *rho, double *B, double *V, double *free_energy,
                  const int *adjptr, int *adjcol, int *adjbod, double *Woff)
{
  for (int i = 0; i < ncon; i ++) if (master[i] == slave[i]) return -1; /* self-contact: outside the rigid contact path */

  double *Hm = calloc ((size_t) ncon * 18, sizeof (double)), *Hs = calloc ((size_t) ncon * 18, sizeof (double));
  double *Pm = calloc ((size_t) ncon * 18, sizeof (double)), *Ps = calloc ((size_t) ncon * 18, sizeof (double));
  double fe = 0.0;

  for (int i = 0; i < ncon; i ++)
  {
    const double *bs = base + 9*i;
    double H[18], X[3], *Wi = W + 9*i, *Bi = B + 3*i, *Vi = V + 3*i;
    int m = master[i], s = slave[i];

    /* update_V_and_B (ldy.c:364-395): V = H_m u_m(t) - H_s u_s(t), B likewise with the free velocity */
    Vi[0] = Vi[1] = Vi[2] = 0.0;
    Bi[0] = Bi[1] = Bi[2] = 0.0;
    rig_H (rot + 9*m, x0 + 3*m, bs, mpnt + 3*i, H);
    h_times (H, velo0 + 6*m, X); Vi[0] += X[0]; Vi[1] += X[1]; Vi[2] += X[2];
    h_times (H, velo + 6*m, X);  Bi[0] += X[0]; Bi[1] += X[1]; Bi[2] += X[2];
    if (!obstacle[m]) { memcpy (Hm + 18*i, H, sizeof H); minv_ht (jinv + 9*m, minv[m], H, Pm + 18*i); }
    if (s >= 0)
    {
      rig_H (rot + 9*s, x0 + 3*s, bs, spnt + 3*i, H);
      h_times (H, velo0 + 6*s, X); Vi[0] -= X[0]; Vi[1] -= X[1]; Vi[2] -= X[2];
      h_times (H, velo + 6*s, X);  Bi[0] -= X[0]; Bi[1] -= X[1]; Bi[2] -= X[2];
      if (!obstacle[s])
      {
        for (int k = 0; k < 18; k ++) H[k] = -H[k]; /* MX_Scale (sH, -1) ldy.c:685 */
        memcpy (Hs + 18*i, H, sizeof H);
        minv_ht (jinv + 9*s, minv[s], H, Ps + 18*i);
      }
    }

    /* W_ii = h (H_m M_m^-1 H_m^T + H_s M_s^-1 H_s^T) (ldy.c:662-715) */
    for (int k = 0; k < 9; k ++) Wi[k] = 0.0;
    hp_add (Hm + 18*i, Pm + 18*i, Wi);
    if (s >= 0) hp_add (Hs + 18*i, Ps + 18*i, Wi);
    for (int k = 0; k < 9; k ++) Wi[k] *= step;

    rho[i] = 1.0 / sym3_max_eig (Wi);  /* ldy.c:719-724 */
    inv3 (Wi, A + 9*i);                /* ldy.c:726-727 */
    const double *Ai = A + 9*i;        /* free energy ldy.c:729-736 */
    double Q0 = Ai[0]*Bi[0] + Ai[3]*Bi[1] + Ai[6]*Bi[2];
    double Q1 = Ai[1]*Bi[0] + Ai[4]*Bi[1] + Ai[7]*Bi[2];
    double Q2 = Ai[2]*Bi[0] + Ai[5]*Bi[1] + Ai[8]*Bi[2];
    fe += Q0*Bi[0] + Q1*Bi[1] + Q2*Bi[2];
  }
  *free_energy = 0.5 * fe;

  /* adjacency (LOCDYN_Insert order restated as: master body, then slave body, ascending rows) */
  int *bptr, *brow;
  body_rows (nbod, obstacle, ncon, master, slave, &bptr, &brow);
  for (int i = 0; i < ncon; i ++)
  {
    int k = adjptr[i];
    int bods[2] = {master[i], slave[i]};
    for (int t = 0; t < 2; t ++)
    {
      int b = bods[t];
      if (b < 0 || obstacle[b]) continue;
      for (int q = bptr[b]; q < bptr[b+1]; q ++)
        if (brow[q] != i) { adjcol[k] = brow[q]; adjbod[k] = b; k ++; }
    }
  }

  /* off-diagonal blocks: upper triangle W_ij = h left_i right_j (ldy.c:738-794), lower = transpose (ldy.c:829-844) */
  for (int i = 0; i < ncon; i ++)
    for (int k = adjptr[i]; k < adjptr[i+1]; k ++)
    {
      int j = adjcol[k], b = adjbod[k];
      if (j < i) continue;
      const double *left = (b == master[i]) ? Hm + 18*i : Hs + 18*i;
      const double *right = (b == master[j]) ? Pm + 18*j : Ps + 18*j;
      double *Wk = Woff + 9*(size_t)k;
      for (int q = 0; q < 9; q ++) Wk[q] = 0.0;
      hp_add (left, right, Wk);
      for (int q = 0; q < 9; q ++) Wk[q] *= step;
    }
  for (int i = 0; i < ncon; i ++)
    for (int k = adjptr[i]; k < adjptr[i+1]; k ++)
    {
      int j = adjcol[k], b = adjbod[k];
      if (j > i) continue;
      int q;
      for (q = adjptr[j]; q < adjptr[j+1] && !(adjcol[q] == i && adjbod[q] == b); q ++);
      const double *U = Woff + 9*(size_t)q;
      double *Wk = Woff + 9*(size_t)k;
      Wk[0] = U[0]; Wk[1] = U[3]; Wk[2] = U[6];   /* TNCOPY */
      Wk[3] = U[1]; Wk[4] = U[4]; Wk[5] = U[7];
      Wk[6] = U[2]; Wk[7] = U[5]; Wk[8] = U[8];
    }

  free (bptr); free (brow);
  free (Hm); free (Hs); free (Pm); free (Ps);
  return 0;
}

uint64_t orc_jp_priority (uint64_t seed, int i)
{
  uint64_t z = seed + 0x9E3779B97F4A7C15ull * ((uint64_t) i + 1ull); /* splitmix64 finaliser */
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return (z & 0xFFFFFFFF00000000ull) | (uint64_t) (uint32_t) i;
}

static const uint64_t *sort_keys;
static int by_priority_desc (const void *a, const void *b)
{
  uint64_t x = sort_keys[*(const int*)a], y = sort_keys[*(const int*)b];
  return x < y ? 1 : x > y ? -1 : 0;
}

/* greedy colouring in the given row order (smallest colour no coloured neighbour holds) */
int orc_colour_ordered (int n, const int *adjptr, const int *adjcol, const int *order, int maxcolours, int *colour)
{
  unsigned char *used = calloc ((size_t) maxcolours + 1, 1);
  int ncolours = 0;
  for (int i = 0; i < n; i ++) colour[i] = -1;
  for (int t = 0; t < n; t ++)
  {
    int i = order[t], c;
    for (int k = adjptr[i]; k < adjptr[i+1]; k ++) { int cj = colour[adjcol[k]]; if (cj >= 0) used[cj] = 1; }
    for (c = 0; c < maxcolours && used[c]; c ++);
    if (c >= maxcolours) { ncolours = -1; break; }
    colour[i] = c;
    if (c + 1 > ncolours) ncolours = c + 1;
    for (int k = adjptr[i]; k < adjptr[i+1]; k ++) { int cj = colour[adjcol[k]]; if (cj >= 0) used[cj] = 0; }
  }
  free (used);
  return ncolours;
}

int orc_colour (int n, const int *adjptr, const int *adjcol, uint64_t seed, int maxcolours, int *colour)
{
  uint64_t *key = malloc (((size_t) n + 1) * sizeof (uint64_t));
  int *order = malloc (((size_t) n + 1) * sizeof (int));
  unsigned char *used = calloc ((size_t) maxcolours + 1, 1);
  int ncolours = 0;

  for (int i = 0; i < n; i ++) { key[i] = orc_jp_priority (seed, i); order[i] = i; colour[i] = -1; }
  sort_keys = key;
  qsort (order, (size_t) n, sizeof (int), by_priority_desc);

  for (int t = 0; t < n; t ++)
  {
    int i = order[t], c;
    for (int k = adjptr[i]; k < adjptr[i+1]; k ++)
    {
      int cj = colour[adjcol[k]];
      if (cj >= 0) used[cj] = 1;
    }
    for (c = 0; c < maxcolours && used[c]; c ++);
    if (c >= maxcolours) { ncolours = -1; break; }
    colour[i] = c;
    if (c + 1 > ncolours) ncolours = c + 1;
    for (int k = adjptr[i]; k < adjptr[i+1]; k ++)
    {
      int cj = colour[adjcol[k]];
      if (cj >= 0) used[cj] = 0;
    }
  }

  free (used); free (order); free (key);
  return ncolours;
}
