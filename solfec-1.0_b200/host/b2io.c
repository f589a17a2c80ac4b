/* b2io.c -- the local dynamics' interchange formats (host C):
 *
 *   LOCDYN_W_MatrixMarket  ldy.c:1005-1052 -> b2gs_write_w_matrix_market,
 *                                            b2gs_locdyn_w_matrix_market
 *   LOCDYN_Dump            ldy.c:892-1002  -> b2gs_write_locdyn_dump,
 *                                            b2gs_locdyn_dump
 *
 * The text is the reference's, character for character: the same printf
 * formats, rows in list order, and in the dump the off-diagonal blocks of one
 * neighbour summed and the neighbours ordered as the reference's map orders
 * them (dumpcmp, ldy.c:330-361: spatial point, sorted body ids, kind, normal).
 * The b2gs_write_* functions take host arrays in caller (list) order; the
 * b2gs_locdyn_* functions download an assembled local dynamics and its
 * current state from the device first. Only contact rows exist on this path,
 * so every row's kind is CONTACT.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/b2_device.h"
#include "../../include/solfec_b200.h"

int b2gs_write_w_matrix_market (const char *path, int n, const double *W, const int *adjptr, const int *adjcol,
                                const double *Woff)
{
  FILE *f;
  long long nnz;
  if (!path || n < 0 || (n > 0 && (!W || !adjptr))) return B2DEV_EINVAL;
  nnz = 9LL * n + 9LL * (n > 0 ? adjptr[n] : 0);
  if (!(f = fopen (path, "w"))) return B2DEV_EINVAL;
  fprintf (f, "%%%%MatrixMarket matrix coordinate real general\n");
  fprintf (f, "%d  %d  %lld\n", 3 * n, 3 * n, nnz);
  for (int r = 0; r < n; r ++)
  {
    const int row = 3 * r + 1;  /* con->num of the r-th row of the list */
    for (int i = 0; i < 3; i ++)
      for (int j = 0; j < 3; j ++) fprintf (f, "%d  %d  %.15g\n", row + i, row + j, W[9 * (size_t) r + 3 * j + i]);
    for (int k = adjptr[r]; k < adjptr[r + 1]; k ++)
    {
      const int col = 3 * adjcol[k] + 1;
      for (int i = 0; i < 3; i ++)
        for (int j = 0; j < 3; j ++) fprintf (f, "%d  %d  %.15g\n", row + i, col + j, Woff[9 * (size_t) k + 3 * j + i]);
    }
  }
  return fclose (f) == 0 ? B2DEV_OK : B2DEV_EINVAL;
}

/* the reference's dump order of two constraints (dumpcmp, ldy.c:330-361) */
typedef struct { const double *point, *base; const int *mid, *sid; } dumpkey;

static int dump_cmp (const dumpkey *K, int a, int b)
{
  for (int i = 0; i < 3; i ++)
  {
    if (K->point [3 * a + i] < K->point [3 * b + i]) return -1;
    if (K->point [3 * a + i] > K->point [3 * b + i]) return 1;
  }
  int ia [2] = {K->mid [a], K->sid [a]}, ib [2] = {K->mid [b], K->sid [b]};
  int sa [2] = {ia [0] < ia [1] ? ia [0] : ia [1], ia [0] < ia [1] ? ia [1] : ia [0]};
  int sb [2] = {ib [0] < ib [1] ? ib [0] : ib [1], ib [0] < ib [1] ? ib [1] : ib [0]};
  for (int i = 0; i < 2; i ++)
  {
    if (sa [i] < sb [i]) return -1;
    if (sa [i] > sb [i]) return 1;
  }
  /* same kind (CONTACT) */
  for (int i = 6; i < 9; i ++)
  {
    if (K->base [9 * a + i] < K->base [9 * b + i]) return -1;
    if (K->base [9 * a + i] > K->base [9 * b + i]) return 1;
  }
  return 0;
}

static void print_head (FILE *f, const char *lead, const double *p, int mid, int sid, const double *base, const double *W)
{
  fprintf (f, "%sCONTACT (%.6g, %.6g, %.6g) (%d, %d) [%.6g, %.6g, %.6g, %.6g, %.6g, %.6g, %.6g, %.6g, %.6g] "
              "[%.6g, %.6g, %.6g, %.6g, %.6g, %.6g, %.6g, %.6g, %.6g]",
    lead, p [0], p [1], p [2], mid, sid,
    base [0], base [1], base [2], base [3], base [4], base [5], base [6], base [7], base [8],
    W [0], W [1], W [2], W [3], W [4], W [5], W [6], W [7], W [8]);
}

int b2gs_write_locdyn_dump (const char *path, int n, const double *point, const int *master_id, const int *slave_id,
                            const double *base, const double *W, const double *B, const double *V, const double *U,
                            const double *R, const int *adjptr, const int *adjcol, const double *Woff)
{
  dumpkey K = {point, base, master_id, slave_id};
  FILE *f;
  int maxdeg = 0, *nb = NULL, *ord = NULL;
  double *sum = NULL;
  if (!path || n < 0) return B2DEV_EINVAL;
  if (n > 0 && (!point || !master_id || !slave_id || !base || !W || !B || !V || !U || !R || !adjptr))
    return B2DEV_EINVAL;
  for (int r = 0; r < n; r ++) if (adjptr [r + 1] - adjptr [r] > maxdeg) maxdeg = adjptr [r + 1] - adjptr [r];
  nb = malloc (sizeof (int) * (maxdeg + 1));
  ord = malloc (sizeof (int) * (maxdeg + 1));
  sum = malloc (sizeof (double) * 9 * (maxdeg + 1));
  if (!nb || !ord || !sum || !(f = fopen (path, "w"))) { free (nb); free (ord); free (sum); return B2DEV_EINVAL; }
  for (int r = 0; r < n; r ++)
  {
    const double *w = W + 9 * (size_t) r, *b = B + 3 * (size_t) r, *v = V + 3 * (size_t) r;
    const double *u = U + 3 * (size_t) r, *rr = R + 3 * (size_t) r;
    int m = 0;
    print_head (f, "", point + 3 * (size_t) r, master_id [r], slave_id [r], base + 9 * (size_t) r, w);
    fprintf (f, " (%.6g, %.6g, %.6g) (%.6g, %.6g, %.6g) (%.6g, %.6g, %.6g) (%.6g, %.6g, %.6g)",
             b [0], b [1], b [2], v [0], v [1], v [2], u [0], u [1], u [2], rr [0], rr [1], rr [2]);
    /* the row's blocks summed per neighbour, in the list order of the blocks (NNADD onto zero) */
    for (int k = adjptr [r]; k < adjptr [r + 1]; k ++)
    {
      int q = 0;
      while (q < m && dump_cmp (&K, nb [q], adjcol [k]) != 0) q ++;
      if (q == m) { nb [m] = adjcol [k]; memset (sum + 9 * m, 0, sizeof (double) * 9); m ++; }
      for (int e = 0; e < 9; e ++) sum [9 * q + e] = sum [9 * q + e] + Woff [9 * (size_t) k + e];
    }
    /* neighbours in the map's order (insertion sort on dumpcmp; rows have a few tens of neighbours) */
    for (int q = 0; q < m; q ++)
    {
      int p = q;
      while (p > 0 && dump_cmp (&K, nb [ord [p - 1]], nb [q]) > 0) { ord [p] = ord [p - 1]; p --; }
      ord [p] = q;
    }
    for (int t = 0; t < m; t ++)
    {
      const int q = ord [t], c = nb [q];
      print_head (f, " => ", point + 3 * (size_t) c, master_id [c], slave_id [c], base + 9 * (size_t) c, sum + 9 * q);
    }
    fprintf (f, "\n");
  }
  free (nb); free (ord); free (sum);
  return fclose (f) == 0 ? B2DEV_OK : B2DEV_EINVAL;
}

/* the assembled local dynamics in caller order, from the device */
typedef struct { int n; long long K; double *W, *A, *rho, *B, *V, *Woff, *R, *U; int *adjptr, *adjcol; } ldydata;

static void ldy_free (ldydata *d)
{
  free (d->W); free (d->A); free (d->rho); free (d->B); free (d->V); free (d->Woff); free (d->R); free (d->U);
  free (d->adjptr); free (d->adjcol);
}

static int ldy_download (b2gs_locdyn *ldy, ldydata *d, int with_state)
{
  int nc, rc;
  double fe;
  memset (d, 0, sizeof *d);
  if ((rc = b2gs_locdyn_sizes (ldy, &d->n, &d->K, &nc, &fe)) != B2DEV_OK) return rc;
  const size_t n1 = (size_t) d->n + 1, k1 = (size_t) d->K + 1;
  d->W = malloc (sizeof (double) * 9 * n1); d->A = malloc (sizeof (double) * 9 * n1);
  d->rho = malloc (sizeof (double) * n1); d->B = malloc (sizeof (double) * 3 * n1);
  d->V = malloc (sizeof (double) * 3 * n1); d->Woff = malloc (sizeof (double) * 9 * k1);
  d->R = malloc (sizeof (double) * 3 * n1); d->U = malloc (sizeof (double) * 3 * n1);
  d->adjptr = malloc (sizeof (int) * n1); d->adjcol = malloc (sizeof (int) * k1);
  if (!d->W || !d->A || !d->rho || !d->B || !d->V || !d->Woff || !d->R || !d->U || !d->adjptr || !d->adjcol)
  { ldy_free (d); return B2DEV_EINVAL; }
  rc = b2dev_get_locdyn (b2gs_locdyn_device (ldy), d->W, d->A, d->rho, d->B, d->V, d->adjptr, d->adjcol, d->Woff, &fe);
  if (rc == B2DEV_OK && with_state) rc = b2gs_locdyn_get_state (ldy, d->R, d->U, NULL, 0);
  if (rc != B2DEV_OK) ldy_free (d);
  return rc;
}

int b2gs_locdyn_w_matrix_market (b2gs_locdyn *ldy, const char *path)
{
  ldydata d;
  int rc;
  if (!ldy || !path) return B2DEV_EINVAL;
  if ((rc = ldy_download (ldy, &d, 0)) != B2DEV_OK) return rc;
  rc = b2gs_write_w_matrix_market (path, d.n, d.W, d.adjptr, d.adjcol, d.Woff);
  ldy_free (&d);
  return rc;
}

int b2gs_locdyn_dump (b2gs_locdyn *ldy, const char *path, const double *point, const int *master_id,
                      const int *slave_id, const double *base)
{
  ldydata d;
  int rc;
  if (!ldy || !path) return B2DEV_EINVAL;
  if ((rc = ldy_download (ldy, &d, 1)) != B2DEV_OK) return rc;
  rc = b2gs_write_locdyn_dump (path, d.n, point, master_id, slave_id, base, d.W, d.B, d.V, d.U, d.R, d.adjptr,
                               d.adjcol, d.Woff);
  ldy_free (&d);
  return rc;
}
