/*
 * ref_harness.c -- TEST INFRASTRUCTURE (oracle/_ref build). Not part of the product.
 *
 * Flat-array entry into the reference's own serial GAUSS_SEIDEL_Solve
 * (bgs.c:913-1069). It builds the LOCDYN/DIAB/OFFB/CON/DOM/SOLFEC records the
 * solver reads (ldy.h:44-90, dom.h:77-129) from plain arrays, runs the
 * unmodified solver, and copies R, U, per-constraint merit, iterations, error
 * and histories back out.
 *
 * Row order: rows are linked into ldy->dia in array order, so the solver visits
 * them in that order (bgs.c:950). Off-diagonal blocks of row i are linked into
 * dia->adj in the order adjptr[i]..adjptr[i+1]-1 (bgs.c:957 walks that list).
 * Every row is a CONTACT with a SIGNORINI_COULOMB material; the cohesion value
 * passed per row is the product SURFACE_MATERIAL_Cohesion_Get(mat) * area that
 * dbs.c:500 and scf.c:37 form (area is set to 1).
 */
#include <stdlib.h>
#include <string.h>
#include "sol.h"
#include "dom.h"
#include "ldy.h"
#include "bgs.h"
#include "err.h"

static int ncallbacks_seen;
static void count_callback (void *data) { (void)data; ncallbacks_seen ++; }

/* constraint kinds (dom.h:98) and Z[4] per row for the next ref_gs_solve
 * (NULL: every row a contact); each row's base is the identity, so riglnk's
 * base^T Z is Z itself */
static const int *g_kind = NULL;
static const double *g_Z = NULL;

void ref_gs_set_kinds (const int *kind, const double *Z)
{
  g_kind = kind;
  g_Z = Z;
}

int ref_gs_solve (int n, const int *adjptr, const int *adjcol, const double *Woff,
                  const double *W, const double *A, const double *rho, const double *B, const double *V,
                  const double *gap, const double *friction, const double *restitution, const double *cohesion,
                  double *R, double *U, double *conmerit,
                  double free_energy, int dynamic, double step,
                  double epsilon, int maxiter, double meritval, int failure,
                  double diagepsilon, int diagmaxiter, int diagsolver, int reverse,
                  int *out_iters, int *out_error, double *out_merit,
                  double *rerhist, double *merhist, int *out_ncallbacks)
{
  SOLFEC *sol = calloc (1, sizeof (SOLFEC));
  DOM *dom = calloc (1, sizeof (DOM));
  LOCDYN *ldy = calloc (1, sizeof (LOCDYN));
  BODY *bod = calloc (1, sizeof (BODY));
  CON *con = calloc (n > 0 ? n : 1, sizeof (CON));
  DIAB *dia = calloc (n > 0 ? n : 1, sizeof (DIAB));
  SURFACE_MATERIAL *mat = calloc (n > 0 ? n : 1, sizeof (SURFACE_MATERIAL));
  double *state = calloc (n > 0 ? n : 1, sizeof (double));
  int nblk = n > 0 ? adjptr[n] : 0;
  OFFB *blk = calloc (nblk > 0 ? nblk : 1, sizeof (OFFB));
  int thrown = 0;

  sol->kind = GAUSS_SEIDEL_SOLVER;
  dom->solfec = sol;
  dom->dynamic = (short) dynamic;
  dom->step = step;
  dom->verbose = 0;
  dom->ldy = ldy;
  bod->dom = dom;
  ldy->dom = dom;
  ldy->free_energy = free_energy;
  ldy->dia = n > 0 ? &dia[0] : NULL;
  dom->con = n > 0 ? &con[0] : NULL;

  for (int i = 0; i < n; i ++)
  {
    CON *c = &con[i];
    DIAB *d = &dia[i];
    memcpy (c->R, R + 3*i, 3 * sizeof (double));
    memcpy (c->U, U + 3*i, 3 * sizeof (double));
    memcpy (c->V, V + 3*i, 3 * sizeof (double));
    c->dia = d;
    c->gap = gap[i];
    c->area = 1.0;
    c->kind = CONTACT;
    if (g_kind && g_kind[i])
    {
      c->kind = g_kind[i];
      for (int q = 0; q < 4; q ++) c->Z[q] = g_Z[4*i + q];
      for (int q = 0; q < 9; q ++) c->base[q] = (q % 4 == 0) ? 1.0 : 0.0;
    }
    mat[i].model = SIGNORINI_COULOMB;
    mat[i].friction = friction[i];
    mat[i].restitution = restitution[i];
    state[i] = cohesion[i];
    c->mat.base = &mat[i];
    c->mat.state = &state[i];
    c->master = bod;
    c->slave = bod;
    c->id = (unsigned) i + 1;
    c->prev = i > 0 ? &con[i-1] : NULL;
    c->next = i + 1 < n ? &con[i+1] : NULL;

    d->R = c->R;
    d->U = c->U;
    d->V = c->V;
    memcpy (d->W, W + 9*i, 9 * sizeof (double));
    memcpy (d->A, A + 9*i, 9 * sizeof (double));
    memcpy (d->B, B + 3*i, 3 * sizeof (double));
    d->rho = rho[i];
    d->con = c;
    d->p = i > 0 ? &dia[i-1] : NULL;
    d->n = i + 1 < n ? &dia[i+1] : NULL;
    d->adj = NULL;
    for (int k = adjptr[i+1] - 1; k >= adjptr[i]; k --) /* prepend backwards => list order == array order */
    {
      OFFB *b = &blk[k];
      memcpy (b->W, Woff + 9*k, 9 * sizeof (double));
      b->dia = &dia[adjcol[k]];
      b->bod = bod;
      b->n = d->adj;
      d->adj = b;
    }
  }

  GAUSS_SEIDEL *gs = GAUSS_SEIDEL_Create (epsilon, maxiter, meritval, (GSFAIL) failure,
                                          diagepsilon, diagmaxiter, (DIAS) diagsolver, NULL, count_callback);
  gs->reverse = reverse ? GS_ON : GS_OFF;
  gs->verbose = 0;
  ncallbacks_seen = 0;

  int code = 0;
  TRY ()
  {
    GAUSS_SEIDEL_Solve (gs, ldy);
  }
  CATCHANY (code)
  {
    thrown = code;
  }
  ENDTRY ()

  for (int i = 0; i < n; i ++)
  {
    memcpy (R + 3*i, con[i].R, 3 * sizeof (double));
    memcpy (U + 3*i, con[i].U, 3 * sizeof (double));
    if (conmerit) conmerit[i] = con[i].merit;
  }
  *out_iters = gs->iters;
  *out_error = (int) gs->error;
  *out_merit = dom->merit;
  if (out_ncallbacks) *out_ncallbacks = ncallbacks_seen;
  int nh = gs->iters; /* completed iterations; each wrote rerhist/merhist (bgs.c:1031-1032) */
  if (rerhist && gs->rerhist) memcpy (rerhist, gs->rerhist, (size_t) nh * sizeof (double));
  if (merhist && gs->merhist) memcpy (merhist, gs->merhist, (size_t) nh * sizeof (double));

  GAUSS_SEIDEL_Destroy (gs);
  free (blk); free (state); free (mat); free (dia); free (con);
  free (bod); free (ldy); free (dom); free (sol);
  return thrown;
}
