/*
 * b2gs.c -- host side of the B200 contact-solve path, in C.
 *
 * Implements the reference's solver object and its run-time semantics on top
 * of the thin device ABI (b2_device.h):
 *  - GAUSS_SEIDEL_Create defaults (bgs.c:443-472) and the diagepsilon /
 *    diagmaxiter defaults of the Python constructor (lng.c:4335-4342);
 *  - the merit switch: merit is evaluated only when meritval < 1 and nomerit
 *    is off (bgs.c:927);
 *  - failure actions (bgs.c:971-1013, 1053-1068): CONTINUE runs the diagonal
 *    solver fallback chain on the device; EXIT returns the THROW code the
 *    reference raises; CALLBACK calls gs->callback(gs->data) once per
 *    diagonal failure and once for divergence. The device cannot call back in
 *    the middle of a sweep, so the callbacks are made on this thread after the
 *    solve, in the same number;
 *  - history buffers sized to maxiter (bgs.c:933-934), iteration history
 *    (bgs.c:1038-1047), error strings (bgs.c:1073-1136).
 * No longjmp crosses the CUDA runtime: a Solfec integration maps the returned
 * THROW code onto its own THROW after this call returns.
 */
#include <float.h>
#include <limits.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../../include/b2_device.h"
#include "../../include/solfec_b200.h"

struct b2gs_solver
{
  double epsilon, meritval, diagepsilon;
  int maxiter, diagmaxiter, diagsolver, failure;
  void *data;
  b2gs_callback callback;
  int error, iters, reverse, variant, nomerit, precision, grid, stage_blocks;
  int *itershist, itershistcount, itershistsize;
  double *rerhist, *merhist;
  int iters_mixed;
  double solve_ms, merit_input;
  b2dev_solve_report last;
};

struct b2gs_locdyn
{
  b2dev_ctx *dev;
  double merit;
  uint64_t colour_seed;
};

static char host_err[512] = "";

const char* b2gs_last_error (void)
{
  if (host_err[0]) return host_err;
  return b2dev_last_error ();
}

static double default_diagepsilon (double epsilon, double meritval)
{
  double m = meritval < 1E-4 ? meritval : 1E-4;
  double d = 0.01 * (epsilon < m ? epsilon : m);   /* lng.c:4335-4339 */
  return d < DBL_EPSILON ? DBL_EPSILON : d;
}

b2gs_solver* b2gs_create (double epsilon, int maxiter, double meritval, int failure,
                          double diagepsilon, int diagmaxiter, int diagsolver,
                          void *data, b2gs_callback callback)
{
  b2gs_solver *gs;

  if (!(epsilon > 0.0) || maxiter <= 0 || !(meritval > 0.0) || failure < 0 || failure > 2 ||
      diagsolver < 0 || diagsolver > 3 || (failure == B2GS_FAILURE_CALLBACK && !callback))
  {
    snprintf (host_err, sizeof host_err, "b2gs_create: invalid parameters");
    return NULL;
  }
  gs = calloc (1, sizeof (b2gs_solver));
  if (!gs) return NULL;
  gs->epsilon = epsilon;
  gs->maxiter = maxiter;
  gs->meritval = meritval;
  gs->failure = failure;
  gs->diagepsilon = diagepsilon > 0.0 ? diagepsilon : default_diagepsilon (epsilon, meritval);
  gs->diagmaxiter = diagmaxiter > 0 ? diagmaxiter : (maxiter / 100 > 100 ? maxiter / 100 : 100); /* lng.c:4341-4342 */
  gs->diagsolver = diagsolver;
  gs->data = data;
  gs->callback = callback;
  gs->error = B2GS_OK;
  gs->reverse = B2GS_OFF;
  gs->variant = B2GS_FULL;
  gs->nomerit = 0;
  gs->precision = B2GS_FP64;
  gs->itershistcount = -1;
  return gs;
}

int b2gs_get_opts (b2gs_solver *gs, b2dev_solve_opts *o)
{
  if (!gs || !o) return B2DEV_EINVAL;
  memset (o, 0, sizeof *o);
  o->epsilon = gs->epsilon;
  o->meritval = gs->meritval;
  o->diagepsilon = gs->diagepsilon;
  o->maxiter = gs->maxiter;
  o->diagmaxiter = gs->diagmaxiter;
  o->diagsolver = gs->diagsolver;
  o->failure = gs->failure;
  o->reverse = gs->reverse;
  o->nomerit = gs->nomerit ? 1 : gs->meritval >= 1.0 ? 1 : 0;  /* bgs.c:927 */
  o->precision = gs->precision;
  o->grid = gs->grid;
  o->stage_blocks = gs->stage_blocks;
  return 0;
}

int b2gs_solve (b2gs_solver *gs, b2gs_locdyn *ldy)
{
  b2dev_solve_opts o;
  b2dev_solve_report rep;
  int rc, nomerit;

  host_err[0] = '\0';
  if (!gs || !ldy) return B2DEV_EINVAL;
  b2gs_get_opts (gs, &o);
  nomerit = o.nomerit;

  free (gs->rerhist);
  free (gs->merhist);
  gs->rerhist = calloc ((size_t) gs->maxiter, sizeof (double));   /* bgs.c:933-934 */
  gs->merhist = calloc ((size_t) gs->maxiter, sizeof (double));
  if (!gs->rerhist || !gs->merhist) return B2DEV_ECUDA;

  rc = b2dev_solve (ldy->dev, &o, &rep, gs->rerhist, gs->merhist);
  if (rc != B2DEV_OK) return rc;

  gs->last = rep;
  gs->iters = rep.iters;
  gs->iters_mixed = rep.iters_mixed;
  gs->solve_ms = rep.ms_device;
  gs->merit_input = rep.merit_input;
  gs->error = rep.last_fail_kind == 1 ? B2GS_DIAGONAL_DIVERGED : rep.last_fail_kind == 2 ? B2GS_DIAGONAL_FAILED : B2GS_OK;
  ldy->merit = nomerit ? 0.0 : rep.merit;

  if (rep.thrown) return B2GS_ERR_GAUSS_SEIDEL_DIAGONAL_DIVERGED;  /* bgs.c:1007 */

  if (gs->failure == B2GS_FAILURE_CALLBACK)
    for (int k = 0; k < rep.nfailures; k ++) gs->callback (gs->data);  /* bgs.c:1009-1011 */

  if (gs->itershistcount >= 0)  /* bgs.c:1038-1047 */
  {
    if (gs->itershistcount >= gs->itershistsize)
    {
      int *h = realloc (gs->itershist, (size_t) (gs->itershistsize + 1024) * sizeof (int));
      if (!h) return B2DEV_ECUDA;
      gs->itershist = h;
      gs->itershistsize += 1024;
    }
    gs->itershist[gs->itershistcount ++] = gs->iters;
  }

  if (gs->iters >= gs->maxiter)  /* bgs.c:1053-1068 */
  {
    gs->error = B2GS_DIVERGED;
    switch (gs->failure)
    {
    case B2GS_FAILURE_CONTINUE: break;
    case B2GS_FAILURE_EXIT: return B2GS_ERR_GAUSS_SEIDEL_DIVERGED;
    case B2GS_FAILURE_CALLBACK: gs->callback (gs->data); break;
    }
  }
  return 0;
}

const char* b2gs_failure_string (b2gs_solver *gs)
{
  switch (gs->failure)
  {
  case B2GS_FAILURE_CONTINUE: return "FAILURE_CONTINUE";
  case B2GS_FAILURE_EXIT: return "FAILURE_EXIT";
  case B2GS_FAILURE_CALLBACK: return "FAILURE_CALLBACK";
  }
  return NULL;
}

const char* b2gs_diagsolver_string (b2gs_solver *gs)
{
  switch (gs->diagsolver)
  {
  case B2GS_PROJECTED_GRADIENT: return "PROJECTED_GRADIENT";
  case B2GS_DE_SAXCE_FENG: return "DE_SAXCE_FENG";
  case B2GS_SEMISMOOTH_NEWTON: return "SEMISMOOTH_NEWTON";
  case B2GS_PROJECTED_NEWTON: return "PROJECTED_NEWTON";
  }
  return NULL;
}

const char* b2gs_error_string (b2gs_solver *gs)
{
  switch (gs->error)
  {
  case B2GS_OK: return "OK";
  case B2GS_DIVERGED: return "DIVERGED";
  case B2GS_DIAGONAL_DIVERGED: return "DIAGONAL_DIVERGED";
  case B2GS_DIAGONAL_FAILED: return "DIAGONAL_FAILED";
  }
  return NULL;
}

const char* b2gs_reverse_string (b2gs_solver *gs)
{
  return gs->reverse == B2GS_ON ? "ON" : gs->reverse == B2GS_OFF ? "OFF" : NULL;
}

const char* b2gs_variant_string (b2gs_solver *gs)
{
  switch (gs->variant)
  {
  case B2GS_FULL: return "FULL";
  case B2GS_MIDDLE_JACOBI: return "MIDDLE_JACOBI";
  case B2GS_BOUNDARY_JACOBI: return "BOUNDARY_JACOBI";
  }
  return NULL;
}

int b2gs_write_state (b2gs_solver *gs, char *buf, int buflen)
{
  return snprintf (buf, (size_t) buflen, "GSITERS %d\n", gs->iters);
}

void b2gs_destroy (b2gs_solver *gs)
{
  if (!gs) return;
  free (gs->rerhist);
  free (gs->merhist);
  free (gs->itershist);
  free (gs);
}

int b2gs_get_iters (b2gs_solver *gs) { return gs->iters; }
int b2gs_get_error (b2gs_solver *gs) { return gs->error; }
const double* b2gs_get_rerhist (b2gs_solver *gs) { return gs->rerhist; }
const double* b2gs_get_merhist (b2gs_solver *gs) { return gs->merhist; }
const int* b2gs_get_itershist (b2gs_solver *gs, int *count)
{
  if (count) *count = gs->itershistcount < 0 ? 0 : gs->itershistcount;
  return gs->itershist;
}
void b2gs_set_itershist (b2gs_solver *gs, int on)
{
  if (on && gs->itershistcount < 0) gs->itershistcount = 0;
  if (!on) gs->itershistcount = -1;
}
void b2gs_set_reverse (b2gs_solver *gs, int onoff) { gs->reverse = onoff ? B2GS_ON : B2GS_OFF; }
void b2gs_set_variant (b2gs_solver *gs, int variant) { if (variant >= 0 && variant <= 2) gs->variant = variant; }
void b2gs_set_nomerit (b2gs_solver *gs, int nomerit) { gs->nomerit = nomerit ? 1 : 0; }
void b2gs_set_params (b2gs_solver *gs, double epsilon, int maxiter, double meritval, double diagepsilon, int diagmaxiter)
{
  if (epsilon > 0.0) gs->epsilon = epsilon;
  if (maxiter > 0) gs->maxiter = maxiter;
  if (meritval > 0.0) gs->meritval = meritval;
  if (diagepsilon > 0.0) gs->diagepsilon = diagepsilon;
  if (diagmaxiter > 0) gs->diagmaxiter = diagmaxiter;
}
void b2gs_set_precision (b2gs_solver *gs, int precision) { gs->precision = precision == B2GS_MIXED ? B2GS_MIXED : B2GS_FP64; }
void b2gs_set_grid (b2gs_solver *gs, int blocks) { gs->grid = blocks > 0 ? blocks : 0; }
void b2gs_set_stage_blocks (b2gs_solver *gs, int blocks) { gs->stage_blocks = blocks > 0 ? blocks : 0; }
int b2gs_get_iters_mixed (b2gs_solver *gs) { return gs->iters_mixed; }
double b2gs_get_solve_ms (b2gs_solver *gs) { return gs->solve_ms; }
double b2gs_get_merit_input (b2gs_solver *gs) { return gs->merit_input; }
int b2gs_get_report (b2gs_solver *gs, void *report, int nbytes)
{
  if (!gs || !report || nbytes < (int) sizeof (b2dev_solve_report)) return B2DEV_EINVAL;
  memcpy (report, &gs->last, sizeof (b2dev_solve_report));
  return 0;
}

/* ---- local dynamics ---- */

b2gs_locdyn* b2gs_locdyn_create (int device, void *stream)
{
  b2gs_locdyn *ldy = calloc (1, sizeof (b2gs_locdyn));
  if (!ldy) return NULL;
  ldy->dev = b2dev_create (device, stream);
  if (!ldy->dev)
  {
    free (ldy);
    return NULL;
  }
  ldy->colour_seed = 0x5EEDC0105ull;
  return ldy;
}

void b2gs_locdyn_destroy (b2gs_locdyn *ldy)
{
  if (!ldy) return;
  b2dev_destroy (ldy->dev);
  free (ldy);
}

void b2gs_locdyn_set_colour_seed (b2gs_locdyn *ldy, uint64_t seed)
{
  ldy->colour_seed = seed;
  b2dev_set_colour_order (ldy->dev, 0);  /* seeded Jones-Plassmann priorities */
}

void* b2gs_locdyn_device (b2gs_locdyn *ldy) { return ldy ? (void*) ldy->dev : NULL; }

int b2gs_locdyn_update_begin (b2gs_locdyn *ldy, const b2gs_bodies *bod, const b2gs_contacts *con,
                              double step, int dynamic)
{
  int rc;
  host_err[0] = '\0';
  if (!ldy || !bod || !con) return B2DEV_EINVAL;
  if (bod->on_device != con->on_device)
  {
    snprintf (host_err, sizeof host_err, "bodies and contacts must both be host or both be device arrays");
    return B2DEV_EINVAL;
  }
  rc = b2dev_upload_scene (ldy->dev, bod->nbod, bod->rot, bod->x0, bod->jinv, bod->minv, bod->velo, bod->velo0,
                           bod->obstacle, con->ncon, con->master, con->slave, con->mpnt, con->spnt, con->base,
                           con->gap, con->friction, con->restitution, con->cohesion, con->on_device);
  if (rc != B2DEV_OK) return rc;
  return b2dev_assemble (ldy->dev, step, dynamic, ldy->colour_seed);
}

int b2gs_locdyn_update_begin_resident (b2gs_locdyn *ldy, double step, int dynamic)
{
  host_err[0] = '\0';
  if (!ldy) return B2DEV_EINVAL;
  return b2dev_assemble (ldy->dev, step, dynamic, ldy->colour_seed);
}

int b2gs_locdyn_set (b2gs_locdyn *ldy, int n, const double *W, const double *A, const double *rho,
                     const double *B, const double *V, const double *gap, const double *friction,
                     const double *restitution, const double *cohesion, const int *adjptr, const int *adjcol,
                     const double *Woff, double free_energy, double step, int dynamic, int on_device)
{
  host_err[0] = '\0';
  if (!ldy) return B2DEV_EINVAL;
  return b2dev_upload_locdyn (ldy->dev, n, W, A, rho, B, V, gap, friction, restitution, cohesion, adjptr, adjcol,
                              Woff, free_energy, step, dynamic, ldy->colour_seed, on_device);
}

int b2gs_locdyn_set_state (b2gs_locdyn *ldy, const double *R, const double *U, int on_device)
{
  return b2dev_set_state (ldy->dev, R, U, on_device);
}

int b2gs_locdyn_get_state (b2gs_locdyn *ldy, double *R, double *U, double *conmerit, int on_device)
{
  return b2dev_get_state (ldy->dev, R, U, conmerit, on_device);
}

double b2gs_locdyn_merit (b2gs_locdyn *ldy) { return ldy->merit; }

int b2gs_locdyn_sizes (b2gs_locdyn *ldy, int *n, long long *nblocks, int *ncolours, double *free_energy)
{
  return b2dev_sizes (ldy->dev, n, nblocks, ncolours, free_energy);
}

int b2gs_locdyn_order (b2gs_locdyn *ldy, int *order) { return b2dev_get_order (ldy->dev, order); }
