/*
 * ref_stubs.c -- TEST INFRASTRUCTURE (oracle/_ref build). Not part of the product.
 *
 * Link stubs that let the reference's own solver translation units
 * (bgs.c dbs.c scf.c mrf.c mem.c err.c alg.c, compiled unmodified from the
 * reference tree) link into a shared library without the rest of Solfec:
 *  - PBF_Int / PBF_Label: called only by GAUSS_SEIDEL_Write_State (bgs.c:1139);
 *    output files are out of scope, so they do nothing.
 *  - springcallback / PENALTY_Spring_Dashpot_Contact: reached only for SPRING
 *    constraints and SPRING_DASHPOT materials (dbs.c:525-531, mrf.c:147);
 *    those kinds are outside the contact path, so they abort loudly.
 *  - SURFACE_MATERIAL_Cohesion_Get: the three-line state getter of sps.c:356;
 *    restated here so sps.c (and its map/set/pack dependencies) stay out.
 *  - dgesv_ / dposv_: no LAPACK is installed; both route to lu_small.c.
 */
#include <stdio.h>
#include <stdlib.h>
#include "dom.h"
#include "pbf.h"
#include "sps.h"
#include "../lu_small.h"

void PBF_Int (PBF *bf, int *value, unsigned int length) { (void)bf; (void)value; (void)length; }
int PBF_Label (PBF *bf, const char *label) { (void)bf; (void)label; return 1; }

double springcallback (void *call, double stroke, double velocity)
{
  (void)call; (void)stroke; (void)velocity;
  fprintf (stderr, "oracle/_ref: SPRING constraints are outside the contact path\n");
  abort ();
}

int PENALTY_Spring_Dashpot_Contact (CON *con, short implicit, double step, double gap, double spring, double dashpot, double hpow,
                             double friction, double cohesion, double *W, double *B, double *V, double *U, double *R)
{
  (void)con; (void)implicit; (void)step; (void)gap; (void)spring; (void)dashpot; (void)hpow;
  (void)friction; (void)cohesion; (void)W; (void)B; (void)V; (void)U; (void)R;
  fprintf (stderr, "oracle/_ref: SPRING_DASHPOT materials are outside the contact path\n");
  abort ();
}

double SURFACE_MATERIAL_Cohesion_Get (SURFACE_MATERIAL_STATE *mat)
{
  return mat->state ? mat->state [0] : 0.0; /* sps.c:33 COHESION == 0 */
}

int dgesv_ (int *n, int *nrhs, double *a, int *lda, int *ipiv, double *b, int *ldb, int *info)
{
  if (*nrhs != 1 || *lda != *n || *ldb != *n) { fprintf (stderr, "oracle/_ref: dgesv_ stub handles nrhs=1, lda=ldb=n only\n"); abort (); }
  *info = orc_dgesv (*n, a, ipiv, b);
  return 0;
}

int dposv_ (char *uplo, int *n, int *nrhs, double *a, int *lda, double *b, int *ldb, int *info)
{
  if (*uplo != 'U' || *nrhs != 1 || *lda != *n || *ldb != *n) { fprintf (stderr, "oracle/_ref: dposv_ stub handles 'U', nrhs=1, lda=ldb=n only\n"); abort (); }
  *info = orc_dposv (*n, a, b);
  return 0;
}
