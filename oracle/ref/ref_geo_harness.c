/*
 * ref_geo_harness.c -- TEST INFRASTRUCTURE (oracle/_ref build). Not part of the product.
 *
 * Flat-array entry into the reference's own contact geometry (goc.c with
 * sph.c, cvx.c, gjk.c and their dependencies, compiled unmodified from the
 * reference tree into _ref/libref_geo.so): gobjcontact for a sphere pair or a
 * convex and a sphere, built from plain arrays, returning the state, the two
 * points, the normal, the gap and the surface pair. The checker of
 * oracle/oracle_detect.c.
 *
 * The link stubs at the end stand for the body, FEM, mesh and bulk-material
 * code that the sphere and convex paths of goc.c never reach; they abort.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "goc.h"
#include "box.h"
#include "sph.h"
#include "cvx.h"
#include "bod.h"
#include "msh.h"
#include "fem.h"
#include "mat.h"

/* action: 0 CONTACT_DETECT, 1 CONTACT_UPDATE; sphere a is the first object */
int ref_gobj_sphere_sphere (int action, const double *ca, double ra, int sa, const double *cb, double rb, int sb,
                            double *onepnt, double *twopnt, double *normal, double *gap, int *spair)
{
  SPHERE a, b;
  double area = 0.0;
  TRI *tri = NULL;
  int ntri = 0, state;
  memset (&a, 0, sizeof a);
  memset (&b, 0, sizeof b);
  memcpy (a.cur_center, ca, sizeof (double [3])); a.cur_radius = ra; a.surface = sa;
  memcpy (b.cur_center, cb, sizeof (double [3])); b.cur_radius = rb; b.surface = sb;
  state = gobjcontact (action ? CONTACT_UPDATE : CONTACT_DETECT, AABB_SPHERE_SPHERE, NULL, &a, NULL, &b,
                       onepnt, twopnt, normal, gap, &area, spair, &tri, &ntri);
  free (tri);
  return state;
}

/* a convex of nver vertices ver[3 nver] with nfac faces fac (per face its
 * vertex count, then vertex indices) and a surface per face, and a sphere;
 * sphere_first selects AABB_SPHERE_CONVEX (the sphere as the first object)
 * over AABB_CONVEX_SPHERE */
int ref_gobj_convex_sphere (int action, int sphere_first, int nver, const double *ver, int nfac, const int *fac,
                            const int *surf, const double *c, double r, int s,
                            double *onepnt, double *twopnt, double *normal, double *gap, int *spair)
{
  CONVEX *cvx = CONVEX_Create (NULL, (double *) ver, nver, (int *) fac, nfac, (int *) surf, 0);
  SPHERE b;
  double area = 0.0;
  TRI *tri = NULL;
  int ntri = 0, state;
  memset (&b, 0, sizeof b);
  memcpy (b.cur_center, c, sizeof (double [3])); b.cur_radius = r; b.surface = s;
  if (sphere_first)
    state = gobjcontact (action ? CONTACT_UPDATE : CONTACT_DETECT, AABB_SPHERE_CONVEX, NULL, &b, NULL, cvx,
                         onepnt, twopnt, normal, gap, &area, spair, &tri, &ntri);
  else
    state = gobjcontact (action ? CONTACT_UPDATE : CONTACT_DETECT, AABB_CONVEX_SPHERE, NULL, cvx, NULL, &b,
                         onepnt, twopnt, normal, gap, &area, spair, &tri, &ntri);
  free (tri);
  CONVEX_Destroy (cvx);
  return state;
}

/* ---- link stubs: code the sphere and convex paths of goc.c do not reach ---- */

static void unreachable (const char *what)
{
  fprintf (stderr, "oracle/_ref: %s is outside the sphere and convex contact paths\n", what);
  abort ();
}

void BODY_Cur_Point (BODY *bod, SGP *sgp, double *X, double *x)
{ (void)bod; (void)sgp; (void)X; (void)x; unreachable ("BODY_Cur_Point"); }
int ELEMENT_Planes (MESH *msh, ELEMENT *ele, double *pla, int *sur, int *ver)
{ (void)msh; (void)ele; (void)pla; (void)sur; (void)ver; unreachable ("ELEMENT_Planes"); return 0; }
int ELEMENT_Vertices (MESH *msh, ELEMENT *ele, double *ver)
{ (void)msh; (void)ele; (void)ver; unreachable ("ELEMENT_Vertices"); return 0; }
void FEM_Cur_Point_Ext (BODY *bod, ELEMENT *ele, double *X, double *point, double *x)
{ (void)bod; (void)ele; (void)X; (void)point; (void)x; unreachable ("FEM_Cur_Point_Ext"); }
BULK_MATERIAL* MATSET_Find (MATSET *set, char *label)
{ (void)set; (void)label; unreachable ("MATSET_Find"); return NULL; }
