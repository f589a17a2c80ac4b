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
#include "hyb.h"
#include "ext/predicates.h"

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

/* the reference initialises the robust predicates once at start-up
 * (solfec.c:295); the hull of the convex-convex path depends on them */
static void predicates_ready (void)
{
  static int done = 0;
  if (!done) { exactinit (); done = 1; }
}

/* two convexes (vertices, faces as count then vertex indices, surface per face):
 * gobjcontact for AABB_CONVEX_CONVEX (detect_convex_convex, goc.c:280-306, or
 * update_convex_convex): state, points, normal, gap, area and surface pair */
int ref_gobj_convex_convex (int action, int nva, const double *va, int nfa, const int *fa, const int *sa,
                            int nvb, const double *vb, int nfb, const int *fb, const int *sb,
                            double *onepnt, double *twopnt, double *normal, double *gap, double *area, int *spair)
{
  predicates_ready ();
  CONVEX *a = CONVEX_Create (NULL, (double *) va, nva, (int *) fa, nfa, (int *) sa, 0);
  CONVEX *b = CONVEX_Create (NULL, (double *) vb, nvb, (int *) fb, nfb, (int *) sb, 0);
  TRI *tri = NULL;
  int ntri = 0, state;
  *area = 0.0;
  state = gobjcontact (action ? CONTACT_UPDATE : CONTACT_DETECT, AABB_CONVEX_CONVEX, NULL, a, NULL, b,
                       onepnt, twopnt, normal, gap, area, spair, &tri, &ntri);
  free (tri);
  CONVEX_Destroy (a);
  CONVEX_Destroy (b);
  return state;
}

/* ---- the reference's CPU detection of a sphere set: its hybrid broad phase
 * (hyb.c:317) over the spheres' boxes (SPHERE_Extents, sph.c:240-252) and
 * detect_sphere_sphere (gobjcontact) for every overlap of spheres of different
 * bodies (the body filter of box.c:107-108). Insertion into the domain and the
 * sparsification are not included. Returns the number of contacts; the first
 * cap sphere pairs (i << 32 | j, i < j, ascending) go to pairs (may be NULL). */

typedef struct { SPHERE *sph; const int *body; long long *pair; size_t n, cap; } hyb_state;

/* one call per reported overlap; the reference's overlap_create skips a pair
 * whose contact exists already (contact_exists, dom.c:333-346), as hybrid can
 * report a pair more than once: the detected pairs are recorded and counted
 * once at the end */
static void hyb_overlap (void *data, BOX *one, BOX *two)
{
  hyb_state *h = data;
  SPHERE *a = one->sgp->gobj, *b = two->sgp->gobj;
  const long long i = a - h->sph, j = b - h->sph;
  double onepnt [3], twopnt [3], normal [3], gap, area;
  int spair [2], ntri = 0;
  TRI *tri = NULL;
  if (h->body [i] == h->body [j]) return;
  if (gobjcontact (CONTACT_DETECT, AABB_SPHERE_SPHERE, NULL, a, NULL, b, onepnt, twopnt, normal, &gap, &area, spair,
                   &tri, &ntri))
  {
    if (h->n == h->cap) { h->cap = h->cap ? 2 * h->cap : 1024; h->pair = realloc (h->pair, sizeof (long long) * h->cap); }
    h->pair [h->n ++] = i < j ? (i << 32) | j : (j << 32) | i;
  }
  free (tri);
}

static int llcmp (const void *x, const void *y)
{
  const long long a = *(const long long *) x, b = *(const long long *) y;
  return a < b ? -1 : a > b;
}

long long ref_detect_spheres_hybrid (int n, const double *centre, const double *radius, const int *body,
                                     long long *pairs, long long cap)
{
  SPHERE *sph = calloc ((size_t) n + 1, sizeof (SPHERE));
  SGP *sgp = calloc ((size_t) n + 1, sizeof (SGP));
  BOX *box = calloc ((size_t) n + 1, sizeof (BOX));
  BOX **ptr = calloc ((size_t) n + 1, sizeof (BOX *));
  hyb_state h = {sph, body, NULL, 0, 0};
  long long count = 0;
  for (int i = 0; i < n; i ++)
  {
    memcpy (sph [i].cur_center, centre + 3 * (size_t) i, sizeof (double [3]));
    sph [i].cur_radius = radius [i];
    sgp [i].gobj = &sph [i];
    sgp [i].kind = GOBJ_SPHERE;
    sgp [i].box = &box [i];
    box [i].kind = GOBJ_SPHERE;
    box [i].sgp = &sgp [i];
    SPHERE_Extents (NULL, &sph [i], box [i].extents);
    ptr [i] = &box [i];
  }
  hybrid (ptr, n, &h, hyb_overlap);
  qsort (h.pair, h.n, sizeof (long long), llcmp);
  for (size_t k = 0; k < h.n; k ++)
    if (k == 0 || h.pair [k] != h.pair [k - 1])
    {
      if (pairs && count < cap) pairs [count] = h.pair [k];
      count ++;
    }
  free (h.pair); free (ptr); free (box); free (sgp); free (sph);
  return count;
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
