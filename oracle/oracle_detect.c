/*
 * oracle_detect.c -- TEST INFRASTRUCTURE. Not part of the product.
 *
 * CPU restatement of the reference's contact update and detection for pairs of
 * spheres held by rigid bodies, the checker of the device detection
 * (solfec-1.0_b200/csrc/b2_detect.cuh). One call is the contact part of
 * DOM_Update_Begin (dom.c:3700-3790) for a scene of spheres:
 *
 *  - sphere centres moved with their bodies: SPHERE_Update (sph.c:322-344)
 *    with BODY_Cur_Point (bod.c:1702-1716);
 *  - contacts of the previous step updated with their master and slave kept
 *    (update_contact, dom.c:430-484, update_sphere_sphere, goc.c:658-677) and
 *    removed when the spheres separated;
 *  - new contacts for every other pair of spheres of different bodies, not
 *    both obstacles (box.c:104-108), whose gap gjk_sphere_sphere (gjk.c:560-584)
 *    finds below GEOMETRIC_EPSILON (detect_sphere_sphere, goc.c:421-456), with
 *    the master chosen by the point order of the centres (goc.c:409-419,
 *    dom.c:386-404);
 *  - insert_contact (dom.c:315-330): spatial point, referential points
 *    (BODY_Ref_Point, bod.c:1736-1750), local base (localbase, dom.c:133-151),
 *    gap, surface material (SPSET_Find, sps.c:152-184, resolved by the caller
 *    into a symmetric table of friction and restitution);
 *  - convex obstacles (orc_detect): vertices moved with their bodies and face
 *    planes recomputed (CONVEX_Update, cvx.c:1362-1396; computeplanes,
 *    cvx.c:72-89); a sphere within r + GEOMETRIC_EPSILON of a hull by
 *    gjk_convex_point (gjk.c:510-556) makes a contact with the convex as the
 *    slave (detect_convex_sphere / update_convex_sphere, goc.c:308-349,
 *    555-597; nearest_normal and nearest_surface, goc.c:87-122);
 *  - sparsify_contacts (dom.c:2956-3054): a new contact whose spatial point
 *    lies within 2 mindist (max-norm) of another contact of one of its bodies is
 *    removed when that contact is old or comes later in the list. Sphere
 *    contacts all have area 1, so the area branches never apply.
 *
 * The reference finds candidate pairs with an AABB sweep (hyb.c) over extents
 * inflated by GEOMETRIC_EPSILON (sph.c:240-252); every pair whose gap is below
 * GEOMETRIC_EPSILON overlaps there, so the candidates only prune and this
 * restatement uses a sweep along x with a wider margin.
 *
 * Order: contacts are listed by pair (i, j), i < j, ascending, where a convex c
 * counts as object nsph + c. The
 * reference lists them in insertion order (broad-phase callback order), which
 * depends on its AABB algorithm; the same order also stands in for the
 * reference's contact ids in the sparsification tie-break.
 *
 * gjk_sphere_sphere and gjk_convex_point here are checked bit for bit against
 * the reference's own gjk.c, compiled into oracle/_ref.
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define GEPS 1E-6 /* GEOMETRIC_EPSILON, alg.c:24 */

/* gjk.c:560-584 */
double orc_gjk_sphere_sphere (const double *a, double ra, const double *b, double rb, double *p, double *q)
{
  double d[3], dlen, deno;
  d[0] = a[0] - b[0]; d[1] = a[1] - b[1]; d[2] = a[2] - b[2];
  dlen = sqrt (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
  if (dlen == 0.0)
  {
    memcpy (p, a, sizeof (double) * 3);
    memcpy (q, b, sizeof (double) * 3);
    return 0.0;
  }
  deno = ra / dlen;
  for (int k = 0; k < 3; k++) p[k] = a[k] - deno * d[k];
  deno = rb / dlen;
  for (int k = 0; k < 3; k++) q[k] = b[k] + deno * d[k];
  deno = ra + rb;
  if (dlen > deno) return dlen - deno;
  for (int k = 0; k < 3; k++) p[k] = .5 * (p[k] + q[k]);
  memcpy (q, p, sizeof (double) * 3);
  return 0.0;
}

/* ---- convex polyhedra: GJK distance to a point (gjk.c:510-556) with Johnson's
 * sub-algorithm as gjk.c:213-330 evaluates it: the sub-simplices of the current
 * simplex are tried in a fixed order (singletons, pairs, triples, the whole) and
 * the first whose barycentric weights (delta) are positive on its members and
 * non-positive off them gives the projection of the origin. */

typedef struct { double w[3]; const double *a, *b; } simplex_pt;

/* sub-simplex masks in the order they are tried (bit i = simplex vertex i) and
 * how many of them a simplex of n vertices tries */
static const int sub_mask[15] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 11, 13, 14, 15};
static const int sub_count[5] = {0, 0, 3, 7, 15};

static int popcount4 (int s) { return (s & 1) + ((s >> 1) & 1) + ((s >> 2) & 1) + ((s >> 3) & 1); }

static int johnson (simplex_pt *w, int n, double *l, double *v)
{
  double dot[4][4], delta[16][4], sum;
  if (n == 1)
  {
    l[0] = 1.0;
    v[0] = w[0].w[0]; v[1] = w[0].w[1]; v[2] = w[0].w[2];
    return 1;
  }
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++)
    {
      dot[i][j] = w[i].w[0] * w[j].w[0] + w[i].w[1] * w[j].w[1] + w[i].w[2] * w[j].w[2];
      dot[j][i] = dot[i][j];
    }
  for (int m = 0; m < sub_count[n]; m++)
  {
    const int s = sub_mask[m];
    int ok = 1, k = -1;
    if (popcount4 (s) == 1)
    {
      for (int i = 0; i < n; i++) if (s & (1 << i)) { delta[s][i] = 1.0; k = i; break; }
      for (int j = 0; j < n; j++)
        if (!(s & (1 << j)))
        {
          delta[s][j] = dot[k][k] - dot[k][j];
          if (delta[s][j] > 0.0) ok = 0;
        }
    }
    else
    {
      for (int i = 0; i < n; i++)
        if (s & (1 << i))
        {
          if (k < 0) k = i;
          delta[s][i] = delta[s & ~(1 << i)][i];
          if (delta[s][i] <= 0.0) ok = 0;
        }
      for (int j = 0; j < n; j++)
        if (!(s & (1 << j)))
        {
          delta[s][j] = 0.0;
          for (int i = 0; i < n; i++)
            if (s & (1 << i)) delta[s][j] += delta[s][i] * (dot[i][k] - dot[i][j]);
          if (delta[s][j] > 0.0) ok = 0;
        }
    }
    if (ok)
    {
      int o = 0;
      sum = 0.0;
      for (int i = 0; i < n; i++)
        if (s & (1 << i))
        {
          w[o] = w[i];
          l[o] = delta[s][i];
          sum += l[o];
          o++;
        }
      v[0] = v[1] = v[2] = 0.0;
      for (int i = 0; i < o; i++)
      {
        l[i] /= sum;
        for (int c = 0; c < 3; c++) v[c] = v[c] + l[i] * w[i].w[c];
      }
      return o;
    }
  }
  return 0;
}

/* gjk_convex_point (gjk.c:510-556): distance from point p to the hull of the
 * na vertices a, and the nearest hull point q */
double orc_gjk_convex_point (const double *a, int na, const double *p, double *q)
{
  simplex_pt w[4];
  double v[3], vlen, delta, mi = 0.0, l[4];
  int toofar = 1, n = 0, j = 0;
  const int k = 4 * na * na;
  v[0] = a[0] - p[0]; v[1] = a[1] - p[1]; v[2] = a[2] - p[2];
  vlen = sqrt (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  while (toofar && vlen > GEPS && n < 4 && j++ < k)
  {
    double dmin = DBL_MAX;
    const double *best = NULL;
    for (int t = 0; t < na; t++)
    {
      const double *c = a + 3 * t;
      const double d = c[0] * v[0] + c[1] * v[1] + c[2] * v[2];
      if (d < dmin) { dmin = d; best = c; }
    }
    w[n].a = best;
    w[n].w[0] = best[0] - p[0]; w[n].w[1] = best[1] - p[1]; w[n].w[2] = best[2] - p[2];
    delta = (v[0] * w[n].w[0] + v[1] * w[n].w[1] + v[2] * w[n].w[2]) / vlen;
    mi = mi > delta ? mi : delta;
    toofar = (vlen - mi) > GEPS;
    if (toofar)
    {
      n = johnson (w, n + 1, l, v);
      vlen = sqrt (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
  }
  if (n)
  {
    q[0] = q[1] = q[2] = 0.0;
    for (n--; n >= 0; n--)
      for (int c = 0; c < 3; c++) q[c] = q[c] + l[n] * w[n].a[c];
  }
  else { q[0] = a[0]; q[1] = a[1]; q[2] = a[2]; }
  return vlen;
}

/* gjk (gjk.c:340-391): distance of two polytopes (vertex sets a, b) and their
 * nearest points p in a and q in b; the support points are the first vertex
 * with the smallest (a) or largest (b) projection on the search direction */
double orc_gjk_polytopes (const double *a, int na, const double *b, int nb, double *p, double *q)
{
  simplex_pt w[4];
  double v[3], vlen, delta, mi = 0.0, l[4];
  int toofar = 1, n = 0, j = 0;
  const int k = (na + nb) * (na + nb);
  v[0] = a[0] - b[0]; v[1] = a[1] - b[1]; v[2] = a[2] - b[2];
  vlen = sqrt (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  while (toofar && vlen > GEPS && n < 4 && j++ < k)
  {
    double dmin = DBL_MAX, dmax = -DBL_MAX;
    const double *sa = NULL, *sb = NULL;
    for (int t = 0; t < na; t++)
    {
      const double *c = a + 3 * t, d = c[0] * v[0] + c[1] * v[1] + c[2] * v[2];
      if (d < dmin) { dmin = d; sa = c; }
    }
    for (int t = 0; t < nb; t++)
    {
      const double *c = b + 3 * t, d = c[0] * v[0] + c[1] * v[1] + c[2] * v[2];
      if (d > dmax) { dmax = d; sb = c; }
    }
    w[n].a = sa;
    w[n].b = sb;
    w[n].w[0] = sa[0] - sb[0]; w[n].w[1] = sa[1] - sb[1]; w[n].w[2] = sa[2] - sb[2];
    delta = (v[0] * w[n].w[0] + v[1] * w[n].w[1] + v[2] * w[n].w[2]) / vlen;
    mi = mi > delta ? mi : delta;
    toofar = (vlen - mi) > GEPS;
    if (toofar)
    {
      n = johnson (w, n + 1, l, v);
      vlen = sqrt (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
  }
  if (n)
  {
    p[0] = p[1] = p[2] = 0.0;
    q[0] = q[1] = q[2] = 0.0;
    for (n--; n >= 0; n--)
      for (int c = 0; c < 3; c++)
      {
        p[c] = p[c] + l[n] * w[n].a[c];
        q[c] = q[c] + l[n] * w[n].b[c];
      }
  }
  else
  {
    p[0] = a[0]; p[1] = a[1]; p[2] = a[2];
    q[0] = b[0]; q[1] = b[1]; q[2] = b[2];
  }
  return vlen;
}

/* computeplanes (cvx.c:72-89): per face the unit normal of (b - a) x (c - b)
 * over its first three vertices, and a point of the face (its first vertex,
 * as CONVEX_Planes, cvx.c:1412-1427, lists it); fac = per face its vertex
 * count then its vertex indices */
void orc_convex_planes (int nfac, const int *fac, const double *cur, double *pla)
{
  for (int f = 0, m = 0; f < nfac; f++, m += fac[m] + 1)
  {
    const double *a = cur + 3 * fac[m + 1], *b = cur + 3 * fac[m + 2], *c = cur + 3 * fac[m + 3];
    double ba[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, cb[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
    double *nl = pla + 6 * f, len;
    nl[0] = ba[1] * cb[2] - ba[2] * cb[1];
    nl[1] = ba[2] * cb[0] - ba[0] * cb[2];
    nl[2] = ba[0] * cb[1] - ba[1] * cb[0];
    len = sqrt (nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
    nl[0] /= len; nl[1] /= len; nl[2] /= len;
    nl[3] = a[0]; nl[4] = a[1]; nl[5] = a[2];
  }
}

/* nearest_normal and nearest_surface, goc.c:87-122 */
static const double *nearest_normal (const double *pnt, const double *pla, int n)
{
  double max = -DBL_MAX;
  const double *ret = NULL;
  for (; n > 0; n--, pla += 6)
  {
    const double v[3] = {pnt[0] - pla[3], pnt[1] - pla[4], pnt[2] - pla[5]};
    const double d = pla[0] * v[0] + pla[1] * v[1] + pla[2] * v[2];
    if (d > max) { ret = pla; max = d; }
  }
  return ret;
}

static int nearest_surface (const double *pnt, const double *pla, const int *sur, int n)
{
  double min = DBL_MAX;
  int ret = sur[0];
  for (; n > 0; n--, pla += 6, sur++)
  {
    const double v[3] = {pnt[0] - pla[3], pnt[1] - pla[4], pnt[2] - pla[5]};
    const double d = pla[0] * v[0] + pla[1] * v[1] + pla[2] * v[2];
    if (fabs (d) < min) { min = fabs (d); ret = *sur; }
  }
  return ret;
}

/* localbase, dom.c:133-151: the normal as the third column, the first column
 * e_x x n normalised (e_y x n when that is shorter than GEOMETRIC_EPSILON) and
 * the second their cross product */
void orc_localbase (const double *n, double *loc)
{
  const double e[2][3] = {{1., 0., 0.}, {0., 1., 0.}};
  double len;
  loc[6] = n[0]; loc[7] = n[1]; loc[8] = n[2];
  loc[0] = e[0][1] * n[2] - e[0][2] * n[1];
  loc[1] = e[0][2] * n[0] - e[0][0] * n[2];
  loc[2] = e[0][0] * n[1] - e[0][1] * n[0];
  len = sqrt (loc[0] * loc[0] + loc[1] * loc[1] + loc[2] * loc[2]);
  if (len < GEPS)
  {
    loc[0] = e[1][1] * n[2] - e[1][2] * n[1];
    loc[1] = e[1][2] * n[0] - e[1][0] * n[2];
    loc[2] = e[1][0] * n[1] - e[1][1] * n[0];
    len = sqrt (loc[0] * loc[0] + loc[1] * loc[1] + loc[2] * loc[2]);
  }
  loc[0] /= len; loc[1] /= len; loc[2] /= len;
  loc[3] = loc[1] * n[2] - loc[2] * n[1];
  loc[4] = loc[2] * n[0] - loc[0] * n[2];
  loc[5] = loc[0] * n[1] - loc[1] * n[0];
}

/* BODY_Cur_Point (bod.c:1702-1716): x = c + R (X - X0), R column-major */
static void cur_point (const double *R, const double *c, const double *X0, const double *X, double *x)
{
  double A[3] = {X[0] - X0[0], X[1] - X0[1], X[2] - X0[2]};
  x[0] = c[0] + (R[0] * A[0] + R[3] * A[1] + R[6] * A[2]);
  x[1] = c[1] + (R[1] * A[0] + R[4] * A[1] + R[7] * A[2]);
  x[2] = c[2] + (R[2] * A[0] + R[5] * A[1] + R[8] * A[2]);
}

/* BODY_Ref_Point (bod.c:1736-1750): X = X0 + R^T (x - c) */
static void ref_point (const double *R, const double *c, const double *X0, const double *x, double *X)
{
  double a[3] = {x[0] - c[0], x[1] - c[1], x[2] - c[2]};
  X[0] = X0[0] + (R[0] * a[0] + R[1] * a[1] + R[2] * a[2]);
  X[1] = X0[1] + (R[3] * a[0] + R[4] * a[1] + R[5] * a[2]);
  X[2] = X0[2] + (R[6] * a[0] + R[7] * a[1] + R[8] * a[2]);
}

/* pntcmp, goc.c:409-419 */
static int pntcmp (const double *a, const double *b)
{
  for (int i = 0; i < 3; i++)
  {
    if (a[i] < b[i]) return -1;
    else if (a[i] > b[i]) return 1;
  }
  return 0;
}

void orc_sphere_centres (int nsph, const int *sbody, const double *sref, const double *rot, const double *x,
                         const double *x0, double *cur)
{
  for (int s = 0; s < nsph; s++)
  {
    const int b = sbody[s];
    cur_point (rot + 9 * (size_t) b, x + 3 * (size_t) b, x0 + 3 * (size_t) b, sref + 3 * (size_t) s, cur + 3 * (size_t) s);
  }
}

/* BODY_Ref_Point for a list of spatial points, each of its body */
void orc_ref_points (int n, const int *body, const double *pts, const double *rot, const double *x,
                     const double *x0, double *out)
{
  for (int k = 0; k < n; k++)
  {
    const int b = body[k];
    ref_point (rot + 9 * (size_t) b, x + 3 * (size_t) b, x0 + 3 * (size_t) b, pts + 3 * (size_t) k, out + 3 * (size_t) k);
  }
}

typedef struct { long long key; int slave_lo; double R[3], U[3]; } prevrec;

static int prevcmp (const void *a, const void *b)
{
  long long x = ((const prevrec *) a)->key, y = ((const prevrec *) b)->key;
  return x < y ? -1 : x > y;
}

typedef struct { double lo; int s; } sweeprec;

static int sweepcmp (const void *a, const void *b)
{
  const sweeprec *x = a, *y = b;
  if (x->lo < y->lo) return -1;
  if (x->lo > y->lo) return 1;
  return x->s - y->s;
}

typedef struct { int i, j; } pairrec;

static int paircmp (const void *a, const void *b)
{
  const pairrec *x = a, *y = b;
  if (x->i != y->i) return x->i - y->i;
  return x->j - y->j;
}

/* convex obstacles of orc_detect: per convex its body, vertices cvert[3 *
 * (cvptr[c] .. cvptr[c+1]-1)] in the body's referential frame, faces
 * fac[cfptr[c] ..] (per face its vertex count, then indices into the convex's
 * vertices) and a surface id per face csurf[csptr[c] .. csptr[c+1]-1] */
typedef struct
{
  int n;
  const int *body, *vptr, *fptr, *fac, *sptr, *surf;
  const double *vert;
  double *cur, *pla;   /* current vertices and planes (6 per face) */
} convexes;

static int detect_all (int nsph, const int *sbody, const double *sref, const double *rad, const int *surf,
                       convexes *cv,
                       int nbod, const double *rot, const double *x, const double *x0, const int *obst,
                       int nsurf, const double *mat,
                       int nprev, const long long *prevkey, const int *prevslave_lo, const double *prevR,
                       const double *prevU, int cap,
                       long long *key, int *slave_lo, int *master, int *slave, double *point, double *mpnt,
                       double *spnt, double *base, double *gap, double *friction, double *restitution,
                       double *R0, double *U0, int *isnew)
{
  double *cur = malloc (sizeof (double) * 3 * (size_t) (nsph + 1));
  sweeprec *sw = malloc (sizeof (sweeprec) * (size_t) (nsph + 1));
  prevrec *pv = malloc (sizeof (prevrec) * (size_t) (nprev + 1));
  size_t pcap = 1024, np = 0;
  pairrec *pairs = malloc (sizeof (pairrec) * pcap);
  int ret = 0;
  (void) nbod;
  orc_sphere_centres (nsph, sbody, sref, rot, x, x0, cur);
  for (int k = 0; k < nprev; k++)
  {
    pv[k].key = prevkey[k]; pv[k].slave_lo = prevslave_lo[k];
    for (int q = 0; q < 3; q++) { pv[k].R[q] = prevR ? prevR[3 * k + q] : 0.0; pv[k].U[q] = prevU ? prevU[3 * k + q] : 0.0; }
  }
  qsort (pv, nprev, sizeof (prevrec), prevcmp);

  /* candidate pairs: sweep along x with a margin above GEOMETRIC_EPSILON */
  for (int s = 0; s < nsph; s++) { sw[s].lo = cur[3 * s] - rad[s]; sw[s].s = s; }
  qsort (sw, nsph, sizeof (sweeprec), sweepcmp);
  for (int a = 0; a < nsph; a++)
  {
    const int i = sw[a].s;
    const double hi = cur[3 * i] + rad[i] + 4 * GEPS;
    for (int b = a + 1; b < nsph && sw[b].lo <= hi; b++)
    {
      int s1 = i, s2 = sw[b].s;
      double p[3], q[3];
      if (s1 > s2) { int t = s1; s1 = s2; s2 = t; }
      if (sbody[s1] == sbody[s2]) continue;
      if (obst[sbody[s1]] && obst[sbody[s2]]) continue;
      if (orc_gjk_sphere_sphere (cur + 3 * s1, rad[s1], cur + 3 * s2, rad[s2], p, q) < GEPS)
      {
        if (np == pcap) { pcap *= 2; pairs = realloc (pairs, sizeof (pairrec) * pcap); }
        pairs[np].i = s1; pairs[np].j = s2; np++;
      }
    }
  }
  /* sphere-convex pairs: every pair tested (the candidate boxes of the
   * reference overlap for every pair the distance test accepts) */
  for (int c = 0; c < cv->n; c++)
  {
    const int nv = cv->vptr[c + 1] - cv->vptr[c], bc = cv->body[c];
    const double *vc = cv->cur + 3 * (size_t) cv->vptr[c];
    for (int i = 0; i < nsph; i++)
    {
      double q[3];
      if (sbody[i] == bc) continue;
      if (obst[sbody[i]] && obst[bc]) continue;
      if (orc_gjk_convex_point (vc, nv, cur + 3 * i, q) < rad[i] + GEPS)
      {
        if (np == pcap) { pcap *= 2; pairs = realloc (pairs, sizeof (pairrec) * pcap); }
        pairs[np].i = i; pairs[np].j = nsph + c; np++;
      }
    }
  }
  qsort (pairs, np, sizeof (pairrec), paircmp);

  /* contacts in pair order */
  {
    const size_t n = np;
    int *keep = malloc (sizeof (int) * (n + 1));
    int *bcnt = calloc ((size_t) nbod + 1, sizeof (int)), *bptr = malloc (sizeof (int) * ((size_t) nbod + 2));
    int *blist = malloc (sizeof (int) * (2 * n + 1));
    long long *k_ = malloc (sizeof (long long) * (n + 1));
    int *sl_ = malloc (sizeof (int) * (n + 1)), *ms_ = malloc (sizeof (int) * (n + 1)), *sv_ = malloc (sizeof (int) * (n + 1));
    int *nw_ = malloc (sizeof (int) * (n + 1));
    double *pt_ = malloc (sizeof (double) * 3 * (n + 1)), *mp_ = malloc (sizeof (double) * 3 * (n + 1));
    double *sp_ = malloc (sizeof (double) * 3 * (n + 1)), *bs_ = malloc (sizeof (double) * 9 * (n + 1));
    double *gp_ = malloc (sizeof (double) * (n + 1)), *fr_ = malloc (sizeof (double) * (n + 1));
    double *rs_ = malloc (sizeof (double) * (n + 1));
    double *r0_ = malloc (sizeof (double) * 3 * (n + 1)), *u0_ = malloc (sizeof (double) * 3 * (n + 1));
    size_t out = 0;
    for (size_t c = 0; c < n && ret == 0; c++)
    {
      const int i = pairs[c].i, j = pairs[c].j;
      prevrec probe, *hit;
      int lo_is_slave, s, m;
      double p[3], q[3], nrm[3], len;
      probe.key = ((long long) i << 32) | (long long) j;
      hit = nprev ? bsearch (&probe, pv, nprev, sizeof (prevrec), prevcmp) : NULL;
      if (j >= nsph)
      {
        /* detect_convex_sphere / update_convex_sphere (goc.c:308-349, 555-597):
         * the convex is the slave (its outward normal), the sphere the master */
        const int cx = j - nsph, bc = cv->body[cx], bi = sbody[i];
        const int nv = cv->vptr[cx + 1] - cv->vptr[cx], nf = cv->sptr[cx + 1] - cv->sptr[cx];
        const double *vc = cv->cur + 3 * (size_t) cv->vptr[cx], *pla = cv->pla + 6 * (size_t) cv->sptr[cx];
        const int *fs = cv->surf + cv->sptr[cx];
        const double *cc = cur + 3 * i;
        double one[3], two[3], dot, ln;
        int ns = 0;
        while (ns < nf && fs[ns] != -INT_MAX) ns++;
        orc_gjk_convex_point (vc, nv, cc, one);
        nrm[0] = cc[0] - one[0]; nrm[1] = cc[1] - one[1]; nrm[2] = cc[2] - one[2];
        dot = nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2];
        if (dot == 0.0)
        {
          const double *nn = nearest_normal (one, pla, ns);
          ln = rad[i];
          if (!nn) { ret = -2; break; }
          nrm[0] = nn[0]; nrm[1] = nn[1]; nrm[2] = nn[2];
        }
        else
        {
          const double il = 1.0 / (ln = sqrt (dot));
          nrm[0] *= il; nrm[1] *= il; nrm[2] *= il;
        }
        for (int v = 0; v < 3; v++) two[v] = cc[v] + (-rad[i]) * nrm[v];
        k_[c] = probe.key;
        sl_[c] = 0;
        ms_[c] = bi;
        sv_[c] = bc;
        nw_[c] = hit == NULL;
        dot = ln - rad[i];
        gp_[c] = dot < 0.0 ? dot : 0.0;
        memcpy (pt_ + 3 * c, two, sizeof (double) * 3);
        ref_point (rot + 9 * (size_t) bi, x + 3 * (size_t) bi, x0 + 3 * (size_t) bi, two, mp_ + 3 * c);
        ref_point (rot + 9 * (size_t) bc, x + 3 * (size_t) bc, x0 + 3 * (size_t) bc, one, sp_ + 3 * c);
        orc_localbase (nrm, bs_ + 9 * c);
        {
          const int s0 = nearest_surface (one, pla, fs, ns);
          const size_t t = (size_t) s0 * (size_t) nsurf + (size_t) surf[i];
          fr_[c] = mat[2 * t];
          rs_[c] = mat[2 * t + 1];
        }
        for (int v = 0; v < 3; v++)
        {
          r0_[3 * c + v] = hit ? hit->R[v] : 0.0;
          u0_[3 * c + v] = hit ? hit->U[v] : 0.0;
        }
        continue;
      }
      if (hit) lo_is_slave = hit->slave_lo;                        /* update: roles kept */
      else lo_is_slave = pntcmp (cur + 3 * i, cur + 3 * j) <= 0;   /* detection: lower centre is the slave */
      s = lo_is_slave ? i : j;
      m = lo_is_slave ? j : i;
      orc_gjk_sphere_sphere (cur + 3 * s, rad[s], cur + 3 * m, rad[m], p, q);
      nrm[0] = p[0] - cur[3 * s]; nrm[1] = p[1] - cur[3 * s + 1]; nrm[2] = p[2] - cur[3 * s + 2];
      len = sqrt (nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
      if (!(len > 0.0)) { ret = -1; break; } /* coincident centres: no normal */
      nrm[0] /= len; nrm[1] /= len; nrm[2] /= len;
      k_[c] = probe.key;
      sl_[c] = lo_is_slave;
      ms_[c] = sbody[m];
      sv_[c] = sbody[s];
      nw_[c] = hit == NULL;
      {
        /* sphere_sphere_gap, goc.c:52-61 */
        double xx[3] = {cur[3 * m] - cur[3 * s], cur[3 * m + 1] - cur[3 * s + 1], cur[3 * m + 2] - cur[3 * s + 2]};
        double d = xx[0] * nrm[0] + xx[1] * nrm[1] + xx[2] * nrm[2], e = rad[s] + rad[m];
        gp_[c] = e > d ? d - e : 0;
      }
      memcpy (pt_ + 3 * c, q, sizeof (double) * 3);
      ref_point (rot + 9 * (size_t) sbody[m], x + 3 * (size_t) sbody[m], x0 + 3 * (size_t) sbody[m], q, mp_ + 3 * c);
      ref_point (rot + 9 * (size_t) sbody[s], x + 3 * (size_t) sbody[s], x0 + 3 * (size_t) sbody[s], p, sp_ + 3 * c);
      orc_localbase (nrm, bs_ + 9 * c);
      {
        const size_t t = (size_t) surf[s] * (size_t) nsurf + (size_t) surf[m];
        fr_[c] = mat[2 * t];
        rs_[c] = mat[2 * t + 1];
      }
      for (int v = 0; v < 3; v++)
      {
        r0_[3 * c + v] = hit ? hit->R[v] : 0.0;
        u0_[3 * c + v] = hit ? hit->U[v] : 0.0;
      }
    }
    if (ret == 0)
    {
      /* sparsify_contacts: per body, its contacts */
      for (size_t c = 0; c < n; c++) { bcnt[ms_[c]]++; bcnt[sv_[c]]++; }
      bptr[0] = 0;
      for (int b = 0; b < nbod; b++) bptr[b + 1] = bptr[b] + bcnt[b];
      for (int b = 0; b < nbod; b++) bcnt[b] = bptr[b];
      for (size_t c = 0; c < n; c++) { blist[bcnt[ms_[c]]++] = (int) c; blist[bcnt[sv_[c]]++] = (int) c; }
      for (size_t c = 0; c < n; c++)
      {
        keep[c] = 1;
        if (!nw_[c]) continue;
        const int bb[2] = {ms_[c], sv_[c]};
        for (int t = 0; t < 2 && keep[c]; t++)
          for (int u = bptr[bb[t]]; u < bptr[bb[t] + 1]; u++)
          {
            const int a = blist[u];
            double dd, mx = 0.0;
            if (a == (int) c) continue;
            for (int v = 0; v < 3; v++) { dd = fabs (pt_[3 * c + v] - pt_[3 * (size_t) a + v]); if (dd > mx) mx = dd; }
            if (mx < 2.0 * GEPS && ((int) c < a || !nw_[a])) { keep[c] = 0; break; }
          }
      }
      for (size_t c = 0; c < n; c++)
      {
        if (!keep[c]) continue;
        if ((int) out < cap)
        {
          key[out] = k_[c]; slave_lo[out] = sl_[c]; master[out] = ms_[c]; slave[out] = sv_[c];
          memcpy (point + 3 * out, pt_ + 3 * c, sizeof (double) * 3);
          memcpy (mpnt + 3 * out, mp_ + 3 * c, sizeof (double) * 3);
          memcpy (spnt + 3 * out, sp_ + 3 * c, sizeof (double) * 3);
          memcpy (base + 9 * out, bs_ + 9 * c, sizeof (double) * 9);
          gap[out] = gp_[c]; friction[out] = fr_[c]; restitution[out] = rs_[c];
          memcpy (R0 + 3 * out, r0_ + 3 * c, sizeof (double) * 3);
          memcpy (U0 + 3 * out, u0_ + 3 * c, sizeof (double) * 3);
          isnew[out] = nw_[c];
        }
        out++;
      }
      ret = (int) out;
    }
    free (keep); free (bcnt); free (bptr); free (blist); free (k_); free (sl_); free (ms_); free (sv_); free (nw_);
    free (pt_); free (mp_); free (sp_); free (bs_); free (gp_); free (fr_); free (rs_); free (r0_); free (u0_);
  }
  free (cur); free (sw); free (pv); free (pairs);
  return ret;
}

int orc_detect_spheres (int nsph, const int *sbody, const double *sref, const double *rad, const int *surf,
                        int nbod, const double *rot, const double *x, const double *x0, const int *obst,
                        int nsurf, const double *mat,
                        int nprev, const long long *prevkey, const int *prevslave_lo, const double *prevR,
                        const double *prevU, int cap,
                        long long *key, int *slave_lo, int *master, int *slave, double *point, double *mpnt,
                        double *spnt, double *base, double *gap, double *friction, double *restitution,
                        double *R0, double *U0, int *isnew)
{
  convexes none;
  memset (&none, 0, sizeof none);
  return detect_all (nsph, sbody, sref, rad, surf, &none, nbod, rot, x, x0, obst, nsurf, mat, nprev, prevkey,
                     prevslave_lo, prevR, prevU, cap, key, slave_lo, master, slave, point, mpnt, spnt, base, gap,
                     friction, restitution, R0, U0, isnew);
}

int orc_detect (int nsph, const int *sbody, const double *sref, const double *rad, const int *surf,
                int nconv, const int *cbody, const int *cvptr, const double *cvert, const int *cfptr, const int *fac,
                const int *csptr, const int *csurf,
                int nbod, const double *rot, const double *x, const double *x0, const int *obst,
                int nsurf, const double *mat,
                int nprev, const long long *prevkey, const int *prevslave_lo, const double *prevR,
                const double *prevU, int cap,
                long long *key, int *slave_lo, int *master, int *slave, double *point, double *mpnt,
                double *spnt, double *base, double *gap, double *friction, double *restitution,
                double *R0, double *U0, int *isnew)
{
  convexes cv;
  int ret;
  cv.n = nconv; cv.body = cbody; cv.vptr = cvptr; cv.vert = cvert; cv.fptr = cfptr; cv.fac = fac;
  cv.sptr = csptr; cv.surf = csurf;
  cv.cur = malloc (sizeof (double) * 3 * (size_t) (nconv ? cvptr[nconv] + 1 : 1));
  cv.pla = malloc (sizeof (double) * 6 * (size_t) (nconv ? csptr[nconv] + 1 : 1));
  for (int c = 0; c < nconv; c++)
  {
    const int b = cbody[c];
    for (int v = cvptr[c]; v < cvptr[c + 1]; v++)
      cur_point (rot + 9 * (size_t) b, x + 3 * (size_t) b, x0 + 3 * (size_t) b, cvert + 3 * (size_t) v,
                 cv.cur + 3 * (size_t) v);
    orc_convex_planes (csptr[c + 1] - csptr[c], fac + cfptr[c], cv.cur + 3 * (size_t) cvptr[c],
                       cv.pla + 6 * (size_t) csptr[c]);
  }
  ret = detect_all (nsph, sbody, sref, rad, surf, &cv, nbod, rot, x, x0, obst, nsurf, mat, nprev, prevkey,
                    prevslave_lo, prevR, prevU, cap, key, slave_lo, master, slave, point, mpnt, spnt, base, gap,
                    friction, restitution, R0, U0, isnew);
  free (cv.cur);
  free (cv.pla);
  return ret;
}
