// b2_cvi.cuh -- contact between two convex polyhedra: detect_convex_convex and
// update_convex_convex (goc.c:280-306, goc.c:527-553). The intersection of the
// two convexes (cvi, cvi.c:118-230) is the polar of the convex hull of the
// polar points of their face planes: the quickhull of those points (hull,
// hul.c:560-779), its polarisation (TRI_Polarise, tri.c:352-447), and the
// contact point, normal, surface pair, area and gap of the intersection
// polytope (point_normal_spair_area_gap, goc.c:148-277).
//
// Callable from device code (one thread per convex pair) and host code. Every
// structure lives in fixed-size arrays of the caller's frame, linked by 16-bit
// indices where the reference links heap records by pointer; the reference
// compares those pointers only for identity and walks its sets and maps in
// address order, which is the input order of the points here, so index links
// reproduce its lists exactly. Capacities: 32 planes of both convexes
// together; a larger pair, or a hull that outgrows the pools, reports
// kCviOverflow instead of a contact.
//
// The hull decides visibility by the sign of orient3d alone (hul.c compares
// it with zero: its running maxima start at 0.0 and are never raised), so the
// exact sign reproduces it: the floating-point determinant when it clears
// Shewchuk's static error bound (the first stage of the reference's
// ext/predicates.c orient3d), else the exact sign of the 4 x 4 determinant
// from exact triple products summed as a floating-point expansion.
// Arithmetic follows the reference's macros (alg.h) operation by operation
// and is built without fused multiply-adds.
#pragma once

#include <cfloat>
#include <cmath>

#include "b2_gjk.cuh"

namespace b2 {
namespace cvi {

constexpr int kMaxPlanes = 32;                 // polar points (planes of both convexes)
constexpr int kMaxHullFaces = 2 * kMaxPlanes;  // faces of a hull of n points: at most 2 n - 4
constexpr int kMaxFaces = 2 * kMaxHullFaces;   // live faces while a step adds its cone
constexpr int kMaxEdges = 3 * kMaxFaces;
constexpr int kMaxPfv = 3 * kMaxHullFaces;     // polar face vertices: 3 per hull triangle
constexpr int kCviOverflow = -1;

// ---- exact orientation sign -------------------------------------------------

// floating-point expansions (Shewchuk, "Adaptive precision floating-point
// arithmetic and fast robust geometric predicates", 1997): a sum of
// non-overlapping doubles in increasing magnitude, exact as a whole
B2_HD inline void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  const double bv = s - a;
  const double av = s - bv;
  e = (a - av) + (b - bv);
}

B2_HD inline void split27(double a, double& hi, double& lo) {
  const double c = 134217729.0 * a;  // 2^27 + 1
  const double big = c - a;
  hi = c - big;
  lo = a - hi;
}

B2_HD inline void two_product(double a, double b, double& p, double& e) {
  p = a * b;
  double ah, al, bh, bl;
  split27(a, ah, al);
  split27(b, bh, bl);
  const double e1 = p - ah * bh;
  const double e2 = e1 - al * bh;
  const double e3 = e2 - ah * bl;
  e = al * bl - e3;
}

// h (len n) += b, zero components dropped (Grow-Expansion); returns the length
B2_HD inline int grow_expansion(double* h, int n, double b) {
  double q = b;
  int m = 0;
  for (int i = 0; i < n; i++) {
    double s, e;
    two_sum(q, h[i], s, e);
    q = s;
    if (e != 0.0) h[m++] = e;
  }
  if (q != 0.0) h[m++] = q;
  return m;
}

// h += s * x * y * z exactly (the product as four doubles: x y = p + e exactly,
// then p z and e z exactly)
B2_HD inline int add_triple(double* h, int n, double s, double x, double y, double z) {
  double p, e, p1, e1, p2, e2;
  two_product(x, y, p, e);
  two_product(p, z, p1, e1);
  two_product(e, z, p2, e2);
  n = grow_expansion(h, n, s * e2);
  n = grow_expansion(h, n, s * p2);
  n = grow_expansion(h, n, s * e1);
  return grow_expansion(h, n, s * p1);
}

// h += s * det [p; q; r] (rows)
B2_HD inline int add_det3(double* h, int n, double s, const double* p, const double* q, const double* r) {
  n = add_triple(h, n, s, p[0], q[1], r[2]);
  n = add_triple(h, n, -s, p[0], q[2], r[1]);
  n = add_triple(h, n, s, p[1], q[2], r[0]);
  n = add_triple(h, n, -s, p[1], q[0], r[2]);
  n = add_triple(h, n, s, p[2], q[0], r[1]);
  return add_triple(h, n, -s, p[2], q[1], r[0]);
}

// exact sign of orient3d (a, b, c, d) = det [a - d; b - d; c - d], which is the
// 4 x 4 determinant with rows (x, 1) expanded along its last column
B2_HD B2_NOINLINE static double orient3d_exact_sign(const double* a, const double* b, const double* c, const double* d) {
  double h[160];  // a non-overlapping expansion of doubles spans at most ~2100 bits / component
  int n = 0;
  n = add_det3(h, n, -1.0, b, c, d);
  n = add_det3(h, n, 1.0, a, c, d);
  n = add_det3(h, n, -1.0, a, b, d);
  n = add_det3(h, n, 1.0, a, b, c);
  if (n == 0) return 0.0;
  return h[n - 1] > 0.0 ? 1.0 : (h[n - 1] < 0.0 ? -1.0 : 0.0);
}

// orient3d, ext/predicates.c:1252-1300: positive when d lies below the plane of
// (a, b, c) oriented counter-clockwise from above; its sign only
B2_HD inline double orient3d(const double* a, const double* b, const double* c, const double* d) {
  const double adx = a[0] - d[0], bdx = b[0] - d[0], cdx = c[0] - d[0];
  const double ady = a[1] - d[1], bdy = b[1] - d[1], cdy = c[1] - d[1];
  const double adz = a[2] - d[2], bdz = b[2] - d[2], cdz = c[2] - d[2];
  const double bdxcdy = bdx * cdy, cdxbdy = cdx * bdy;
  const double cdxady = cdx * ady, adxcdy = adx * cdy;
  const double adxbdy = adx * bdy, bdxady = bdx * ady;
  const double det = adz * (bdxcdy - cdxbdy) + bdz * (cdxady - adxcdy) + cdz * (adxbdy - bdxady);
  const double permanent = (fabs(bdxcdy) + fabs(cdxbdy)) * fabs(adz) + (fabs(cdxady) + fabs(adxcdy)) * fabs(bdz) +
                           (fabs(adxbdy) + fabs(bdxady)) * fabs(cdz);
  // o3derrboundA = (7 + 56 eps) eps, eps = 2^-53 (exactinit)
  const double eps = 1.1102230246251565e-16;
  const double errbound = ((7.0 + 56.0 * eps) * eps) * permanent;
  if (det > errbound || -det > errbound) return det;
  return orient3d_exact_sign(a, b, c, d);
}

// ---- quickhull of the polar points (hul.c) ----------------------------------

struct HEdge {
  short v0, v1;  // vertices (point indices), counter-clockwise in the face
  short f;       // the neighbouring face through this edge
  short n;       // next edge of the face
};

struct HFace {
  double pla[4];
  short v;       // list of outside points (vertex records)
  short w;       // the chosen outside point
  short e;       // edge list
  short n;       // next face
  short tri;     // output triangle
  char marked;
};

struct HVert {
  short p;  // point index
  short n;  // next record
};

struct OutTri {
  double out[3];  // face normal (not normalised)
  short ver[3];   // point indices, counter-clockwise
  short adj[3];   // adj[0] across ver[0]-ver[1], adj[1] across ver[1]-ver[2], adj[2] across ver[2]-ver[0]
};

struct Hull {
  const double* y;  // points [3 n]
  int n;
  HFace face[kMaxFaces];
  HEdge edge[kMaxEdges];
  HVert vert[kMaxPlanes];
  short free_face[kMaxFaces], free_edge[kMaxEdges];
  int nfree_face, nfree_edge, used_face, used_edge, used_vert;
  bool overflow;

  B2_HD const double* P(int i) const { return y + 3 * i; }

  B2_HD int new_face() {
    int f;
    if (nfree_face) f = free_face[--nfree_face];
    else if (used_face < kMaxFaces) f = used_face++;
    else { overflow = true; return -1; }
    HFace& F = face[f];
    F.pla[0] = F.pla[1] = F.pla[2] = F.pla[3] = 0.0;
    F.v = F.w = F.e = F.n = F.tri = -1;
    F.marked = 0;
    return f;
  }
  B2_HD int new_edge() {
    int e;
    if (nfree_edge) e = free_edge[--nfree_edge];
    else if (used_edge < kMaxEdges) e = used_edge++;
    else { overflow = true; return -1; }
    edge[e].v0 = edge[e].v1 = edge[e].f = edge[e].n = -1;
    return e;
  }
  B2_HD void free_f(int f) { free_face[nfree_face++] = (short)f; }
  B2_HD void free_e(int e) { free_edge[nfree_edge++] = (short)e; }

  // orient, hul.c:61-73: orient3d (c, b, a, d) over the face's first two edges
  B2_HD double orient(int f, int d) const {
    const HEdge& e1 = edge[face[f].e];
    const HEdge& e2 = edge[e1.n];
    return orient3d(P(e2.v1), P(e1.v1), P(e1.v0), P(d));
  }

  // setplane, hul.c:76-90
  B2_HD bool setplane(int f) {
    const HEdge& e1 = edge[face[f].e];
    const HEdge& e2 = edge[e1.n];
    const double *a0 = P(e1.v0), *a1 = P(e1.v1), *b0 = P(e2.v0), *b1 = P(e2.v1);
    const double ba[3] = {a1[0] - a0[0], a1[1] - a0[1], a1[2] - a0[2]};
    const double cb[3] = {b1[0] - b0[0], b1[1] - b0[1], b1[2] - b0[2]};
    double* pla = face[f].pla;
    pla[0] = ba[1] * cb[2] - ba[2] * cb[1];
    pla[1] = ba[2] * cb[0] - ba[0] * cb[2];
    pla[2] = ba[0] * cb[1] - ba[1] * cb[0];
    pla[3] = -(a0[0] * pla[0] + a0[1] * pla[1] + a0[2] * pla[2]);
    double m = fabs(pla[0]);
    if (m < fabs(pla[1])) m = fabs(pla[1]);
    if (m < fabs(pla[2])) m = fabs(pla[2]);
    return m != 0.0;
  }

  B2_HD int othere(int f, int g) const {  // edge of f whose neighbour is g
    for (int e = face[f].e; e >= 0; e = edge[e].n)
      if (edge[e].f == g) return e;
    return -1;
  }
  B2_HD int otherv(int f, int p, int q) const {  // vertex of f other than p and q
    for (int e = face[f].e; e >= 0; e = edge[e].n)
      if (edge[e].v0 != p && edge[e].v0 != q) return edge[e].v0;
    return -1;
  }
  B2_HD int edge_from(int f, int v) const {
    for (int e = face[f].e; e >= 0; e = edge[e].n)
      if (edge[e].v0 == v) return e;
    return -1;
  }
  B2_HD int edge_to(int f, int v) const {
    for (int e = face[f].e; e >= 0; e = edge[e].n)
      if (edge[e].v1 == v) return e;
    return -1;
  }

  // mendface, hul.c:150-228: a face whose vertices are colinear is flipped
  // with its neighbour across the edge that contains the middle vertex
  B2_HD B2_NOINLINE bool mendface(int f) {
    int e, c = -1;
    for (e = face[f].e; e >= 0; e = edge[e].n) {
      const int a = edge[e].v0, b = edge[e].v1;
      if ((c = otherv(f, a, b)) < 0) return false;
      const double *A = P(a), *B = P(b), *C = P(c);
      const double u[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
      const double v[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
      const double l0 = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      const double l1 = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      const double d = u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
      if (d >= 0 && l1 <= l0) break;  // c in [a, b]
    }
    if (e < 0) return false;
    const int a = c, g = edge[e].f;
    const int h = othere(g, f);
    if (h < 0) return false;
    const int b = otherv(g, edge[h].v0, edge[h].v1);
    if (b < 0) return false;
    const int x = edge_from(f, a);
    if (x < 0) return false;
    const int yv = edge_to(g, b);
    if (yv < 0) return false;
    const int z = edge_from(g, b);
    if (z < 0) return false;
    const int w = edge_to(f, a);
    if (w < 0) return false;
    int o = othere(edge[yv].f, g);
    if (o < 0) return false;
    edge[o].f = (short)f;
    o = othere(edge[w].f, f);
    if (o < 0) return false;
    edge[o].f = (short)g;
    edge[e].v0 = (short)b; edge[e].v1 = (short)a;
    edge[h].v0 = (short)a; edge[h].v1 = (short)b;
    edge[e].n = -1; edge[yv].n = (short)e; edge[x].n = (short)yv; face[f].e = (short)x;
    edge[h].n = -1; edge[w].n = (short)h; edge[z].n = (short)w; face[g].e = (short)z;
    return setplane(f) && setplane(g);
  }

  // simplex_vertices, hul.c:239-343: the input points sorted by x (stably, as
  // glibc's qsort orders equal keys), points inside the 10 eps box of an
  // earlier sorted point dropped, then four well separated points in input
  // order; the rest (input order) pushed onto a list, so it runs backwards
  B2_HD B2_NOINLINE bool simplex_vertices(int sv[4], int& list) {
    short order[kMaxPlanes];
    bool alive[kMaxPlanes];
    for (int i = 0; i < n; i++) { order[i] = (short)i; alive[i] = true; }
    for (int i = 1; i < n; i++) {  // insertion sort: stable
      const short k = order[i];
      const double key = P(k)[0];
      int j = i - 1;
      while (j >= 0 && P(order[j])[0] > key) { order[j + 1] = order[j]; j--; }
      order[j + 1] = k;
    }
    const double d = 10 * kGeomEps;
    for (int pp = 0, pn; pp < n; pp = pn) {
      int pq;
      pn = n;
      const double* A = P(order[pp]);
      for (pq = pp + 1; pq < n && P(order[pq])[0] - d < A[0] + d; pq++) {
        const double* B = P(order[pq]);
        int i;
        for (i = 1; i < 3; i++)
          if (B[i] - d >= A[i] + d || B[i] + d <= A[i] - d) break;
        if (i == 3) alive[order[pq]] = false;
        else if (pn == n) pn = pq;
      }
      if (pn == n) pn = pq;
    }
    int j = 0;
    for (int p = 0; p < n && j < 4; p++) {
      if (!alive[p]) continue;
      const double* X = P(p);
      double u[3] = {0.0, 0.0, 0.0};
      int i;
      for (i = 0; i < j; i++) {
        const double* S = P(sv[i]);
        u[0] = S[0] - X[0]; u[1] = S[1] - X[1]; u[2] = S[2] - X[2];
        double m = fabs(u[0]);
        if (m < fabs(u[1])) m = fabs(u[1]);
        if (m < fabs(u[2])) m = fabs(u[2]);
        if (m < 2.0 * kGeomEps) break;  // too close
      }
      if (i != j) continue;
      if (j == 2) {
        const double *S0 = P(sv[0]), *S1 = P(sv[1]);
        const double a[3] = {S1[0] - S0[0], S1[1] - S0[1], S1[2] - S0[2]};
        const double b[3] = {u[1] * a[2] - u[2] * a[1], u[2] * a[0] - u[0] * a[2], u[0] * a[1] - u[1] * a[0]};
        double m = fabs(b[0]);
        if (m < fabs(b[1])) m = fabs(b[1]);
        if (m < fabs(b[2])) m = fabs(b[2]);
        if (m < kGeomEps) continue;  // colinear
      } else if (j == 3) {
        const double *S0 = P(sv[0]), *S1 = P(sv[1]), *S2 = P(sv[2]);
        const double a[3] = {S1[0] - S0[0], S1[1] - S0[1], S1[2] - S0[2]};
        const double b[3] = {S2[0] - S1[0], S2[1] - S1[1], S2[2] - S1[2]};
        const double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
        const double dd = u[0] * c[0] + u[1] * c[1] + u[2] * c[2];
        if ((dd > 0 ? dd : -dd) < kGeomEps) continue;  // coplanar
      }
      sv[j++] = p;
      alive[p] = false;
    }
    if (j != 4) return false;
    list = -1;
    for (int p = 0; p < n; p++) {
      if (!alive[p]) continue;
      const int x = used_vert++;
      vert[x].p = (short)p;
      vert[x].n = (short)list;
      list = x;
    }
    return true;
  }

  // simplex, hul.c:346-456: four faces (a b c), (b d c), (d a c), (d b a), each
  // turned over when the remaining vertex is in front of it
  B2_HD B2_NOINLINE int simplex(int a, int b, int c, int d) {
    int e[12], f[4];
    for (int i = 0; i < 12; i++) e[i] = new_edge();
    for (int i = 0; i < 4; i++) f[i] = new_face();
    if (overflow) return -1;
    const int verts[12][2] = {{a, b}, {b, c}, {c, a}, {b, d}, {d, c}, {c, b},
                              {d, a}, {a, c}, {c, d}, {d, b}, {b, a}, {a, d}};
    const int nbr[12] = {3, 1, 2, 3, 2, 0, 3, 0, 1, 1, 0, 2};
    for (int i = 0; i < 12; i++) {
      edge[e[i]].v0 = (short)verts[i][0];
      edge[e[i]].v1 = (short)verts[i][1];
      edge[e[i]].f = (short)f[nbr[i]];
      edge[e[i]].n = (i % 3 == 2) ? -1 : (short)e[i + 1];
    }
    for (int i = 0; i < 4; i++) face[f[i]].e = (short)e[3 * i];
    face[f[0]].n = (short)f[1];
    face[f[1]].n = (short)f[2];
    face[f[2]].n = (short)f[3];
    const int other[4] = {d, a, b, c};
    for (int i = 0; i < 4; i++) {
      if (!setplane(f[i])) return -1;
      if (orient(f[i], other[i]) > 0.0) {  // reverse the edges and the plane
        for (int g = face[f[i]].e; g >= 0; g = edge[g].n) {
          const short t = edge[g].v0; edge[g].v0 = edge[g].v1; edge[g].v1 = t;
        }
        const int e0 = face[f[i]].e, e1 = edge[e0].n, e2 = edge[e1].n;
        edge[e2].n = (short)e1;
        edge[e1].n = (short)e0;
        edge[e0].n = -1;
        face[f[i]].e = (short)e2;
        face[f[i]].pla[0] *= -1.0; face[f[i]].pla[1] *= -1.0; face[f[i]].pla[2] *= -1.0;
        face[f[i]].pla[3] *= -1.0;
      }
    }
    return f[0];
  }

  // nextaround, hul.c:474-487: the face across the edge of f that ends at v
  B2_HD int nextaround(int f, int v) const {
    for (int e = face[f].e; e >= 0; e = edge[e].n)
      if (edge[e].v1 == v) return edge[e].f;
    return -1;
  }

  // testsimplex, hul.c:527-553
  B2_HD B2_NOINLINE bool testsimplex(int h) const {
    for (; h >= 0; h = face[h].n)
      for (int e = face[h].e; e >= 0; e = edge[e].n)
        for (int i = 0; i < 2; i++) {
          const int v = i ? edge[e].v1 : edge[e].v0;
          int nn = 1, f;
          for (f = nextaround(h, v); f >= 0 && f != h && nn < 4; f = nextaround(f, v)) nn++;
          if (f < 0 || nn != 3) return false;
        }
    return true;
  }

  // mark, hul.c:460-471: faces visible from point v, depth first through the
  // edges in list order; g = the last face met that v does not see
  B2_HD B2_NOINLINE void mark(int f0, int v, int& g) {
    short fs[kMaxFaces], es[kMaxFaces];
    int top = 0;
    const double d0 = orient(f0, v);
    if (!face[f0].marked && d0 > 0.0) {
      face[f0].marked = 1;
      fs[0] = (short)f0; es[0] = face[f0].e; top = 1;
    } else if (d0 <= 0.0) {
      g = f0;
    }
    while (top > 0) {
      const int e = es[top - 1];
      if (e < 0) { top--; continue; }
      es[top - 1] = edge[e].n;
      const int f = edge[e].f;
      const double d = orient(f, v);
      if (!face[f].marked && d > 0.0) {
        face[f].marked = 1;
        if (top >= kMaxFaces) { overflow = true; return; }
        fs[top] = (short)f; es[top] = face[f].e; top++;
      } else if (d <= 0.0) {
        g = f;
      }
    }
  }

  // nextonridge, hul.c:491-524
  B2_HD int nextonridge(int e, int* g) const {
    if (g) {
      const int v = edge[e].v1;
      int f = edge[e].f, nn;
      for (nn = 1, f = nextaround(f, v); f >= 0 && face[f].marked && nn < n; f = nextaround(f, v)) nn++;
      if (f < 0 || nn == n) return -1;
      for (e = face[f].e; e >= 0 && edge[e].v0 != v; e = edge[e].n) {}
      *g = f;
      return e;
    }
    for (; e >= 0 && !face[edge[e].f].marked; e = edge[e].n) {}
    return e;
  }

  // the points of the list l above face f go to f's outside set: the last of
  // them becomes f->w and the earlier choices move to f->v (hul.c:580-603 and
  // 683-708, whose running maximum stays 0)
  B2_HD B2_NOINLINE void take_outside(int f, short& l) {
    int z = -1, x = l;
    while (x >= 0) {
      const int yv = vert[x].n;
      if (orient(f, vert[x].p) > 0.0) {
        if (face[f].w >= 0) {
          vert[face[f].w].n = face[f].v;
          face[f].v = face[f].w;
        }
        face[f].w = (short)x;
        if (z >= 0) vert[z].n = (short)yv;
        else l = (short)yv;
      } else {
        z = x;
      }
      x = yv;
    }
  }

  // hull, hul.c:560-779: the hull's faces as triangles, counter-clockwise
  // seen from outside, with their adjacency; returns the count or -1
  B2_HD B2_NOINLINE int build(const double* pts, int npts, OutTri* tri) {
    y = pts; n = npts;
    nfree_face = nfree_edge = used_face = used_edge = used_vert = 0;
    overflow = false;
    if (n > kMaxPlanes) { overflow = true; return -1; }
    int sv[4], list;
    if (!simplex_vertices(sv, list)) return -1;
    int h = simplex(sv[0], sv[1], sv[2], sv[3]);
    if (h < 0 || !testsimplex(h)) return -1;
    short l = (short)list;
    for (int f = h; f >= 0; f = face[f].n) take_outside(f, l);
    int f;
    for (f = h; f >= 0 && face[f].w < 0; f = face[f].n) {}
    while (f >= 0) {
      int g = -1;
      mark(f, vert[face[f].w].p, g);
      if (overflow) return -1;
      int k, e;
      if (g < 0 || (k = e = nextonridge(face[g].e, nullptr)) < 0) return -1;
      int ehead = -1, etail = -1, head = -1, tail = -1;
      const int top = vert[face[f].w].p;
      do {
        const int cur = new_face();
        if (tail < 0) tail = cur;
        int i = new_edge();
        if (overflow) return -1;
        edge[i].v0 = edge[e].v1;
        edge[i].v1 = edge[e].v0;
        edge[i].f = (short)g;
        face[cur].e = (short)i;
        const int jj = new_edge();
        if (overflow) return -1;
        edge[jj].v0 = (short)top;
        edge[jj].v1 = edge[e].v1;
        edge[jj].n = face[cur].e; face[cur].e = (short)jj;
        i = new_edge();
        if (overflow) return -1;
        edge[i].v0 = edge[e].v0;
        edge[i].v1 = (short)top;
        edge[i].n = face[cur].e; face[cur].e = (short)i;
        if (head >= 0) {
          edge[i].f = (short)head;
          edge[ehead].f = (short)cur;
        } else {
          etail = i;
        }
        face[cur].n = (short)head; head = cur;
        ehead = jj;
        const int old = e;
        if ((e = nextonridge(old, &g)) < 0) return -1;
        edge[old].f = (short)cur;
      } while (e != k);
      edge[ehead].f = (short)tail;
      edge[etail].f = (short)head;
      face[f].w = -1;  // the top point's record is released
      for (g = head; g >= 0; g = face[g].n)
        if (!setplane(g) && !mendface(g)) return -1;
      for (int m = h; m >= 0; m = face[m].n) {
        if (!face[m].marked) continue;
        if (face[m].w >= 0) {
          vert[face[m].w].n = face[m].v;
          face[m].v = face[m].w;
        }
        if (face[m].v >= 0)
          for (g = head; g >= 0; g = face[g].n) take_outside(g, face[m].v);
      }
      int survivors = -1;
      for (int m = h, nx; m >= 0; m = nx) {
        nx = face[m].n;
        if (face[m].marked) {
          for (int x = face[m].e, xn; x >= 0; x = xn) { xn = edge[x].n; free_e(x); }
          free_f(m);
        } else {
          face[m].n = (short)survivors;
          survivors = m;
        }
      }
      face[tail].n = (short)survivors;
      h = head;
      for (f = h; f >= 0 && face[f].w < 0; f = face[f].n) {}
    }
    int m = 0;
    for (f = h; f >= 0; f = face[f].n) m++;
    if (m > kMaxHullFaces) { overflow = true; return -1; }
    int t = 0;
    for (f = h; f >= 0; f = face[f].n, t++) {
      const int e = face[f].e, k = edge[e].n, i = edge[k].n;
      OutTri& T = tri[t];
      T.out[0] = face[f].pla[0]; T.out[1] = face[f].pla[1]; T.out[2] = face[f].pla[2];
      T.ver[0] = edge[e].v0; T.ver[1] = edge[k].v0; T.ver[2] = edge[i].v0;
      T.adj[0] = T.adj[1] = T.adj[2] = -1;
      const int nb[3] = {edge[e].f, edge[k].f, edge[i].f};
      for (int q = 0; q < 3; q++) {
        const int s = face[nb[q]].tri;
        if (s < 0) continue;
        int a, b;  // TRI_Addadj, tri.c:107-118
        for (a = 0; a < 3 && tri[s].adj[a] >= 0; a++) {}
        for (b = 0; b < 3 && T.adj[b] >= 0; b++) {}
        if (a >= 3 || b >= 3) return -1;
        tri[s].adj[a] = (short)t;
        T.adj[b] = (short)s;
      }
      face[f].tri = (short)t;
    }
    for (t = m - 1; t >= 0; t--) {  // TRI_Sortadj, tri.c:79-104
      OutTri& T = tri[t];
      const int ed[3][2] = {{T.ver[0], T.ver[1]}, {T.ver[1], T.ver[2]}, {T.ver[2], T.ver[0]}};
      short out[3] = {-1, -1, -1};
      for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
          const int s = T.adj[j];
          if (s < 0) continue;
          int cnt = 0;
          for (int q = 0; q < 3; q++)
            if (tri[s].ver[q] == ed[i][0] || tri[s].ver[q] == ed[i][1]) cnt++;
          if (cnt == 2) { out[i] = (short)s; T.adj[j] = -1; }
        }
      T.adj[0] = out[0]; T.adj[1] = out[1]; T.adj[2] = out[2];
    }
    return m;
  }
};

// the triangle after t counter-clockwise around its vertex v (tri.c:59-64)
B2_HD inline int tri_nextaround(const OutTri* tri, int t, int v) {
  if (v == tri[t].ver[0]) return tri[t].adj[2];
  if (v == tri[t].ver[1]) return tri[t].adj[0];
  return tri[t].adj[1];
}

struct Polar {
  short coord[kMaxPfv];  // vertex of the polar face: a hull triangle
  short nl[kMaxPfv];     // the face's normal: a polar point
  short next[kMaxPfv];   // next vertex, counter-clockwise
  int nfaces;            // heads: entries 0 .. nfaces - 1
};

// TRI_Polarise, tri.c:352-447: one polar face per hull vertex, in point
// order, listing the hull triangles around it (from the first triangle that
// holds it); the polar vertex of triangle t is out / -d, d the smallest
// -<out, ver> over its vertices, clamped to -eps
B2_HD B2_NOINLINE static bool polarise(const OutTri* tri, int m, const double* y, double* w, Polar& P, int npts) {
  short first[kMaxPlanes];
  for (int i = 0; i < npts; i++) first[i] = -1;
  int cnt = 0;
  for (int t = 0; t < m; t++)
    for (int i = 0; i < 3; i++) {
      const int v = tri[t].ver[i];
      if (first[v] >= 0) continue;
      cnt++;
      int s, j;
      for (s = tri_nextaround(tri, t, v), j = 0; s >= 0 && s != t && j < m; s = tri_nextaround(tri, s, v), j++) cnt++;
      if (s < 0 || j >= m) return false;
      first[v] = (short)t;
    }
  if (cnt > kMaxPfv) return false;
  for (int t = 0; t < m; t++) {
    const double* o = tri[t].out;
    double d = 0.0;
    for (int i = 0; i < 3; i++) {
      const double* q = y + 3 * tri[t].ver[i];
      const double x = -(o[0] * q[0] + o[1] * q[1] + o[2] * q[2]);
      if (x < d) d = x;
    }
    if (d > kGeomEps) return false;
    if (d > -kGeomEps) d = -kGeomEps;
    w[3 * t] = o[0] / -d; w[3 * t + 1] = o[1] / -d; w[3 * t + 2] = o[2] / -d;
  }
  int i = 0;
  for (int v = 0; v < npts; v++) {
    if (first[v] < 0) continue;
    int t = first[v];
    P.coord[i] = (short)t; P.nl[i] = (short)v;
    int q = i;
    for (const int s = t; (t = tri_nextaround(tri, t, v)) != s;) {
      const int p = --cnt;
      P.coord[p] = (short)t; P.nl[p] = (short)v;
      P.next[q] = (short)p;
      q = p;
    }
    P.next[q] = (short)i;
    i++;
  }
  P.nfaces = i;
  return true;
}

// nearest_surface, goc.c:107-126
B2_HD inline int nearest_surface(const double* pnt, const double* pla, const int* sur, int n) {
  double min = DBL_MAX;
  int ret = sur[0];
  for (int f = 0; f < n; f++, pla += 6) {
    const double v0 = pnt[0] - pla[3], v1 = pnt[1] - pla[4], v2 = pnt[2] - pla[5];
    const double d = pla[0] * v0 + pla[1] * v1 + pla[2] * v2;
    if (fabs(d) < min) { min = fabs(d); ret = sur[f]; }
  }
  return ret;
}

struct Convex {
  const double* v;  // vertices [3 nv]
  int nv;
  const double* pla;  // planes [6 np]: unit normal, point
  int np;
  const int* sur;  // surface id per plane
  int ns;          // planes on the surface (the first ns)
};

struct Contact {
  double point[3], normal[3], area, gap;
  int spair[2];
};

// per-thread scratch of one convex pair
struct Scratch {
  Hull hull;
  OutTri tri[kMaxHullFaces];
  Polar pol;
  double yy[3 * kMaxPlanes];
  double pv[3 * kMaxHullFaces];
};

// detect_convex_convex (update = false) and update_convex_convex (update =
// true, c.spair holds the current pair): 0 no contact; 1, or 2 when an update
// changed the surface pair; kCviOverflow past the capacities above
B2_HD B2_NOINLINE static int convex_convex(const Convex& A, const Convex& B, bool update, Contact& c, Scratch& s) {
  double p[3], q[3];
  // cvi, cvi.c:118-230 (NON_REGULARIZED: the closest point p is not refined)
  const double dist = gjk_polytopes(A.v, A.nv, B.v, B.nv, p, q);
  if (dist > kGeomEps) return 0;
  const int npts = A.np + B.np;
  if (npts > kMaxPlanes) return kCviOverflow;
  double e[6] = {DBL_MAX, DBL_MAX, DBL_MAX, -DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int k = 0; k < 2; k++) {  // vertices_extents, cvi.c:68-101
    const Convex& X = k ? B : A;
    for (int i = 0; i < X.nv; i++)
      for (int j = 0; j < 3; j++) {
        const double x = X.v[3 * i + j];
        if (x < e[j]) e[j] = x;
        if (x > e[3 + j]) e[3 + j] = x;
      }
  }
  for (int j = 0; j < 3; j++) { e[j] -= kGeomEps; e[3 + j] += kGeomEps; }
  for (int k = 0, i = 0; k < 2; k++) {  // the planes moved to p = 0, as polar points
    const Convex& X = k ? B : A;
    for (int f = 0; f < X.np; f++, i++) {
      const double* nl = X.pla + 6 * f;
      const double t[3] = {nl[3] - p[0], nl[4] - p[1], nl[5] - p[2]};
      double d = -(nl[0] * t[0] + nl[1] * t[1] + nl[2] * t[2]);
      if (d > -kGeomEps) d = -kGeomEps;
      s.yy[3 * i] = nl[0] / -d; s.yy[3 * i + 1] = nl[1] / -d; s.yy[3 * i + 2] = nl[2] / -d;
    }
  }
  const int m = s.hull.build(s.yy, npts, s.tri);
  if (m < 0) return s.hull.overflow ? kCviOverflow : 0;
  if (!polarise(s.tri, m, s.yy, s.pv, s.pol, npts)) return 0;
  int nver = 0;
  for (int k = 0; k < s.pol.nfaces; k++) {
    nver++;
    for (int w = s.pol.next[k]; w != k; w = s.pol.next[w]) nver++;
  }
  if (nver - s.pol.nfaces * 2 <= 3) return 0;
  for (int k = 0; k < m; k++) {  // back to the old origin, within the extents
    double* x = s.pv + 3 * k;
    x[0] = x[0] + p[0]; x[1] = x[1] + p[1]; x[2] = x[2] + p[2];
    if (x[0] < e[0] || x[1] < e[1] || x[2] < e[2] || x[0] > e[3] || x[1] > e[4] || x[2] > e[5]) return 0;
  }
  // point_normal_spair_area_gap, goc.c:148-277, over the triangle fans of the
  // polar faces (cvi.c:205-219) as they are produced
  double normal[3] = {0.0, 0.0, 0.0}, point[3] = {0.0, 0.0, 0.0}, area = 0.0;
  for (int k = 0; k < s.pol.nfaces; k++) {
    const int nlk = s.pol.nl[k];
    double out[3] = {s.yy[3 * nlk], s.yy[3 * nlk + 1], s.yy[3 * nlk + 2]};
    const double len = sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
    out[0] /= len; out[1] /= len; out[2] /= len;
    int flg = nlk + 1;
    if (flg > A.np) flg = -(flg - A.np);
    const bool on_a = flg > 0 && flg < A.ns + 1;
    const bool on_b = flg < 0 && -flg < B.ns + 1;
    const double* v0 = s.pv + 3 * s.pol.coord[k];
    for (int w = s.pol.next[k], z = s.pol.next[w]; z != k; w = s.pol.next[w], z = s.pol.next[z]) {
      const double* v1 = s.pv + 3 * s.pol.coord[w];
      const double* v2 = s.pv + 3 * s.pol.coord[z];
      const double ab[3] = {v0[0] - v1[0], v0[1] - v1[1], v0[2] - v1[2]};
      const double cb[3] = {v2[0] - v1[0], v2[1] - v1[1], v2[2] - v1[2]};
      const double nl[3] = {ab[1] * cb[2] - ab[2] * cb[1], ab[2] * cb[0] - ab[0] * cb[2], ab[0] * cb[1] - ab[1] * cb[0]};
      const double a = 0.5 * sqrt(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
      const double b = a * a;
      if (on_a) for (int j = 0; j < 3; j++) normal[j] = normal[j] + b * out[j];
      if (on_b) for (int j = 0; j < 3; j++) normal[j] = normal[j] - b * out[j];
      double mid[3];
      for (int j = 0; j < 3; j++) mid[j] = .333333333333333 * (v0[j] + v1[j] + v2[j]);
      for (int j = 0; j < 3; j++) point[j] = point[j] + a * mid[j];
      area += a;
    }
  }
  for (int j = 0; j < 3; j++) point[j] /= area;
  {
    const double len = sqrt(normal[0] * normal[0] + normal[1] * normal[1] + normal[2] * normal[2]);
    normal[0] /= len; normal[1] /= len; normal[2] /= len;
  }
  area *= 0.5;
  double tmp[3];
  if (gjk_convex_point(A.v, A.nv, point, tmp) > kGeomEps || gjk_convex_point(B.v, B.nv, point, tmp) > kGeomEps)
    return 0;
  int state = 1;
  if (!update) {
    c.spair[0] = nearest_surface(point, A.pla, A.sur, A.ns);
    c.spair[1] = nearest_surface(point, B.pla, B.sur, B.ns);
  } else {
    int j;
    if ((j = nearest_surface(point, A.pla, A.sur, A.ns)) != c.spair[0]) c.spair[0] = j, state = 2;
    if ((j = nearest_surface(point, B.pla, B.sur, B.ns)) != c.spair[1]) c.spair[1] = j, state = 2;
  }
  double neg = DBL_MAX, pos = -DBL_MAX, gap;
  for (int k = 0; k < m; k++) {
    const double* x = s.pv + 3 * k;
    const double a = normal[0] * x[0] + normal[1] * x[1] + normal[2] * x[2];
    if (a > pos) pos = a;
    if (a < neg) neg = a;
  }
  if (neg == DBL_MAX || pos == -DBL_MAX) gap = 0.0;
  else gap = neg - pos;
  if (gap < -kGeomEps) {  // the convexes moved apart by the penetration along the normal
    const double a = -gap;
    double* aa = s.yy;  // the polar points and polar vertices are no longer needed
    double* tb = s.pv;
    if (A.nv > kMaxPlanes || B.nv > kMaxHullFaces) return kCviOverflow;
    for (int i = 0; i < A.nv; i++)
      for (int j = 0; j < 3; j++) aa[3 * i + j] = A.v[3 * i + j] - a * normal[j];
    for (int i = 0; i < B.nv; i++)
      for (int j = 0; j < 3; j++) tb[3 * i + j] = B.v[3 * i + j] + a * normal[j];
    const double b = gjk_polytopes(aa, A.nv, tb, B.nv, p, q) - 2 * a;
    gap = b < 0.0 ? b : 0.0;
  }
  for (int j = 0; j < 3; j++) { c.point[j] = point[j]; c.normal[j] = normal[j]; }
  c.area = area;
  c.gap = gap;
  const double sanity = point[0] + point[1] + point[2] + normal[0] + normal[1] + normal[2] + area + gap;
  if (!(fabs(sanity) <= DBL_MAX)) return 0;  // not finite
  return state;
}

}  // namespace cvi
}  // namespace b2
