// b2_gjk.cuh -- the reference's GJK distance routines (gjk.c) for the
// contact geometry, callable from device and host code: Johnson's
// sub-algorithm, the distance from a point to a convex hull
// (gjk_convex_point) and between two convex hulls (gjk). Built without fused
// multiply-adds, they reproduce the reference's arithmetic bit for bit.
#pragma once

#include <cfloat>
#include <cmath>

#if defined(__CUDACC__)
#define B2_HD __host__ __device__
#define B2_NOINLINE __noinline__
#else
#define B2_HD
#define B2_NOINLINE __attribute__((noinline))
#endif

namespace b2 {

constexpr double kGeomEps = 1e-6;  // GEOMETRIC_EPSILON, alg.c:24

// Johnson's sub-algorithm as gjk.c:213-330 evaluates it: sub-simplices tried
// in a fixed order (singletons, pairs, triples, the whole simplex), the first
// whose barycentric weights are positive on its members and non-positive off
// them gives the projection of the origin. w[i] holds a Minkowski point and
// wa[i] the index of its hull vertex.
B2_HD B2_NOINLINE static int johnson_project(double (*w)[3], int* wa, int n, double* l, double* v) {
  const int sub_mask[15] = {1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 12, 11, 13, 14, 15};
  const int sub_count[5] = {0, 0, 3, 7, 15};
  double dot[4][4], delta[16][4];
  if (n == 1) {
    l[0] = 1.0;
    v[0] = w[0][0]; v[1] = w[0][1]; v[2] = w[0][2];
    return 1;
  }
  for (int i = 0; i < n; i++)
    for (int j = i; j < n; j++) {
      dot[i][j] = w[i][0] * w[j][0] + w[i][1] * w[j][1] + w[i][2] * w[j][2];
      dot[j][i] = dot[i][j];
    }
  for (int m = 0; m < sub_count[n]; m++) {
    const int s = sub_mask[m];
    bool ok = true;
    int k = -1;
    if ((s & (s - 1)) == 0) {
      for (int i = 0; i < n; i++)
        if (s & (1 << i)) { delta[s][i] = 1.0; k = i; break; }
      for (int j = 0; j < n; j++)
        if (!(s & (1 << j))) {
          delta[s][j] = dot[k][k] - dot[k][j];
          if (delta[s][j] > 0.0) ok = false;
        }
    } else {
      for (int i = 0; i < n; i++)
        if (s & (1 << i)) {
          if (k < 0) k = i;
          delta[s][i] = delta[s & ~(1 << i)][i];
          if (delta[s][i] <= 0.0) ok = false;
        }
      for (int j = 0; j < n; j++)
        if (!(s & (1 << j))) {
          delta[s][j] = 0.0;
          for (int i = 0; i < n; i++)
            if (s & (1 << i)) delta[s][j] += delta[s][i] * (dot[i][k] - dot[i][j]);
          if (delta[s][j] > 0.0) ok = false;
        }
    }
    if (ok) {
      int o = 0;
      double sum = 0.0;
      for (int i = 0; i < n; i++)
        if (s & (1 << i)) {
          w[o][0] = w[i][0]; w[o][1] = w[i][1]; w[o][2] = w[i][2];
          wa[o] = wa[i];
          l[o] = delta[s][i];
          sum += l[o];
          o++;
        }
      v[0] = v[1] = v[2] = 0.0;
      for (int i = 0; i < o; i++) {
        l[i] /= sum;
        for (int c = 0; c < 3; c++) v[c] = v[c] + l[i] * w[i][c];
      }
      return o;
    }
  }
  return 0;
}

// gjk_convex_point, gjk.c:510-556: distance from p to the hull of the na
// vertices a[3 na] and the nearest hull point q (an upper bound of the exact
// distance within GEOMETRIC_EPSILON)
B2_HD B2_NOINLINE static double gjk_convex_point(const double* a, int na, const double* p, double* q) {
  double w[4][3], v[3], l[4], mi = 0.0;
  int wa[4];
  int n = 0, j = 0;
  bool toofar = true;
  const int k = 4 * na * na;
  v[0] = a[0] - p[0]; v[1] = a[1] - p[1]; v[2] = a[2] - p[2];
  double vlen = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  while (toofar && vlen > kGeomEps && n < 4 && j++ < k) {
    double dmin = DBL_MAX;
    int best = 0;
    for (int t = 0; t < na; t++) {
      const double d = a[3 * t] * v[0] + a[3 * t + 1] * v[1] + a[3 * t + 2] * v[2];
      if (d < dmin) { dmin = d; best = t; }
    }
    wa[n] = best;
    w[n][0] = a[3 * best] - p[0]; w[n][1] = a[3 * best + 1] - p[1]; w[n][2] = a[3 * best + 2] - p[2];
    const double delta = (v[0] * w[n][0] + v[1] * w[n][1] + v[2] * w[n][2]) / vlen;
    mi = mi > delta ? mi : delta;
    toofar = (vlen - mi) > kGeomEps;
    if (toofar) {
      n = johnson_project(w, wa, n + 1, l, v);
      vlen = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
  }
  if (n) {
    q[0] = q[1] = q[2] = 0.0;
    for (n--; n >= 0; n--)
      for (int c = 0; c < 3; c++) q[c] = q[c] + l[n] * a[3 * wa[n] + c];
  } else {
    q[0] = a[0]; q[1] = a[1]; q[2] = a[2];
  }
  return vlen;
}

// gjk, gjk.c:340-391: distance of the hulls of the na vertices a[3 na] and the
// nb vertices b[3 nb] and their nearest points p (in a) and q (in b). The
// support points are the first vertex of a with the smallest, and of b with
// the largest, projection on the search direction.
B2_HD B2_NOINLINE static double gjk_polytopes(const double* a, int na, const double* b, int nb, double* p, double* q) {
  double w[4][3], v[3], l[4], mi = 0.0;
  int wa[4], wb[4];
  int n = 0, j = 0;
  bool toofar = true;
  const int k = (na + nb) * (na + nb);
  v[0] = a[0] - b[0]; v[1] = a[1] - b[1]; v[2] = a[2] - b[2];
  double vlen = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  while (toofar && vlen > kGeomEps && n < 4 && j++ < k) {
    double dmin = DBL_MAX, dmax = -DBL_MAX;
    int sa = 0, sb = 0;
    for (int t = 0; t < na; t++) {
      const double d = a[3 * t] * v[0] + a[3 * t + 1] * v[1] + a[3 * t + 2] * v[2];
      if (d < dmin) { dmin = d; sa = t; }
    }
    for (int t = 0; t < nb; t++) {
      const double d = b[3 * t] * v[0] + b[3 * t + 1] * v[1] + b[3 * t + 2] * v[2];
      if (d > dmax) { dmax = d; sb = t; }
    }
    wa[n] = sa;
    wb[n] = sb;
    for (int c = 0; c < 3; c++) w[n][c] = a[3 * sa + c] - b[3 * sb + c];
    const double delta = (v[0] * w[n][0] + v[1] * w[n][1] + v[2] * w[n][2]) / vlen;
    mi = mi > delta ? mi : delta;
    toofar = (vlen - mi) > kGeomEps;
    if (toofar) {
      // johnson_project keeps one index per simplex point: carry both
      // supports in one int (a index in the low 16 bits)
      int wab[4];
      for (int i = 0; i <= n; i++) wab[i] = wa[i] | (wb[i] << 16);
      n = johnson_project(w, wab, n + 1, l, v);
      for (int i = 0; i < n; i++) { wa[i] = wab[i] & 0xffff; wb[i] = wab[i] >> 16; }
      vlen = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    }
  }
  if (n) {
    p[0] = p[1] = p[2] = 0.0;
    q[0] = q[1] = q[2] = 0.0;
    for (n--; n >= 0; n--)
      for (int c = 0; c < 3; c++) {
        p[c] = p[c] + l[n] * a[3 * wa[n] + c];
        q[c] = q[c] + l[n] * b[3 * wb[n] + c];
      }
  } else {
    for (int c = 0; c < 3; c++) { p[c] = a[c]; q[c] = b[c]; }
  }
  return vlen;
}

}  // namespace b2
