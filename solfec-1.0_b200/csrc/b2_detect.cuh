// b2_detect.cuh -- contact update and detection between spheres of rigid bodies,
// and between spheres and convex obstacles (the contact part of
// DOM_Update_Begin, dom.c:3700-3790, for those pairs).
//
//   k_sph_centres   SPHERE_Update with BODY_Cur_Point (sph.c:322-344,
//                   bod.c:1702-1716); largest radius for the cell size
//   k_sph_cells     uniform grid cell of each centre (edge 2 r_max + 2 eps) and
//                   its hash bucket
//   k_sph_buckets   first and last sorted sphere of each bucket
//   k_cvx_update    convex obstacles moved with their bodies (CONVEX_Update,
//                   cvx.c:1362-1396): vertices, face planes, bounding box
//   k_sph_pairs     per sphere i, the spheres j > i of the 27 surrounding cells
//                   whose gjk_sphere_sphere gap (gjk.c:560-584) is below
//                   GEOMETRIC_EPSILON (goc.c:431), bodies different and not
//                   both obstacles (box.c:104-108): counted, then written
//   k_sph_sort_seg  the pairs of each sphere in ascending j (list order)
//   k_cvx_pairs     per sphere, the convexes whose gjk_convex_point distance
//                   (gjk.c:510-556) is below r + GEOMETRIC_EPSILON (goc.c:319),
//                   after a box test, with the same body filters: counted,
//                   then written after the sphere's sphere partners
//   k_sph_contacts  one contact per pair: roles kept from the previous step
//                   (update_contact, dom.c:430-484; update_sphere_sphere,
//                   goc.c:658-677) or set by the centres' point order
//                   (detect_sphere_sphere, goc.c:421-456); spatial point,
//                   normal, gap (goc.c:52-61), referential points
//                   (BODY_Ref_Point, bod.c:1736-1750), local base (localbase,
//                   dom.c:133-151), surface material, carried R and U; for a
//                   convex partner detect_convex_sphere (goc.c:308-349)
//   k_sph_body_*    per body, its contacts (sparsification neighbourhoods)
//   k_sph_sparsify  sparsify_contacts (dom.c:2956-3054) for sphere contacts
//                   (area 1): a new contact within 2 mindist (max-norm) of an
//                   old contact, or of a later new one, of one of its bodies
//   k_sph_compact   the kept contacts into the scene arrays
//
// Every pair with gap below GEOMETRIC_EPSILON has its centres within
// r_i + r_j + eps < cell edge along each axis, so the 27 cells around a sphere
// hold all its candidates; the reference's inflated AABBs (sph.c:240-252) also
// overlap for every such pair, so the grid replaces its broad phase exactly.
// Arithmetic follows the reference's macros (alg.h) operation by operation;
// the library is built without fused multiply-adds, so results match the
// oracle bit for bit.
#pragma once

#include <cfloat>
#include <cstdint>

#include "b2_cvi.cuh"
#include "b2_gjk.cuh"

namespace b2 {

struct SphereDev {
  int nsph, nbod;
  const int* body;      // body of each sphere
  const double* ref;    // referential centre [3]
  const double* rad;    // radius
  const int* surf;      // surface id
  double* cur;          // current centre [3]
  int4* cell;           // grid cell (x, y, z, unused)
  unsigned int* hkey;   // hash bucket of the cell
};

__device__ __forceinline__ void cur_point(const double* R, const double* c, const double* X0, const double* X,
                                          double* x) {
  const double A0 = X[0] - X0[0], A1 = X[1] - X0[1], A2 = X[2] - X0[2];
  x[0] = c[0] + (R[0] * A0 + R[3] * A1 + R[6] * A2);
  x[1] = c[1] + (R[1] * A0 + R[4] * A1 + R[7] * A2);
  x[2] = c[2] + (R[2] * A0 + R[5] * A1 + R[8] * A2);
}

__device__ __forceinline__ void ref_point(const double* R, const double* c, const double* X0, const double* x,
                                          double* X) {
  const double a0 = x[0] - c[0], a1 = x[1] - c[1], a2 = x[2] - c[2];
  X[0] = X0[0] + (R[0] * a0 + R[1] * a1 + R[2] * a2);
  X[1] = X0[1] + (R[3] * a0 + R[4] * a1 + R[5] * a2);
  X[2] = X0[2] + (R[6] * a0 + R[7] * a1 + R[8] * a2);
}

// gjk_sphere_sphere, gjk.c:560-584: gap and the closest points p (on a), q (on b)
__device__ __forceinline__ double gjk_spheres(const double* a, double ra, const double* b, double rb, double* p,
                                              double* q) {
  const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  const double dlen = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  if (dlen == 0.0) {
    p[0] = a[0]; p[1] = a[1]; p[2] = a[2];
    q[0] = b[0]; q[1] = b[1]; q[2] = b[2];
    return 0.0;
  }
  double deno = ra / dlen;
  p[0] = a[0] - deno * d0; p[1] = a[1] - deno * d1; p[2] = a[2] - deno * d2;
  deno = rb / dlen;
  q[0] = b[0] + deno * d0; q[1] = b[1] + deno * d1; q[2] = b[2] + deno * d2;
  deno = ra + rb;
  if (dlen > deno) return dlen - deno;
  p[0] = .5 * (p[0] + q[0]); p[1] = .5 * (p[1] + q[1]); p[2] = .5 * (p[2] + q[2]);
  q[0] = p[0]; q[1] = p[1]; q[2] = p[2];
  return 0.0;
}

// the gap alone (the same operations as gjk_spheres up to its return value)
__device__ __forceinline__ double gjk_spheres_gap(const double* a, double ra, const double* b, double rb) {
  const double d0 = a[0] - b[0], d1 = a[1] - b[1], d2 = a[2] - b[2];
  const double dlen = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
  const double deno = ra + rb;
  return dlen > deno ? dlen - deno : 0.0;
}

// localbase, dom.c:133-151
__device__ __forceinline__ void local_base(const double* n, double* loc) {
  const double e0[3] = {1., 0., 0.}, e1[3] = {0., 1., 0.};
  loc[6] = n[0]; loc[7] = n[1]; loc[8] = n[2];
  loc[0] = e0[1] * n[2] - e0[2] * n[1];
  loc[1] = e0[2] * n[0] - e0[0] * n[2];
  loc[2] = e0[0] * n[1] - e0[1] * n[0];
  double len = sqrt(loc[0] * loc[0] + loc[1] * loc[1] + loc[2] * loc[2]);
  if (len < kGeomEps) {
    loc[0] = e1[1] * n[2] - e1[2] * n[1];
    loc[1] = e1[2] * n[0] - e1[0] * n[2];
    loc[2] = e1[0] * n[1] - e1[1] * n[0];
    len = sqrt(loc[0] * loc[0] + loc[1] * loc[1] + loc[2] * loc[2]);
  }
  loc[0] /= len; loc[1] /= len; loc[2] /= len;
  loc[3] = loc[1] * n[2] - loc[2] * n[1];
  loc[4] = loc[2] * n[0] - loc[0] * n[2];
  loc[5] = loc[0] * n[1] - loc[1] * n[0];
}

// pntcmp, goc.c:409-419
__device__ __forceinline__ int point_cmp(const double* a, const double* b) {
  for (int i = 0; i < 3; i++) {
    if (a[i] < b[i]) return -1;
    if (a[i] > b[i]) return 1;
  }
  return 0;
}

// ---- convex obstacles (detect_convex_sphere, goc.c:308-349) ----

struct ConvexDev {
  int n;
  const int* body;     // body of each convex
  const int* vptr;     // vertices of convex c: vptr[c] .. vptr[c+1]-1
  const double* vert;  // referential vertices [3]
  const int* fptr;     // faces of convex c in fac[fptr[c] ..]: count, then vertex indices
  const int* fac;
  const int* sptr;     // faces of convex c: sptr[c] .. sptr[c+1]-1 (surface ids, planes)
  const int* surf;
  const int* nsurf_face;  // faces before the first internal one (surface -INT_MAX)
  double* cur;         // current vertices [3]
  double* pla;         // per face unit normal and first vertex [6]
  double* box;         // per convex min[3], max[3] of the current vertices
};

// computeplanes (cvx.c:72-89) in CONVEX_Planes' layout, current vertices from
// the body (CONVEX_Update, cvx.c:1362-1396) and the bounding box: one thread
// per convex (obstacles and other large shapes are few)
__global__ void k_cvx_update(ConvexDev cv, const double* rot, const double* xb, const double* x0) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cv.n) return;
  const int b = cv.body[c];
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int v = cv.vptr[c]; v < cv.vptr[c + 1]; v++) {
    double x[3];
    cur_point(rot + 9 * (size_t)b, xb + 3 * (size_t)b, x0 + 3 * (size_t)b, cv.vert + 3 * (size_t)v, x);
    for (int k = 0; k < 3; k++) {
      cv.cur[3 * (size_t)v + k] = x[k];
      lo[k] = x[k] < lo[k] ? x[k] : lo[k];
      hi[k] = x[k] > hi[k] ? x[k] : hi[k];
    }
  }
  for (int k = 0; k < 3; k++) { cv.box[6 * c + k] = lo[k]; cv.box[6 * c + 3 + k] = hi[k]; }
  const double* cur = cv.cur + 3 * (size_t)cv.vptr[c];
  for (int f = cv.sptr[c], m = cv.fptr[c]; f < cv.sptr[c + 1]; f++, m += cv.fac[m] + 1) {
    const double* a = cur + 3 * cv.fac[m + 1];
    const double* bb = cur + 3 * cv.fac[m + 2];
    const double* cc = cur + 3 * cv.fac[m + 3];
    const double ba0 = bb[0] - a[0], ba1 = bb[1] - a[1], ba2 = bb[2] - a[2];
    const double cb0 = cc[0] - bb[0], cb1 = cc[1] - bb[1], cb2 = cc[2] - bb[2];
    double* nl = cv.pla + 6 * (size_t)f;
    nl[0] = ba1 * cb2 - ba2 * cb1;
    nl[1] = ba2 * cb0 - ba0 * cb2;
    nl[2] = ba0 * cb1 - ba1 * cb0;
    const double len = sqrt(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
    nl[0] /= len; nl[1] /= len; nl[2] /= len;
    nl[3] = a[0]; nl[4] = a[1]; nl[5] = a[2];
  }
}

// nearest_normal and nearest_surface, goc.c:87-122
__device__ __forceinline__ int nearest_plane_max(const double* pnt, const double* pla, int n) {
  double max = -DBL_MAX;
  int ret = -1;
  for (int f = 0; f < n; f++, pla += 6) {
    const double v0 = pnt[0] - pla[3], v1 = pnt[1] - pla[4], v2 = pnt[2] - pla[5];
    const double d = pla[0] * v0 + pla[1] * v1 + pla[2] * v2;
    if (d > max) { ret = f; max = d; }
  }
  return ret;
}

__device__ __forceinline__ int nearest_surface_id(const double* pnt, const double* pla, const int* sur, int n) {
  double min = DBL_MAX;
  int ret = sur[0];
  for (int f = 0; f < n; f++, pla += 6) {
    const double v0 = pnt[0] - pla[3], v1 = pnt[1] - pla[4], v2 = pnt[2] - pla[5];
    const double d = pla[0] * v0 + pla[1] * v1 + pla[2] * v2;
    if (fabs(d) < min) { min = fabs(d); ret = sur[f]; }
  }
  return ret;
}

// CONTACT_EXCLUDE_BODIES (lng.c:8817-8852; the nobody set of box.c:116-118):
// excluded body pairs as min << 32 | max keys in ascending order
struct PairFilter {
  const long long* body_pairs;
  int n;
};

__device__ __forceinline__ bool body_pair_excluded(const PairFilter& f, int a, int b) {
  if (f.n == 0) return false;
  const long long key = ((long long)(a < b ? a : b) << 32) | (long long)(a < b ? b : a);
  int lo = 0, hi = f.n - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const long long v = f.body_pairs[mid];
    if (v == key) return true;
    if (v < key) lo = mid + 1; else hi = mid - 1;
  }
  return false;
}

// CONTACT_EXCLUDE_SURFACES (lng.c:8855-8872; dom.c:379-389): a new contact of
// an excluded surface pair is not created (nosurf[s1 * nsurf + s2], symmetric,
// or null); UNPHYSICAL_PENETRATION (lng.c:9175-9191): a contact whose gap is
// at or below depth (negative; -DBL_MAX unless set) sets bad flag 128, where
// the reference stops (dom.c:374, 461, 3792)
struct ContactRules {
  const unsigned char* nosurf;
  double depth;
};

__device__ __forceinline__ unsigned int cell_hash(int x, int y, int z, unsigned int mask) {
  return (((unsigned int)x * 73856093u) ^ ((unsigned int)y * 19349663u) ^ ((unsigned int)z * 83492791u)) & mask;
}

// bad flags (bit or): 1 a radius not positive and finite or a centre not finite,
// 2 a centre too far from the origin for the grid, 4 two coincident centres,
// 8 a surface id out of range, 16 a body index out of range, 32 a convex
// without a finite face plane
__global__ void k_sph_centres(SphereDev s, const double* rot, const double* xb, const double* x0,
                              unsigned long long* rmax_bits, int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long rb = 0;  // this thread's radius bits (positive doubles order as integers)
  if (i < s.nsph) {
    const int b = s.body[i];
    if (b < 0 || b >= s.nbod) {
      atomicOr(bad, 16);
    } else {
      double c[3];
      cur_point(rot + 9 * (size_t)b, xb + 3 * (size_t)b, x0 + 3 * (size_t)b, s.ref + 3 * (size_t)i, c);
      s.cur[3 * (size_t)i] = c[0]; s.cur[3 * (size_t)i + 1] = c[1]; s.cur[3 * (size_t)i + 2] = c[2];
      const double r = s.rad[i];
      if (!(r > 0.0) || !isfinite(r) || !isfinite(c[0]) || !isfinite(c[1]) || !isfinite(c[2])) atomicOr(bad, 1);
      else rb = (unsigned long long)__double_as_longlong(r);
    }
  }
  // the largest radius: a warp maximum, then one atomic per warp (every lane
  // of the warp reaches the shuffles: the block size is a multiple of 32)
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long v = __shfl_xor_sync(0xffffffffu, rb, o);
    rb = v > rb ? v : rb;
  }
  if ((threadIdx.x & 31) == 0 && rb) atomicMax(rmax_bits, rb);
}

__global__ void k_sph_cells(SphereDev s, const unsigned long long* rmax_bits, unsigned int mask, int* sidx,
                            int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.nsph) return;
  const double h = 2.0 * __longlong_as_double((long long)*rmax_bits) + 2.0 * kGeomEps;
  int q[3];
  for (int k = 0; k < 3; k++) {
    const double f = floor(s.cur[3 * (size_t)i + k] / h);
    if (!(fabs(f) < 1.0e9)) { atomicOr(bad, 2); q[k] = 0; }
    else q[k] = (int)f;
  }
  s.cell[i] = make_int4(q[0], q[1], q[2], 0);
  s.hkey[i] = cell_hash(q[0], q[1], q[2], mask);
  sidx[i] = i;
}

__global__ void k_sph_buckets(int n, const unsigned int* key, int* bstart, int* bend) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const unsigned int k = key[t];
  if (t == 0 || key[t - 1] != k) bstart[k] = t;
  if (t == n - 1 || key[t + 1] != k) bend[k] = t + 1;
}

// WRITE = false: count[i] = pairs (i, j > i); WRITE = true: their j at off[i]..
template <bool WRITE>
__global__ void k_sph_pairs(SphereDev s, const int* obst, PairFilter pf, const int* sorted, const int* bstart,
                            const int* bend, unsigned int mask, int* count, const int* off, int* pj) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= s.nsph) return;
  const int i = sorted[t];
  const int4 ci = s.cell[i];
  const int bi = s.body[i];
  if (bi < 0 || bi >= s.nbod) return;  // reported by k_sph_centres
  const bool oi = obst[bi] != 0;
  const double a[3] = {s.cur[3 * (size_t)i], s.cur[3 * (size_t)i + 1], s.cur[3 * (size_t)i + 2]};
  const double ra = s.rad[i];
  int cnt = 0;
  int w = WRITE ? off[i] : 0;
  for (int dz = -1; dz <= 1; dz++)
    for (int dy = -1; dy <= 1; dy++)
      for (int dx = -1; dx <= 1; dx++) {
        const int nx = ci.x + dx, ny = ci.y + dy, nz = ci.z + dz;
        const unsigned int hb = cell_hash(nx, ny, nz, mask);
        const int u0 = bstart[hb], u1 = bend[hb];
        for (int u = u0; u < u1; u++) {
          const int j = sorted[u];
          if (j <= i) continue;
          const int4 cj = s.cell[j];
          if (cj.x != nx || cj.y != ny || cj.z != nz) continue;  // another cell in the same bucket
          const int bj = s.body[j];
          if (bj < 0 || bj >= s.nbod || bj == bi || (oi && obst[bj]) || body_pair_excluded(pf, bi, bj)) continue;
          const double b[3] = {s.cur[3 * (size_t)j], s.cur[3 * (size_t)j + 1], s.cur[3 * (size_t)j + 2]};
          if (gjk_spheres_gap(a, ra, b, s.rad[j]) < kGeomEps) {
            if (WRITE) pj[w++] = j;
            cnt++;
          }
        }
      }
  if (!WRITE) count[i] = cnt;
}

// convex partners of sphere i (pair index nsph + c): a box test first (the
// distance test accepts only spheres within r + eps of the hull), then the
// gjk_convex_point distance. WRITE = false: ccount[i]; WRITE = true: written
// after the sphere's sphere partners, at off[i] + scount[i]
template <bool WRITE>
__global__ void k_cvx_pairs(SphereDev s, ConvexDev cv, const int* obst, PairFilter pf, int* ccount, const int* off,
                            const int* scount, int* pj) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.nsph) return;
  const int bi = s.body[i];
  if (bi < 0 || bi >= s.nbod) return;  // reported by k_sph_centres
  const bool oi = obst[bi] != 0;
  const double a[3] = {s.cur[3 * (size_t)i], s.cur[3 * (size_t)i + 1], s.cur[3 * (size_t)i + 2]};
  const double ra = s.rad[i];
  int cnt = 0;
  int w = WRITE ? off[i] + scount[i] : 0;
  for (int c = 0; c < cv.n; c++) {
    const int bc = cv.body[c];
    if (bc == bi || (oi && obst[bc]) || body_pair_excluded(pf, bi, bc)) continue;
    const double* bx = cv.box + 6 * (size_t)c;
    bool near = true;
    for (int k = 0; k < 3; k++)
      if (a[k] < bx[k] - ra - 2.0 * kGeomEps || a[k] > bx[3 + k] + ra + 2.0 * kGeomEps) near = false;
    if (!near) continue;
    double q[3];
    if (gjk_convex_point(cv.cur + 3 * (size_t)cv.vptr[c], cv.vptr[c + 1] - cv.vptr[c], a, q) < ra + kGeomEps) {
      if (WRITE) pj[w++] = s.nsph + c;
      cnt++;
    }
  }
  if (!WRITE) ccount[i] = cnt;
}

__global__ void k_add_counts(int n, const int* a, int* b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] += a[i];
}

// Sum of the per-sphere pair counts in 64 bits (the scan that follows runs in
// int, so the host checks this total first): one atomic per warp.
__global__ void k_count_total(int n, const int* cnt, unsigned long long* total) {
  unsigned long long s = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += (unsigned)cnt[i];
#pragma unroll
  for (int d = 16; d >= 1; d >>= 1) s += __shfl_down_sync(0xffffffffu, s, d);
  if ((threadIdx.x & 31) == 0 && s) atomicAdd(total, s);
}

__global__ void k_sph_sort_seg(int nsph, const int* off, int* pj, int* pi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nsph) return;
  const int b = off[i], e = off[i + 1];
  for (int k = b + 1; k < e; k++) {  // a sphere has a few tens of pairs at most
    const int v = pj[k];
    int m = k - 1;
    while (m >= b && pj[m] > v) { pj[m + 1] = pj[m]; m--; }
    pj[m + 1] = v;
  }
  for (int k = b; k < e; k++) pi[k] = i;
}

struct ContactOut {
  int* master; int* slave; double* point; double* mpnt; double* spnt; double* base; double* gap;
  double* fric; double* rest; double* coh; double* R0; double* U0; long long* key; int* slave_lo; int* isnew;
  double* area;
};

__global__ void k_sph_contacts(int npair, SphereDev s, ConvexDev cv, const int* pi, const int* pj, const double* rot,
                               const double* xb, const double* x0, int nsurf, const double* mat, ContactRules cr,
                               int nprev, const long long* prevkey, const int* prevslave_lo, const double* prevR,
                               const double* prevU, ContactOut o, int* bad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= npair) return;
  const int i = pi[k], j = pj[k];
  const long long key = ((long long)i << 32) | (long long)j;
  int hit = -1;
  {  // the previous step's contacts are in ascending key order
    int lo = 0, hi = nprev - 1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      const long long v = prevkey[mid];
      if (v == key) { hit = mid; break; }
      if (v < key) lo = mid + 1; else hi = mid - 1;
    }
  }
  if (j >= s.nsph) {
    // detect_convex_sphere / update_convex_sphere (goc.c:308-349, 555-597):
    // the convex is the slave (its outward normal), the sphere the master
    const int c = j - s.nsph, bc = cv.body[c], bi = s.body[i];
    o.master[k] = bi;
    o.slave[k] = bc;
    o.key[k] = key;
    o.slave_lo[k] = 0;
    o.isnew[k] = hit < 0;
    const double* cc = s.cur + 3 * (size_t)i;
    const double r = s.rad[i];
    const double* pla = cv.pla + 6 * (size_t)cv.sptr[c];
    const int* fs = cv.surf + cv.sptr[c];
    const int ns = cv.nsurf_face[c];
    double one[3], n[3], len;
    gjk_convex_point(cv.cur + 3 * (size_t)cv.vptr[c], cv.vptr[c + 1] - cv.vptr[c], cc, one);
    n[0] = cc[0] - one[0]; n[1] = cc[1] - one[1]; n[2] = cc[2] - one[2];
    const double dot = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
    if (dot == 0.0) {  // centre on the hull: the normal of the plane it is furthest out of
      const int f = nearest_plane_max(one, pla, ns);
      len = r;
      if (f < 0) { atomicOr(bad, 32); n[0] = n[1] = 0.0; n[2] = 1.0; }
      else { n[0] = pla[6 * f]; n[1] = pla[6 * f + 1]; n[2] = pla[6 * f + 2]; }
    } else {
      len = sqrt(dot);
      const double il = 1.0 / len;
      n[0] *= il; n[1] *= il; n[2] *= il;
    }
    double two[3];
    for (int v = 0; v < 3; v++) two[v] = cc[v] + (-r) * n[v];
    const double g = len - r;
    o.gap[k] = g < 0.0 ? g : 0.0;
    for (int v = 0; v < 3; v++) o.point[3 * (size_t)k + v] = two[v];
    double X[3];
    ref_point(rot + 9 * (size_t)bi, xb + 3 * (size_t)bi, x0 + 3 * (size_t)bi, two, X);
    for (int v = 0; v < 3; v++) o.mpnt[3 * (size_t)k + v] = X[v];
    ref_point(rot + 9 * (size_t)bc, xb + 3 * (size_t)bc, x0 + 3 * (size_t)bc, one, X);
    for (int v = 0; v < 3; v++) o.spnt[3 * (size_t)k + v] = X[v];
    double loc[9];
    local_base(n, loc);
    for (int v = 0; v < 9; v++) o.base[9 * (size_t)k + v] = loc[v];
    const int s1 = nearest_surface_id(one, pla, fs, ns), s2 = s.surf[i];
    if (o.gap[k] <= cr.depth) atomicOr(bad, 128);
    if (s1 < 0 || s1 >= nsurf || s2 < 0 || s2 >= nsurf) {
      atomicOr(bad, 8);
      o.fric[k] = o.rest[k] = 0.0;
    } else {
      const size_t t = (size_t)s1 * nsurf + s2;
      o.fric[k] = mat[2 * t];
      o.rest[k] = mat[2 * t + 1];
      if (hit < 0 && cr.nosurf && cr.nosurf[t]) o.master[k] = o.slave[k] = -1;  // an excluded surface pair
    }
    o.coh[k] = 0.0;
    o.area[k] = 1.0;  // detect_convex_sphere, goc.c:341
    for (int v = 0; v < 3; v++) {
      o.R0[3 * (size_t)k + v] = hit >= 0 ? prevR[3 * (size_t)hit + v] : 0.0;
      o.U0[3 * (size_t)k + v] = hit >= 0 ? prevU[3 * (size_t)hit + v] : 0.0;
    }
    return;
  }
  const double* ci = s.cur + 3 * (size_t)i;
  const double* cj = s.cur + 3 * (size_t)j;
  const int lo_slave = hit >= 0 ? prevslave_lo[hit] : (point_cmp(ci, cj) <= 0 ? 1 : 0);
  const int sv = lo_slave ? i : j, ms = lo_slave ? j : i;
  const double* cs = s.cur + 3 * (size_t)sv;
  const double* cm = s.cur + 3 * (size_t)ms;
  const double rs = s.rad[sv], rm = s.rad[ms];
  const int bm = s.body[ms], bs = s.body[sv];
  // every index array of the contact is written before anything is checked:
  // the body lists of the sparsification read them
  o.master[k] = bm;
  o.slave[k] = bs;
  o.key[k] = key;
  o.slave_lo[k] = lo_slave;
  o.isnew[k] = hit < 0;
  double p[3], q[3], n[3];
  gjk_spheres(cs, rs, cm, rm, p, q);
  n[0] = p[0] - cs[0]; n[1] = p[1] - cs[1]; n[2] = p[2] - cs[2];
  const double len = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
  if (!(len > 0.0)) atomicOr(bad, 4);  // coincident centres: the normal is not finite, the call fails
  n[0] /= len; n[1] /= len; n[2] /= len;
  double g;
  {  // sphere_sphere_gap, goc.c:52-61
    const double x0_ = cm[0] - cs[0], x1_ = cm[1] - cs[1], x2_ = cm[2] - cs[2];
    const double d = x0_ * n[0] + x1_ * n[1] + x2_ * n[2];
    const double e = rs + rm;
    g = e > d ? d - e : 0;
  }
  for (int v = 0; v < 3; v++) o.point[3 * (size_t)k + v] = q[v];
  double X[3];
  ref_point(rot + 9 * (size_t)bm, xb + 3 * (size_t)bm, x0 + 3 * (size_t)bm, q, X);
  for (int v = 0; v < 3; v++) o.mpnt[3 * (size_t)k + v] = X[v];
  ref_point(rot + 9 * (size_t)bs, xb + 3 * (size_t)bs, x0 + 3 * (size_t)bs, p, X);
  for (int v = 0; v < 3; v++) o.spnt[3 * (size_t)k + v] = X[v];
  double loc[9];
  local_base(n, loc);
  for (int v = 0; v < 9; v++) o.base[9 * (size_t)k + v] = loc[v];
  o.gap[k] = g;
  if (g <= cr.depth) atomicOr(bad, 128);
  const int s1 = s.surf[sv], s2 = s.surf[ms];
  if (s1 < 0 || s1 >= nsurf || s2 < 0 || s2 >= nsurf) {
    atomicOr(bad, 8);
    o.fric[k] = o.rest[k] = 0.0;
  } else {
    const size_t t = (size_t)s1 * nsurf + s2;
    o.fric[k] = mat[2 * t];
    o.rest[k] = mat[2 * t + 1];
    if (hit < 0 && cr.nosurf && cr.nosurf[t]) o.master[k] = o.slave[k] = -1;  // an excluded surface pair
  }
  o.coh[k] = 0.0;
  o.area[k] = 1.0;  // detect_sphere_sphere, goc.c:436
  for (int v = 0; v < 3; v++) {
    o.R0[3 * (size_t)k + v] = hit >= 0 ? prevR[3 * (size_t)hit + v] : 0.0;
    o.U0[3 * (size_t)k + v] = hit >= 0 ? prevU[3 * (size_t)hit + v] : 0.0;
  }
}

// ---- convex-convex pairs (detect_convex_convex / update_convex_convex) ----
//
// Broad phase: a uniform grid over the centres of the convexes' boxes, its
// cell edge the largest box side of the ordinary convexes plus
// 2 GEOMETRIC_EPSILON; convexes whose box side exceeds kLargeConvex times the
// mean (floors, walls) are listed apart and tested against every convex.
// Two convexes within GEOMETRIC_EPSILON of each other have overlapping
// eps-inflated boxes (CONVEX_Extents, cvx.c:1236-1260), so their centres lie
// in neighbouring cells; a candidate pair then passes the box test and, in
// k_cc_gjk, the GJK distance test of cvi (cvi.c:128-129, gjk of the lower
// convex first), which leaves the narrow phase only pairs that touch. Pairs of one body and
// pairs of two obstacles are left out (box.c:104-108). A pair is keyed by its
// convexes c1 < c2 as (nsph + c1) << 32 | (nsph + c2); the first object of the
// reference's gobjcontact is c1 (the slave, holding the outward normal), the
// second c2 (the master), in detection and update alike (overlap_create,
// dom.c:392-399; update_contact, dom.c:446-450).

constexpr double kLargeConvex = 4.0;

// ext[c] = the largest side of convex c's box; sum += ext[c]
__global__ void k_cc_extent(ConvexDev cv, double* ext, double* sum) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cv.n) return;
  const double* b = cv.box + 6 * c;
  double e = b[3] - b[0];
  if (b[4] - b[1] > e) e = b[4] - b[1];
  if (b[5] - b[2] > e) e = b[5] - b[2];
  ext[c] = e;
  atomicAdd(sum, e);
}

__device__ __forceinline__ bool cc_large(const double* ext, const double* sum, int n, int c) {
  return ext[c] > kLargeConvex * (*sum / n);
}

// the largest side among ordinary convexes (bits of a non-negative double);
// the large ones listed
__global__ void k_cc_classify(int n, const double* ext, const double* sum, unsigned long long* emax, int* large,
                              int* nlarge) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  if (cc_large(ext, sum, n, c)) large[atomicAdd(nlarge, 1)] = c;
  else atomicMax(emax, (unsigned long long)__double_as_longlong(ext[c]));
}

// grid cell of an ordinary convex's box centre and its bucket; a large
// convex goes to bucket mask + 1, which no cell probes. Bad flag 2: a centre
// too far from the origin for the grid.
__global__ void k_cc_cells(ConvexDev cv, const double* ext, const double* sum, const unsigned long long* emax,
                           unsigned int mask, int4* cell, unsigned int* hkey, int* idx, int* bad) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cv.n) return;
  idx[c] = c;
  if (cc_large(ext, sum, cv.n, c)) {
    cell[c] = make_int4(0, 0, 0, 1);
    hkey[c] = mask + 1;
    return;
  }
  const double h = __longlong_as_double((long long)*emax) + 2.0 * kGeomEps;
  const double* b = cv.box + 6 * c;
  int q[3];
  for (int k = 0; k < 3; k++) {
    const double f = floor(0.5 * (b[k] + b[3 + k]) / h);
    if (!(fabs(f) < 1.0e9)) { atomicOr(bad, 2); q[k] = 0; }
    else q[k] = (int)f;
  }
  cell[c] = make_int4(q[0], q[1], q[2], 0);
  hkey[c] = cell_hash(q[0], q[1], q[2], mask);
}

__device__ __forceinline__ bool cc_candidate(const ConvexDev& cv, const int* obst, const PairFilter& pf, int i,
                                             int j) {
  const int bi = cv.body[i], bj = cv.body[j];
  if (bi == bj || (obst[bi] && obst[bj]) || body_pair_excluded(pf, bi, bj)) return false;
  const double* a = cv.box + 6 * i;
  const double* b = cv.box + 6 * j;
  for (int k = 0; k < 3; k++)
    if (!(b[k] - kGeomEps <= a[3 + k] + kGeomEps && a[k] - kGeomEps <= b[3 + k] + kGeomEps)) return false;
  return true;
}

// keep[t] = 1 when the convexes of candidate key t are within GEOMETRIC_EPSILON
// (gjk with the lower convex first, as cvi calls it); cls[t] = a work class of
// the pair for the narrow phase: its plane count, how many of its face normals
// are parallel across the two convexes (aligned boxes make coplanar polar
// points, turned ones do not), along how many axes the two are offset (face,
// edge or corner neighbours) and whether they are apart or overlap, so that a
// warp takes pairs of one kind
__global__ void k_cc_gjk(int n, int nsph, ConvexDev cv, const long long* keys, unsigned char* keep,
                         unsigned int* cls) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const long long key = keys[t];
  const int lo = (int)(key >> 32) - nsph, hi = (int)(key & 0xFFFFFFFFLL) - nsph;
  double p[3], q[3];
  const double dist = gjk_polytopes(cv.cur + 3 * (size_t)cv.vptr[lo], cv.vptr[lo + 1] - cv.vptr[lo],
                                    cv.cur + 3 * (size_t)cv.vptr[hi], cv.vptr[hi + 1] - cv.vptr[hi], p, q);
  keep[t] = dist <= kGeomEps;
  const double* ba = cv.box + 6 * lo;
  const double* bb = cv.box + 6 * hi;
  int sep = 0;  // axes along which the boxes' centres are further apart than a quarter of their summed sides
  for (int k = 0; k < 3; k++) {
    const double da = ba[3 + k] - ba[k], db = bb[3 + k] - bb[k];
    sep += fabs((ba[k] + ba[3 + k]) - (bb[k] + bb[3 + k])) > 0.5 * (da + db);
  }
  const int na = cv.sptr[lo + 1] - cv.sptr[lo], nb = cv.sptr[hi + 1] - cv.sptr[hi];
  const double* pa = cv.pla + 6 * (size_t)cv.sptr[lo];
  const double* pb = cv.pla + 6 * (size_t)cv.sptr[hi];
  int par = 0;
  for (int a = 0; a < na; a++)
    for (int b = 0; b < nb; b++) {
      const double d = pa[6 * a] * pb[6 * b] + pa[6 * a + 1] * pb[6 * b + 1] + pa[6 * a + 2] * pb[6 * b + 2];
      par += fabs(d) > 1.0 - 1e-12;
    }
  cls[t] = ((unsigned int)(na + nb) << 16) | ((unsigned int)(par < 255 ? par : 255) << 8) | ((unsigned int)sep << 1) |
           (unsigned int)(dist > 0.0);
}

// per sorted position t (convex i = sorted[t]): its partners j > i of the 27
// cells around it (ordinary convexes), and the large convexes l (a large i
// pairs only with large l > i). WRITE = false: cnt[t]; WRITE = true: the keys
// from off[t].
template <bool WRITE>
__global__ void k_cc_pairs(ConvexDev cv, const int* obst, PairFilter pf, int nsph, const int* sorted, const int4* cell,
                           const int* bstart, const int* bend, unsigned int mask, const int* large, int nlarge,
                           int* cnt, const int* off, long long* keys) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cv.n) return;
  const int i = sorted[t];
  const int4 ci = cell[i];
  int found = 0, w = WRITE ? off[t] : 0;
  auto emit = [&](int j) {
    if (WRITE) {
      const long long lo = nsph + (i < j ? i : j), hi = nsph + (i < j ? j : i);
      keys[w++] = (lo << 32) | hi;
    }
    found++;
  };
  if (ci.w == 0) {
    for (int dz = -1; dz <= 1; dz++)
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          const int nx = ci.x + dx, ny = ci.y + dy, nz = ci.z + dz;
          const unsigned int hb = cell_hash(nx, ny, nz, mask);
          for (int u = bstart[hb]; u < bend[hb]; u++) {
            const int j = sorted[u];
            if (j <= i) continue;
            const int4 cj = cell[j];
            if (cj.x != nx || cj.y != ny || cj.z != nz) continue;  // another cell in the same bucket
            if (cc_candidate(cv, obst, pf, i, j)) emit(j);
          }
        }
  }
  for (int u = 0; u < nlarge; u++) {
    const int l = large[u];
    if (l == i || (ci.w != 0 && l < i)) continue;
    if (cc_candidate(cv, obst, pf, i, l)) emit(l);
  }
  if (!WRITE) cnt[t] = found;
}

// the contact of candidate pair t (slot k0 + t of the staged arrays): the
// polyhedral intersection of its convexes (b2_cvi.cuh); a pair without a
// contact keeps master = slave = -1 and is dropped by the sparsification. Bad
// flags: 8 a surface id out of the material table, 64 a pair over the
// intersection's capacity (32 planes of both convexes together).
__global__ void __launch_bounds__(64) k_cc_contacts(int ncc, int k0, int nsph, const int* order, ConvexDev cv,
                                                    const long long* ckey,
                                                    const double* rot, const double* xb, const double* x0, int nsurf,
                                                    const double* mat, ContactRules cr, int nprev,
                                                    const long long* prevkey,
                                                    const double* prevR, const double* prevU, ContactOut o, int* bad) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= ncc) return;
  const int t = order[w];  // pairs run in work-class order, results go to their key-order slots
  const int k = k0 + t;
  const long long key = ckey[t];
  const int c1 = (int)(key >> 32) - nsph, c2 = (int)(key & 0xFFFFFFFFLL) - nsph;
  int hit = -1;
  {
    int lo = 0, hi = nprev - 1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1;
      const long long v = prevkey[mid];
      if (v == key) { hit = mid; break; }
      if (v < key) lo = mid + 1; else hi = mid - 1;
    }
  }
  o.key[k] = key;
  o.slave_lo[k] = 1;
  o.isnew[k] = hit < 0;
  o.master[k] = o.slave[k] = -1;
  cvi::Convex A, B;
  const int cc[2] = {c1, c2};
  for (int e = 0; e < 2; e++) {
    cvi::Convex& X = e ? B : A;
    const int c = cc[e];
    X.v = cv.cur + 3 * (size_t)cv.vptr[c];
    X.nv = cv.vptr[c + 1] - cv.vptr[c];
    X.pla = cv.pla + 6 * (size_t)cv.sptr[c];
    X.np = cv.sptr[c + 1] - cv.sptr[c];
    X.sur = cv.surf + cv.sptr[c];
    X.ns = cv.nsurf_face[c];
  }
  cvi::Scratch scratch;
  cvi::Contact ct;
  // update_convex_convex differs from detect_convex_convex only in its return
  // value (2 when the surface pair changed); the contact data are the same
  const int state = cvi::convex_convex(A, B, false, ct, scratch);
  if (state <= 0) {
    if (state == cvi::kCviOverflow) atomicOr(bad, 64);
    return;
  }
  const int bs = cv.body[c1], bm = cv.body[c2];
  o.master[k] = bm;
  o.slave[k] = bs;
  for (int v = 0; v < 3; v++) o.point[3 * (size_t)k + v] = ct.point[v];
  double X[3];
  ref_point(rot + 9 * (size_t)bm, xb + 3 * (size_t)bm, x0 + 3 * (size_t)bm, ct.point, X);
  for (int v = 0; v < 3; v++) o.mpnt[3 * (size_t)k + v] = X[v];
  ref_point(rot + 9 * (size_t)bs, xb + 3 * (size_t)bs, x0 + 3 * (size_t)bs, ct.point, X);
  for (int v = 0; v < 3; v++) o.spnt[3 * (size_t)k + v] = X[v];
  double loc[9];
  local_base(ct.normal, loc);
  for (int v = 0; v < 9; v++) o.base[9 * (size_t)k + v] = loc[v];
  o.gap[k] = ct.gap;
  o.area[k] = ct.area;
  if (ct.gap <= cr.depth) atomicOr(bad, 128);
  const int s1 = ct.spair[0], s2 = ct.spair[1];
  if (s1 < 0 || s1 >= nsurf || s2 < 0 || s2 >= nsurf) {
    atomicOr(bad, 8);
    o.fric[k] = o.rest[k] = 0.0;
  } else {
    const size_t u = (size_t)s1 * nsurf + s2;
    o.fric[k] = mat[2 * u];
    o.rest[k] = mat[2 * u + 1];
    if (hit < 0 && cr.nosurf && cr.nosurf[u]) o.master[k] = o.slave[k] = -1;  // an excluded surface pair
  }
  o.coh[k] = 0.0;
  for (int v = 0; v < 3; v++) {
    o.R0[3 * (size_t)k + v] = hit >= 0 ? prevR[3 * (size_t)hit + v] : 0.0;
    o.U0[3 * (size_t)k + v] = hit >= 0 ? prevU[3 * (size_t)hit + v] : 0.0;
  }
}

// body indices come from k_sph_contacts, which takes them from the checked
// sphere bodies; the range tests below keep a corrupted entry from addressing
// outside the per-body arrays
__global__ void k_sph_body_count(int n, int nb, const int* master, const int* slave, int* bcnt, int* bad) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int m = master[k], s = slave[k];
  if (m == -1 && s == -1) return;  // a convex pair without a contact
  if (m < 0 || m >= nb || s < 0 || s >= nb) { atomicOr(bad, 16); return; }
  atomicAdd(bcnt + m, 1);
  atomicAdd(bcnt + s, 1);
}

__global__ void k_sph_body_fill(int n, int nb, const int* master, const int* slave, int* cursor, int* blist) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int m = master[k], s = slave[k];
  if (m < 0 || m >= nb || s < 0 || s >= nb) return;
  blist[atomicAdd(cursor + m, 1)] = k;
  blist[atomicAdd(cursor + s, 1)] = k;
}

// the objects of a contact as keyed (sphere i, or convex c as nsph + c): the
// slave's and the master's
__device__ __forceinline__ void contact_objects(long long key, int slave_lo, int& sobj, int& mobj) {
  const int i = (int)(key >> 32), j = (int)(key & 0xFFFFFFFFLL);
  sobj = slave_lo ? i : j;
  mobj = slave_lo ? j : i;
}

// gobj_adjacent for two objects: convexes of one body that touched when they
// were set up (CONVEX_Adjacent, cvx.c:1399-1409); spheres have no adjacency here
__device__ __forceinline__ bool objects_adjacent(int x, int y, int nsph, const int* aptr, const int* alist) {
  if (x < nsph || y < nsph || !aptr) return false;
  const int cy = y - nsph;
  for (int u = aptr[cy]; u < aptr[cy + 1]; u++)
    if (alist[u] == x - nsph) return true;
  return false;
}

// sparsify_contacts, dom.c:2956-3054: keep[k] = 0 for a convex pair without a
// contact and for a new contact whose area is below minarea; a new contact
// whose area is below threshold times that of another contact of its bodies
// goes when the two contacts join the same pair of bodies through adjacent
// objects; otherwise it goes when its point lies within margin (max-norm) of
// the other contact's point and the other one is old or comes later in key
// order (the reference compares contact ids, given in creation order). The
// decision does not depend on the order of the body lists.
__global__ void k_sph_sparsify(int n, int nb, const int* master, const int* slave, const int* isnew,
                               const double* point, const double* area, const long long* key, const int* slave_lo,
                               int nsph, const int* aptr, const int* alist, const int* bptr, const int* blist,
                               double margin, double threshold, double minarea, int* keep) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  int kp = 1;
  const int m = master[k], s = slave[k];
  if (m == -1 && s == -1) {
    kp = 0;
  } else if (isnew[k] && m >= 0 && m < nb && s >= 0 && s < nb) {
    const double p0 = point[3 * (size_t)k], p1 = point[3 * (size_t)k + 1], p2 = point[3 * (size_t)k + 2];
    const double ak = area[k];
    int so, mo;
    contact_objects(key[k], slave_lo[k], so, mo);
    if (ak < minarea) kp = 0;
    const int bb[2] = {m, s};
    for (int t = 0; t < 2 && kp; t++)
      for (int u = bptr[bb[t]]; u < bptr[bb[t] + 1]; u++) {
        const int a = blist[u];
        if (a == k || a < 0 || a >= n) continue;
        if (ak < threshold * area[a]) {
          int sa, ma;
          contact_objects(key[a], slave_lo[a], sa, ma);
          if (m == master[a] && s == slave[a]) {
            if (objects_adjacent(mo, ma, nsph, aptr, alist)) { kp = 0; break; }
          } else if (m == slave[a] && s == master[a]) {
            if (objects_adjacent(mo, sa, nsph, aptr, alist)) { kp = 0; break; }
          }
          continue;
        }
        const double e0 = fabs(p0 - point[3 * (size_t)a]), e1 = fabs(p1 - point[3 * (size_t)a + 1]),
                     e2 = fabs(p2 - point[3 * (size_t)a + 2]);
        double mx = 0.0;
        if (e0 > mx) mx = e0;
        if (e1 > mx) mx = e1;
        if (e2 > mx) mx = e2;
        if (mx < margin && (k < a || !isnew[a])) { kp = 0; break; }
      }
  }
  keep[k] = kp;
}

// scatter kept contact k to slot pos[k] of the output arrays
__global__ void k_sph_compact(int n, const int* keep, const int* pos, ContactOut in, ContactOut out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n || !keep[k]) return;
  const int d = pos[k];
  out.master[d] = in.master[k];
  out.slave[d] = in.slave[k];
  out.key[d] = in.key[k];
  out.slave_lo[d] = in.slave_lo[k];
  out.isnew[d] = in.isnew[k];
  out.gap[d] = in.gap[k];
  out.fric[d] = in.fric[k];
  out.rest[d] = in.rest[k];
  out.coh[d] = in.coh[k];
  out.area[d] = in.area[k];
  for (int v = 0; v < 3; v++) {
    out.point[3 * (size_t)d + v] = in.point[3 * (size_t)k + v];
    out.mpnt[3 * (size_t)d + v] = in.mpnt[3 * (size_t)k + v];
    out.spnt[3 * (size_t)d + v] = in.spnt[3 * (size_t)k + v];
    out.R0[3 * (size_t)d + v] = in.R0[3 * (size_t)k + v];
    out.U0[3 * (size_t)d + v] = in.U0[3 * (size_t)k + v];
  }
  for (int v = 0; v < 9; v++) out.base[9 * (size_t)d + v] = in.base[9 * (size_t)k + v];
}

}  // namespace b2
