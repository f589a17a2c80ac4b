// Test harness: csrc/b2_cvi.cuh (the convex-convex contact of the device
// kernels) compiled for the host, behind a flat-array entry like the
// reference harness's ref_gobj_convex_convex, so CPU tests can compare the
// restatement itself with the reference's gobjcontact on many random pairs.
#include <vector>

#include "b2_cvi.cuh"

using namespace b2;

// computeplanes (cvx.c:72-89), as k_cvx_update computes them
static void planes(int nfac, const int* fac, const double* cur, double* pla) {
  for (int f = 0, m = 0; f < nfac; f++, m += fac[m] + 1) {
    const double *a = cur + 3 * fac[m + 1], *b = cur + 3 * fac[m + 2], *c = cur + 3 * fac[m + 3];
    const double ba[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]}, cb[3] = {c[0] - b[0], c[1] - b[1], c[2] - b[2]};
    double* nl = pla + 6 * f;
    nl[0] = ba[1] * cb[2] - ba[2] * cb[1];
    nl[1] = ba[2] * cb[0] - ba[0] * cb[2];
    nl[2] = ba[0] * cb[1] - ba[1] * cb[0];
    const double len = sqrt(nl[0] * nl[0] + nl[1] * nl[1] + nl[2] * nl[2]);
    nl[0] /= len; nl[1] /= len; nl[2] /= len;
    nl[3] = a[0]; nl[4] = a[1]; nl[5] = a[2];
  }
}

static cvi::Scratch scratch;

extern "C" int cvi_host_pair(int update, int nva, const double* va, int nfa, const int* fa, const int* sa, int nvb,
                             const double* vb, int nfb, const int* fb, const int* sb, double* point, double* normal,
                             double* gap, double* area, int* spair) {
  std::vector<double> pa(6 * nfa), pb(6 * nfb);
  planes(nfa, fa, va, pa.data());
  planes(nfb, fb, vb, pb.data());
  const cvi::Convex A{va, nva, pa.data(), nfa, sa, nfa}, B{vb, nvb, pb.data(), nfb, sb, nfb};
  cvi::Contact c;
  c.spair[0] = spair[0];
  c.spair[1] = spair[1];
  const int st = cvi::convex_convex(A, B, update != 0, c, scratch);
  if (st > 0) {
    for (int j = 0; j < 3; j++) { point[j] = c.point[j]; normal[j] = c.normal[j]; }
    *gap = c.gap;
    *area = c.area;
    spair[0] = c.spair[0];
    spair[1] = c.spair[1];
  }
  return st;
}

extern "C" double cvi_host_orient3d(const double* a, const double* b, const double* c, const double* d) {
  return cvi::orient3d(a, b, c, d);
}
