// b2_bilateral.cuh -- per-step update of the bilateral constraints on the
// device bodies, the constraint part of DOM_Update_Begin (dom.c:3716-3732),
// run after BODY_Dynamic_Step_Begin has moved the bodies to t + h/2 and
// before the local dynamics is assembled from them.
//
//   RIGLNK  update_riglnk (dom.c:524-550): the link vector m - s between the
//           master's current point and the slave's (or the fixed spatial
//           point spnt when there is no slave), gap = |m - s| - length, base
//           from the link direction; the row's Z[0..2] receives the link
//           vector in that base, as the diagonal solver forms it (dbs.c:409,
//           TVMUL), Z[3] keeps the length.
//   FIXDIR  update_fixdir (dom.c:487-500) with a slave body: the constraint
//           point follows the slave's referential point, the master's
//           referential point is moved under it, and the base is built from
//           the master's current image (BODY_Cur_Vector, bod.c:1775-1781) of
//           the referential direction held in Z[0..2].
//   FIXPNT, VELODIR, VELODIR3 and FIXDIR without a slave only move their
//   spatial point, which the solve does not read; their prescribed values
//   come with the kinds.
//
// Arithmetic follows the reference's macros (SUB, LEN, SCALE, NVMUL, TVMUL)
// operation by operation; built without fused multiply-adds.
#pragma once

#include "b2_detect.cuh"
#include "b2_diag.cuh"

namespace b2 {

__global__ void k_constraints_update(int n, int nbod, const int* kind, const int* master, const int* slave,
                                     const double* rot, const double* x, const double* x0, double* mpnt,
                                     const double* spnt, double* base, double* gap, double* Z, int* bad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int k = kind[i];
  const int m = master[i], s = slave[i];
  if ((k == CON_RIGLNK || k == CON_FIXDIR) && (m < 0 || m >= nbod || s < -1 || s >= nbod)) {
    atomicExch(bad, 1);  // invalid body index: the row is left as it is
    return;
  }
  if (k == CON_RIGLNK) {
    double pm[3], ps[3];
    cur_point(rot + 9 * (size_t)m, x + 3 * (size_t)m, x0 + 3 * (size_t)m, mpnt + 3 * (size_t)i, pm);
    if (s >= 0) {
      cur_point(rot + 9 * (size_t)s, x + 3 * (size_t)s, x0 + 3 * (size_t)s, spnt + 3 * (size_t)i, ps);
    } else {
      ps[0] = spnt[3 * (size_t)i]; ps[1] = spnt[3 * (size_t)i + 1]; ps[2] = spnt[3 * (size_t)i + 2];
    }
    const double v[3] = {pm[0] - ps[0], pm[1] - ps[1], pm[2] - ps[2]};
    double nv[3] = {v[0], v[1], v[2]};
    double len = sqrt(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2]);
    double* Zi = Z + 4 * (size_t)i;
    gap[i] = len - Zi[3];
    len = 1.0 / len;
    nv[0] *= len; nv[1] *= len; nv[2] *= len;
    double b[9];
    local_base(nv, b);
#pragma unroll
    for (int q = 0; q < 9; q++) base[9 * (size_t)i + q] = b[q];
    Zi[0] = b[0] * v[0] + b[1] * v[1] + b[2] * v[2];
    Zi[1] = b[3] * v[0] + b[4] * v[1] + b[5] * v[2];
    Zi[2] = b[6] * v[0] + b[7] * v[1] + b[8] * v[2];
  } else if (k == CON_FIXDIR && s >= 0) {
    double p[3], X[3];
    cur_point(rot + 9 * (size_t)s, x + 3 * (size_t)s, x0 + 3 * (size_t)s, spnt + 3 * (size_t)i, p);
    ref_point(rot + 9 * (size_t)m, x + 3 * (size_t)m, x0 + 3 * (size_t)m, p, X);
    mpnt[3 * (size_t)i] = X[0]; mpnt[3 * (size_t)i + 1] = X[1]; mpnt[3 * (size_t)i + 2] = X[2];
    const double* R = rot + 9 * (size_t)m;
    const double* d = Z + 4 * (size_t)i;
    const double nv[3] = {R[0] * d[0] + R[3] * d[1] + R[6] * d[2], R[1] * d[0] + R[4] * d[1] + R[7] * d[2],
                          R[2] * d[0] + R[5] * d[1] + R[8] * d[2]};
    double b[9];
    local_base(nv, b);
#pragma unroll
    for (int q = 0; q < 9; q++) base[9 * (size_t)i + q] = b[q];
  }
}

// The bilateral constraints kept across detections as rows n0 .. n0+nc-1 of
// the detection's output, after its contacts: bodies, points and frame as
// set up, gap 0 until b2dev_update_constraints, no material, key -1 (never
// matched by the next detection), kind and Z into the caller-order kind
// planes; R, U carried from the previous detection's constraint rows when
// pR is given (the same constraints), else zero.
__global__ void k_constraints_append(int n0, int nc, const int* kind, const int* master, const int* slave,
                                     const double* mpnt, const double* spnt, const double* base, const double* Z,
                                     const double* pR, const double* pU, ContactOut o, int* kind_c, double* Z_c) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nc) return;
  const size_t i = (size_t)n0 + j;
  o.master[i] = master[j];
  o.slave[i] = slave[j];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    o.point[3 * i + q] = mpnt[3 * (size_t)j + q];
    o.mpnt[3 * i + q] = mpnt[3 * (size_t)j + q];
    o.spnt[3 * i + q] = spnt[3 * (size_t)j + q];
    o.R0[3 * i + q] = pR ? pR[3 * (size_t)j + q] : 0.0;
    o.U0[3 * i + q] = pU ? pU[3 * (size_t)j + q] : 0.0;
  }
#pragma unroll
  for (int q = 0; q < 9; q++) o.base[9 * i + q] = base[9 * (size_t)j + q];
  o.gap[i] = 0.0;
  o.fric[i] = o.rest[i] = o.coh[i] = 0.0;
  o.key[i] = -1;
  o.slave_lo[i] = 0;
  o.isnew[i] = 0;
  o.area[i] = 0.0;
  kind_c[i] = kind[j];
#pragma unroll
  for (int q = 0; q < 4; q++) Z_c[4 * i + q] = Z[4 * (size_t)j + q];
}

}  // namespace b2
