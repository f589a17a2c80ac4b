"""Golden vectors of the reference's own contact geometry: gobjcontact
(goc.c:1362) for sphere pairs and for a convex and a sphere, computed by the
reference sources compiled into oracle/_ref/libref_geo.so (oracle/Makefile,
harness oracle/ref/ref_geo_harness.c). Inputs are seeded; the fixture holds
inputs and outputs as exact float64 bit patterns (hex), so the oracle's
restatement can be checked where the reference cannot be built. Run where the
reference build exists; the tests read only detect_ref.json."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, '..', '..', 'oracle'))
sys.path.insert(0, os.path.join(HERE, '..', '..', 'solfec-1.0_b200'))

import oracle  # noqa: E402
from solfec_b200 import scenes  # noqa: E402


def hx(a):
    return [float(v).hex() for v in np.atleast_1d(np.asarray(a, dtype=np.float64))]


def main():
    rng = np.random.default_rng(2024)
    spheres = []
    for t in range(40):
        a = rng.normal(size=3)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        ra, rb = rng.uniform(0.05, 1.0, 2)
        b = a + d * (ra + rb) * rng.choice([0.9, 0.999, 1.0, 1.0 + 5e-7, 1.0 + 3e-6])
        for update in (0, 1):
            st, one, two, nrm, gap, sp = oracle.ref_gobj_sphere_sphere(a, ra, 1, b, rb, 2, update=bool(update))
            spheres.append(dict(update=update, a=hx(a), ra=hx(ra), b=hx(b), rb=hx(rb), state=int(st),
                                onepnt=hx(one), twopnt=hx(two), normal=hx(nrm), gap=hx(gap)))
    convex = []
    for t in range(24):
        lo = rng.normal(size=3)
        hi = lo + rng.uniform(0.2, 2.0, 3)
        ver, fac = scenes.box_convex(lo, hi)
        R = np.linalg.qr(rng.normal(size=(3, 3)))[0]
        if np.linalg.det(R) < 0:
            R[:, 0] = -R[:, 0]
        ver = (ver - lo) @ R.T + lo
        surf = np.arange(6, dtype=np.int32) + 10
        face = rng.integers(6)
        cen = ver.mean(0)
        pla = oracle.convex_planes(fac, ver)
        r = rng.uniform(0.05, 0.5)
        c = pla[face, 3:6] + 0.25 * (ver[fac[5 * face + 2]] - pla[face, 3:6]) + pla[face, :3] * r * \
            rng.choice([0.9, 0.99999, 1.0 + 5e-7, 1.0 + 3e-6])
        if t % 8 == 0:
            c = cen + 0.01 * rng.normal(size=3)   # centre inside the convex
        for sphere_first in (0, 1):
            for update in (0, 1):
                st, one, two, nrm, gap, sp = oracle.ref_gobj_convex_sphere(ver, fac, surf, c, r, 3, bool(sphere_first),
                                                                           bool(update))
                convex.append(dict(sphere_first=sphere_first, update=update, ver=hx(ver.reshape(-1)),
                                   fac=[int(v) for v in fac], surf=[int(v) for v in surf], c=hx(c), r=hx(r),
                                   state=int(st), onepnt=hx(one), twopnt=hx(two), normal=hx(nrm), gap=hx(gap),
                                   spair=[int(v) for v in sp]))
    out = dict(source='gobjcontact of the reference (goc.c, gjk.c, cvx.c, sph.c) compiled into oracle/_ref/libref_geo.so',
               sphere_sphere=spheres, convex_sphere=convex)
    path = os.path.join(HERE, 'detect_ref.json')
    with open(path, 'w') as f:
        json.dump(out, f)
    print(path, len(spheres), 'sphere cases,', len(convex), 'convex cases')


if __name__ == '__main__':
    main()
