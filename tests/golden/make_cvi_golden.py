"""Golden contacts of the convex-convex path: for the seeded convex piles of
solfec_b200.scenes.convex_pile, the reference's own gobjcontact
(detect_convex_convex, goc.c:280-306, compiled from the reference sources into
oracle/_ref/libref_geo.so) for every pair of convexes c1 < c2 of different
bodies, not both obstacles, with the first object c1. Writes convex/pile_ref.npz:
per scene the pair keys (c1, c2) with a contact and per contact the point,
normal, gap, area and surface pair. Needs oracle/_ref built."""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, 'solfec-1.0_b200'), os.path.join(ROOT, 'oracle')]

import oracle as O  # noqa: E402
from solfec_b200 import scenes  # noqa: E402

# (seed, convex_pile keyword arguments)
CASES = [(1, {}), (2, dict(nx=4, ny=3, nz=2, hulls=12)), (3, dict(nx=4, ny=3, nz=2, hulls=12))]


def reference_pairs(seed, kw):
    sc, cv = scenes.convex_pile(seed=seed, **kw)
    conv = scenes.convex_list(cv)
    keys, point, normal, gap, area, spair = [], [], [], [], [], []
    for i in range(len(conv)):
        for j in range(i + 1, len(conv)):
            if cv['body'][i] == cv['body'][j] or (sc.obstacle[cv['body'][i]] and sc.obstacle[cv['body'][j]]):
                continue
            st, pt, nrm, g, a, sp = O.ref_gobj_convex_convex(*conv[i], *conv[j])
            if st > 0:
                keys.append((i, j)); point.append(pt); normal.append(nrm); gap.append(g); area.append(a)
                spair.append(sp)
    return dict(keys=np.array(keys, np.int32), point=np.array(point), normal=np.array(normal),
                gap=np.array(gap), area=np.array(area), spair=np.array(spair, np.int32))


def main():
    if not O.geo_available():
        sys.exit('build oracle/_ref first (the reference geometry library)')
    out = {}
    for seed, kw in CASES:
        for name, v in reference_pairs(seed, kw).items():
            out['s%d_%s' % (seed, name)] = v
    np.savez_compressed(os.path.join(HERE, 'convex', 'pile_ref.npz'), **out)


if __name__ == '__main__':
    main()
