"""Convex-convex contact detection on the device (csrc/b2_cvi.cuh and the
convex pairs of csrc/b2_detect.cuh) against the reference's own gobjcontact
(goc.c detect_convex_convex) over every pair of seeded scenes of convex
bodies, as recorded in tests/golden/convex/pile_ref.npz by make_cvi_golden.py
from the reference compiled from its sources (tests/test_detect_cpu.py checks
the fixture against that build): the contact set, and per contact its point,
normal, gap, area and surface-pair material, bit for bit; the sparsification
rule (dom.c:2956-3054) restated over the reference's contacts.

Every body sits at the origin with the identity rotation, so the device's
current vertices are the referential ones exactly and both sides see the same
numbers. The lower convex of a pair is the reference's first object (slave)."""
import os

import numpy as np
import pytest

from solfec_b200 import LOCDYN, scenes
from solfec_b200.detect import CONVEXES, bodies_only
from solfec_b200.dynamics import RIGID_DYNAMICS

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'convex', 'pile_ref.npz')
NSURF = 7


def same_bits(a, b):
    a = np.asarray(a, float).ravel(); b = np.asarray(b, float).ravel()
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def material():
    m = np.zeros((NSURF, NSURF, 2))
    for a in range(NSURF):
        for b in range(NSURF):
            m[a, b, 0] = 0.1 + 0.01 * (min(a, b) * NSURF + max(a, b))   # distinct friction per surface pair
    return m


def run_device(sc, cv, sparsify=None, detect_twice=False):
    J = np.tile(np.eye(3).reshape(9), (sc.nbod, 1))
    mass = np.ones(sc.nbod)
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    RIGID_DYNAMICS(ldy, J, mass, sc.x)
    det = CONVEXES(ldy, cv, material())
    if sparsify:
        det.sparsify(**sparsify)
    det.detect()
    first = det.contacts()
    out = first
    if detect_twice:
        det.detect()
        out = det.contacts()
    ldy.close()
    return first, out


def reference_contacts(seed):
    """The reference's contacts of convex_pile(seed): {(c1, c2): (state,
    point, normal, gap, area, spair)}."""
    g = np.load(GOLDEN)
    f = lambda name: g['s%d_%s' % (seed, name)]
    return {tuple(int(v) for v in k): (1, f('point')[t], f('normal')[t], f('gap')[t], f('area')[t], f('spair')[t])
            for t, k in enumerate(f('keys'))}


def sparsify_keep(keys, contacts, bodies, threshold=0.01, minarea=0.0, mindist=1e-6):
    """sparsify_contacts (dom.c:2956-3054) over new contacts listed in key
    order (a contact's id order): convexes of different bodies are never
    adjacent here, so a contact of relatively small area is kept."""
    keep = []
    for k, key in enumerate(keys):
        st, pt, nrm, gap, area, sp = contacts[key]
        m, s = bodies[key]
        ok = area >= minarea
        for a, other in enumerate(keys):
            if not ok:
                break
            if a == k or not (set(bodies[other]) & {m, s}):
                continue
            if area < threshold * contacts[other][4]:
                continue
            d = np.abs(pt - contacts[other][1]).max()
            if d < 2 * mindist and k < a:
                ok = False
        keep.append(ok)
    return keep


def check_scene(seed, sc, cv, min_contacts):
    ref = reference_contacts(seed)
    keys = sorted(ref)
    bodies = {key: (cv['body'][key[1]], cv['body'][key[0]]) for key in keys}   # (master, slave)
    keep = sparsify_keep(keys, ref, bodies)
    expect = [key for key, k in zip(keys, keep) if k]
    assert len(expect) >= min_contacts
    first, again = run_device(sc, cv, detect_twice=True)
    ns = 0
    got = [(int(k >> 32) - ns, int(k & 0xFFFFFFFF) - ns) for k in first['key']]
    assert got == expect
    mat = material()
    for t, key in enumerate(expect):
        st, pt, nrm, gap, area, sp = ref[key]
        assert first['master'][t] == cv['body'][key[1]] and first['slave'][t] == cv['body'][key[0]]
        assert first['slave_lo'][t] == 1 and first['isnew'][t] == 1
        assert same_bits(first['point'][t], pt), key
        assert same_bits(first['base'][t, 6:9], nrm), key
        assert same_bits(first['gap'][t], gap) and same_bits(first['area'][t], area), key
        assert same_bits(first['mpnt'][t], pt) and same_bits(first['spnt'][t], pt)
        assert first['friction'][t] == mat[sp[0], sp[1], 0], key
    # a second detection on unmoved bodies updates every contact in place
    assert np.array_equal(again['key'], first['key']) and not again['isnew'].any()
    for name in ('point', 'base', 'gap', 'area', 'friction'):
        assert same_bits(again[name], first[name]), name
    return len(expect)


def test_convex_lattice_contacts_equal_reference():
    """A 5 x 4 x 3 lattice of boxes with jittered sizes and positions (faces
    touching, slightly overlapping or slightly apart), rotated boxes and
    random hulls among them, on a floor obstacle."""
    sc, cv = scenes.convex_pile(seed=1)
    n = check_scene(1, sc, cv, min_contacts=60)
    assert n >= 60


@pytest.mark.parametrize('seed', [2, 3])
def test_convex_pile_contacts_equal_reference(seed):
    sc, cv = scenes.convex_pile(seed=seed, nx=4, ny=3, nz=2, hulls=12)
    check_scene(seed, sc, cv, min_contacts=25)
