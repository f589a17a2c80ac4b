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

import oracle
from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, scenes
from solfec_b200._lib import lib
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


def expected_step(sc, cv, st, prev, mat, threshold=0.01, mindist=1e-6):
    """The contacts the reference's DOM_Update_Begin makes of the convexes at
    the device's body state st (rotations, mass centres): gobjcontact of the
    compiled reference for every pair on the current vertices (cur_point of
    the oracle), kept contacts carrying their R and U, new ones sparsified."""
    if not oracle.geo_available():
        pytest.skip('reference geometry build unavailable')
    vbody = np.repeat(cv['body'], np.diff(cv['vptr']))
    cur = oracle.sphere_centres(vbody, cv['vert'], st['rot'], st['x'], sc.x0)
    conv = [(cur[cv['vptr'][c]:cv['vptr'][c + 1]], f, s_) for c, (_, f, s_) in enumerate(scenes.convex_list(cv))]
    found = {}
    for i in range(len(conv)):
        for j in range(i + 1, len(conv)):
            if sc.obstacle[cv['body'][i]] and sc.obstacle[cv['body'][j]]:
                continue
            r = oracle.ref_gobj_convex_convex(*conv[i], *conv[j])
            if r[0] > 0:
                found[(i, j)] = r
    keys = sorted(found)
    pkeys = {} if prev is None else {int(k): t for t, k in enumerate(prev['key'])}
    key64 = [(i << 32) | j for i, j in keys]
    isnew = [k not in pkeys for k in key64]
    body = {key: (cv['body'][key[1]], cv['body'][key[0]]) for key in keys}
    keep = []
    for t, key in enumerate(keys):
        ok = True
        if isnew[t]:
            m, s_ = body[key]
            for a, other in enumerate(keys):
                if a == t or not (set(body[other]) & {m, s_}):
                    continue
                if found[key][4] < threshold * found[other][4]:
                    continue
                if np.abs(found[key][1] - found[other][1]).max() < 2 * mindist and (t < a or not isnew[a]):
                    ok = False
                    break
        keep.append(ok)
    out = {n: [] for n in ('key', 'slave_lo', 'master', 'slave', 'point', 'mpnt', 'spnt', 'base', 'gap', 'area',
                           'friction', 'restitution', 'R', 'U', 'isnew')}
    for t, key in enumerate(keys):
        if not keep[t]:
            continue
        st_, pt, nrm, gap, area, sp = found[key]
        m, s_ = body[key]
        out['key'].append(key64[t]); out['slave_lo'].append(1); out['master'].append(m); out['slave'].append(s_)
        out['point'].append(pt)
        out['mpnt'].append(oracle.ref_points([m], [pt], st['rot'], st['x'], sc.x0)[0])
        out['spnt'].append(oracle.ref_points([s_], [pt], st['rot'], st['x'], sc.x0)[0])
        out['base'].append(oracle.localbase(nrm)); out['gap'].append(gap); out['area'].append(area)
        out['friction'].append(mat[sp[0], sp[1], 0]); out['restitution'].append(mat[sp[0], sp[1], 1])
        hit = pkeys.get(key64[t])
        out['R'].append(np.zeros(3) if hit is None or 'R' not in prev else prev['R'][hit])
        out['U'].append(np.zeros(3) if hit is None or 'U' not in prev else prev['U'][hit])
        out['isnew'].append(int(hit is None))
    return {k: np.array(v) for k, v in out.items()}


def same_contacts(dev, exp):
    assert dev['key'].shape[0] == exp['key'].shape[0], (dev['key'].shape, exp['key'].shape)
    if exp['key'].shape[0] == 0:
        return
    for k, b in exp.items():
        a = np.asarray(dev[k])
        if a.dtype.kind == 'f':
            assert np.array_equal(a.view(np.uint64), np.ascontiguousarray(b, np.float64).reshape(a.shape)
                                  .view(np.uint64)), k
        else:
            assert np.array_equal(a.astype(np.int64), b.astype(np.int64).reshape(a.shape)), k


def test_convex_time_loop_matches_reference_every_step():
    """Boxes and hulls dropped onto a floor: at every step the device's
    contact update and detection on its own body state equals the reference's
    gobjcontact over all pairs, with the R and U of the device solve carried
    for kept contacts, as the bodies fall, land, settle and rotate."""
    sc, cv, J, mass = scenes.convex_drop()
    mat = np.zeros((3, 3, 2))
    mat[..., 0] = [[0.3, 0.4, 0.5], [0.4, 0.6, 0.7], [0.5, 0.7, 0.2]]
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    det = CONVEXES(ldy, cv, mat)
    gs = GAUSS_SEIDEL_SOLVER(1e-6, 300)
    prev = None
    counts = []
    h = sc.step
    for k in range(60):
        dyn.step_begin(h, (0.0, 0.0, -9.81))
        st = dyn.state()
        nc, nn = det.detect()
        dev = det.contacts()
        same_contacts(dev, expected_step(sc, cv, st, prev, mat))
        counts.append((nc, nn))
        if nc > 0:
            assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, 1) == 0
            det.carry_state()
            gs.solve(ldy)
            R, U, _ = ldy.get_state()
            prev = dict(key=dev['key'], R=R, U=U)
        else:
            prev = dict(key=dev['key'])
        dyn.step_end(h)
    kept = sum(nc - nn for nc, nn in counts)
    assert max(nc for nc, _ in counts) >= 8 and kept > 100, counts
    assert np.all(dyn.state()['x'][sc.obstacle == 0, 2] > 0.3)   # resting on the floor, not through it
    ldy.close()


def test_hexahedra_geometry_contacts_equal_reference():
    """The perturbed cubes and walls of the config-3 scene (8 x 8 x 3 of them):
    the device detection at the scene's state equals the reference's
    gobjcontact over all pairs, face, edge and corner contacts alike."""
    sc = scenes.hexahedra_lattice(nx=8, ny=8, nz=3)
    cv = scenes.hexahedra_geometry(nx=8, ny=8, nz=3)
    J = np.tile(np.eye(3).reshape(9), (sc.nbod, 1))
    mat = np.zeros((1, 1, 2)); mat[0, 0, 0] = 0.4
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    dyn = RIGID_DYNAMICS(ldy, J, np.ones(sc.nbod), sc.x)
    det = CONVEXES(ldy, cv, mat)
    det.detect()
    dev = det.contacts()
    exp = expected_step(sc, cv, dyn.state(), None, mat)
    same_contacts(dev, exp)
    assert dev['key'].shape[0] > 400
    ldy.close()


def test_exclusions_and_penetration_depth():
    """CONTACT_EXCLUDE_BODIES and CONTACT_EXCLUDE_SURFACES on the seeded pile:
    the contacts are the reference's without the excluded body pairs and
    without new contacts of the excluded surface pairs; UNPHYSICAL_PENETRATION
    below the pile's deepest gap fails the detection, above it passes."""
    from solfec_b200 import DeviceError
    sc, cv = scenes.convex_pile(seed=1)
    ref = reference_contacts(1)
    keys = sorted(ref)
    body = cv['body']
    ex_bodies = {tuple(sorted((int(body[i]), int(body[j])))) for (i, j) in keys[::7]}
    ex_surf = {(1, 4), (2, 2)}
    excluded = lambda key: (tuple(sorted((int(body[key[0]]), int(body[key[1]])))) in ex_bodies
                            or tuple(sorted((int(ref[key][5][0]), int(ref[key][5][1])))) in ex_surf)
    left = [key for key in keys if not excluded(key)]
    assert 0 < len(left) < len(keys) - len(ex_bodies)
    bodies = {key: (body[key[1]], body[key[0]]) for key in left}
    keep = sparsify_keep(left, ref, bodies)
    expect = [key for key, k in zip(left, keep) if k]
    J = np.tile(np.eye(3).reshape(9), (sc.nbod, 1))
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    RIGID_DYNAMICS(ldy, J, np.ones(sc.nbod), sc.x)
    det = CONVEXES(ldy, cv, material())
    det.exclude_bodies(sorted(ex_bodies))
    det.exclude_surfaces(sorted(ex_surf))
    det.detect()
    dev = det.contacts()
    assert [(int(k >> 32), int(k & 0xFFFFFFFF)) for k in dev['key']] == expect
    for t, key in enumerate(expect):
        assert same_bits(dev['point'][t], ref[key][1]) and same_bits(dev['gap'][t], ref[key][3])
    deepest = -min(ref[k][3] for k in keys)
    det.unphysical_penetration(1.5 * deepest)
    det.detect()
    det.unphysical_penetration(0.5 * deepest)
    with pytest.raises(DeviceError, match='penetration'):
        det.detect()
    ldy.close()
