"""CPU tests of the sphere contact detection oracle (oracle/oracle_detect.c):
gjk_sphere_sphere pinned bit for bit to the reference's own gjk.c (compiled
into oracle/_ref), the restated contact formulas against an independent
vectorised restatement, and the update, filter and sparsification rules of
dom.c and box.c on hand-built cases."""
import os

import numpy as np
import pytest

import oracle
from solfec_b200 import scenes

MAT = np.array([[[0.3, 0.0]]])
EPS = 1e-6


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.skipif(not oracle.ref_available(), reason='reference build unavailable')
def test_gjk_sphere_sphere_pinned_to_reference():
    rng = np.random.default_rng(11)
    for t in range(3000):
        a = rng.normal(size=3)
        scale = [1e-7, 1e-3, 0.1, 1.0][t % 4]
        b = a + rng.normal(size=3) * scale
        ra, rb = rng.uniform(0.01, 1.0, 2)
        if t % 5 == 0:   # touching within GEOMETRIC_EPSILON
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            b = a + d * (ra + rb + rng.uniform(-2e-6, 2e-6))
        if t % 97 == 0:
            b = a.copy()
        g1, p1, q1 = oracle.gjk_sphere_sphere(a, ra, b, rb, 'oracle')
        g2, p2, q2 = oracle.gjk_sphere_sphere(a, ra, b, rb, 'ref')
        assert _bits([g1]) == _bits([g2]) and np.array_equal(_bits(p1), _bits(p2)) and np.array_equal(_bits(q1), _bits(q2))


def test_localbase_frame():
    rng = np.random.default_rng(3)
    ns = [np.array([1.0, 0, 0]), np.array([-1.0, 0, 0]), np.array([0, 0, 1.0])]
    ns += [v / np.linalg.norm(v) for v in rng.normal(size=(50, 3))]
    for n in ns:
        L = oracle.localbase(n).reshape(3, 3).T   # column-major storage
        assert np.array_equal(L[:, 2], n)
        assert np.allclose(L.T @ L, np.eye(3), atol=1e-14)
    # e_x x n vanishes for n = e_x: the reference falls back to e_y x n
    L = oracle.localbase([1.0, 0, 0]).reshape(3, 3).T
    assert np.array_equal(L[:, 0], [0.0, 0.0, -1.0])


def _numpy_contacts(cur, rad, sbody, obst):
    """Independent restatement: all pairs by brute force, the reference's
    formulas in numpy, the lower centre (point order) as the slave."""
    n = cur.shape[0]
    I, J = np.triu_indices(n, 1)
    keep = (sbody[I] != sbody[J]) & ~((obst[sbody[I]] != 0) & (obst[sbody[J]] != 0))
    I, J = I[keep], J[keep]
    d = cur[I] - cur[J]
    dlen = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    deno = rad[I] + rad[J]
    g = np.where(dlen > deno, dlen - deno, 0.0)
    m = g < EPS
    I, J = I[m], J[m]
    lo_slave = np.array([tuple(cur[i]) <= tuple(cur[j]) for i, j in zip(I, J)], dtype=bool)
    s = np.where(lo_slave, I, J)
    mm = np.where(lo_slave, J, I)
    d = cur[s] - cur[mm]
    dlen = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
    p = cur[s] - (rad[s] / dlen)[:, None] * d
    q = cur[mm] + (rad[mm] / dlen)[:, None] * d
    over = ~(dlen > rad[s] + rad[mm])
    mid = .5 * (p + q)
    p = np.where(over[:, None], mid, p)
    q = np.where(over[:, None], mid, q)
    nrm = p - cur[s]
    ln = np.sqrt(nrm[:, 0] * nrm[:, 0] + nrm[:, 1] * nrm[:, 1] + nrm[:, 2] * nrm[:, 2])
    nrm = nrm / ln[:, None]
    x = cur[mm] - cur[s]
    dd = x[:, 0] * nrm[:, 0] + x[:, 1] * nrm[:, 1] + x[:, 2] * nrm[:, 2]
    e = rad[s] + rad[mm]
    gap = np.where(e > dd, dd - e, 0.0)
    return dict(key=(I.astype(np.int64) << 32) | J, slave_lo=lo_slave.astype(np.int32), point=q, gap=gap,
                normal=nrm, master=sbody[mm], slave=sbody[s])


def test_oracle_matches_vectorised_restatement(scene_cache):
    sc = scene_cache('spheres_lattice')
    sp = scenes.sphere_shapes(sc)
    got = oracle.detect_spheres(sp['body'], sp['centre'], sp['radius'], sp['surface'], sc.rot, sc.x, sc.x0,
                                sc.obstacle, MAT)
    cur = oracle.sphere_centres(sp['body'], sp['centre'], sc.rot, sc.x, sc.x0)
    ref = _numpy_contacts(cur, sp['radius'], sp['body'], sc.obstacle)
    assert got['key'].shape[0] > 1000
    assert np.array_equal(got['key'], ref['key'])
    assert np.array_equal(got['slave_lo'], ref['slave_lo'])
    assert np.array_equal(got['master'], ref['master']) and np.array_equal(got['slave'], ref['slave'])
    for k in ('point', 'gap'):
        assert np.array_equal(_bits(got[k]), _bits(ref[k])), k
    assert np.array_equal(_bits(got['base'][:, 6:9]), _bits(ref['normal']))
    assert np.all(got['friction'] == 0.3) and np.all(got['isnew'] == 1)
    # referential points map back onto the spatial ones
    R = sc.rot.reshape(-1, 3, 3).transpose(0, 2, 1)
    xm = sc.x[got['master']] + np.einsum('nij,nj->ni', R[got['master']], got['mpnt'] - sc.x0[got['master']])
    assert np.allclose(xm, got['point'], atol=1e-12)


def _two_spheres(c0, c1, r=(0.5, 0.5), obst=(0, 0), body=(0, 1)):
    nb = max(body) + 1
    rot = np.tile(np.eye(3).reshape(9), (nb, 1))
    x = np.zeros((nb, 3))
    x0 = np.zeros((nb, 3))
    sref = np.array([c0, c1], float)
    return dict(sbody=np.array(body), sref=sref, rad=np.array(r, float), surf=np.zeros(2, np.int32), rot=rot, x=x,
                x0=x0, obst=np.array(obst[:nb]))


def _detect(c, prev=None):
    return oracle.detect_spheres(c['sbody'], c['sref'], c['rad'], c['surf'], c['rot'], c['x'], c['x0'], c['obst'],
                                 MAT, prev)


def test_update_keeps_roles_and_drops_separated():
    # sphere 0 below sphere 1 (equal x and y): sphere 0 is the slave
    c = _two_spheres([0, 0, 0], [0, 0, 0.999])
    a = _detect(c)
    assert a['key'].tolist() == [1] and a['slave_lo'].tolist() == [1] and a['isnew'].tolist() == [1]
    # the centres swap heights: a fresh detection would make sphere 1 the slave,
    # the update keeps sphere 0 as the slave (update_contact keeps the roles)
    c2 = _two_spheres([0, 0, 0.999], [0, 0, 0])
    assert _detect(c2)['slave_lo'].tolist() == [0]
    prev = dict(a, R=np.array([[1.0, 2.0, 3.0]]), U=np.array([[4.0, 5.0, 6.0]]))
    b = _detect(c2, prev)
    assert b['slave_lo'].tolist() == [1] and b['isnew'].tolist() == [0]
    assert b['R'].tolist() == [[1.0, 2.0, 3.0]] and b['U'].tolist() == [[4.0, 5.0, 6.0]]
    assert b['slave'].tolist() == [0] and b['master'].tolist() == [1]
    # separated by more than GEOMETRIC_EPSILON: removed; within it: kept with gap 0
    assert _detect(_two_spheres([0, 0, 0], [0, 0, 1.0 + 2e-6]), prev)['key'].shape[0] == 0
    k = _detect(_two_spheres([0, 0, 0], [0, 0, 1.0 + 5e-7]), prev)
    assert k['key'].shape[0] == 1 and k['gap'][0] == 0.0


def test_filters_same_body_and_obstacle_pairs():
    assert _detect(_two_spheres([0, 0, 0], [0, 0, 0.9], body=(0, 0)))['key'].shape[0] == 0
    assert _detect(_two_spheres([0, 0, 0], [0, 0, 0.9], obst=(1, 1)))['key'].shape[0] == 0
    assert _detect(_two_spheres([0, 0, 0], [0, 0, 0.9], obst=(1, 0)))['key'].shape[0] == 1


def test_coincident_centres_rejected():
    with pytest.raises(ValueError):
        _detect(_two_spheres([0, 0, 0], [0, 0, 0]))


def _three():
    # sphere 0 touches spheres 1 and 2, whose contact points with it lie within
    # 2 mindist of each other; 1 and 2 (other bodies) overlap too
    nb = 3
    rot = np.tile(np.eye(3).reshape(9), (nb, 1))
    sref = np.array([[0, 0, 0], [0.999, 0, 0], [0.999 + 1e-7, 0, 0]], float)
    return dict(sbody=np.arange(3), sref=sref, rad=np.full(3, 0.5), surf=np.zeros(3, np.int32), rot=rot,
                x=np.zeros((3, 3)), x0=np.zeros((3, 3)), obst=np.zeros(3, np.int32))


def test_sparsify_duplicate_points():
    c = _three()
    out = _detect(c)
    # pairs (0,1), (0,2), (1,2): the earlier of the two new contacts of sphere 0
    # with duplicate points, (0,1), is removed (sparsify_contacts keeps the later id)
    assert out['key'].tolist() == [(0 << 32) | 2, (1 << 32) | 2]
    # with (0,1) an old contact, the new (0,2) goes instead
    first = _detect(_two_spheres([0, 0, 0], [0.999, 0, 0]))
    prev = dict(key=first['key'], slave_lo=first['slave_lo'])
    out = _detect(c, prev)
    assert out['key'].tolist() == [1, (1 << 32) | 2] and out['isnew'].tolist() == [0, 1]


# ---------------------------------------------------------------- convex obstacles

@pytest.mark.skipif(not oracle.ref_available(), reason='reference build unavailable')
def test_gjk_convex_point_pinned_to_reference():
    rng = np.random.default_rng(12)
    for t in range(3000):
        box = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float) * rng.uniform(0.2, 2, 3)
        box += rng.normal(size=box.shape) * 0.05
        R = np.linalg.qr(rng.normal(size=(3, 3)))[0]
        a = box @ R.T + rng.normal(size=3)
        p = a.mean(0) + rng.normal(size=3) * [0.05, 0.5, 1.0, 3.0][t % 4]   # inside, near and far
        d1, q1 = oracle.gjk_convex_point(a, p, 'oracle')
        d2, q2 = oracle.gjk_convex_point(a, p, 'ref')
        assert _bits([d1]) == _bits([d2]) and np.array_equal(_bits(q1), _bits(q2))


def test_box_planes_point_outward():
    v, f = scenes.box_convex([0, 0, 0], [1, 2, 3])
    pla = oracle.convex_planes(f, v)
    assert np.array_equal(pla[:, :3], np.array([[-1, 0, 0], [1, 0, 0], [0, -1, 0], [0, 1, 0], [0, 0, -1], [0, 0, 1.0]]))
    for k in range(6):   # each plane's point lies on its face
        axis = k // 2
        assert pla[k, 3 + axis] == (v[:, axis].max() if k % 2 else v[:, axis].min())


def _box_contacts(shift, prev=None):
    sc, sp, J, mass = scenes.spheres_in_box()
    n = sp['body'].shape[0]
    x = sc.x.copy()
    x[:n] += shift
    out = oracle.detect_spheres(sp['body'], sp['centre'], sp['radius'], sp['surface'], sc.rot, x, sc.x0, sc.obstacle,
                                MAT, prev, convex=sp['convex'])
    return sc, sp, x, out


def test_spheres_on_box_floor():
    sc, sp, x, out = _box_contacts([0.0, 0.0, -0.00201])   # the lowest layer 10 um into the floor
    n = sp['body'].shape[0]
    j = out['key'] & 0xFFFFFFFF
    wall = j >= n
    floor_body = n   # the first convex, the floor
    assert wall.sum() == 25 and np.all(out['slave'][wall] == floor_body)
    assert np.all(out['master'][wall] == (out['key'][wall] >> 32))
    assert np.all(out['slave_lo'][wall] == 0)
    assert np.allclose(out['gap'][wall], -1e-5, atol=1e-12)
    nrm = out['base'][wall][:, 6:9]
    assert np.allclose(nrm, [0, 0, 1], atol=1e-12)
    ctr = x[out['master'][wall]]
    assert np.allclose(out['point'][wall], ctr - 0.05 * nrm, atol=1e-15)
    assert np.allclose(out['spnt'][wall][:, 2], 0.0, atol=1e-12)   # on the floor's top face (referential = spatial)


def test_box_side_wall_and_update():
    # shifted 3.5 mm towards the +x wall (clearance 2 mm, jitter up to 1 mm):
    # the whole last column touches it; the update carries R
    sc, sp, x, out = _box_contacts([0.0035, 0.0, 0.0])
    n = sp['body'].shape[0]
    j = out['key'] & 0xFFFFFFFF
    side = j == n + 2   # the +x wall
    assert side.sum() == 15 and np.all(out['isnew'] == 1)
    assert np.allclose(out['base'][side][:, 6:9], [-1, 0, 0], atol=1e-12)
    prev = dict(key=out['key'], slave_lo=out['slave_lo'], R=np.arange(3 * len(j), dtype=float).reshape(-1, 3),
                U=np.zeros((len(j), 3)))
    sc, sp, x2, out2 = _box_contacts([0.0036, 0.0, 0.0], prev)
    assert np.array_equal(out2['key'], out['key']) and np.all(out2['isnew'] == 0)
    assert np.array_equal(out2['R'], prev['R'])


# ---------------------------------------------------------------- pinned to the reference's gobjcontact

def _same_bits(a, b):
    return np.array_equal(_bits(np.atleast_1d(a)), _bits(np.atleast_1d(b)))


@pytest.mark.skipif(not oracle.geo_available(), reason='reference build unavailable')
def test_sphere_contacts_pinned_to_reference_gobjcontact(scene_cache):
    """Every contact the oracle forms on the settled lattice equals the
    reference's own detect_sphere_sphere (gobjcontact, CONTACT_DETECT) bit for
    bit, whichever sphere the broad phase hands over first: roles, normal,
    gap and both points; and a pair the oracle leaves out is no contact there."""
    from scipy.spatial import cKDTree
    sc = scene_cache('spheres_lattice')
    sp = scenes.sphere_shapes(sc)
    out = oracle.detect_spheres(sp['body'], sp['centre'], sp['radius'], sp['surface'], sc.rot, sc.x, sc.x0,
                                sc.obstacle, MAT)
    cur = oracle.sphere_centres(sp['body'], sp['centre'], sc.rot, sc.x, sc.x0)
    rad = sp['radius']
    found = set()
    for k in range(out['key'].shape[0]):
        i, j = int(out['key'][k] >> 32), int(out['key'][k] & 0xFFFFFFFF)
        found.add((i, j))
        for first, second in ((i, j), (j, i)):
            st, one, two, nrm, gap, _ = oracle.ref_gobj_sphere_sphere(cur[first], rad[first], 0, cur[second],
                                                                       rad[second], 0)
            assert st in (1, 2)
            master = second if st == 1 else first   # dom.c:386-404
            mpt, spt = (two, one) if st == 1 else (one, two)
            assert sp['body'][master] == out['master'][k]
            assert _same_bits(nrm, out['base'][k, 6:9]) and _same_bits(gap, out['gap'][k])
            assert _same_bits(mpt, out['point'][k])
    near = cKDTree(cur).query_pairs(2 * rad.max() + 1e-5, output_type='ndarray')
    left = [(int(a), int(b)) for a, b in near if (int(a), int(b)) not in found][:300]
    assert left
    for a, b in left:
        assert oracle.ref_gobj_sphere_sphere(cur[a], rad[a], 0, cur[b], rad[b], 0)[0] == 0


@pytest.mark.skipif(not oracle.geo_available(), reason='reference build unavailable')
def test_sphere_update_pinned_to_reference_gobjcontact():
    """Kept contacts after the centres moved (roles kept): the reference's
    update_sphere_sphere (CONTACT_UPDATE, slave first) gives the oracle's
    normal, gap and points bit for bit, also where the centres' point order
    has flipped."""
    rng = np.random.default_rng(21)
    for t in range(200):
        a = rng.normal(size=3)
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        c = _two_spheres(a, a + d * rng.uniform(0.95, 1.0), r=(0.5, 0.5))
        first = _detect(c)
        assert first['key'].shape[0] == 1
        b = a + d * rng.uniform(0.9, 1.0) * np.where(rng.uniform() < 0.5, 1, -1)   # may swap the point order
        c2 = _two_spheres(a, b, r=(0.5, 0.5))
        out = _detect(c2, dict(key=first['key'], slave_lo=first['slave_lo']))
        assert out['key'].shape[0] == 1 and out['isnew'][0] == 0
        s, m = (0, 1) if first['slave_lo'][0] else (1, 0)
        cs = [a, b]
        st, one, two, nrm, gap, _ = oracle.ref_gobj_sphere_sphere(cs[s], 0.5, 0, cs[m], 0.5, 0, update=True)
        assert st == 1
        assert _same_bits(nrm, out['base'][0, 6:9]) and _same_bits(gap, out['gap'][0])
        assert _same_bits(two, out['point'][0])


@pytest.mark.skipif(not oracle.geo_available(), reason='reference build unavailable')
def test_convex_contacts_pinned_to_reference_gobjcontact():
    """Spheres pressed into the floor and a side wall of the box: every
    sphere-wall contact equals the reference's detect_convex_sphere
    (gobjcontact with the convex first and with the sphere first) and
    update_convex_sphere bit for bit; spheres the oracle leaves out touch no
    wall there."""
    sc, sp, x, out = _box_contacts([0.0035, 0.0, -0.0021])
    cv = sp['convex']
    n = sp['body'].shape[0]
    cur = oracle.sphere_centres(sp['body'], sp['centre'], sc.rot, x, sc.x0)
    walls = {}
    for c in range(cv['body'].shape[0]):
        b = cv['body'][c]
        X = cv['vert'][cv['vptr'][c]:cv['vptr'][c + 1]]
        A = X - sc.x0[b]   # the walls do not rotate: R (X - X0) is X - X0 exactly
        walls[c] = (x[b] + A, cv['fac'][cv['fptr'][c]:cv['fptr'][c + 1]], cv['surf'][cv['sptr'][c]:cv['sptr'][c + 1]])
    seen = set()
    for k in range(out['key'].shape[0]):
        i, j = int(out['key'][k] >> 32), int(out['key'][k] & 0xFFFFFFFF)
        if j < n:
            continue
        c = j - n
        seen.add((i, c))
        ver, fac, surf = walls[c]
        for sphere_first in (False, True):
            for update in (False, True):
                st, one, two, nrm, gap, spair = oracle.ref_gobj_convex_sphere(ver, fac, surf, cur[i], 0.05, 0,
                                                                              sphere_first, update)
                assert st == (2 if sphere_first and not update else 1)
                mpt = one if sphere_first else two
                assert _same_bits(nrm, out['base'][k, 6:9]) and _same_bits(gap, out['gap'][k])
                assert _same_bits(mpt, out['point'][k])
    assert len(seen) >= 40
    for i in range(n):
        for c in walls:
            if (i, c) not in seen:
                ver, fac, surf = walls[c]
                assert oracle.ref_gobj_convex_sphere(ver, fac, surf, cur[i], 0.05, 0)[0] == 0


@pytest.mark.skipif(not oracle.geo_available(), reason='reference build unavailable')
def test_reference_broad_phase_finds_the_oracle_pairs(scene_cache):
    """The reference's own broad phase (hyb.c hybrid over the eps-inflated
    sphere boxes) with detect_sphere_sphere per overlap finds exactly the
    oracle's sphere pairs on the settled lattice and on an overlapping grid."""
    for sc in (scene_cache('spheres_lattice'), scenes.spheres_grid(12)):
        sp = scenes.sphere_shapes(sc, friction=0.3)
        out = oracle.detect_spheres(sp['body'], sp['centre'], sp['radius'], sp['surface'], sc.rot, sc.x, sc.x0,
                                    sc.obstacle, MAT)
        cur = oracle.sphere_centres(sp['body'], sp['centre'], sc.rot, sc.x, sc.x0)
        ref = oracle.ref_detect_spheres_hybrid(cur, sp['radius'], sp['body'], pairs=True)
        assert ref.shape[0] > 1000 and np.array_equal(ref, out['key'])


# ---------------------------------------------------------------- golden vectors of the reference's gobjcontact

def _unhex(v):
    return np.array([float.fromhex(x) for x in v])


def _golden():
    import json
    import os
    return json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'detect_ref.json')))


def test_oracle_sphere_pairs_match_golden_gobjcontact():
    """tests/golden/detect_ref.json (made by make_detect_golden.py from the
    reference's own gobjcontact): each sphere pair, detected fresh or updated
    with the first sphere as the slave, gives the oracle's contact bit for bit."""
    eye = np.tile(np.eye(3).reshape(9), (2, 1))
    z = np.zeros((2, 3))
    for case in _golden()['sphere_sphere']:
        a, b = _unhex(case['a']), _unhex(case['b'])
        ra, rb = _unhex(case['ra'])[0], _unhex(case['rb'])[0]
        prev = dict(key=np.array([1], np.int64), slave_lo=np.array([1], np.int32)) if case['update'] else None
        out = oracle.detect_spheres([0, 1], np.stack([a, b]), [ra, rb], [0, 0], eye, z, z, [0, 0], MAT, prev)
        if case['state'] == 0:
            assert out['key'].shape[0] == 0
            continue
        assert out['key'].shape[0] == 1
        st = case['state']
        assert out['master'][0] == (1 if st == 1 else 0)
        assert _same_bits(out['base'][0, 6:9], _unhex(case['normal'])) and _same_bits(out['gap'], _unhex(case['gap']))
        assert _same_bits(out['point'][0], _unhex(case['twopnt'] if st == 1 else case['onepnt']))


def test_oracle_convex_sphere_matches_golden_gobjcontact():
    """Each convex-sphere case of the fixture (convex or sphere first, detect
    or update, centres near faces, edges and inside) gives the oracle's contact
    bit for bit: normal, gap, master point, and the convex point."""
    eye = np.tile(np.eye(3).reshape(9), (2, 1))
    z = np.zeros((2, 3))
    for case in _golden()['convex_sphere']:
        ver = _unhex(case['ver']).reshape(-1, 3)
        fac = np.array(case['fac'], np.int32)
        surf = np.array(case['surf'], np.int32)
        c, r = _unhex(case['c']), _unhex(case['r'])[0]
        cv = dict(body=[1], vptr=[0, ver.shape[0]], vert=ver, fptr=[0, fac.shape[0]], fac=fac, sptr=[0, surf.shape[0]],
                  surf=surf)
        mat = np.zeros((16, 16, 2))
        out = oracle.detect_spheres([0], c[None], [r], [3], eye, z, z, [0, 1], mat, None, convex=cv)
        if case['state'] == 0:
            assert out['key'].shape[0] == 0
            continue
        assert out['key'].shape[0] == 1 and out['master'][0] == 0 and out['slave'][0] == 1
        mpt, cpt = (case['onepnt'], case['twopnt']) if case['sphere_first'] else (case['twopnt'], case['onepnt'])
        assert _same_bits(out['base'][0, 6:9], _unhex(case['normal'])) and _same_bits(out['gap'], _unhex(case['gap']))
        assert _same_bits(out['point'][0], _unhex(mpt))
        assert _same_bits(out['spnt'][0], _unhex(cpt))   # referential = spatial here


@pytest.mark.skipif(not oracle.ref_available(), reason='reference build unavailable')
def test_gjk_polytopes_pinned_to_reference():
    """gjk of two polytopes (the first step of the reference's convex-convex
    intersection, cvi.c:131) restated bit for bit: separated, touching and
    overlapping pairs of perturbed, rotated hexahedra."""
    rng = np.random.default_rng(13)
    base = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float)
    for t in range(2000):
        def hexa():
            h = base * rng.uniform(0.2, 2, 3) + rng.normal(size=(8, 3)) * 0.05
            return h @ np.linalg.qr(rng.normal(size=(3, 3)))[0].T
        a, b = hexa(), hexa()
        b += a.mean(0) - b.mean(0) + rng.normal(size=3) * [0.3, 1.0, 3.0][t % 3]
        d1, p1, q1 = oracle.gjk_polytopes(a, b, 'oracle')
        d2, p2, q2 = oracle.gjk_polytopes(a, b, 'ref')
        assert _bits([d1]) == _bits([d2]) and np.array_equal(_bits(p1), _bits(p2)) and np.array_equal(_bits(q1), _bits(q2))


def test_clumps_of_spheres():
    """Bodies made of several spheres (clumps): spheres of one body never touch
    each other (box.c:107-108), and two bodies touching through two sphere
    pairs get two contacts between the same bodies."""
    nb = 2
    rot = np.tile(np.eye(3).reshape(9), (nb, 1))
    # body 0: spheres at x = 0 and x = 0.9 (overlapping each other); body 1: the same shifted up by 0.95
    sref = np.array([[0, 0, 0], [0.9, 0, 0], [0, 0, 0.95], [0.9, 0, 0.95]], float)
    out = oracle.detect_spheres([0, 0, 1, 1], sref, np.full(4, 0.5), np.zeros(4, np.int32), rot, np.zeros((2, 3)),
                                np.zeros((2, 3)), np.zeros(2, np.int32), MAT)
    pairs = [(int(k >> 32), int(k & 0xFFFFFFFF)) for k in out['key']]
    assert (0, 1) not in pairs and (2, 3) not in pairs
    assert (0, 2) in pairs and (1, 3) in pairs
    assert set(zip(out['master'].tolist(), out['slave'].tolist())) <= {(0, 1), (1, 0)}


@pytest.mark.skipif(not oracle.geo_available(), reason='reference build unavailable')
def test_convex_convex_golden_pinned_to_reference():
    """tests/golden/convex/pile_ref.npz (make_cvi_golden.py) holds exactly the
    reference's gobjcontact results (detect_convex_convex, goc.c:280-306) for
    every convex pair of the seeded convex piles, bit for bit."""
    import importlib.util
    spec = importlib.util.spec_from_file_location('make_cvi_golden', os.path.join(os.path.dirname(
        os.path.abspath(__file__)), 'golden', 'make_cvi_golden.py'))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'convex', 'pile_ref.npz'))
    for seed, kw in gen.CASES:
        now = gen.reference_pairs(seed, kw)
        assert now['keys'].shape[0] > 20
        for name, v in now.items():
            stored = g['s%d_%s' % (seed, name)]
            assert stored.shape == v.shape and np.array_equal(stored.view(np.uint8), v.view(np.uint8)), (seed, name)


def _cvi_host_lib(tmp_path_factory):
    """tests/cvi_host_harness.cpp: csrc/b2_cvi.cuh built for the host with
    g++ (no fused multiply-adds, as the device build)."""
    import ctypes as C
    import subprocess
    here = os.path.dirname(os.path.abspath(__file__))
    csrc = os.path.join(os.path.dirname(here), 'solfec-1.0_b200', 'csrc')
    out = str(tmp_path_factory.mktemp('cvi') / 'libcvi_host.so')
    subprocess.check_call(['g++', '-O2', '-ffp-contract=off', '-fPIC', '-shared', '-I', csrc, '-o', out,
                           os.path.join(here, 'cvi_host_harness.cpp')])
    lib = C.CDLL(out)
    dp = np.ctypeslib.ndpointer(np.float64, flags='C')
    ip = np.ctypeslib.ndpointer(np.int32, flags='C')
    lib.cvi_host_pair.restype = C.c_int
    lib.cvi_host_pair.argtypes = [C.c_int, C.c_int, dp, C.c_int, ip, ip, C.c_int, dp, C.c_int, ip, ip, dp, dp, dp,
                                  dp, ip]
    lib.cvi_host_orient3d.restype = C.c_double
    lib.cvi_host_orient3d.argtypes = [dp, dp, dp, dp]
    return lib


@pytest.fixture(scope='module')
def cvi_host(tmp_path_factory):
    return _cvi_host_lib(tmp_path_factory)


def test_cvi_orientation_sign_exact(cvi_host):
    """The hull's orientation test (csrc/b2_cvi.cuh orient3d) has the exact
    sign of the determinant on near-degenerate inputs, against rational
    arithmetic: coplanar points, points a rounding away from a plane,
    collinear points, widely scaled points."""
    from fractions import Fraction as F
    rng = np.random.default_rng(3)
    zeros = 0
    for t in range(4000):
        k = t % 4
        if k == 0:
            pts = [np.array([rng.uniform(-1, 1) * 10.0 ** rng.integers(-3, 6), rng.uniform(-1, 1), 0.3])
                   for _ in range(4)]
        elif k == 1:
            a, b, c = (rng.normal(size=3) * 1e4 for _ in range(3))
            u, v = rng.uniform(size=2)
            d = a + u * (b - a) + v * (c - a)
            pts = [a, b, c, d + rng.choice([0.0, 1e-12, -1e-12]) * rng.normal(size=3)]
        elif k == 2:
            a, dv = rng.normal(size=3), rng.normal(size=3)
            pts = [a + s * dv for s in rng.uniform(-1, 1, 4)]
        else:
            pts = [rng.normal(size=3) * 10.0 ** rng.integers(-6, 6) for _ in range(4)]
        pts = [np.ascontiguousarray(p, float) for p in pts]
        M = [[F(x) - F(y) for x, y in zip(p, pts[3])] for p in pts[:3]]
        e = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0])
             + M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]))
        s = cvi_host.cvi_host_orient3d(*pts)
        zeros += e == 0
        assert ((e > 0) - (e < 0)) == ((s > 0) - (s < 0)), t
    assert zeros > 500


def _random_hull(rng, centre, npts):
    V, faces = scenes.hull_faces(centre + rng.normal(size=(npts, 3)) * 0.5)
    fac = np.array(sum(([3] + list(f) for f in faces), []), np.int32)
    return V, fac, len(faces)


@pytest.mark.skipif(not oracle.geo_available(), reason='reference build unavailable')
def test_cvi_restatement_equals_reference_on_random_pairs(cvi_host):
    """csrc/b2_cvi.cuh, built for the host, against the reference's own
    gobjcontact (detect_convex_convex and update_convex_convex) on random
    pairs: stacked and offset boxes (touching exactly, within and past eps,
    overlapping), perturbed hexahedra side by side, turned boxes, coincident
    side planes, and random hulls of 5 to 8 points. State, point, normal, gap,
    area and surface pair equal bit for bit."""
    rng = np.random.default_rng(7)
    fac_box = np.array(sum(([4] + list(f) for f in scenes.HEX_FACES), []), np.int32)

    def box(c, h, pert=0.0, R=None):
        v = np.array([[(-h[0], h[0])[i], (-h[1], h[1])[j], (-h[2], h[2])[k]] for k in (0, 1) for j in (0, 1)
                      for i in (0, 1)])
        v = v + rng.uniform(-pert, pert, v.shape) * h
        return (v @ R.T if R is not None else v) + c

    def turn():
        w = rng.normal(size=3)
        a = np.linalg.norm(w)
        K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
        return np.eye(3) + np.sin(a) / a * K + (1 - np.cos(a)) / a ** 2 * K @ K

    contacts = 0
    for t in range(1200):
        kind = t % 5
        h = 0.5 * rng.uniform(0.5, 1.5, 3)
        if kind == 0:
            a = box(np.zeros(3), h)
            b = box(np.array([rng.uniform(-.5, .5), rng.uniform(-.5, .5),
                              2 * h[2] + rng.choice([0.0, -1e-3, -1e-2, 1e-7, -1e-7])]), h)
            fa = fb = fac_box
        elif kind == 1:
            a = box(np.zeros(3), h, 0.1)
            b = box(np.array([2 * h[0] + rng.uniform(-0.05, 0.02), rng.uniform(-0.1, 0.1), 0.0]), h, 0.1)
            fa = fb = fac_box
        elif kind == 2:
            a = box(np.zeros(3), h, R=turn())
            b = box(rng.uniform(-1.2, 1.2, 3), h, R=turn())
            fa = fb = fac_box
        elif kind == 3:
            a = box(np.zeros(3), h)
            b = box(np.array([0.0, 0.0, 2 * h[2] - rng.choice([0.0, 1e-3, 0.25])]), h)
            fa = fb = fac_box
        else:
            a, fa, _ = _random_hull(rng, np.zeros(3), int(rng.integers(5, 9)))
            b, fb, _ = _random_hull(rng, rng.uniform(-0.8, 0.8, 3), int(rng.integers(5, 9)))
        sa = np.arange(1, 1 + (6 if fa is fac_box else fa.shape[0] // 4), dtype=np.int32)
        sb = np.arange(11, 11 + (6 if fb is fac_box else fb.shape[0] // 4), dtype=np.int32)
        for update in (False, True):
            r = oracle.ref_gobj_convex_convex(a, fa, sa, b, fb, sb, update=update, spair=(sa[0], sb[0]))
            va = np.ascontiguousarray(a, float).ravel()
            vb = np.ascontiguousarray(b, float).ravel()
            pt, nr, g, ar = np.zeros(3), np.zeros(3), np.zeros(1), np.zeros(1)
            sp = np.array([sa[0], sb[0]], np.int32)
            st = cvi_host.cvi_host_pair(int(update), va.size // 3, va, sa.size, fa, sa, vb.size // 3, vb, sb.size,
                                        fb, sb, pt, nr, g, ar, sp)
            assert st == r[0], (t, update)
            if st > 0:
                contacts += 1
                for mine, ref in ((pt, r[1]), (nr, r[2]), (g[0], r[3]), (ar[0], r[4])):
                    assert np.array_equal(np.asarray(mine, float).view(np.uint64),
                                          np.asarray(ref, float).view(np.uint64)), (t, update)
                assert np.array_equal(sp, r[5]), (t, update)
    assert contacts > 1500
