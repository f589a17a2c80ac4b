"""GPU tests of the sphere contact update and detection (csrc/b2_detect.cuh
through the C ABI b2dev_spheres_setup / b2dev_detect_spheres): bit-for-bit
parity of every contact array with the CPU restatement
oracle/oracle_detect.c on settled packings (1000 equal spheres, 20000
polydisperse spheres), and inside a device time loop where bodies move,
contacts appear, persist with their roles and carried R and U, and separate."""
import dataclasses

import numpy as np
import pytest

import oracle
from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, DeviceError, scenes
from solfec_b200._lib import lib
from solfec_b200.detect import SPHERES, bodies_only, run_spheres
from solfec_b200.dynamics import RIGID_DYNAMICS

pytestmark = pytest.mark.gpu

KEYS = ['key', 'slave_lo', 'master', 'slave', 'point', 'mpnt', 'spnt', 'base', 'gap', 'friction', 'restitution',
        'R', 'U', 'isnew']


def _same(dev, orc):
    assert dev['key'].shape[0] == orc['key'].shape[0]
    for k in KEYS:
        a, b = np.asarray(dev[k]), np.asarray(orc[k])
        if a.dtype.kind == 'f':
            assert np.array_equal(a.view(np.uint64), np.ascontiguousarray(b, dtype=np.float64).view(np.uint64)), k
        else:
            assert np.array_equal(a.astype(np.int64), b.astype(np.int64)), k


def _oracle(sp, rot, x, x0, obst, prev=None):
    mat = np.asarray(sp['material'], float).reshape(1, 1, 2)
    return oracle.detect_spheres(sp['body'], sp['centre'], sp['radius'], sp['surface'], rot, x, x0, obst, mat, prev)


def _detect_scene(sc):
    sp = scenes.sphere_shapes(sc)
    J, mass = scenes.sphere_inertia(sc)
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    RIGID_DYNAMICS(ldy, J, mass, sc.x)
    sph = SPHERES(ldy, **sp)
    nc, nn = sph.detect()
    dev = sph.contacts()
    cur = sph.centres()
    orc = _oracle(sp, sc.rot, sc.x, sc.x0, sc.obstacle)
    assert nc == nn == orc['key'].shape[0]
    assert np.array_equal(cur, oracle.sphere_centres(sp['body'], sp['centre'], sc.rot, sc.x, sc.x0))
    _same(dev, orc)
    ldy.close()
    return nc


def test_detect_lattice_matches_oracle(scene_cache):
    assert _detect_scene(scene_cache('spheres_lattice')) > 1000


def test_detect_polydisperse_matches_oracle(scene_cache):
    assert _detect_scene(scene_cache('spheres_polydisperse')) > 10000


def test_time_loop_matches_oracle_every_step():
    """Spheres falling onto a bed of fixed spheres: every step's detection on
    the device bodies equals the oracle's, given the previous step's contacts
    and the R and U of the device solve."""
    sc, sp, J, mass = scenes.spheres_on_bed()
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    sph = SPHERES(ldy, **sp)
    gs = GAUSS_SEIDEL_SOLVER(1e-6, 200, diagsolver='SEMISMOOTH_NEWTON')
    prev = None
    seen_new = seen_kept = seen_dropped = 0
    h = sc.step
    for k in range(120):
        dyn.step_begin(h, (0.0, 0.0, -9.81))
        st = dyn.state()
        nc, nn = sph.detect()
        dev = sph.contacts()
        orc = _oracle(sp, st['rot'], st['x'], sc.x0, sc.obstacle, prev)
        _same(dev, orc)
        if prev is not None:
            seen_dropped += int(np.setdiff1d(prev['key'], dev['key']).shape[0])
        seen_new += nn
        seen_kept += nc - nn
        if nc > 0:
            assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, 1) == 0
            sph.carry_state()
            R0, U0, _ = ldy.get_state()
            assert np.array_equal(R0, dev['R']) and np.array_equal(U0, dev['U'])
            gs.solve(ldy)
            R, U, _ = ldy.get_state()
            prev = dict(key=dev['key'], slave_lo=dev['slave_lo'], R=R, U=U)
        else:
            prev = dict(key=dev['key'], slave_lo=dev['slave_lo'])
        dyn.step_end(h)
    assert seen_new > 0 and seen_kept > 0
    # the spheres rest on the bed: no deep interpenetration, none fell through
    assert dev['gap'].min() > -2e-3, dev['gap'].min()
    assert np.all(dyn.state()['x'][sc.obstacle == 0, 2] > 0.04)
    ldy.close()


def test_run_spheres_loop():
    sc, sp, J, mass = scenes.spheres_on_bed(seed=6, n_side=4, layers=2)
    gs = GAUSS_SEIDEL_SOLVER(1e-6, 200)
    counts = []
    dyn, sph, ldy = run_spheres(sc, sp, gs, 80, J, mass, gravity=(0.0, 0.0, -9.81),
                                callback=lambda k, d, s, l: counts.append(s.ncon))
    assert max(counts) > 0 and counts[0] == 0
    assert np.all(dyn.state()['x'][sc.obstacle == 0, 2] > 0.04)
    ldy.close()


def _pair_scene(dz):
    """spheres_on_bed with body 1 moved onto body 0 (dz above it); every
    sphere centred on its body, so the current centres are exact."""
    sc, sp, J, mass = scenes.spheres_on_bed(seed=7, n_side=2, layers=1)
    x = sc.x.copy()
    x[1] = x[0] + np.array([0.0, 0.0, dz])
    sc = dataclasses.replace(sc, x=x, x0=x.copy())
    sp = dict(sp, centre=x.copy())
    return sc, sp, J, mass


def _setup(sc, J, mass):
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    RIGID_DYNAMICS(ldy, J, mass, sc.x)
    return ldy


def test_detect_errors_reported():
    sc, sp, J, mass = _pair_scene(0.0)   # coincident centres of two bodies
    ldy = _setup(sc, J, mass)
    with pytest.raises(DeviceError, match='coincide'):
        SPHERES(ldy, **sp).detect()
    ldy.close()
    sc, sp, J, mass = _pair_scene(0.09)  # one contact, surface 3 of a one-surface table
    ldy = _setup(sc, J, mass)
    with pytest.raises(DeviceError, match='surface'):
        SPHERES(ldy, **dict(sp, surface=np.full(sp['body'].shape[0], 3, np.int32))).detect()
    with pytest.raises(DeviceError, match='symmetric'):
        SPHERES(ldy, **dict(sp, material=np.array([[[0.1, 0.0], [0.2, 0.0]], [[0.3, 0.0], [0.1, 0.0]]])))
    s = SPHERES(ldy, **sp)
    assert s.detect() == (1, 1)
    ldy.close()


def test_sparsified_contacts_match_oracle():
    """Sphere 0 touches spheres 1 and 2, whose centres lie 1e-7 apart: the two
    contact points are duplicates and the earlier new contact is removed
    (the compaction path; without removals the staged arrays are taken over)."""
    sc, sp, J, mass = scenes.spheres_on_bed(seed=7, n_side=2, layers=1)
    x = sc.x.copy()
    x[1] = x[0] + np.array([0.099, 0.0, 0.0])
    x[2] = x[1] + np.array([1e-7, 0.0, 0.0])
    sc = dataclasses.replace(sc, x=x, x0=x.copy())
    sp = dict(sp, centre=x.copy())
    ldy = _setup(sc, J, mass)
    s = SPHERES(ldy, **sp)
    assert s.detect() == (2, 2)
    dev = s.contacts()
    assert dev['key'].tolist() == [(0 << 32) | 2, (1 << 32) | 2]
    _same(dev, _oracle(sp, sc.rot, sc.x, sc.x0, sc.obstacle))
    ldy.close()


def _oracle_box(sp, rot, x, x0, obst, prev=None):
    mat = np.asarray(sp['material'], float).reshape(1, 1, 2)
    return oracle.detect_spheres(sp['body'], sp['centre'], sp['radius'], sp['surface'], rot, x, x0, obst, mat, prev,
                                 convex=sp['convex'])


def test_box_walls_match_oracle():
    """Spheres pressed into the floor and a side wall of a box of convex walls:
    sphere-convex contacts (GJK closest points, planes, nearest surface) equal
    the oracle bit for bit."""
    sc, sp, J, mass = scenes.spheres_in_box()
    n = sp['body'].shape[0]
    x = sc.x.copy()
    x[:n] += np.array([0.0035, 0.0, -0.0021])
    sc = dataclasses.replace(sc, x=x)
    ldy = _setup(sc, J, mass)
    s = SPHERES(ldy, **sp)
    nc, nn = s.detect()
    dev = s.contacts()
    orc = _oracle_box(sp, sc.rot, sc.x, sc.x0, sc.obstacle)
    assert nc == nn == orc['key'].shape[0] and int(((dev['key'] & 0xFFFFFFFF) >= n).sum()) >= 25 + 15
    _same(dev, orc)
    ldy.close()


def test_box_time_loop_matches_oracle_every_step():
    """Spheres dropped into the box: every step's contacts (sphere-sphere and
    sphere-wall) equal the oracle's on the device bodies, with the carried R, U."""
    sc, sp, J, mass = scenes.spheres_in_box(n_side=4, layers=3)
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    sph = SPHERES(ldy, **sp)
    gs = GAUSS_SEIDEL_SOLVER(1e-6, 200)
    prev = None
    walls = 0
    h = sc.step
    for k in range(80):
        dyn.step_begin(h, (0.0, 0.0, -9.81))
        st = dyn.state()
        nc, nn = sph.detect()
        dev = sph.contacts()
        _same(dev, _oracle_box(sp, st['rot'], st['x'], sc.x0, sc.obstacle, prev))
        walls = max(walls, int(((dev['key'] & 0xFFFFFFFF) >= sp['body'].shape[0]).sum()))
        if nc > 0:
            assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, 1) == 0
            sph.carry_state()
            gs.solve(ldy)
            R, U, _ = ldy.get_state()
            prev = dict(key=dev['key'], slave_lo=dev['slave_lo'], R=R, U=U)
        else:
            prev = dict(key=dev['key'], slave_lo=dev['slave_lo'])
        dyn.step_end(h)
    assert walls >= 16   # the lowest layer rests on the floor
    assert np.all(dyn.state()['x'][:sp['body'].shape[0], 2] > 0.04)
    ldy.close()


def _clump_scene(offsets0, offsets1, dz):
    """spheres_on_bed with bodies 0 and 1 made clumps (several spheres each,
    at the given offsets from the body's centre) and body 1 placed dz above
    body 0; every rotation the identity, so referential and current centres
    agree. Bodies 2 and 3 carry no shapes; the bed spheres keep theirs."""
    sc, sp, J, mass = scenes.spheres_on_bed(seed=7, n_side=2, layers=1)
    nb = sc.nbod
    x = sc.x.copy()
    x[1] = x[0] + np.array([0.0, 0.0, dz])
    sc = dataclasses.replace(sc, rot=np.tile(np.eye(3).reshape(9), (nb, 1)), x=x, x0=x.copy())
    o0, o1 = np.asarray(offsets0, float), np.asarray(offsets1, float)
    bed = np.arange(4, nb)
    body = np.concatenate([np.zeros(len(o0)), np.ones(len(o1)), bed]).astype(np.int32)
    centre = np.concatenate([x[0] + o0, x[1] + o1, x[bed]])
    radius = np.concatenate([np.full(len(o0) + len(o1), 0.05), sp['radius'][bed]])
    sp = dict(sp, body=body, centre=centre, radius=radius, surface=np.zeros(body.shape[0], np.int32))
    return sc, sp, J, mass


@pytest.mark.parametrize('variant', ['two_contacts', 'duplicate_points'])
def test_clumps_match_oracle(variant):
    """Bodies made of several spheres: spheres of one body never touch each
    other (box.c:107-108); two bodies touching through two sphere pairs get
    two contacts between the same bodies; when those two contact points lie
    within 2 mindist of each other the sparsification removes one (the
    compaction path; otherwise the staged arrays are taken over). Every array
    equals the oracle's bit for bit."""
    if variant == 'two_contacts':  # overlapping spheres inside each body, two body-to-body contacts
        sc, sp, J, mass = _clump_scene([[0, 0, 0], [-0.09, 0, 0]], [[0, 0, 0], [-0.09, 0, 0]], 0.099)
    else:                          # body 0's two spheres 1e-7 apart: duplicate contact points with body 1
        sc, sp, J, mass = _clump_scene([[0, 0, 0], [1e-7, 0, 0]], [[0, 0, 0]], 0.099)
    ldy = _setup(sc, J, mass)
    s = SPHERES(ldy, **sp)
    nc, nn = s.detect()
    dev = s.contacts()
    orc = _oracle(sp, sc.rot, sc.x, sc.x0, sc.obstacle)
    _same(dev, orc)
    body = sp['body']
    pi, pj = dev['key'] >> 32, dev['key'] & 0xFFFFFFFF
    assert not np.any(body[pi] == body[pj])                       # no contact inside a clump
    assert set(zip(dev['master'].tolist(), dev['slave'].tolist())) <= {(0, 1), (1, 0)}
    if variant == 'two_contacts':
        assert nc == nn == 2 and pi.tolist() == [0, 1] and pj.tolist() == [2, 3]
    else:
        assert nc == nn == 1                                      # of two touching pairs, one contact is kept
    # a second detection updates the kept contacts with their roles
    nc2, nn2 = s.detect()
    assert nc2 == nc and nn2 == 0
    _same(s.contacts(), _oracle(sp, sc.rot, sc.x, sc.x0, sc.obstacle,
                                dict(key=dev['key'], slave_lo=dev['slave_lo'])))
    ldy.close()


def test_excluded_body_pairs_spheres(scene_cache):
    """CONTACT_EXCLUDE_BODIES on the settled 1000-sphere lattice: the contacts
    are the oracle's without the excluded body pairs, bit for bit."""
    sc = scene_cache('spheres_lattice')
    sp = scenes.sphere_shapes(sc)
    J, mass = scenes.sphere_inertia(sc)
    orc = _oracle(sp, sc.rot, sc.x, sc.x0, sc.obstacle)
    key = orc['key']
    bi = sp['body'][(key >> 32).astype(np.int64)]
    j = (key & 0xFFFFFFFF).astype(np.int64)
    bj = np.where(j < sp['body'].shape[0], sp['body'][np.minimum(j, sp['body'].shape[0] - 1)], -1)
    pairs = np.stack([bi, bj], axis=1)[::5]
    pairs = pairs[pairs[:, 1] >= 0]
    ex = {tuple(sorted(map(int, p))) for p in pairs}
    keep = np.array([tuple(sorted((int(a), int(b)))) not in ex for a, b in zip(bi, bj)])
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    RIGID_DYNAMICS(ldy, J, mass, sc.x)
    sph = SPHERES(ldy, **sp)
    sph.exclude_bodies(pairs)
    sph.detect()
    dev = sph.contacts()
    _same(dev, {k: np.asarray(v)[keep] for k, v in orc.items()})
    assert keep.sum() < keep.shape[0]
    ldy.close()
