"""GPU tests of the device rigid time integration (csrc/b2_rigid.cuh through
the C ABI b2dev_rigid_*): bitwise parity with the CPU restatement
oracle/rigid_oracle.py (BODY_Dynamic_Step_Begin / End, bod.c:1313-1493), and
the reference's own end-to-end pins of tests/block-sliding.py:64-80 through
the full device step (integrator, assembly, Gauss-Seidel solve)."""
import dataclasses
import json
import os

import numpy as np
import pytest

import oracle
import rigid_oracle as ro
from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, scenes
from solfec_b200.dynamics import RIGID_DYNAMICS, run_fixed_contacts
from solfec_b200._lib import lib

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _scene_with_spin(seed, omega):
    sc = scenes.spheres_small(seed, 60)
    rng = np.random.default_rng(seed)
    nb = sc.nbod
    velo = sc.velo.copy()
    velo[:, 0:3] = rng.normal(size=(nb, 3)) * omega
    velo[sc.obstacle != 0] = 0.0
    sc = dataclasses.replace(sc, velo=np.ascontiguousarray(velo), velo0=np.ascontiguousarray(velo))
    ob = sc.obstacle != 0  # walls: zero inverse inertia and mass (never accelerated)
    J = np.stack([np.eye(3).reshape(9) if o else np.linalg.inv(j.reshape(3, 3).T).T.reshape(9)
                  for j, o in zip(sc.jinv, ob)])
    mass = np.where(ob, 1.0, 1.0 / np.where(ob, 1.0, sc.minv))
    schemes = [('RIG_POS', 'RIG_NEG', 'RIG_IMP')[b % 3] for b in range(nb)]
    loads = rng.normal(size=(nb, 9))
    return sc, J, mass, schemes, loads


def _oracle_bodies(sc, J, mass, schemes, flags=None):
    from solfec_b200.dynamics import SCHEMES
    return ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle,
                     [SCHEMES[s] for s in schemes], flags)


@pytest.mark.parametrize('omega,exact', [(5.0, True), (900.0, False)])
def test_rigid_step_parity(omega, exact):
    """Device begin/end against the oracle on 60 bodies with the three schemes
    (NEW1, NEW2, NEW3's Newton solve), every seventh body with
    BODY_DISABLE_ROTATION, obstacles, point loads and random reactions:
    bitwise while the rotation of a half step stays below ten degrees (Taylor
    branch of the exponential map and its derivatives), within 1e-12 relative
    above it (sin/cos of two libraries)."""
    sc, J, mass, schemes, loads = _scene_with_spin(11, omega)
    h = 1e-3
    g = (0.0, 0.0, -9.81)
    ldy = LOCDYN()
    ldy.update_begin(sc)
    off = np.arange(sc.nbod) % 7 == 3
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x, schemes, disable_rotation=off)
    bd = _oracle_bodies(sc, J, mass, schemes, np.where(off, ro.BODY_DISABLE_ROTATION, 0))

    def same(a, b):
        a, b = np.asarray(a, float), np.asarray(b, float)
        if exact:
            assert np.array_equal(a, b), np.abs(a - b).max()
        else:
            assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * max(1.0, np.abs(b).max()))

    dyn.step_begin(h, g, loads)
    ro.step_begin(bd, h, g, loads)
    st = dyn.state()
    for k in ('rot', 'x', 'velo', 'velo0'):
        same(st[k], np.array(getattr(bd, k)))

    assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, 1) == 0
    rng = np.random.default_rng(3)
    R = rng.normal(size=(sc.ncon, 3))
    ldy.set_state(R, np.zeros((sc.ncon, 3)))
    dyn.step_end(h)
    ro.step_end(bd, h, sc.master, sc.slave, sc.mpnt, sc.spnt, sc.base, R)
    st = dyn.state()
    for k in ('rot', 'x', 'velo'):
        same(st[k], np.array(getattr(bd, k)))
    ldy.close()


def test_rigid_rejects_unknown_scheme():
    sc, J, mass, _, _ = _scene_with_spin(2, 1.0)
    ldy = LOCDYN()
    ldy.update_begin(sc)
    with pytest.raises(ValueError):
        RIGID_DYNAMICS(ldy, J, mass, sc.x, 'RIG_FOO')
    sch = np.full(sc.nbod, 3, dtype=np.int32)  # no such scheme, through the C ABI
    from solfec_b200._lib import ptr
    Jc = np.ascontiguousarray(J); mc = np.ascontiguousarray(mass); xc = np.ascontiguousarray(sc.x)
    assert lib().b2dev_rigid_setup(ldy.device_context, ptr(Jc), ptr(mc), ptr(xc), ptr(sch), 0) != 0
    ldy.close()


def test_new3_failure_reported():
    """A NEW3 body whose Newton Jacobian is singular (zero inertia under a
    referential torque), where the reference stops the program
    (ERR_BOD_NEW3_SINGULAR_JACOBIAN, bod.c:196): the device records it and the
    next state read raises; the oracle reports the same."""
    from solfec_b200 import DeviceError
    sc, J, mass, _, _ = _scene_with_spin(5, 1.0)
    J = J.copy()
    b = int(np.nonzero(sc.obstacle == 0)[0][0])
    J[b] = 0.0
    loads = np.zeros((sc.nbod, 9)); loads[b, 6] = 1.0
    sc = dataclasses.replace(sc, master=np.zeros(0, np.int32), slave=np.zeros(0, np.int32), mpnt=np.zeros((0, 3)),
                             spnt=np.zeros((0, 3)), base=np.zeros((0, 9)), gap=np.zeros(0), friction=np.zeros(0),
                             restitution=np.zeros(0), cohesion=np.zeros(0))
    ldy = LOCDYN()
    ldy.update_begin(sc)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x, 'RIG_IMP')
    dyn.step_begin(1e-3, (0.0, 0.0, 0.0), loads)
    dyn.step_end(1e-3)
    with pytest.raises(DeviceError, match='NEW3'):
        dyn.state()
    ldy.close()
    bd = _oracle_bodies(sc, J, mass, ['RIG_IMP'] * sc.nbod)
    none = (np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
    ro.step_begin(bd, 1e-3, (0.0, 0.0, 0.0), loads)
    ro.step_end(bd, 1e-3, [], [], *none)
    assert bd.failures == 1


def test_block_sliding_device():
    """The reference's block-sliding test (tests/block-sliding.py): 8001 steps
    of the device step on the restated scene. The first 1000 steps equal the
    CPU restatement (oracle integrator and oracle Gauss-Seidel) bitwise; the
    six trajectory values the reference pins hold to its 1e-3 tolerance."""
    sc, J, mass = scenes.block_sliding()
    ref = json.load(open(os.path.join(HERE, 'golden', 'block_sliding_ref.json')))
    nsteps = max(p['index'] for p in ref['pins']) + 1
    X, V = [], []

    def cb(k, t, dyn, ldy):
        st = dyn.state()
        X.append(st['x'][1, 0])
        V.append(st['velo'][1, 3])

    gs = GAUSS_SEIDEL_SOLVER(1e-3, 1000)
    dyn, ldy = run_fixed_contacts(sc, gs, nsteps, J, mass, gravity=(0.0, 0.0, -9.81),
                                  loads=scenes.block_sliding_loads, callback=cb)
    ldy.close()
    X, V = np.array(X), np.array(V)
    for p in ref['pins']:
        val = X[p['index']] if p['quantity'] == 'x' else V[p['index']]
        assert abs(val - p['value']) / max(1.0, p['value']) <= ref['tolerance'], (p, val)

    # CPU restatement of the same 1000 steps
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    R = np.zeros(3 * sc.ncon)
    U = np.zeros(3 * sc.ncon)
    t, h = 0.0, sc.step
    Xc, Vc = [], []
    for _ in range(1000):
        ro.step_begin(bd, h, (0.0, 0.0, -9.81), scenes.block_sliding_loads(t + 0.5 * h))
        cur = dataclasses.replace(sc, rot=np.array(bd.rot), velo=np.array(bd.velo), velo0=np.array(bd.velo0))
        out = oracle.solve(oracle.assemble(cur), R, U, epsilon=1e-3, maxiter=1000)
        R, U = out['R'], out['U']
        ro.step_end(bd, h, sc.master, sc.slave, sc.mpnt, sc.spnt, sc.base, R.reshape(-1, 3))
        t += h
        Xc.append(bd.x[1][0])
        Vc.append(bd.velo[1][3])
    assert np.array_equal(X[:1000], np.array(Xc))
    assert np.array_equal(V[:1000], np.array(Vc))


def test_projectile_device():
    """The reference's tests/projectile.py on the device integrator (no
    contacts): the pinned x distance within its 0.5%, and every step equal to
    the CPU restatement bitwise."""
    sc, J, mass = scenes.projectile()
    ldy = LOCDYN()
    ldy.update_begin(sc)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    g = (0.0, 0.0, -scenes.PROJECTILE_GRAVITY)
    for _ in range(1024):
        u = dyn.state()['velo'][0]
        dyn.step_begin(sc.step, g, scenes.projectile_loads(mass[0], u))
        dyn.step_end(sc.step)
        ro.step_begin(bd, sc.step, g, scenes.projectile_loads(bd.mass[0], bd.velo[0]))
        ro.step_end(bd, sc.step, [], [], np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
        st = dyn.state()
        assert np.array_equal(st['x'][0], np.array(bd.x[0])) and np.array_equal(st['velo'][0], np.array(bd.velo[0]))
    ldy.close()
    ref = json.load(open(os.path.join(HERE, 'golden', 'projectile_ref.json')))
    x_in = st['x'][0, 0] / 0.0254
    assert abs(x_in - ref['value']) / ref['value'] < ref['tolerance'], x_in
