"""CPU tests of the rigid time-integration oracle (oracle/rigid_oracle.py):
the reference's own end-to-end pins (tests/block-sliding.py:64-80) through
the restated integrator and the restated (and, when built, the compiled
reference) Gauss-Seidel solver, and properties of the schemes."""
import dataclasses
import json
import math
import os

import numpy as np
import pytest

import oracle
import rigid_oracle as ro
from solfec_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))


def run_block_sliding_cpu(nsteps, impl='oracle'):
    sc, J, mass = scenes.block_sliding()
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    h = sc.step
    R = np.zeros(3 * sc.ncon)
    U = np.zeros(3 * sc.ncon)
    X, V = [], []
    t = 0.0
    for _ in range(nsteps):
        ro.step_begin(bd, h, (0.0, 0.0, -9.81), scenes.block_sliding_loads(t + 0.5 * h))
        cur = dataclasses.replace(sc, rot=np.array(bd.rot), velo=np.array(bd.velo), velo0=np.array(bd.velo0))
        out = oracle.solve(oracle.assemble(cur), R, U, epsilon=1e-3, maxiter=1000, impl=impl)
        R, U = out['R'], out['U']
        ro.step_end(bd, h, sc.master, sc.slave, sc.mpnt, sc.spnt, sc.base, R.reshape(-1, 3))
        t += h
        X.append(bd.x[1][0])
        V.append(bd.velo[1][3])
    return np.array(X), np.array(V)


def check_pins(X, V):
    ref = json.load(open(os.path.join(HERE, 'golden', 'block_sliding_ref.json')))
    for p in ref['pins']:
        val = X[p['index']] if p['quantity'] == 'x' else V[p['index']]
        err = abs(val - p['value']) / max(1.0, p['value'])
        assert err <= ref['tolerance'], (p, val, err)


@pytest.mark.parametrize('impl', ['oracle', 'ref'])
def test_block_sliding_pins_cpu(impl):
    if impl == 'ref' and not oracle.ref_available():
        pytest.skip('compiled reference solver not built')
    X, V = run_block_sliding_cpu(8001, impl)
    check_pins(X, V)


def run_arch_cpu(ratio, nsteps=750, impl='oracle'):
    """The masonry arch of tests/arch.py as fixed contacts: 750 steps of 1 ms
    under gravity, GAUSS_SEIDEL_SOLVER (1E-4, 10000) warm-started from the
    previous reactions. Returns the kinetic energy of the voussoirs after the
    last step (ENERGY (solfec) [0])."""
    sc, J, mass = scenes.masonry_arch(ratio)
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    R = np.zeros(3 * sc.ncon)
    U = np.zeros(3 * sc.ncon)
    for _ in range(nsteps):
        ro.step_begin(bd, sc.step, (0.0, 0.0, -9.81))
        cur = dataclasses.replace(sc, rot=np.array(bd.rot), x=np.array(bd.x), velo=np.array(bd.velo),
                                  velo0=np.array(bd.velo0))
        out = oracle.solve(oracle.assemble(cur), R, U, epsilon=1e-4, maxiter=10000, impl=impl)
        R, U = out['R'], out['U']
        ro.step_end(bd, sc.step, sc.master, sc.slave, sc.mpnt, sc.spnt, sc.base, R.reshape(-1, 3))
    return sum(ro.kinetic_energy(bd, b) for b in range(bd.nbod) if not bd.obstacle[b])


@pytest.mark.parametrize('impl', ['oracle', 'ref'])
def test_masonry_arch_threshold_cpu(impl):
    """The reference's pass criterion (tests/arch.py:132): after 750 steps the
    arch of thickness ratio 0.1095 is at rest (kinetic energy below 1e-4) and
    the one of ratio 0.1094 collapses (above 1e-3)."""
    if impl == 'ref' and not oracle.ref_available():
        pytest.skip('compiled reference solver not built')
    e1 = run_arch_cpu(0.1095, impl=impl)
    e2 = run_arch_cpu(0.1094, impl=impl)
    assert e1 < 1e-4 and e2 > 1e-3, (e1, e2)


def test_projectile_pin_cpu():
    """The reference's tests/projectile.py: drag load -m v and gravity, no
    contacts; the x distance after the run in inches within 0.5% of 86.138
    (the exact value, 2.54 (1 - exp(-1.976)) m)."""
    sc, J, mass = scenes.projectile()
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    for _ in range(1024):
        L = scenes.projectile_loads(bd.mass[0], bd.velo[0])
        ro.step_begin(bd, sc.step, (0.0, 0.0, -scenes.PROJECTILE_GRAVITY), L)
        ro.step_end(bd, sc.step, [], [], np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
    ref = json.load(open(os.path.join(HERE, 'golden', 'projectile_ref.json')))
    x_in = bd.x[0][0] / 0.0254
    assert abs(x_in - ref['value']) / ref['value'] < ref['tolerance'], x_in


def run_constrained_cpu(sc, J, mass, kinds, Z, gravity, nsteps, callback, impl='oracle', **kw):
    """Time loop of a scene whose rows are bilateral constraints: step begin,
    the constraints' update (update_riglnk / update_fixdir), assembly, the
    solve with the constraint kinds, step end; callback(k, t, bd) after step k
    stops the loop by returning False. Returns the last step index."""
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    mpnt, base, gap, Zc = sc.mpnt.copy(), sc.base.copy(), sc.gap.copy(), np.array(Z, dtype=float)
    R = np.zeros(3 * sc.ncon)
    U = np.zeros(3 * sc.ncon)
    t = 0.0
    for k in range(1, nsteps + 1):
        ro.step_begin(bd, sc.step, gravity)
        ro.update_constraints(bd, kinds, sc.master, sc.slave, mpnt, sc.spnt, base, gap, Zc)
        cur = dataclasses.replace(sc, rot=np.array(bd.rot), x=np.array(bd.x), velo=np.array(bd.velo),
                                  velo0=np.array(bd.velo0), mpnt=mpnt, base=base, gap=gap)
        out = oracle.solve(oracle.assemble(cur), R, U, kinds=kinds, Z=Zc, impl=impl, **kw)
        R, U = out['R'], out['U']
        ro.step_end(bd, sc.step, sc.master, sc.slave, mpnt, sc.spnt, base, R.reshape(-1, 3))
        t += sc.step
        if callback(k, t, bd) is False:
            return k
    return nsteps


class PendulumPeriod:
    """The termination callback of tests/math-pendulum.py:21-38: the time of
    the fifth sign change of the ball's vertical velocity (velo[5]), counting
    the start, i.e. one full period from the horizontal."""

    def __init__(self):
        self.previous, self.howmany, self.period = 0.0, 0, None

    def __call__(self, k, t, bd):
        v = bd.velo[0][5]
        if v * self.previous <= 0:
            if self.howmany > 3:
                self.period = t
                return False
            self.howmany += 1
        self.previous = v
        return True


class PinnedBarSwing:
    """The callback of tests/pinned-bar.py:35-45: the angular velocity about
    y (velo[1]) when the mass centre's x (conf[9]) first reaches 0."""

    def __init__(self):
        self.omega = None

    def __call__(self, k, t, bd):
        if bd.x[0][0] <= 0:
            self.omega = bd.velo[0][1]
            return False
        return True


def pin(name):
    return json.load(open(os.path.join(HERE, 'golden', name)))


@pytest.mark.parametrize('impl', ['oracle', 'ref'])
def test_math_pendulum_period_cpu(impl):
    """The reference's tests/math-pendulum.py: a ball on a rigid link
    (RIGLNK to a fixed point) released from the horizontal under gravity pi^2,
    GAUSS_SEIDEL_SOLVER (1E-3, 1000, failure = 'EXIT'); the period within 1%
    of 2.36 s; the link length held to 1e-6."""
    if impl == 'ref' and not oracle.ref_available():
        pytest.skip('compiled reference solver not built')
    sc, J, mass, kinds, Z = scenes.math_pendulum()
    cb = PendulumPeriod()
    lengths = []

    def watch(k, t, bd):
        x = bd.x[0]
        lengths.append(math.sqrt(x[0] ** 2 + x[1] ** 2 + (x[2] - 1.0) ** 2))
        return cb(k, t, bd)
    run_constrained_cpu(sc, J, mass, kinds, Z, (0.0, 0.0, -scenes.MATH_PENDULUM_GRAVITY), 2600, watch, impl,
                        epsilon=1e-3, maxiter=1000, failure='EXIT')
    ref = pin('math_pendulum_ref.json')
    assert cb.period is not None and abs(cb.period - ref['value']) / ref['value'] < ref['tolerance'], cb.period
    assert np.abs(np.array(lengths) - 1.0).max() < 1e-6


@pytest.mark.parametrize('impl', ['oracle', 'ref'])
def test_pinned_bar_cpu(impl):
    """The reference's tests/pinned-bar.py: a bar hinged by two FIX_POINT
    constraints, released at 30 degrees, GAUSS_SEIDEL_SOLVER (1E-3, 1000,
    failure = 'EXIT'); the angular velocity about y as the mass centre passes
    x = 0 within 1% of 2.121 rad/s; the hinge points do not move."""
    if impl == 'ref' and not oracle.ref_available():
        pytest.skip('compiled reference solver not built')
    sc, J, mass, kinds, Z = scenes.pinned_bar()
    cb = PinnedBarSwing()
    drift = []

    def watch(k, t, bd):
        for p in sc.mpnt:
            q = ro.cur_point(bd, 0, [float(v) for v in p])
            drift.append(max(abs(q[i] - p[i]) for i in range(3)))
        return cb(k, t, bd)
    run_constrained_cpu(sc, J, mass, kinds, Z, (0.0, 0.0, -scenes.PINNED_BAR_GRAVITY), 500, watch, impl,
                        epsilon=1e-3, maxiter=1000, failure='EXIT')
    ref = pin('pinned_bar_ref.json')
    assert cb.omega is not None and abs(cb.omega - ref['value']) / ref['value'] < ref['tolerance'], cb.omega
    assert max(drift) < 1e-6, max(drift)


def double_pendulum_energy(bd):
    """Total energy as tests/double-pendulum.py:93-97 forms it: the kinetic
    energy plus m g max(z, 0) of both balls."""
    g = scenes.DOUBLE_PENDULUM_GRAVITY
    return sum(ro.kinetic_energy(bd, b) + bd.mass[b] * g * max(bd.x[b][2], 0.0) for b in range(2))


def double_pendulum_step_cpu(bd, sc, sph, cons, state, impl='oracle', **kw):
    """One step of the double pendulum on the CPU restatements: step begin,
    the links' update, contact update and detection (oracle_detect.c, carried
    R, U by pair key), the rows (contacts, then the links), assembly, solve
    with the kinds, step end. state: the carried detection, link frames and
    link reactions (updated in place). Returns (detection, rows, R, U, out)."""
    h = sc.step
    ro.step_begin(bd, h, (0.0, 0.0, -scenes.DOUBLE_PENDULUM_GRAVITY))
    cm, cb, cg, cZ = state['mpnt'], state['base'], state['gap'], state['Z']
    ro.update_constraints(bd, cons['kinds'], cons['master'], cons['slave'], cm, cons['spnt'], cb, cg, cZ)
    det = oracle.detect_spheres(sph['body'], sph['centre'], sph['radius'], sph['surface'], np.array(bd.rot),
                                np.array(bd.x), sc.x0, sc.obstacle, sph['material'], state['prev'],
                                convex=sph['convex'])
    n1, nc = det['key'].shape[0], cons['kinds'].shape[0]
    rows = dataclasses.replace(
        sc, rot=np.array(bd.rot), x=np.array(bd.x), velo=np.array(bd.velo), velo0=np.array(bd.velo0),
        master=np.concatenate([det['master'], cons['master']]).astype(np.int32),
        slave=np.concatenate([det['slave'], cons['slave']]).astype(np.int32),
        mpnt=np.concatenate([det['mpnt'].reshape(-1, 3), cm]), spnt=np.concatenate([det['spnt'].reshape(-1, 3),
                                                                                     cons['spnt']]),
        base=np.concatenate([det['base'].reshape(-1, 9), cb]), gap=np.concatenate([det['gap'], cg]),
        friction=np.concatenate([det['friction'], np.zeros(nc)]),
        restitution=np.concatenate([det['restitution'], np.zeros(nc)]), cohesion=np.zeros(n1 + nc))
    kinds = np.concatenate([np.zeros(n1, np.int32), cons['kinds']])
    Z = np.concatenate([np.zeros((n1, 4)), cZ])
    R0 = np.concatenate([det['R'].reshape(-1, 3), state['R']])
    U0 = np.concatenate([det['U'].reshape(-1, 3), state['U']])
    order = kw.pop('order', None)
    ld = oracle.assemble(rows)
    if order is None:
        order = np.arange(n1 + nc)
    out = oracle.solve(ld.permuted(order), R0[order].ravel(), U0[order].ravel(), kinds=kinds[order], Z=Z[order],
                       impl=impl, **kw)
    R = np.empty((n1 + nc, 3)); U = np.empty((n1 + nc, 3))
    R[order] = out['R'].reshape(-1, 3); U[order] = out['U'].reshape(-1, 3)
    state['R'], state['U'] = R[n1:], U[n1:]
    state['prev'] = dict(key=det['key'], slave_lo=det['slave_lo'], R=R[:n1], U=U[:n1])
    ro.step_end(bd, h, rows.master, rows.slave, rows.mpnt, rows.spnt, rows.base, R)
    return det, rows, R, U, out


def double_pendulum_state(cons):
    n = cons['kinds'].shape[0]
    return dict(prev=None, mpnt=np.array(cons['mpnt'], float).reshape(n, 3).copy(),
                base=np.array(cons['base'], float).reshape(n, 9).copy(), gap=np.zeros(n),
                Z=np.array(cons['Z'], float).reshape(n, 4).copy(), R=np.zeros((n, 3)), U=np.zeros((n, 3)))


def check_double_pendulum_pins(tot):
    """tests/double-pendulum.py:93-115: the total energy shifted by its last
    value, at the pinned indices, within 1e-3 relative to max(1, value)."""
    ref = pin('double_pendulum_ref.json')
    tot = np.asarray(tot) - tot[-1]
    for p in ref['pins']:
        err = abs(tot[p['index']] - p['value']) / max(1.0, p['value'])
        assert err <= ref['tolerance'], (p, tot[p['index']], err)


@pytest.mark.parametrize('impl', ['oracle', 'ref'])
def test_double_pendulum_energy_cpu(impl):
    """The reference's tests/double-pendulum.py: two balls on rigid links
    (RIGLNK to a fixed point and between the balls) strike a fixed box
    (sphere-convex contacts, restitution 0.1) over 2.5 s of 1 ms steps,
    GAUSS_SEIDEL_SOLVER (1E-3, 1000, failure = 'EXIT'); the total energy at
    the five pinned indices within the test's 1e-3."""
    if impl == 'ref' and not oracle.ref_available():
        pytest.skip('compiled reference solver not built')
    sc, sph, cons, J, mass = scenes.double_pendulum()
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    state = double_pendulum_state(cons)
    tot, hits = [double_pendulum_energy(bd)], 0
    for _ in range(2500):
        det, _, _, _, _ = double_pendulum_step_cpu(bd, sc, sph, cons, state, impl, epsilon=1e-3, maxiter=1000,
                                                   failure='EXIT')
        hits += int(det['key'].shape[0] > 0)
        tot.append(double_pendulum_energy(bd))
    assert hits > 5  # the balls strike the box
    check_double_pendulum_pins(tot)


def test_expmap_rotation():
    rng = np.random.default_rng(5)
    for scale in (1e-6, 1e-2, 0.17, 0.18, 1.0, 3.0):
        for _ in range(20):
            w = rng.normal(size=3)
            w *= scale / np.linalg.norm(w)
            R = np.array(ro.expmap(list(w))).reshape(3, 3).T  # row-major
            assert np.abs(R @ R.T - np.eye(3)).max() < 1e-14
            assert abs(np.linalg.det(R) - 1.0) < 1e-14
            a = np.linalg.norm(w)
            K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
            Rr = np.eye(3) + math.sin(a) / a * K + (1 - math.cos(a)) / a ** 2 * K @ K
            assert np.abs(R - Rr).max() < 1e-14
            assert np.allclose(R @ w, w, atol=1e-15 * max(1.0, a))  # the axis is fixed


def _spinning_body(scheme):
    J = np.diag([0.4, 0.7, 1.1]).reshape(9)
    jinv = np.linalg.inv(J.reshape(3, 3)).reshape(9)
    return ro.Bodies(rot=np.eye(3).reshape(1, 9), x=[[0.0, 0.0, 0.0]], velo=[[0.3, 2.0, -0.5, 0.0, 0.0, 0.0]],
                     J=J[None], jinv=jinv[None], mass=[2.0], minv=[0.5], x0=[[0.0, 0.0, 0.0]], obstacle=[0],
                     scheme=[scheme])


def test_neg_scheme_conserves_angular_momentum():
    """NEW2 (RIG_NEG) conserves the spatial angular momentum of a free body
    exactly up to rounding (bod.h:83)."""
    bd = _spinning_body(ro.SCH_RIG_NEG)
    L0 = np.array(ro.spatial_angular_momentum(bd, 0))
    for _ in range(2000):
        ro.step_begin(bd, 1e-3)
        ro.step_end(bd, 1e-3, [], [], np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
    L = np.array(ro.spatial_angular_momentum(bd, 0))
    assert np.linalg.norm(L - L0) / np.linalg.norm(L0) < 1e-12
    Rm = np.array(bd.rot[0]).reshape(3, 3)
    assert np.abs(Rm @ Rm.T - np.eye(3)).max() < 1e-12


def test_pos_scheme_energy_bounded():
    """NEW1 (RIG_POS): a free body's kinetic energy stays within a small
    drift over many steps."""
    bd = _spinning_body(ro.SCH_RIG_POS)
    e0 = ro.kinetic_energy(bd, 0)
    for _ in range(2000):
        ro.step_begin(bd, 1e-3)
        ro.step_end(bd, 1e-3, [], [], np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
    assert abs(ro.kinetic_energy(bd, 0) - e0) / e0 < 1e-3


def test_free_fall_is_exact():
    """Constant gravity: the half-step position updates integrate a constant
    acceleration exactly (x = x0 + v0 t + g t^2 / 2 up to rounding)."""
    bd = ro.Bodies(rot=np.eye(3).reshape(1, 9), x=[[0.0, 0.0, 1.0]], velo=[[0.0, 0.0, 0.0, 0.5, 0.0, 0.0]],
                   J=np.eye(3).reshape(1, 9), jinv=np.eye(3).reshape(1, 9), mass=[3.0], minv=[1.0 / 3.0],
                   x0=[[0.0, 0.0, 1.0]], obstacle=[0])
    h, n = 1e-3, 500
    for _ in range(n):
        ro.step_begin(bd, h, (0.0, 0.0, -9.81))
        ro.step_end(bd, h, [], [], np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
    t = n * h
    assert abs(bd.x[0][2] - (1.0 - 0.5 * 9.81 * t * t)) < 1e-12
    assert abs(bd.x[0][0] - 0.5 * t) < 1e-12
    assert abs(bd.velo[0][5] + 9.81 * t) < 1e-12


def test_constraint_force_is_HtR():
    """rig_constraints_force of one contact equals H^T R of the operator
    written out with numpy (spatial force on the master, opposite on the
    slave), H = [base^T R skew(X - X0)^T | base^T] (bod.c:216-228)."""
    rng = np.random.default_rng(7)
    Rm = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    Rm *= np.sign(np.linalg.det(Rm))
    base = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    X0 = rng.normal(size=3)
    X = rng.normal(size=3)
    r = rng.normal(size=3)
    H = np.array(ro.operator_H(list(Rm.T.reshape(9)), list(X0), list(base.T.reshape(9)), list(X)))
    H = H.reshape(6, 3).T  # 3 x 6
    A = X - X0
    S = np.array([[0, -A[2], A[1]], [A[2], 0, -A[0]], [-A[1], A[0], 0]])
    Href = np.hstack([base.T @ Rm @ S.T, base.T])
    assert np.allclose(H, Href, atol=1e-14)
    # one body on one contact: the end-of-step velocity change is h M^-1 H^T r
    bd = ro.Bodies(rot=Rm.T.reshape(1, 9), x=[X0], velo=[[0.0] * 6], J=np.eye(3).reshape(1, 9),
                   jinv=np.eye(3).reshape(1, 9), mass=[1.0], minv=[1.0], x0=[X0], obstacle=[0],
                   scheme=[ro.SCH_RIG_POS])
    ro.step_end(bd, 1.0, [0], [-1], X[None], X[None], base.T.reshape(1, 9), r[None])
    assert np.allclose(np.array(bd.velo[0]), Href.T @ r, atol=1e-13)


def test_expmap123_is_the_derivative_of_expmap():
    """EXPMAP123 (alg.h:1280-1382) restated: the derivatives of the rotation
    matrix with respect to each component, against central differences, in
    the Taylor branch and above ten degrees."""
    rng = np.random.default_rng(11)
    for scale in (1e-9, 1e-3, 0.1, 0.17, 0.5, 2.0):
        for _ in range(10):
            w = rng.normal(size=3)
            w *= scale / np.linalg.norm(w)
            D = ro.expmap123(list(w))
            eps = 1e-6 * max(scale, 1e-3)
            for k in range(3):
                e = np.zeros(3); e[k] = eps
                fd = (np.array(ro.expmap(list(w + e))) - np.array(ro.expmap(list(w - e)))) / (2 * eps)
                assert np.abs(np.array(D[k]) - fd).max() < 1e-6, (scale, k)


def test_dgesv3_solves():
    rng = np.random.default_rng(12)
    for _ in range(200):
        A = rng.normal(size=(3, 3)); b = rng.normal(size=3)
        a = list(A.T.reshape(9)); x = list(b)
        assert ro.dgesv3(a, x) == 0
        assert np.allclose(A @ np.array(x), b, rtol=1e-10, atol=1e-10)
    a = [0.0] * 9
    assert ro.dgesv3(a, [1.0, 2.0, 3.0]) == 1


def tumbling_body(scheme, flags=None):
    J = np.diag([1.0, 2.0, 3.0]).reshape(9)
    return ro.Bodies(np.eye(3).reshape(1, 9), np.zeros((1, 3)), np.array([[0.4, 3.0, 0.2, 0.0, 0.0, 0.0]]),
                     J.reshape(1, 9), np.linalg.inv(J.reshape(3, 3)).reshape(1, 9), [1.0], [1.0], np.zeros((1, 3)),
                     [0], scheme=[scheme], flags=flags)


def test_schemes_match_their_documented_conservation():
    """The three rigid schemes as bod.h:82-84 describes them, on a
    torque-free body tumbling about its unstable middle axis, 10,000 steps of
    0.03: NEW3 (RIG_IMP) keeps the spatial angular momentum R J W to rounding
    and its kinetic energy error bounded (no drift); NEW2 (RIG_NEG, the
    default) keeps the momentum and loses energy steadily; NEW1 (RIG_POS)
    gains energy and does not keep the momentum."""
    none = (np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
    out = {}
    for sch in (ro.SCH_RIG_IMP, ro.SCH_RIG_NEG, ro.SCH_RIG_POS):
        bd = tumbling_body(sch)
        L0 = np.array(ro.spatial_angular_momentum(bd, 0))
        E0 = ro.kinetic_energy(bd, 0)
        dE = []
        for k in range(10000):
            ro.step_begin(bd, 0.03)
            ro.step_end(bd, 0.03, [], [], *none)
            if k % 500 == 499:
                dE.append((ro.kinetic_energy(bd, 0) - E0) / E0)
        assert bd.failures == 0
        L = np.array(ro.spatial_angular_momentum(bd, 0))
        out[sch] = (np.linalg.norm(L - L0) / np.linalg.norm(L0), np.array(dE))
    dL, dE = out[ro.SCH_RIG_IMP]
    assert dL < 1e-12 and np.abs(dE).max() < 1e-3, (dL, dE)
    dL, dE = out[ro.SCH_RIG_NEG]
    assert dL < 1e-12 and dE[-1] < -5e-3 and np.all(np.diff(dE[::4]) < 0), (dL, dE)
    dL, dE = out[ro.SCH_RIG_POS]
    assert dL > 1e-3 and dE[-1] > 5e-3, (dL, dE)


def test_disable_rotation_keeps_orientation():
    """BODY_DISABLE_ROTATION (bod.c:1337-1340, 1450-1453): the rotation stays
    the identity whatever angular velocity the body carries."""
    none = (np.zeros((0, 3)), np.zeros((0, 3)), np.zeros((0, 9)), np.zeros((0, 3)))
    bd = tumbling_body(ro.SCH_RIG_NEG, flags=[ro.BODY_DISABLE_ROTATION])
    for _ in range(50):
        ro.step_begin(bd, 1e-3, (0.0, 0.0, -9.81))
        ro.step_end(bd, 1e-3, [], [], *none)
    assert bd.rot[0] == list(np.eye(3).reshape(9))
    assert bd.x[0][2] < 0.0
