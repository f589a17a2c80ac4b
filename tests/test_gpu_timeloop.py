"""Parity of whole device time loops with the CPU restatements, step after
step: the device integrator (BODY_Dynamic_Step_Begin / End), the assembly on
the device bodies (LOCDYN_Update_Begin), and the Gauss-Seidel solve
warm-started from the previous step, against oracle/rigid_oracle.py, the C
assembly oracle and the C solver oracle run in the device's row order. Body
states, reactions, velocities and iteration counts are bitwise equal at every
step (the half-step rotations stay in the exponential map's Taylor branch).
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
import rigid_oracle as ro
from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, scenes
from solfec_b200._lib import lib
from solfec_b200.dynamics import RIGID_DYNAMICS

pytestmark = pytest.mark.gpu
GRAVITY = (0.0, 0.0, -9.81)


def same_bits(a, b):
    a = np.asarray(a, float).ravel(); b = np.asarray(b, float).ravel()
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def inertia(sc):
    ob = sc.obstacle != 0  # walls: zero inverse inertia and mass (never accelerated)
    J = np.stack([np.eye(3).reshape(9) if o else np.linalg.inv(j.reshape(3, 3).T).T.reshape(9)
                  for j, o in zip(sc.jinv, ob)])
    mass = np.where(ob, 1.0, 1.0 / np.where(ob, 1.0, sc.minv))
    return J, mass


def time_loop_parity(sc, steps, J=None, mass=None, scheme=None, **kw):
    if J is None:
        J, mass = inertia(sc)
    h = float(sc.step)
    ldy = LOCDYN()
    ldy.update_begin(sc)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x, scheme)
    codes = None if scheme is None else [{'RIG_POS': 0, 'RIG_NEG': 1, 'RIG_IMP': 2}[scheme]] * sc.nbod
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle, codes)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    n = sc.ncon
    R = np.zeros((n, 3)); U = np.zeros((n, 3))
    Ro = np.zeros((n, 3)); Uo = np.zeros((n, 3))
    iters = []
    for k in range(steps):
        dyn.step_begin(h, GRAVITY)
        ro.step_begin(bd, h, GRAVITY)
        st = dyn.state()
        for key in ('rot', 'x', 'velo', 'velo0'):
            assert same_bits(st[key], np.array(getattr(bd, key))), (k, key)
        assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, int(sc.dynamic)) == 0
        ldy.set_state(R, U)
        gs.solve(ldy)
        R, U, _ = ldy.get_state()
        cur = dataclasses.replace(sc, rot=np.array(bd.rot), x=np.array(bd.x), velo=np.array(bd.velo),
                                  velo0=np.array(bd.velo0))
        ld = O.assemble(cur)
        order = ldy.order()
        res = O.solve(ld.permuted(order), R=Ro[order].ravel(), U=Uo[order].ravel(), **kw)
        Ro = np.empty((n, 3)); Uo = np.empty((n, 3))
        Ro[order] = res['R'].reshape(-1, 3); Uo[order] = res['U'].reshape(-1, 3)
        assert gs.iters == res['iters'], (k, gs.iters, res['iters'])
        assert same_bits(R, Ro) and same_bits(U, Uo), k
        iters.append(gs.iters)
        dyn.step_end(h)
        ro.step_end(bd, h, sc.master, sc.slave, sc.mpnt, sc.spnt, sc.base, Ro)
    st = dyn.state()
    for key in ('rot', 'x', 'velo'):
        assert same_bits(st[key], np.array(getattr(bd, key))), key
    ldy.close()
    return iters, bd


def test_config1_time_loop(scene_cache):
    """The 1000-sphere lattice of config 1 (FP64, epsilon = meritval = 1e-4),
    20 steps under gravity from its settled state."""
    iters, _ = time_loop_parity(scene_cache('spheres_lattice'), 20, epsilon=1e-4, maxiter=1000, meritval=1e-4)
    assert len(iters) == 20 and min(iters) >= 1


def test_hexahedra_time_loop(scene_cache):
    """A 12 x 12 x 4 hexahedra lattice (the bench's scene shape), 15 steps
    from rest with the bench's stopping rule (merit 1e-4 decides)."""
    iters, _ = time_loop_parity(scene_cache('hexahedra_lattice', nx=12, ny=12, nz=4), 15, epsilon=1.0,
                                maxiter=1000, meritval=1e-4)
    assert iters[0] > iters[-1]


def test_masonry_arch_threshold():
    """The reference's tests/arch.py on the device: 750 steps of each arch,
    GAUSS_SEIDEL_SOLVER (1E-4, 10000), bitwise with the CPU restatements at
    every step, and its pass criterion (tests/arch.py:132): thickness ratio
    0.1095 ends at rest (kinetic energy below 1e-4), 0.1094 collapses (above
    1e-3)."""
    energy = {}
    for ratio in (0.1095, 0.1094):
        sc, J, mass = scenes.masonry_arch(ratio)
        iters, bd = time_loop_parity(sc, 750, J=J, mass=mass, epsilon=1e-4, maxiter=10000)
        assert max(iters) > 1000  # the first steps of an arch at rest need thousands of sweeps
        energy[ratio] = sum(ro.kinetic_energy(bd, b) for b in range(bd.nbod) if not bd.obstacle[b])
    assert energy[0.1095] < 1e-4 and energy[0.1094] > 1e-3, energy


def test_detected_hexahedra_time_loop():
    """The config-3 bodies (8 x 8 x 3 perturbed cubes and their walls) with
    the contacts of the device's convex detection: 8 steps from rest, the
    assembly and solve bitwise with the CPU restatements at every step."""
    from solfec_b200.detect import detected_scene
    sc = scenes.hexahedra_lattice(nx=8, ny=8, nz=3)
    cv = scenes.hexahedra_geometry(nx=8, ny=8, nz=3)
    J, mass = inertia(sc)
    det, con = detected_scene(sc, cv, J, mass, material=(0.4, 0.0))
    assert det.ncon > 400 and np.median(det.gap) < 0.0
    iters, _ = time_loop_parity(det, 8, epsilon=1.0, maxiter=1000, meritval=1e-4)
    assert min(iters) >= 1


def test_masonry_arch_new3_time_loop():
    """The stable arch of tests/arch.py integrated with NEW3 (RIG_IMP, the
    Newton solve of bod.c:163-209) for 300 steps: device and CPU restatement
    bitwise at every step; the arch stays at rest."""
    sc, J, mass = scenes.masonry_arch(0.1095)
    iters, bd = time_loop_parity(sc, 300, J=J, mass=mass, scheme='RIG_IMP', epsilon=1e-4, maxiter=10000)
    assert bd.failures == 0
    assert sum(ro.kinetic_energy(bd, b) for b in range(bd.nbod) if not bd.obstacle[b]) < 1e-4


def constrained_loop_parity(sc, J, mass, kinds, Z, gravity, nsteps, callback, **kw):
    """Device time loop of a scene whose rows are bilateral constraints (step
    begin, b2dev_update_constraints, assembly, solve with the kinds, step
    end) against the CPU restatements, bitwise at every step; callback(k, t,
    bd) on the restated bodies after step k stops the loop with False."""
    h = float(sc.step)
    ldy = LOCDYN()
    ldy.update_begin(sc)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    ldy.set_kinds(kinds, Z)
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    mpnt, base, gap, Zc = sc.mpnt.copy(), sc.base.copy(), sc.gap.copy(), np.array(Z, dtype=float)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    n = sc.ncon
    R = np.zeros((n, 3)); U = np.zeros((n, 3))
    Ro = np.zeros((n, 3)); Uo = np.zeros((n, 3))
    t = 0.0
    for k in range(1, nsteps + 1):
        dyn.step_begin(h, gravity)
        ro.step_begin(bd, h, gravity)
        dyn.update_constraints()
        ro.update_constraints(bd, kinds, sc.master, sc.slave, mpnt, sc.spnt, base, gap, Zc)
        assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, int(sc.dynamic)) == 0
        ldy.set_state(R, U)
        gs.solve(ldy)
        R, U, _ = ldy.get_state()
        cur = dataclasses.replace(sc, rot=np.array(bd.rot), x=np.array(bd.x), velo=np.array(bd.velo),
                                  velo0=np.array(bd.velo0), mpnt=mpnt, base=base, gap=gap)
        order = ldy.order()
        res = O.solve(O.assemble(cur).permuted(order), R=Ro[order].ravel(), U=Uo[order].ravel(), kinds=kinds[order],
                      Z=Zc[order], **kw)
        Ro = np.empty((n, 3)); Uo = np.empty((n, 3))
        Ro[order] = res['R'].reshape(-1, 3); Uo[order] = res['U'].reshape(-1, 3)
        assert gs.iters == res['iters'], (k, gs.iters, res['iters'])
        assert same_bits(R, Ro) and same_bits(U, Uo), k
        dyn.step_end(h)
        ro.step_end(bd, h, sc.master, sc.slave, mpnt, sc.spnt, base, Ro)
        st = dyn.state()
        for key in ('rot', 'x', 'velo'):
            assert same_bits(st[key], np.array(getattr(bd, key))), (k, key)
        t += h
        if callback(k, t, bd) is False:
            break
    ldy.close()
    return k


def test_math_pendulum_period():
    """The reference's tests/math-pendulum.py on the device: a RIGLNK row to
    a fixed point, updated on the device every step, bitwise with the CPU
    restatements at every step of one full swing; the period within 1% of
    2.36 s (the pinned value of the test)."""
    from test_rigid_cpu import PendulumPeriod, pin
    sc, J, mass, kinds, Z = scenes.math_pendulum()
    cb = PendulumPeriod()
    constrained_loop_parity(sc, J, mass, kinds, Z, (0.0, 0.0, -scenes.MATH_PENDULUM_GRAVITY), 2600, cb,
                            epsilon=1e-3, maxiter=1000, failure='EXIT')
    ref = pin('math_pendulum_ref.json')
    assert cb.period is not None and abs(cb.period - ref['value']) / ref['value'] < ref['tolerance'], cb.period


def test_pinned_bar_swing():
    """The reference's tests/pinned-bar.py on the device: two FIXPNT rows
    hinge a bar, bitwise with the CPU restatements at every step; the angular
    velocity about y as the mass centre passes x = 0 within 1% of 2.121."""
    from test_rigid_cpu import PinnedBarSwing, pin
    sc, J, mass, kinds, Z = scenes.pinned_bar()
    cb = PinnedBarSwing()
    constrained_loop_parity(sc, J, mass, kinds, Z, (0.0, 0.0, -scenes.PINNED_BAR_GRAVITY), 500, cb,
                            epsilon=1e-3, maxiter=1000, failure='EXIT')
    ref = pin('pinned_bar_ref.json')
    assert cb.omega is not None and abs(cb.omega - ref['value']) / ref['value'] < ref['tolerance'], cb.omega


def test_math_pendulum_through_run_fixed_contacts():
    """The same pendulum through the time-loop API (dynamics.run_fixed_contacts
    with kinds), the period read from the device bodies."""
    from solfec_b200.dynamics import run_fixed_contacts
    from test_rigid_cpu import pin
    sc, J, mass, kinds, Z = scenes.math_pendulum()
    state = dict(previous=0.0, howmany=0, period=None)

    def cb(k, t, dyn, ldy):
        v = dyn.state()['velo'][0, 5]
        if v * state['previous'] <= 0:
            if state['howmany'] > 3:
                state['period'] = t
                return False
            state['howmany'] += 1
        state['previous'] = v
        return True
    gs = GAUSS_SEIDEL_SOLVER(1e-3, 1000, failure='EXIT')
    dyn, ldy = run_fixed_contacts(sc, gs, 2600, J, mass, gravity=(0.0, 0.0, -scenes.MATH_PENDULUM_GRAVITY),
                                  callback=cb, kinds=kinds, Z=Z)
    ldy.close()
    ref = pin('math_pendulum_ref.json')
    assert state['period'] is not None and abs(state['period'] - ref['value']) / ref['value'] < ref['tolerance']


def test_double_pendulum_energy():
    """The reference's tests/double-pendulum.py on the device: two RIGLNK rows
    kept across detections (b2dev_constraints_setup) after the sphere-box
    contacts of every step's detection, the links' frames refreshed on the
    device, 2500 steps; detection, reactions, iterations and bodies bitwise
    with the CPU restatements at every step, and the total energy at the
    test's five pinned indices within its 1e-3."""
    from solfec_b200.detect import SPHERES, bodies_only
    from test_rigid_cpu import (check_double_pendulum_pins, double_pendulum_energy, double_pendulum_state,
                                double_pendulum_step_cpu)
    sc, sph, cons, J, mass = scenes.double_pendulum()
    h = sc.step
    g = (0.0, 0.0, -scenes.DOUBLE_PENDULUM_GRAVITY)
    ldy = LOCDYN()
    ldy.update_begin(bodies_only(sc))
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    s = SPHERES(ldy, **sph)
    s.set_constraints(**cons)
    gs = GAUSS_SEIDEL_SOLVER(1e-3, 1000, failure='EXIT')
    bd = ro.Bodies(sc.rot, sc.x, sc.velo, J, sc.jinv, mass, sc.minv, sc.x0, sc.obstacle)
    state = double_pendulum_state(cons)
    tot, hits = [double_pendulum_energy(bd)], 0
    for k in range(2500):
        dyn.step_begin(h, g)
        nc, _ = s.detect()
        dyn.update_constraints()
        assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, 1) == 0
        s.carry_state()
        gs.solve(ldy)
        R, U, _ = ldy.get_state()
        det, _, Ro, Uo, out = double_pendulum_step_cpu(bd, sc, sph, cons, state, order=ldy.order(), epsilon=1e-3,
                                                       maxiter=1000, failure='EXIT')
        assert nc == det['key'].shape[0], k
        if nc:
            dev = s.contacts()
            for key in ('key', 'master', 'slave', 'mpnt', 'spnt', 'base', 'gap'):
                assert same_bits(dev[key], det[key]), (k, key)
            hits += 1
        assert gs.iters == out['iters'], (k, gs.iters, out['iters'])
        assert same_bits(R, Ro) and same_bits(U, Uo), k
        dyn.step_end(h)
        st = dyn.state()
        for key in ('rot', 'x', 'velo'):
            assert same_bits(st[key], np.array(getattr(bd, key))), (k, key)
        tot.append(double_pendulum_energy(bd))
    ldy.close()
    assert hits > 5
    check_double_pendulum_pins(tot)
