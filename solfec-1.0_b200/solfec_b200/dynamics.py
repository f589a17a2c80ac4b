"""Rigid-body time stepping on the device around the contact solve.

The reference advances every body with BODY_Dynamic_Step_Begin before the
local dynamics is assembled and with BODY_Dynamic_Step_End after the solve
(bod.c:1313-1493, called from the time loop in sol.c). RIGID_DYNAMICS runs
both on the GPU (csrc/b2_rigid.cuh) on the body arrays the assembly reads, so
a step is

    step_begin -> LOCDYN update (device bodies) -> GAUSS_SEIDEL solve -> step_end

without the bodies leaving the device. run_fixed_contacts keeps the uploaded
contacts (referential points, frames, gaps, materials) for every step, which is
exact for contacts that stay attached to the same material points, e.g. a
block sliding on a flat table; for spheres and convex obstacles,
detect.run_spheres detects and updates the contacts on the device every step.

Schemes: 'RIG_NEG' (NEW2, the reference's default), 'RIG_POS' (NEW1) and
'RIG_IMP' (NEW3). Bilateral constraints (FIXPNT, FIXDIR, VELODIR, VELODIR3,
RIGLNK) ride along as rows of the fixed set with their kinds: every step
updates their frames from the device bodies before the assembly, as
DOM_Update_Begin does (dom.c:3716-3732).
"""
from __future__ import annotations

import numpy as np

from ._lib import lib, ptr
from .solver import LOCDYN, _check

SCHEMES = {'RIG_POS': 0, 'RIG_NEG': 1, 'RIG_IMP': 2}
BODY_DISABLE_ROTATION = 0x0004  # bod.h:144


def _f64(a, n):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if a.shape[0] != n:
        raise ValueError('expected %d values, got %d' % (n, a.shape[0]))
    return a


class RIGID_DYNAMICS:
    """Device time integration of the bodies of a LOCDYN's uploaded scene.

    J: (nbod, 9) referential inertia (column-major); mass: (nbod,); x: (nbod, 3)
    current mass centres; scheme: None (all 'RIG_NEG') or one name per body
    ('RIG_POS' NEW1, 'RIG_NEG' NEW2, 'RIG_IMP' NEW3); disable_rotation: None
    or a boolean per body (BODY_DISABLE_ROTATION).
    """

    def __init__(self, ldy: LOCDYN, J, mass, x, scheme=None, disable_rotation=None):
        self.ldy = ldy
        self.nbod = int(np.asarray(mass).reshape(-1).shape[0])
        nb = self.nbod
        self._J = _f64(J, 9 * nb)
        self._mass = _f64(mass, nb)
        self._x = _f64(x, 3 * nb)
        sch = None
        if scheme is not None:
            names = [scheme] * nb if isinstance(scheme, str) else list(scheme)
            if len(names) != nb:
                raise ValueError('one scheme per body')
            for s in names:
                if s not in SCHEMES:
                    raise ValueError("scheme %r is not one of RIG_POS, RIG_NEG, RIG_IMP" % s)
            sch = np.array([SCHEMES[s] for s in names], dtype=np.int32)
        _check(lib().b2dev_rigid_setup(ldy.device_context, ptr(self._J), ptr(self._mass), ptr(self._x), ptr(sch), 0),
               'b2dev_rigid_setup')
        if disable_rotation is not None:
            flags = np.where(np.asarray(disable_rotation, bool).reshape(-1), BODY_DISABLE_ROTATION, 0).astype(np.int32)
            if flags.shape[0] != nb:
                raise ValueError('one disable_rotation flag per body')
            self._flags = flags
            _check(lib().b2dev_rigid_flags(ldy.device_context, ptr(flags), 0), 'b2dev_rigid_flags')

    def step_begin(self, step: float, gravity=(0.0, 0.0, 0.0), loads=None):
        """BODY_Dynamic_Step_Begin of every body. loads: None or (nbod, 9)
        linear force, spatial torque and referential torque of the point loads
        at time + step/2 (what rig_point_forces_accumulate sums)."""
        g = np.ascontiguousarray(gravity, dtype=np.float64).reshape(3)
        L = None if loads is None else _f64(loads, 9 * self.nbod)
        _check(lib().b2dev_rigid_step_begin(self.ldy.device_context, float(step), ptr(g), ptr(L), 0),
               'BODY_Dynamic_Step_Begin')

    def update_constraints(self):
        """The bilateral constraints' update of DOM_Update_Begin on the device
        bodies (RIGLNK frames, gaps and link vectors; FIXDIR with a slave body)."""
        _check(lib().b2dev_update_constraints(self.ldy.device_context), 'b2dev_update_constraints')

    def step_end(self, step: float):
        """BODY_Dynamic_Step_End of every body with the reactions of the last solve."""
        _check(lib().b2dev_rigid_step_end(self.ldy.device_context, float(step)), 'BODY_Dynamic_Step_End')

    def state(self) -> dict:
        nb = max(self.nbod, 1)
        rot, x, velo, velo0 = np.zeros(9 * nb), np.zeros(3 * nb), np.zeros(6 * nb), np.zeros(6 * nb)
        _check(lib().b2dev_rigid_get(self.ldy.device_context, ptr(rot), ptr(x), ptr(velo), ptr(velo0), 0),
               'b2dev_rigid_get')
        n = self.nbod
        return dict(rot=rot[:9 * n].reshape(n, 9), x=x[:3 * n].reshape(n, 3), velo=velo[:6 * n].reshape(n, 6),
                    velo0=velo0[:6 * n].reshape(n, 6))


def run_fixed_contacts(scene, gs, nsteps: int, J, mass, gravity=(0.0, 0.0, 0.0), loads=None, callback=None,
                       scheme=None, time: float = 0.0, ldy: LOCDYN = None, kinds=None, Z=None):
    """Time loop of a scene whose contacts stay as uploaded.

    Every step: bodies to t + h/2 and free velocities (device), the bilateral
    constraints' frames from the moved bodies (with kinds), local dynamics
    from the device bodies, GAUSS_SEIDEL solve warm-started from the previous
    reactions (the reference keeps con->R between steps), constraint reactions
    and the second half step (device). loads(t) -> (nbod, 9) or None is called
    with t = time + h/2 of each step; callback(k, time, dyn, ldy) after step k
    (k from 1), where a return value of False stops the loop. kinds, Z: the
    rows' constraint kinds and values as LOCDYN.set_kinds takes them (RIGLNK:
    Z[3] the link length; FIXDIR with a slave: Z[0..2] the master's
    referential direction). Returns (RIGID_DYNAMICS, LOCDYN).
    """
    if ldy is None:
        ldy = LOCDYN()
    ldy.update_begin(scene)  # upload of bodies and contacts (and a first assembly)
    dyn = RIGID_DYNAMICS(ldy, J, mass, scene.x, scheme)
    bilateral = kinds is not None and bool(np.any(np.asarray(kinds) != 0))
    if bilateral:
        ldy.set_kinds(kinds, Z)
    h = float(scene.step)
    R = np.zeros((scene.ncon, 3))
    U = np.zeros((scene.ncon, 3))
    t = float(time)
    for k in range(1, int(nsteps) + 1):
        dyn.step_begin(h, gravity, None if loads is None else loads(t + 0.5 * h))
        if bilateral:
            dyn.update_constraints()
        _check(lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, int(scene.dynamic)), 'LOCDYN_Update_Begin')
        ldy.set_state(R, U)
        gs.solve(ldy)
        R, U, _ = ldy.get_state()
        dyn.step_end(h)
        t += h
        if callback is not None and callback(k, t, dyn, ldy) is False:
            break
    return dyn, ldy
