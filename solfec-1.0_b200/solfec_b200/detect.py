"""Contact update and detection between spheres on the device.

In the reference every time step's DOM_Update_Begin (dom.c:3630-3790) moves the
bodies (BODY_Dynamic_Step_Begin), updates the existing contacts
(update_contact, dom.c:430-484), detects new ones over the AABB overlaps of the
shapes (overlap_create, dom.c:348-412, gobjcontact in goc.c) and sparsifies
them (sparsify_contacts, dom.c:2956-3054) before LOCDYN_Update_Begin assembles
the local dynamics. SPHERES does the contact part for sphere shapes of rigid
bodies on the GPU (csrc/b2_detect.cuh), on the device bodies a LOCDYN holds and
RIGID_DYNAMICS moves, so a time step of a sphere scene is

    step_begin -> detect -> LOCDYN update -> carry R, U -> GAUSS_SEIDEL solve -> step_end

with only the contact count crossing to the host. Contacts are listed by sphere
pair (i, j), i < j. Kept contacts carry their R and U from the last solve (the
reference keeps con->R and con->U), new ones start from zero.

Convex obstacles (box walls, say) collide with the spheres as the
reference's detect_convex_sphere does: the closest hull point by GJK
(gjk_convex_point), the convex as the slave, the material of the nearest face's
surface.

Convexes of different bodies collide with one another as the reference's
detect_convex_convex and update_convex_convex do (goc.c:280-306, 527-553): one
contact per pair at the area centre of the surface of the convexes'
intersection polytope (cvi.c, hul.c, tri.c, restated in csrc/b2_cvi.cuh), with
its normal, gap, area and surface pair. Pairs come from a sweep over the
convexes' eps-inflated boxes; the lower convex of a pair is the slave. A
scene of convex bodies alone is a SPHERES with no spheres (CONVEXES).
Sparsification follows CONTACT_SPARSIFY (sparsify).

Materials: a symmetric table (nsurf, nsurf, 2) of friction and restitution per
surface pair (SPSET_Find resolved by the caller). Cohesion is not supported:
the reference gives it only to contacts created at time zero and updates
cohesive contacts differently (dom.c:455-460).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from ._lib import lib, ptr
from .dynamics import RIGID_DYNAMICS
from .solver import LOCDYN, _check


def _i32(a, n):
    a = np.ascontiguousarray(a, dtype=np.int32).reshape(-1)
    if a.shape[0] != n:
        raise ValueError('expected %d values, got %d' % (n, a.shape[0]))
    return a


def _f64(a, n):
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if a.shape[0] != n:
        raise ValueError('expected %d values, got %d' % (n, a.shape[0]))
    return a


def material_table(material) -> np.ndarray:
    """(nsurf, nsurf, 2) friction and restitution from a table or from one
    (friction, restitution) pair for a single surface."""
    m = np.asarray(material, dtype=np.float64)
    if m.shape == (2,):
        m = m.reshape(1, 1, 2)
    if m.ndim != 3 or m.shape[0] != m.shape[1] or m.shape[2] != 2:
        raise ValueError('material: expected (nsurf, nsurf, 2) or (friction, restitution)')
    return np.ascontiguousarray(m)


class SPHERES:
    """Sphere shapes of the bodies of a LOCDYN's device scene.

    body: (nsph,) body of each sphere; centre: (nsph, 3) referential centres;
    radius: (nsph,); surface: (nsph,) surface ids (default 0); material: see
    material_table; convex: None or the keyword arguments of set_convexes
    (convex obstacles, detect_convex_sphere of goc.c:308-349). The LOCDYN's
    bodies need RIGID_DYNAMICS set up (mass centres) before the first detect().
    """

    def __init__(self, ldy: LOCDYN, body, centre, radius, surface=None, material=(0.0, 0.0), convex=None):
        self.ldy = ldy
        self.nsph = int(np.asarray(body).reshape(-1).shape[0])
        n = self.nsph
        self._body = _i32(body, n)
        self._centre = _f64(centre, 3 * n)
        self._radius = _f64(radius, n)
        self._surface = _i32(np.zeros(n) if surface is None else surface, n)
        self._mat = material_table(material)
        self.ncon = 0
        self.nnew = 0
        self.ncons = 0
        _check(lib().b2dev_spheres_setup(ldy.device_context, n, ptr(self._body), ptr(self._centre),
                                         ptr(self._radius), ptr(self._surface), int(self._mat.shape[0]),
                                         ptr(self._mat), 0), 'b2dev_spheres_setup')
        self.nconv = 0
        if convex is not None:
            self.set_convexes(**convex)

    def set_convexes(self, body, vptr, vert, fptr, fac, sptr, surf):
        """Convex obstacles the spheres collide with (b2dev_convexes_setup):
        per convex its body, referential vertices vert[vptr[c]:vptr[c+1]], faces
        fac[fptr[c]:fptr[c+1]] (per face its vertex count then vertex indices,
        counter-clockwise seen from outside) and surface ids surf[sptr[c]:sptr[c+1]]."""
        nc = int(np.asarray(body).reshape(-1).shape[0])
        vptr = _i32(vptr, nc + 1)
        sptr = _i32(sptr, nc + 1)
        fptr = _i32(fptr, nc + 1)
        self._cvx = [_i32(body, nc), vptr, _f64(vert, 3 * int(vptr[-1])), fptr, _i32(fac, int(fptr[-1])), sptr,
                     _i32(surf, int(sptr[-1]))]
        _check(lib().b2dev_convexes_setup(self.ldy.device_context, nc, *[ptr(a) for a in self._cvx]),
               'b2dev_convexes_setup')
        self.nconv = nc

    def set_constraints(self, kinds, master, slave, mpnt, spnt, base, Z):
        """Bilateral constraints kept across detections (b2dev_constraints_setup):
        per constraint its kind (1-5, dom.h:98), master and slave body (-1:
        none, spnt then a spatial point), referential points, base (column-major
        9) and Z (4; RIGLNK: Z[3] the link length). Every detect() lists them
        after its contacts; RIGID_DYNAMICS.update_constraints refreshes RIGLNK
        and two-body FIXDIR frames from the moved bodies."""
        n = int(np.asarray(kinds).reshape(-1).shape[0])
        self._cons = [_i32(kinds, n), _i32(master, n), _i32(slave, n), _f64(mpnt, 3 * n), _f64(spnt, 3 * n),
                      _f64(base, 9 * n), _f64(Z, 4 * n)]
        _check(lib().b2dev_constraints_setup(self.ldy.device_context, n, *[ptr(a) for a in self._cons]),
               'b2dev_constraints_setup')
        self.ncons = n

    def sparsify(self, threshold=0.01, minarea=0.0, mindist=1e-6):
        """CONTACT_SPARSIFY (lng.c:8875-8899) for the sparsification of new
        contacts (sparsify_contacts, dom.c:2956-3054)."""
        _check(lib().b2dev_contact_sparsify(self.ldy.device_context, float(threshold), float(minarea),
                                            float(mindist)), 'CONTACT_SPARSIFY')

    def exclude_bodies(self, pairs):
        """CONTACT_EXCLUDE_BODIES for each (body1, body2) of pairs (replaces earlier ones)."""
        p = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
        self._ex_bodies = p
        _check(lib().b2dev_exclude_bodies(self.ldy.device_context, int(p.shape[0]), ptr(p)),
               'CONTACT_EXCLUDE_BODIES')

    def exclude_surfaces(self, pairs):
        """CONTACT_EXCLUDE_SURFACES for each (surf1, surf2) of pairs (replaces earlier ones)."""
        p = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
        self._ex_surf = p
        _check(lib().b2dev_exclude_surfaces(self.ldy.device_context, int(p.shape[0]), ptr(p)),
               'CONTACT_EXCLUDE_SURFACES')

    def unphysical_penetration(self, depth):
        """UNPHYSICAL_PENETRATION: detection fails on a contact gap at or below -depth."""
        _check(lib().b2dev_unphysical_penetration(self.ldy.device_context, float(depth)), 'UNPHYSICAL_PENETRATION')

    def detect(self):
        """Update and detection of the contacts; returns (contacts, new contacts)."""
        nc, nn = C.c_int(0), C.c_int(0)
        _check(lib().b2dev_detect_spheres(self.ldy.device_context, C.byref(nc), C.byref(nn)), 'contact detection')
        self.ncon, self.nnew = int(nc.value), int(nn.value)
        return self.ncon, self.nnew

    def carry_state(self):
        """Solver state = the carried R and U (after the local dynamics update)."""
        _check(lib().b2dev_detect_carry_state(self.ldy.device_context), 'b2dev_detect_carry_state')

    def contacts(self) -> dict:
        n = self.ncon
        m = max(n, 1)
        out = dict(master=np.zeros(m, np.int32), slave=np.zeros(m, np.int32), point=np.zeros((m, 3)),
                   mpnt=np.zeros((m, 3)), spnt=np.zeros((m, 3)), base=np.zeros((m, 9)), gap=np.zeros(m),
                   friction=np.zeros(m), restitution=np.zeros(m), key=np.zeros(m, np.int64),
                   slave_lo=np.zeros(m, np.int32), isnew=np.zeros(m, np.int32), R=np.zeros((m, 3)),
                   U=np.zeros((m, 3)))
        names = ['master', 'slave', 'point', 'mpnt', 'spnt', 'base', 'gap', 'friction', 'restitution', 'key',
                 'slave_lo', 'isnew', 'R', 'U']
        _check(lib().b2dev_get_contacts(self.ldy.device_context, *[ptr(out[k]) for k in names], 0),
               'b2dev_get_contacts')
        out['area'] = np.zeros(m)
        if n > 0:
            _check(lib().b2dev_get_contact_area(self.ldy.device_context, ptr(out['area']), 0),
                   'b2dev_get_contact_area')
        return {k: v[:n] for k, v in out.items()}

    def centres(self) -> np.ndarray:
        cur = np.zeros((max(self.nsph, 1), 3))
        _check(lib().b2dev_sphere_centres(self.ldy.device_context, ptr(cur), 0), 'b2dev_sphere_centres')
        return cur[:self.nsph]


def CONVEXES(ldy: LOCDYN, convex: dict, material=(0.0, 0.0)) -> SPHERES:
    """Convex shapes of the bodies of a LOCDYN's device scene, no spheres:
    convex = the keyword arguments of SPHERES.set_convexes."""
    e = np.zeros(0)
    return SPHERES(ldy, np.zeros(0, np.int32), np.zeros((0, 3)), e, material=material, convex=convex)


def detected_scene(scene, convex: dict, J, mass, material=(0.0, 0.0), sparsify=None):
    """The scene's bodies with the contacts of one device detection of their
    convexes (the contact part of DOM_Update_Begin at the scene's state):
    master, slave, referential points, local bases, gaps and materials of the
    detected contacts, cohesion 0. Returns (scene, contacts dict with areas)."""
    ldy = LOCDYN()
    try:
        ldy.update_begin(bodies_only(scene))
        RIGID_DYNAMICS(ldy, J, mass, scene.x)
        det = CONVEXES(ldy, convex, material)
        if sparsify:
            det.sparsify(**sparsify)
        det.detect()
        con = det.contacts()
    finally:
        ldy.close()
    n = con['key'].shape[0]
    out = dataclasses.replace(scene, master=con['master'].astype(np.int32), slave=con['slave'].astype(np.int32),
                              mpnt=con['mpnt'], spnt=con['spnt'], base=con['base'], gap=con['gap'],
                              friction=con['friction'], restitution=con['restitution'], cohesion=np.zeros(n))
    return out, con


def bodies_only(scene):
    """The scene's bodies with no contacts (what detection starts from)."""
    e = np.zeros(0)
    return dataclasses.replace(scene, master=np.zeros(0, np.int32), slave=np.zeros(0, np.int32),
                               mpnt=np.zeros((0, 3)), spnt=np.zeros((0, 3)), base=np.zeros((0, 9)), gap=e,
                               friction=e, restitution=e, cohesion=e)


def run_spheres(scene, spheres: dict, gs, nsteps: int, J, mass, gravity=(0.0, 0.0, 0.0), callback=None,
                scheme=None, ldy: LOCDYN = None, constraints: dict = None):
    """Time loop of a sphere scene with contact detection on the device.

    scene: bodies (its contacts are ignored); spheres: keyword arguments of
    SPHERES (body, centre, radius, surface, material, convex); constraints:
    None or the keyword arguments of SPHERES.set_constraints. Every step:
    bodies to t + h/2 and free velocities, contact update and detection, the
    constraints' frames, local dynamics, R and U carried over, GAUSS_SEIDEL
    solve, reactions and second half step. callback(k, dyn, sph, ldy) after
    step k (from 1); False stops the loop. Returns (RIGID_DYNAMICS, SPHERES,
    LOCDYN)."""
    if ldy is None:
        ldy = LOCDYN()
    ldy.update_begin(bodies_only(scene))
    dyn = RIGID_DYNAMICS(ldy, J, mass, scene.x, scheme)
    sph = SPHERES(ldy, **spheres)
    if constraints is not None:
        sph.set_constraints(**constraints)
    h = float(scene.step)
    for k in range(1, int(nsteps) + 1):
        dyn.step_begin(h, gravity)
        nc, _ = sph.detect()
        if sph.ncons > 0:
            dyn.update_constraints()
        if nc + sph.ncons > 0:
            _check(lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, int(scene.dynamic)),
                   'LOCDYN_Update_Begin')
            sph.carry_state()
            gs.solve(ldy)
        dyn.step_end(h)
        if callback is not None and callback(k, dyn, sph, ldy) is False:
            break
    return dyn, sph, ldy
