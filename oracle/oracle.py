"""oracle.py -- TEST INFRASTRUCTURE. Not part of the product.

ctypes binding of the CPU oracle (lib/liboracle.so, the C restatement) and of
the reference's own solver compiled from its sources (_ref/libref_bgs.so).
Only tests/, __graft_entry__.smoke() and the cpu_baseline leg of bench.py
import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}

DS = {'PROJECTED_GRADIENT': 0, 'DE_SAXCE_FENG': 1, 'SEMISMOOTH_NEWTON': 2, 'PROJECTED_NEWTON': 3}
FAIL = {'CONTINUE': 0, 'EXIT': 1, 'CALLBACK': 2}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags='C_CONTIGUOUS')
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags='C_CONTIGUOUS')


def build():
    """Compile the restatement and, where the reference tree is present, the
    reference solver (oracle/Makefile)."""
    subprocess.run(['make', '-s', '-C', HERE], check=True)


def _load(name):
    if name in _LIBS:
        return _LIBS[name]
    path = os.path.join(HERE, {'oracle': 'lib/liboracle.so', 'ref': '_ref/libref_bgs.so',
                               'geo': '_ref/libref_geo.so'}[name])
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    if name == 'geo':
        lib.ref_gobj_sphere_sphere.restype = C.c_int
        lib.ref_gobj_sphere_sphere.argtypes = [C.c_int, _dp, C.c_double, C.c_int, _dp, C.c_double, C.c_int,
                                               _dp, _dp, _dp, _dp, _ip]
        lib.ref_gobj_convex_convex.restype = C.c_int
        lib.ref_gobj_convex_convex.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _ip, _ip, C.c_int, _dp, C.c_int, _ip,
                                               _ip, _dp, _dp, _dp, _dp, _dp, _ip]
        lib.ref_detect_spheres_hybrid.restype = C.c_longlong
        lib.ref_detect_spheres_hybrid.argtypes = [C.c_int, _dp, _dp, _ip, C.c_void_p, C.c_longlong]
        lib.ref_gobj_convex_sphere.restype = C.c_int
        lib.ref_gobj_convex_sphere.argtypes = [C.c_int, C.c_int, C.c_int, _dp, C.c_int, _ip, _ip, _dp, C.c_double,
                                               C.c_int, _dp, _dp, _dp, _dp, _ip]
        _LIBS[name] = lib
        return lib
    solve = lib.orc_gs_solve if name == 'oracle' else lib.ref_gs_solve
    solve.restype = C.c_int
    solve.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                      _dp, _dp, _dp, C.c_double, C.c_int, C.c_double,
                      C.c_double, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                      C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double), _dp, _dp, C.POINTER(C.c_int)]
    if name == 'oracle':
        lib.orc_count_blocks.restype = C.c_int64
        lib.orc_count_blocks.argtypes = [C.c_int, _ip, C.c_int, _ip, _ip, _ip]
        lib.orc_assemble.restype = C.c_int
        lib.orc_assemble.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _ip, C.c_int, _ip, _ip, _dp, _dp, _dp,
                                     C.c_double, _dp, _dp, _dp, _dp, _dp, C.POINTER(C.c_double), _ip, _ip, _ip, _dp]
        lib.orc_colour.restype = C.c_int
        lib.orc_colour.argtypes = [C.c_int, _ip, _ip, C.c_uint64, C.c_int, _ip]
        lib.orc_colour_ordered.restype = C.c_int
        lib.orc_colour_ordered.argtypes = [C.c_int, _ip, _ip, _ip, C.c_int, _ip]
        lib.orc_jp_priority.restype = C.c_uint64
        lib.orc_jp_priority.argtypes = [C.c_uint64, C.c_int]
        lib.orc_merit.restype = C.c_double
        lib.orc_merit.argtypes = [C.c_int, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp,
                                  C.c_double, C.c_int, C.c_double]
    _LIBS[name] = lib
    return lib


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, '_ref/libref_bgs.so'))


class LocalDynamics:
    """Flat local dynamics (the LOCDYN content the solver reads): rows in list
    order with W, A, rho, B, V and contact parameters, plus per-row
    off-diagonal blocks (adjptr/adjcol/Woff)."""

    def __init__(self, W, A, rho, B, V, gap, friction, restitution, cohesion, adjptr, adjcol, Woff,
                 free_energy, step, dynamic=1, adjbod=None):
        c = np.ascontiguousarray
        self.W, self.A, self.rho, self.B, self.V = c(W, float), c(A, float), c(rho, float), c(B, float), c(V, float)
        self.gap, self.friction = c(gap, float), c(friction, float)
        self.restitution, self.cohesion = c(restitution, float), c(cohesion, float)
        self.adjptr, self.adjcol, self.Woff = c(adjptr, np.int32), c(adjcol, np.int32), c(Woff, float)
        self.adjbod = None if adjbod is None else c(adjbod, np.int32)
        self.free_energy, self.step, self.dynamic = float(free_energy), float(step), int(dynamic)

    @property
    def n(self):
        return int(self.rho.shape[0])

    @property
    def nblocks(self):
        return int(self.adjptr[-1])

    def permuted(self, order):
        """Rows re-listed in the given order (order[p] = old row at position p),
        block columns renumbered, each row's blocks kept in their order."""
        order = np.asarray(order, np.int64)
        inv = np.empty_like(order); inv[order] = np.arange(order.size)
        deg = np.diff(self.adjptr)[order]
        ptr = np.zeros(order.size + 1, np.int64); np.cumsum(deg, out=ptr[1:])
        src = np.concatenate([np.arange(self.adjptr[i], self.adjptr[i + 1]) for i in order]) if order.size else np.zeros(0, np.int64)
        src = src.astype(np.int64)
        rows = lambda a, w: a.reshape(-1, w)[order].reshape(-1)  # noqa: E731
        return LocalDynamics(rows(self.W, 9), rows(self.A, 9), self.rho[order], rows(self.B, 3), rows(self.V, 3),
                             self.gap[order], self.friction[order], self.restitution[order], self.cohesion[order],
                             ptr.astype(np.int32), inv[self.adjcol[src]].astype(np.int32),
                             self.Woff.reshape(-1, 9)[src].reshape(-1), self.free_energy, self.step, self.dynamic,
                             None if self.adjbod is None else self.adjbod[src])


def assemble(scene) -> LocalDynamics:
    """Oracle assembly of a scenes.Scene (restated LOCDYN_Update_Begin)."""
    lib = _load('oracle')
    n = scene.ncon
    adjptr = np.zeros(n + 1, np.int32)
    nblk = lib.orc_count_blocks(scene.nbod, scene.obstacle, n, scene.master, scene.slave, adjptr)
    W = np.zeros(9 * n); A = np.zeros(9 * n); rho = np.zeros(n); B = np.zeros(3 * n); V = np.zeros(3 * n)
    adjcol = np.zeros(max(nblk, 1), np.int32); adjbod = np.zeros(max(nblk, 1), np.int32)
    Woff = np.zeros(9 * max(nblk, 1))
    fe = C.c_double(0.0)
    rc = lib.orc_assemble(scene.nbod, scene.rot.ravel(), scene.x0.ravel(), scene.jinv.ravel(), scene.minv,
                          scene.velo.ravel(), scene.velo0.ravel(), scene.obstacle, n, scene.master, scene.slave,
                          scene.mpnt.ravel(), scene.spnt.ravel(), scene.base.ravel(), scene.step,
                          W, A, rho, B, V, C.byref(fe), adjptr, adjcol, adjbod, Woff)
    if rc != 0:
        raise ValueError('oracle assembly rejected the scene (rc=%d)' % rc)
    return LocalDynamics(W, A, rho, B, V, scene.gap, scene.friction, scene.restitution, scene.cohesion,
                         adjptr, adjcol[:nblk], Woff[:9 * nblk], fe.value, scene.step, scene.dynamic, adjbod[:nblk])


def colour(ld: LocalDynamics, seed=None, maxcolours: int = 256):
    """Greedy colouring in decreasing Jones-Plassmann priority (seeded) order,
    or in list order when seed is None (the device's default mode)."""
    lib = _load('oracle')
    col = np.zeros(ld.n, np.int32)
    adjcol = ld.adjcol if ld.nblocks else np.zeros(1, np.int32)
    if seed is None:
        order = np.arange(max(ld.n, 1), dtype=np.int32)
        nc = lib.orc_colour_ordered(ld.n, ld.adjptr, adjcol, order, maxcolours, col)
    else:
        nc = lib.orc_colour(ld.n, ld.adjptr, adjcol, seed, maxcolours, col)
    return nc, col


def colour_order(col):
    """Rows sorted by (colour, row index): the processing order of a
    colour-by-colour sweep."""
    return np.lexsort((np.arange(col.size), col)).astype(np.int64)


def solve(ld: LocalDynamics, R=None, U=None, epsilon=1e-4, maxiter=1000, meritval=1.0, failure='CONTINUE',
          diagepsilon=None, diagmaxiter=None, diagsolver='SEMISMOOTH_NEWTON', reverse=False, impl='oracle',
          kinds=None, Z=None):
    """Run the restated (impl='oracle') or the compiled reference
    (impl='ref') Gauss-Seidel solve on ld in list order. Defaults of
    diagepsilon / diagmaxiter follow lng.c:4335-4342. kinds: None (all
    contacts) or a constraint kind per row (dom.h:98), with Z[n][4] (VELODIR
    value, VELODIR3 values, RIGLNK local link vector and length)."""
    if diagepsilon is None:
        diagepsilon = max(2.220446049250313e-16, 0.01 * min(epsilon, min(meritval, 1e-4)))
    if diagmaxiter is None:
        diagmaxiter = max(100, maxiter // 100)
    lib = _load(impl)
    fn = lib.orc_gs_solve if impl == 'oracle' else lib.ref_gs_solve
    n = ld.n
    R = np.zeros(3 * n) if R is None else np.ascontiguousarray(R, float).copy().reshape(-1)
    U = np.zeros(3 * n) if U is None else np.ascontiguousarray(U, float).copy().reshape(-1)
    conmerit = np.zeros(max(n, 1))
    rer = np.zeros(max(maxiter, 1)); mer = np.zeros(max(maxiter, 1))
    iters, err, ncb = C.c_int(0), C.c_int(0), C.c_int(0)
    merit = C.c_double(0.0)
    adjcol = ld.adjcol if ld.nblocks else np.zeros(1, np.int32)
    Woff = ld.Woff if ld.nblocks else np.zeros(9)
    setk = lib.orc_gs_set_kinds if impl == 'oracle' else lib.ref_gs_set_kinds
    setk.restype = None
    setk.argtypes = [C.c_void_p, C.c_void_p]
    if kinds is not None:
        kinds = np.ascontiguousarray(kinds, dtype=np.int32)
        Zk = np.ascontiguousarray(np.zeros((n, 4)) if Z is None else Z, dtype=np.float64).reshape(n, 4)
        setk(kinds.ctypes.data, Zk.ctypes.data)
    try:
        thrown = _gs_call(fn, n, ld, adjcol, Woff, R, U, conmerit, epsilon, maxiter, meritval, failure, diagepsilon,
                          diagmaxiter, diagsolver, reverse, iters, err, merit, rer, mer, ncb)
    finally:
        setk(None, None)
    k = iters.value
    return dict(R=R, U=U, conmerit=conmerit[:n], iters=k, error=err.value, merit=merit.value,
                rerhist=rer[:k].copy(), merhist=mer[:k].copy(), thrown=thrown, ncallbacks=ncb.value)


def _gs_call(fn, n, ld, adjcol, Woff, R, U, conmerit, epsilon, maxiter, meritval, failure, diagepsilon, diagmaxiter,
             diagsolver, reverse, iters, err, merit, rer, mer, ncb):
    return fn(n, ld.adjptr, adjcol, Woff, ld.W if n else np.zeros(9), ld.A if n else np.zeros(9),
                ld.rho if n else np.zeros(1), ld.B if n else np.zeros(3), ld.V if n else np.zeros(3),
                ld.gap if n else np.zeros(1), ld.friction if n else np.zeros(1),
                ld.restitution if n else np.zeros(1), ld.cohesion if n else np.zeros(1),
                R if n else np.zeros(3), U if n else np.zeros(3), conmerit, ld.free_energy, ld.dynamic, ld.step,
                epsilon, maxiter, meritval, FAIL[failure], diagepsilon, diagmaxiter, DS[diagsolver], int(reverse),
                C.byref(iters), C.byref(err), C.byref(merit), rer, mer, C.byref(ncb))


def merit(ld: LocalDynamics, R):
    lib = _load('oracle')
    U = np.zeros(3 * ld.n); cm = np.zeros(max(ld.n, 1))
    m = lib.orc_merit(ld.n, ld.adjptr, ld.adjcol if ld.nblocks else np.zeros(1, np.int32),
                      ld.Woff if ld.nblocks else np.zeros(9), ld.W, ld.A, ld.B, ld.V, ld.gap, ld.friction,
                      ld.restitution, ld.cohesion, np.ascontiguousarray(R, float).reshape(-1), U, cm,
                      ld.free_energy, ld.dynamic, ld.step)
    return m, U, cm[:ld.n]


# ---------------------------------------------------------------- sphere contact detection

_lp = np.ctypeslib.ndpointer(dtype=np.int64, flags='C_CONTIGUOUS')


def _detect_sigs(lib):
    if getattr(lib, '_detect_ready', False):
        return
    lib.orc_gjk_sphere_sphere.restype = C.c_double
    lib.orc_gjk_sphere_sphere.argtypes = [_dp, C.c_double, _dp, C.c_double, _dp, _dp]
    lib.orc_localbase.restype = None
    lib.orc_localbase.argtypes = [_dp, _dp]
    lib.orc_sphere_centres.restype = None
    lib.orc_sphere_centres.argtypes = [C.c_int, _ip, _dp, _dp, _dp, _dp, _dp]
    lib.orc_ref_points.restype = None
    lib.orc_ref_points.argtypes = [C.c_int, _ip, _dp, _dp, _dp, _dp, _dp]
    lib.orc_detect_spheres.restype = C.c_int
    lib.orc_detect_spheres.argtypes = ([C.c_int, _ip, _dp, _dp, _ip, C.c_int, _dp, _dp, _dp, _ip, C.c_int, _dp,
                                        C.c_int, _lp, _ip, _dp, _dp, C.c_int,
                                        _lp, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip])
    lib.orc_gjk_convex_point.restype = C.c_double
    lib.orc_gjk_convex_point.argtypes = [_dp, C.c_int, _dp, _dp]
    lib.orc_gjk_polytopes.restype = C.c_double
    lib.orc_gjk_polytopes.argtypes = [_dp, C.c_int, _dp, C.c_int, _dp, _dp]
    lib.orc_convex_planes.restype = None
    lib.orc_convex_planes.argtypes = [C.c_int, _ip, _dp, _dp]
    lib.orc_detect.restype = C.c_int
    lib.orc_detect.argtypes = ([C.c_int, _ip, _dp, _dp, _ip, C.c_int, _ip, _ip, _dp, _ip, _ip, _ip, _ip,
                                C.c_int, _dp, _dp, _dp, _ip, C.c_int, _dp,
                                C.c_int, _lp, _ip, _dp, _dp, C.c_int,
                                _lp, _ip, _ip, _ip, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _ip])
    lib._detect_ready = True


def gjk_sphere_sphere(a, ra, b, rb, which='oracle'):
    """(gap, p, q) of gjk_sphere_sphere: the restatement, or the reference's
    gjk.c compiled into _ref (which='ref')."""
    lib = _load(which)
    f = lib.orc_gjk_sphere_sphere if which == 'oracle' else lib.gjk_sphere_sphere
    f.restype = C.c_double
    f.argtypes = [_dp, C.c_double, _dp, C.c_double, _dp, _dp]
    p, q = np.zeros(3), np.zeros(3)
    g = f(np.ascontiguousarray(a, dtype=np.float64), float(ra), np.ascontiguousarray(b, dtype=np.float64),
          float(rb), p, q)
    return g, p, q


def gjk_convex_point(a, p, which='oracle'):
    """(distance, nearest hull point) of gjk_convex_point: the restatement, or
    the reference's gjk.c compiled into _ref (which='ref')."""
    lib = _load(which)
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    if which == 'oracle':
        _detect_sigs(lib)
        f = lib.orc_gjk_convex_point
    else:
        f = lib.gjk_convex_point
        f.restype = C.c_double
        f.argtypes = [_dp, C.c_int, _dp, _dp]
    q = np.zeros(3)
    d = f(a, a.shape[0] // 3, np.ascontiguousarray(p, dtype=np.float64), q)
    return d, q


def gjk_polytopes(a, b, which='oracle'):
    """(distance, p, q) of gjk for two vertex sets: the restatement, or the
    reference's gjk.c compiled into _ref (which='ref')."""
    lib = _load(which)
    a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    b = np.ascontiguousarray(b, dtype=np.float64).reshape(-1)
    if which == 'oracle':
        _detect_sigs(lib)
        f = lib.orc_gjk_polytopes
    else:
        f = lib.gjk
        f.restype = C.c_double
        f.argtypes = [_dp, C.c_int, _dp, C.c_int, _dp, _dp]
    p, q = np.zeros(3), np.zeros(3)
    d = f(a, a.shape[0] // 3, b, b.shape[0] // 3, p, q)
    return d, p, q


def convex_planes(fac, cur):
    """computeplanes: (nfac, 6) unit normal and first vertex per face."""
    lib = _load('oracle')
    _detect_sigs(lib)
    fac = np.ascontiguousarray(fac, dtype=np.int32)
    nf, m = 0, 0
    while m < fac.shape[0]:
        nf += 1
        m += fac[m] + 1
    pla = np.zeros((max(nf, 1), 6))
    lib.orc_convex_planes(nf, fac, np.ascontiguousarray(cur, dtype=np.float64).reshape(-1), pla)
    return pla[:nf]


def localbase(n):
    lib = _load('oracle')
    _detect_sigs(lib)
    loc = np.zeros(9)
    lib.orc_localbase(np.ascontiguousarray(n, dtype=np.float64), loc)
    return loc


def sphere_centres(sbody, sref, rot, x, x0):
    lib = _load('oracle')
    _detect_sigs(lib)
    sbody = np.ascontiguousarray(sbody, dtype=np.int32)
    cur = np.zeros((sbody.shape[0], 3))
    lib.orc_sphere_centres(sbody.shape[0], sbody, np.ascontiguousarray(sref, dtype=np.float64).reshape(-1),
                           np.ascontiguousarray(rot, dtype=np.float64).reshape(-1),
                           np.ascontiguousarray(x, dtype=np.float64).reshape(-1),
                           np.ascontiguousarray(x0, dtype=np.float64).reshape(-1), cur)
    return cur


def ref_points(body, pts, rot, x, x0):
    """BODY_Ref_Point (bod.c:1736-1750) of spatial points pts[k] on bodies body[k]."""
    lib = _load('oracle')
    _detect_sigs(lib)
    body = np.ascontiguousarray(body, dtype=np.int32)
    out = np.zeros((body.shape[0], 3))
    lib.orc_ref_points(body.shape[0], body, np.ascontiguousarray(pts, dtype=np.float64).reshape(-1),
                       np.ascontiguousarray(rot, dtype=np.float64).reshape(-1),
                       np.ascontiguousarray(x, dtype=np.float64).reshape(-1),
                       np.ascontiguousarray(x0, dtype=np.float64).reshape(-1), out)
    return out


def detect_spheres(sbody, sref, radius, surface, rot, x, x0, obstacle, material, prev=None, convex=None):
    """The contact part of DOM_Update_Begin for spheres (oracle_detect.c).
    material: (nsurf, nsurf, 2) friction, restitution. prev: None or a dict
    returned by an earlier call, with 'R' and 'U' set to the reactions and
    velocities to carry over. Returns a dict of contact arrays in pair order."""
    lib = _load('oracle')
    _detect_sigs(lib)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32).reshape(-1)
    sbody, surface, obstacle = i32(sbody), i32(surface), i32(obstacle)
    sref, radius, rot, x, x0 = f64(sref), f64(radius), f64(rot), f64(x), f64(x0)
    mat = np.asarray(material, dtype=np.float64)
    nsurf = mat.shape[0]
    mat = f64(mat)
    nsph, nbod = sbody.shape[0], obstacle.shape[0]
    if prev is None:
        pk, ps, pR, pU, npv = np.zeros(1, np.int64), np.zeros(1, np.int32), np.zeros(3), np.zeros(3), 0
    else:
        npv = prev['key'].shape[0]
        pk = np.ascontiguousarray(prev['key'], dtype=np.int64)
        ps = i32(prev['slave_lo'])
        pR = f64(prev.get('R', np.zeros((npv, 3))))
        pU = f64(prev.get('U', np.zeros((npv, 3))))
        if npv == 0:
            pk, ps, pR, pU = np.zeros(1, np.int64), np.zeros(1, np.int32), np.zeros(3), np.zeros(3)

    if convex is not None:
        cb = i32(convex['body'])
        cvptr, cvert = i32(convex['vptr']), f64(convex['vert'])
        cfptr, fac = i32(convex['fptr']), i32(convex['fac'])
        csptr, csurf = i32(convex['sptr']), i32(convex['surf'])
        nconv = cb.shape[0]
    else:
        nconv = 0
        cb, cvptr, cfptr, csptr = (np.zeros(1, np.int32) for _ in range(4))
        cvert, fac, csurf = np.zeros(3), np.zeros(1, np.int32), np.zeros(1, np.int32)

    def run(cap):
        c1 = max(cap, 1)
        out = dict(key=np.zeros(c1, np.int64), slave_lo=np.zeros(c1, np.int32), master=np.zeros(c1, np.int32),
                   slave=np.zeros(c1, np.int32), point=np.zeros((c1, 3)), mpnt=np.zeros((c1, 3)),
                   spnt=np.zeros((c1, 3)), base=np.zeros((c1, 9)), gap=np.zeros(c1), friction=np.zeros(c1),
                   restitution=np.zeros(c1), R=np.zeros((c1, 3)), U=np.zeros((c1, 3)), isnew=np.zeros(c1, np.int32))
        n = lib.orc_detect(nsph, sbody, sref, radius, surface, nconv, cb, cvptr, cvert, cfptr, fac, csptr, csurf,
                           nbod, rot, x, x0, obstacle, nsurf, mat, npv, pk, ps, pR, pU, cap,
                                   out['key'], out['slave_lo'], out['master'], out['slave'], out['point'],
                                   out['mpnt'], out['spnt'], out['base'], out['gap'], out['friction'],
                                   out['restitution'], out['R'], out['U'], out['isnew'])
        return n, out

    n, out = run(8 * nsph + 16)
    if n == -1:
        raise ValueError('coincident sphere centres')
    if n < 0:
        raise ValueError('a convex without surface faces')
    if n > 8 * nsph + 16:
        n, out = run(n)
    return {k: v[:n] for k, v in out.items()}


# ---------------------------------------------------------------- the reference's own contact geometry

def geo_available() -> bool:
    return os.path.exists(os.path.join(HERE, '_ref/libref_geo.so'))


def ref_gobj_sphere_sphere(ca, ra, sa, cb, rb, sb, update=False):
    """gobjcontact (goc.c:1362) of the reference for spheres a (first) and b:
    (state, onepnt, twopnt, normal, gap, spair)."""
    lib = _load('geo')
    one, two, nrm, gap, sp = np.zeros(3), np.zeros(3), np.zeros(3), np.zeros(1), np.zeros(2, np.int32)
    st = lib.ref_gobj_sphere_sphere(int(update), np.ascontiguousarray(ca, dtype=np.float64), float(ra), int(sa),
                                    np.ascontiguousarray(cb, dtype=np.float64), float(rb), int(sb),
                                    one, two, nrm, gap, sp)
    return st, one, two, nrm, gap[0], sp


def ref_gobj_convex_sphere(ver, fac, surf, c, r, s, sphere_first=False, update=False):
    """gobjcontact of the reference for a convex (vertices, reference face
    layout, surface per face) and a sphere: (state, onepnt, twopnt, normal,
    gap, spair), onepnt on the first object."""
    lib = _load('geo')
    ver = np.ascontiguousarray(ver, dtype=np.float64).reshape(-1)
    fac = np.ascontiguousarray(fac, dtype=np.int32)
    surf = np.ascontiguousarray(surf, dtype=np.int32)
    one, two, nrm, gap, sp = np.zeros(3), np.zeros(3), np.zeros(3), np.zeros(1), np.zeros(2, np.int32)
    st = lib.ref_gobj_convex_sphere(int(update), int(sphere_first), ver.shape[0] // 3, ver, surf.shape[0], fac, surf,
                                    np.ascontiguousarray(c, dtype=np.float64), float(r), int(s), one, two, nrm,
                                    gap, sp)
    return st, one, two, nrm, gap[0], sp


def ref_gobj_convex_convex(va, fa, sa, vb, fb, sb, update=False, spair=(0, 0)):
    """gobjcontact (goc.c:1362) of the reference for two convexes a (first)
    and b, each as vertices, reference face layout (count, then indices) and
    a surface per face: (state, onepnt, normal, gap, area, spair). For an
    update, spair is the contact's current surface pair."""
    lib = _load('geo')
    va = np.ascontiguousarray(va, dtype=np.float64).reshape(-1)
    vb = np.ascontiguousarray(vb, dtype=np.float64).reshape(-1)
    fa = np.ascontiguousarray(fa, dtype=np.int32); fb = np.ascontiguousarray(fb, dtype=np.int32)
    sa = np.ascontiguousarray(sa, dtype=np.int32); sb = np.ascontiguousarray(sb, dtype=np.int32)
    one, two, nrm, gap, area = np.zeros(3), np.zeros(3), np.zeros(3), np.zeros(1), np.zeros(1)
    sp = np.array(spair, np.int32)
    st = lib.ref_gobj_convex_convex(int(update), va.shape[0] // 3, va, sa.shape[0], fa, sa, vb.shape[0] // 3, vb,
                                    sb.shape[0], fb, sb, one, two, nrm, gap, area, sp)
    return st, one, nrm, gap[0], area[0], sp


def ref_detect_spheres_hybrid(centre, radius, body, pairs=False):
    """The reference's CPU detection of a sphere set (hyb.c hybrid broad phase
    and detect_sphere_sphere per overlap): the number of contacts, or with
    pairs=True their sphere-pair keys (i << 32 | j, ascending)."""
    lib = _load('geo')
    n = int(np.asarray(radius).shape[0])
    args = (n, np.ascontiguousarray(centre, dtype=np.float64).reshape(-1),
            np.ascontiguousarray(radius, dtype=np.float64), np.ascontiguousarray(body, dtype=np.int32))
    if not pairs:
        return int(lib.ref_detect_spheres_hybrid(*args, None, 0))
    cap = 16 * n + 16
    out = np.zeros(cap, np.int64)
    m = int(lib.ref_detect_spheres_hybrid(*args, out.ctypes.data_as(C.c_void_p), cap))
    if m > cap:
        out = np.zeros(m, np.int64)
        m = int(lib.ref_detect_spheres_hybrid(*args, out.ctypes.data_as(C.c_void_p), m))
    return out[:m]

