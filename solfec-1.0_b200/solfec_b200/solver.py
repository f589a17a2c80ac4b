"""Python face of the B200 contact-solve path, mirroring the reference's
scripting interface for it:

* ``GAUSS_SEIDEL_SOLVER(epsilon, maxiter, meritval=1.0, failure='CONTINUE',
  diagepsilon=None, diagmaxiter=None, diagsolver='SEMISMOOTH_NEWTON',
  data=None, callback=None)`` -- same keywords, defaults and validation as
  lng_GAUSS_SEIDEL_SOLVER_new (lng.c:4243-4345) and the same attributes as its
  getset table (lng.c:4624-4640: failure, error, iters, itershist, rerhist,
  merhist, epsilon, maxiter, diagepsilon, diagmaxiter, diagsolver, reverse,
  variant, innerloops), plus ``meritval``, ``nomerit`` and ``precision``.
* ``LOCDYN`` -- the device-resident local dynamics and constraint state that
  GAUSS_SEIDEL_Solve reads and writes (ldy.h:81-90, dom.h:79-92).

Everything runs through libsolfec_b200.so (include/solfec_b200.h); there is no
CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from ._lib import CALLBACK, b2dev_solve_report, b2gs_bodies, b2gs_contacts, last_error, lib, ptr

DIAGSOLVERS = ('PROJECTED_GRADIENT', 'DE_SAXCE_FENG', 'SEMISMOOTH_NEWTON', 'PROJECTED_NEWTON')
FAILURES = ('CONTINUE', 'EXIT', 'CALLBACK')
ERRORS = ('OK', 'DIVERGED', 'DIAGONAL_DIVERGED', 'DIAGONAL_FAILED')
ERR_GAUSS_SEIDEL_DIAGONAL_DIVERGED = 44
ERR_GAUSS_SEIDEL_DIVERGED = 45


class SolfecError(RuntimeError):
    """A THROW of the reference solver (err.h code in ``code``)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class DeviceError(RuntimeError):
    pass


def _check(rc, what):
    if rc != 0:
        raise DeviceError('%s failed (status %d): %s' % (what, rc, last_error()))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class LOCDYN:
    """Local dynamics of one step resident on a CUDA device."""

    def __init__(self, device: int = 0, stream=None):
        L = lib()
        self._h = L.b2gs_locdyn_create(int(device), stream)
        if not self._h:
            raise DeviceError('b2gs_locdyn_create: %s' % last_error())
        self.device = int(device)
        self._keep = []

    def close(self):
        if getattr(self, '_h', None):
            lib().b2gs_locdyn_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    @property
    def device_context(self):
        return lib().b2gs_locdyn_device(self._h)

    def set_colour_seed(self, seed: int):
        """Seeded Jones-Plassmann priorities for the next layouts."""
        lib().b2gs_locdyn_set_colour_seed(self._h, int(seed) & 0xFFFFFFFFFFFFFFFF)

    def set_colour_list_order(self):
        """Greedy colouring in list order for the next layouts (the default)."""
        _check(lib().b2dev_set_colour_order(self.device_context, 1), 'b2dev_set_colour_order')

    def set_wait_limit(self, seconds: float):
        """Limit of the solver's bounded device-side waits (0: the default 2 s)."""
        _check(lib().b2dev_set_wait_limit(self.device_context, float(seconds)), 'b2dev_set_wait_limit')

    def colour_reuse_count(self) -> int:
        """Layouts that reused the previous colouring (unchanged contact graph)."""
        return int(lib().b2dev_colour_reuse_count(self.device_context))

    def update_begin(self, scene, step=None, dynamic=None):
        """LOCDYN_Update_Begin on a scenes.Scene (host numpy arrays)."""
        keep = [_f64(scene.rot), _f64(scene.x0), _f64(scene.jinv), _f64(scene.minv), _f64(scene.velo),
                _f64(scene.velo0), _i32(scene.obstacle), _i32(scene.master), _i32(scene.slave), _f64(scene.mpnt),
                _f64(scene.spnt), _f64(scene.base), _f64(scene.gap), _f64(scene.friction),
                _f64(scene.restitution), _f64(scene.cohesion)]
        b = b2gs_bodies(scene.nbod, *[ptr(a) for a in keep[:7]], 0)
        c = b2gs_contacts(scene.ncon, *[ptr(a) for a in keep[7:]], 0)
        rc = lib().b2gs_locdyn_update_begin(self._h, C.byref(b), C.byref(c),
                                            float(scene.step if step is None else step),
                                            int(scene.dynamic if dynamic is None else dynamic))
        _check(rc, 'LOCDYN_Update_Begin')

    def update_begin_arrays(self, bodies: b2gs_bodies, contacts: b2gs_contacts, step: float, dynamic: int = 1):
        """LOCDYN_Update_Begin on caller-built structs (host or device pointers)."""
        _check(lib().b2gs_locdyn_update_begin(self._h, C.byref(bodies), C.byref(contacts), float(step), int(dynamic)),
               'LOCDYN_Update_Begin')

    def set(self, ld):
        """Load an assembled local dynamics (an object with the attributes of
        oracle.LocalDynamics: W, A, rho, B, V, gap, friction, restitution,
        cohesion, adjptr, adjcol, Woff, free_energy, step, dynamic)."""
        arrs = [_f64(ld.W), _f64(ld.A), _f64(ld.rho), _f64(ld.B), _f64(ld.V), _f64(ld.gap), _f64(ld.friction),
                _f64(ld.restitution), _f64(ld.cohesion), _i32(ld.adjptr), _i32(ld.adjcol), _f64(ld.Woff)]
        n = int(arrs[2].shape[0])
        rc = lib().b2gs_locdyn_set(self._h, n, *[ptr(a) for a in arrs], float(ld.free_energy), float(ld.step),
                                   int(ld.dynamic), 0)
        _check(rc, 'b2gs_locdyn_set')

    def set_state_ptr(self, R_ptr, U_ptr, on_device=1):
        """Initial R/U from raw pointers (device pointers when on_device)."""
        _check(lib().b2gs_locdyn_set_state(self._h, R_ptr, U_ptr, int(on_device)), 'b2gs_locdyn_set_state')

    def get_state_ptr(self, R_ptr, U_ptr, cm_ptr=None, on_device=1):
        _check(lib().b2gs_locdyn_get_state(self._h, R_ptr, U_ptr, cm_ptr, int(on_device)), 'b2gs_locdyn_get_state')

    def set_kinds(self, kinds=None, Z=None):
        """Constraint kinds of the rows (dom.h:98: 0 CONTACT, 1 FIXPNT, 2 FIXDIR,
        3 VELODIR, 4 VELODIR3, 5 RIGLNK) with Z[n][4] (VELODIR value, VELODIR3
        values, RIGLNK local link vector and length); None: all contacts. Set
        after the rows are uploaded (an upload or a detection resets them)."""
        n = self.sizes()[0]
        if kinds is None:
            _check(lib().b2dev_set_kinds(self.device_context, n, None, None, 0), 'b2dev_set_kinds')
            return
        k = np.ascontiguousarray(kinds, dtype=np.int32).reshape(-1)
        z = np.ascontiguousarray(np.zeros((k.shape[0], 4)) if Z is None else Z, dtype=np.float64).reshape(-1)
        self._kinds = (k, z)
        _check(lib().b2dev_set_kinds(self.device_context, int(k.shape[0]), ptr(k), ptr(z), 0), 'b2dev_set_kinds')

    def set_state(self, R=None, U=None):
        n = self.sizes()[0]
        Rh = None if R is None else _f64(R).reshape(-1)
        Uh = None if U is None else _f64(U).reshape(-1)
        for a in (Rh, Uh):
            if a is not None and a.shape[0] != 3 * n:
                raise ValueError('state arrays need 3 values per row')
        _check(lib().b2gs_locdyn_set_state(self._h, ptr(Rh), ptr(Uh), 0), 'b2gs_locdyn_set_state')

    def get_state(self):
        n = self.sizes()[0]
        R = np.zeros(3 * n); U = np.zeros(3 * n); cm = np.zeros(max(n, 1))
        _check(lib().b2gs_locdyn_get_state(self._h, ptr(R), ptr(U), ptr(cm), 0), 'b2gs_locdyn_get_state')
        return R.reshape(-1, 3), U.reshape(-1, 3), cm[:n]

    @property
    def merit(self) -> float:
        return float(lib().b2gs_locdyn_merit(self._h))

    def sizes(self):
        n, nb, nc, fe = C.c_int(0), C.c_longlong(0), C.c_int(0), C.c_double(0.0)
        _check(lib().b2gs_locdyn_sizes(self._h, C.byref(n), C.byref(nb), C.byref(nc), C.byref(fe)), 'sizes')
        return n.value, nb.value, nc.value, fe.value

    def order(self):
        n = self.sizes()[0]
        o = np.zeros(max(n, 1), np.int32)
        _check(lib().b2gs_locdyn_order(self._h, ptr(o)), 'order')
        return o[:n]

    def colours(self):
        n = self.sizes()[0]
        col = np.zeros(max(n, 1), np.int32)
        _check(lib().b2dev_get_colours(self.device_context, ptr(col)), 'colours')
        return col[:n]

    def download(self):
        """Assembled data in caller order (W, A, rho, B, V, adjptr, adjcol, Woff, free_energy)."""
        n, K, _, _ = self.sizes()
        W = np.zeros(9 * max(n, 1)); A = np.zeros(9 * max(n, 1)); rho = np.zeros(max(n, 1))
        B = np.zeros(3 * max(n, 1)); V = np.zeros(3 * max(n, 1))
        adjptr = np.zeros(n + 1, np.int32); adjcol = np.zeros(max(K, 1), np.int32); Woff = np.zeros(9 * max(K, 1))
        fe = C.c_double(0.0)
        _check(lib().b2dev_get_locdyn(self.device_context, ptr(W), ptr(A), ptr(rho), ptr(B), ptr(V), ptr(adjptr),
                                      ptr(adjcol), ptr(Woff), C.byref(fe)), 'get_locdyn')
        return dict(W=W[:9 * n], A=A[:9 * n], rho=rho[:n], B=B[:3 * n], V=V[:3 * n], adjptr=adjptr,
                    adjcol=adjcol[:K], Woff=Woff[:9 * K], free_energy=fe.value)

    def w_matrix_market(self, path: str):
        """LOCDYN_W_MatrixMarket (ldy.c:1005-1052) of the assembled local dynamics."""
        _check(lib().b2gs_locdyn_w_matrix_market(self._h, os.fsencode(path)), 'LOCDYN_W_MatrixMarket')

    def dump(self, path: str, point, master_id, slave_id, base):
        """LOCDYN_Dump (ldy.c:892-1002) of the assembled local dynamics and its
        current R, U: point (n, 3) spatial contact points, master_id /
        slave_id (n,) body ids (-1: none), base (n, 9) local frames."""
        n = self.sizes()[0]
        p, b = _f64(point).reshape(-1), _f64(base).reshape(-1)
        mi, si = _i32(master_id).reshape(-1), _i32(slave_id).reshape(-1)
        if p.shape[0] != 3 * n or b.shape[0] != 9 * n or mi.shape[0] != n or si.shape[0] != n:
            raise ValueError('dump: point (n, 3), master_id (n,), slave_id (n,) and base (n, 9) are required')
        _check(lib().b2gs_locdyn_dump(self._h, os.fsencode(path), ptr(p), ptr(mi), ptr(si), ptr(b)), 'LOCDYN_Dump')

    @property
    def assemble_ms(self) -> float:
        return float(lib().b2dev_last_assemble_ms(self.device_context))


class GAUSS_SEIDEL_SOLVER:
    """Block Gauss-Seidel contact solver (bgs.h GAUSS_SEIDEL) on the GPU."""

    def __init__(self, epsilon, maxiter, meritval=1.0, failure='CONTINUE', diagepsilon=None, diagmaxiter=None,
                 diagsolver='SEMISMOOTH_NEWTON', data=None, callback=None):
        # lng.c:4270-4272 type tests: positive epsilon, maxiter, meritval, diagepsilon, diagmaxiter
        if not epsilon > 0:
            raise ValueError('epsilon must be positive')
        if not (isinstance(maxiter, (int, np.integer)) and maxiter > 0):
            raise ValueError('maxiter must be a positive integer')
        if not meritval > 0:
            raise ValueError('meritval must be positive')
        if failure not in FAILURES:
            raise ValueError('Invalid failure action')
        if diagsolver not in DIAGSOLVERS:
            raise ValueError('Invalid diagonal solver')
        if failure == 'CALLBACK' and callback is None:
            raise ValueError('A callback routine must be given with CALLBACK failure action')
        if callback is not None and not callable(callback):
            raise TypeError('callback must be callable')
        if diagepsilon is not None and not diagepsilon > 0:
            raise ValueError('diagepsilon must be positive')
        if diagmaxiter is not None and not diagmaxiter > 0:
            raise ValueError('diagmaxiter must be positive')
        self.data = data
        self.callback = callback
        self._cb_exc = None

        def _tramp(_):
            try:
                self.callback(self.data)
            except Exception as e:  # surfaced after the C call returns
                self._cb_exc = e
        self._cfunc = CALLBACK(_tramp)
        self._h = lib().b2gs_create(float(epsilon), int(maxiter), float(meritval), FAILURES.index(failure),
                                    float(diagepsilon) if diagepsilon is not None else 0.0,
                                    int(diagmaxiter) if diagmaxiter is not None else 0,
                                    DIAGSOLVERS.index(diagsolver), None, self._cfunc)
        if not self._h:
            raise ValueError(last_error())
        self._epsilon, self._maxiter, self._meritval = float(epsilon), int(maxiter), float(meritval)
        self._diagsolver = diagsolver
        self._precision = 'FP64'

    def __del__(self):
        try:
            if getattr(self, '_h', None):
                lib().b2gs_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # ---- solve
    def solve(self, ldy: LOCDYN):
        """GAUSS_SEIDEL_Solve: R and U of ``ldy`` are updated in place; a
        FAILURE_EXIT divergence raises SolfecError with the err.h code."""
        self._cb_exc = None
        rc = lib().b2gs_solve(self._h, ldy.handle)
        if self._cb_exc is not None:
            raise self._cb_exc
        if rc == ERR_GAUSS_SEIDEL_DIAGONAL_DIVERGED:
            raise SolfecError(rc, 'GAUSS_SEIDEL: diagonal block solver diverged (FAILURE_EXIT)')
        if rc == ERR_GAUSS_SEIDEL_DIVERGED:
            raise SolfecError(rc, 'GAUSS_SEIDEL: iterations limit reached (FAILURE_EXIT)')
        _check(rc, 'GAUSS_SEIDEL_Solve')

    # ---- attributes (lng.c:4624-4640)
    @property
    def failure(self):
        return lib().b2gs_failure_string(self._h).decode()

    @property
    def diagsolver(self):
        return lib().b2gs_diagsolver_string(self._h).decode()

    @property
    def error(self):
        return lib().b2gs_error_string(self._h).decode()

    @property
    def iters(self):
        return int(lib().b2gs_get_iters(self._h))

    @property
    def rerhist(self):
        p = lib().b2gs_get_rerhist(self._h)
        return [p[k] for k in range(self.iters)] if p else []

    @property
    def merhist(self):
        p = lib().b2gs_get_merhist(self._h)
        return [p[k] for k in range(self.iters)] if p else []

    @property
    def itershist(self):
        cnt = C.c_int(0)
        p = lib().b2gs_get_itershist(self._h, C.byref(cnt))
        return [p[k] for k in range(cnt.value)] if p else []

    @itershist.setter
    def itershist(self, on):
        lib().b2gs_set_itershist(self._h, 1 if on in (True, 'ON', 1) else 0)

    @property
    def reverse(self):
        return lib().b2gs_reverse_string(self._h).decode()

    @reverse.setter
    def reverse(self, value):
        if value not in ('ON', 'OFF'):
            raise ValueError("reverse must be 'ON' or 'OFF'")
        lib().b2gs_set_reverse(self._h, 1 if value == 'ON' else 0)

    @property
    def variant(self):
        return lib().b2gs_variant_string(self._h).decode()

    @variant.setter
    def variant(self, value):
        names = ('FULL', 'MIDDLE_JACOBI', 'BOUNDARY_JACOBI')
        if value not in names:
            raise ValueError('invalid variant')
        lib().b2gs_set_variant(self._h, names.index(value))

    innerloops = 1  # parallel (MPI) setting; one device sweeps every row

    def _set(self, epsilon=0.0, maxiter=0, meritval=0.0, diagepsilon=0.0, diagmaxiter=0):
        lib().b2gs_set_params(self._h, float(epsilon), int(maxiter), float(meritval), float(diagepsilon),
                              int(diagmaxiter))

    @property
    def epsilon(self):
        return self._epsilon

    @epsilon.setter
    def epsilon(self, v):
        if not v > 0:
            raise ValueError('epsilon must be positive')
        self._epsilon = float(v); self._set(epsilon=v)

    @property
    def maxiter(self):
        return self._maxiter

    @maxiter.setter
    def maxiter(self, v):
        if not v > 0:
            raise ValueError('maxiter must be positive')
        self._maxiter = int(v); self._set(maxiter=v)

    @property
    def meritval(self):
        return self._meritval

    @meritval.setter
    def meritval(self, v):
        if not v > 0:
            raise ValueError('meritval must be positive')
        self._meritval = float(v); self._set(meritval=v)

    @property
    def nomerit(self):
        return self._meritval >= 1.0

    @nomerit.setter
    def nomerit(self, v):
        lib().b2gs_set_nomerit(self._h, 1 if v else 0)

    @property
    def precision(self):
        return self._precision

    @precision.setter
    def precision(self, v):
        if v not in ('FP64', 'MIXED'):
            raise ValueError("precision must be 'FP64' or 'MIXED'")
        self._precision = v
        lib().b2gs_set_precision(self._h, 1 if v == 'MIXED' else 0)

    def set_grid(self, blocks: int):
        lib().b2gs_set_grid(self._h, int(blocks))

    def set_stage_blocks(self, blocks: int):
        """Off-diagonal blocks staged per warp window (0: automatic); small values
        force tiles to be processed in several windows."""
        lib().b2gs_set_stage_blocks(self._h, int(blocks))

    @property
    def iters_mixed(self):
        return int(lib().b2gs_get_iters_mixed(self._h))

    @property
    def solve_ms(self):
        return float(lib().b2gs_get_solve_ms(self._h))

    @property
    def merit_input(self):
        return float(lib().b2gs_get_merit_input(self._h))

    @property
    def report(self) -> dict:
        """Device report of the last solve (kernel times, sweeps, grid)."""
        r = b2dev_solve_report()
        _check(lib().b2gs_get_report(self._h, C.byref(r), C.sizeof(r)), 'b2gs_get_report')
        return {k: (list(getattr(r, k)) if k in ('ms_kernel', 'sweeps_launch') else getattr(r, k))
                for k, _ in r._fields_}

    def write_state(self) -> str:
        buf = C.create_string_buffer(64)
        lib().b2gs_write_state(self._h, buf, 64)
        return buf.value.decode()
