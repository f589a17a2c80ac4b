"""Batched solves: many small independent scenes solved by one persistent
launch, each with its own GAUSS_SEIDEL_Solve stopping decision.

The reference solves one scene per call (bgs.c:913-1069); a user with many
small scenes calls it once per scene. Here the scenes are uploaded as one
union (bodies and contacts concatenated, contacts of scene k touching only
scene k's bodies), the contact graph is coloured and laid out once, and every
scene keeps the reference semantics: its own merit and error, histories,
failure handling and final iterate. The launch sequence is captured into a
CUDA graph and replayed; rows per tile, the persistent grid and the staging
window are chosen by the autotuner (b2dev_autotune_batch).
"""
from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from ._lib import b2dev_batch_report, b2dev_solve_opts, b2dev_solve_report, b2dev_tune_result, last_error, lib


def _check(rc, what):
    if rc != 0:
        raise RuntimeError('%s failed (status %d): %s' % (what, rc, last_error()))


def concat_scenes(scene_list):
    """(union scene, contact offsets [k+1]) of independent scenes with the same
    time step; body indices of scene k are shifted by the bodies before it."""
    from .scenes import Scene
    if not scene_list:
        raise ValueError('no scenes')
    step = scene_list[0].step
    if any(abs(s.step - step) > 0 for s in scene_list):
        raise ValueError('scenes of one batch share the time step')
    boff = np.cumsum([0] + [s.nbod for s in scene_list])
    coff = np.cumsum([0] + [s.ncon for s in scene_list]).astype(np.int32)
    cat = lambda name: np.concatenate([getattr(s, name) for s in scene_list])
    master = np.concatenate([s.master + boff[k] for k, s in enumerate(scene_list)]).astype(np.int32)
    slave = np.concatenate([np.where(s.slave >= 0, s.slave + boff[k], -1) for k, s in enumerate(scene_list)]).astype(np.int32)
    mass = None if any(s.mass is None for s in scene_list) else cat('mass')
    u = Scene(name='batch-%d' % len(scene_list), step=step, dynamic=scene_list[0].dynamic,
              rot=cat('rot'), x=cat('x'), x0=cat('x0'), jinv=cat('jinv'), minv=cat('minv'), velo=cat('velo'),
              velo0=cat('velo0'), obstacle=cat('obstacle'), master=master, slave=slave, mpnt=cat('mpnt'),
              spnt=cat('spnt'), base=cat('base'), gap=cat('gap'), friction=cat('friction'),
              restitution=cat('restitution'), cohesion=cat('cohesion'), mass=mass)
    return u, coff


@dataclasses.dataclass
class BatchResult:
    iters: np.ndarray          # per scene
    merit: np.ndarray
    error: np.ndarray
    merit_input: np.ndarray
    thrown: np.ndarray
    nfailures: np.ndarray
    ms_to_decision: np.ndarray  # device time from launch start to the scene's final decision
    rows: np.ndarray
    ms_device: float            # the whole launch (events)
    sweeps: int
    grid: int


class BatchSolver:
    """Scenes of one batch resident on a device, solved together."""

    def __init__(self, scene_list, device: int = 0, colour_seed=None):
        from .solver import LOCDYN
        self.ldy = LOCDYN(device)
        if colour_seed is not None:
            self.ldy.set_colour_seed(colour_seed)
        self.nprob = len(scene_list)
        self.update(scene_list)
        self.grid = 0
        self.stage_blocks = 0

    @property
    def ctx(self):
        return self.ldy.device_context

    def update(self, scene_list):
        """LOCDYN_Update_Begin of every scene (same contact sets keep the layout
        and the captured graph)."""
        u, off = concat_scenes(scene_list)
        if len(scene_list) != self.nprob:
            raise ValueError('batch size changed')
        self.offsets = off
        _check(lib().b2dev_set_problems(self.ctx, self.nprob, off.ctypes.data_as(C.c_void_p)), 'b2dev_set_problems')
        self.ldy.update_begin(u)
        self.union = u

    def _opts(self, gs):
        o = b2dev_solve_opts()
        _check(lib().b2gs_get_opts(gs.handle if hasattr(gs, 'handle') else gs._h, C.byref(o)), 'b2gs_get_opts')
        o.grid = int(self.grid)
        o.stage_blocks = int(self.stage_blocks)
        return o

    def autotune(self, gs):
        """Choose rows per tile, persistent grid and staging window by timing."""
        r = b2dev_tune_result()
        _check(lib().b2dev_autotune_batch(self.ctx, C.byref(self._opts(gs)), C.byref(r)), 'b2dev_autotune_batch')
        self.grid, self.stage_blocks = r.grid, r.stage_blocks
        trials = [dict(tile_rows=r.trial_rows[i], grid=r.trial_grid[i], stage_blocks=r.trial_stage[i],
                       ms=float(r.trial_ms[i])) for i in range(r.ntrials)]
        return dict(tile_rows=r.tile_rows, grid=r.grid, stage_blocks=r.stage_blocks, ms=float(r.ms), trials=trials)

    def solve(self, gs, use_graph: bool = True, histories: bool = False) -> BatchResult:
        """Solve every scene with the parameters of GAUSS_SEIDEL_SOLVER gs."""
        P = self.nprob
        reps = (b2dev_batch_report * P)()
        tot = b2dev_solve_report()
        o = self._opts(gs)
        rh = np.zeros(P * o.maxiter) if histories else None
        mh = np.zeros(P * o.maxiter) if histories else None
        _check(lib().b2dev_solve_batch(self.ctx, C.byref(o), reps,
                                       None if rh is None else rh.ctypes.data_as(C.c_void_p),
                                       None if mh is None else mh.ctypes.data_as(C.c_void_p),
                                       C.byref(tot), 1 if use_graph else 0), 'b2dev_solve_batch')
        f = lambda name, dt: np.array([getattr(reps[k], name) for k in range(P)], dtype=dt)
        res = BatchResult(iters=f('iters', int), merit=f('merit', float), error=f('error', float),
                          merit_input=f('merit_input', float), thrown=f('thrown', int),
                          nfailures=f('nfailures', int), ms_to_decision=f('ms_to_decision', float),
                          rows=f('rows', int), ms_device=float(tot.ms_device), sweeps=int(tot.sweeps),
                          grid=int(tot.grid))
        if histories:
            res.rerhist = rh.reshape(P, o.maxiter)
            res.merhist = mh.reshape(P, o.maxiter)
        return res

    def state(self):
        """(R, U, per-contact merit) of the union in caller order."""
        return self.ldy.get_state()

    def set_state(self, R=None, U=None):
        self.ldy.set_state(R, U)

    def free_energy(self):
        fe = np.zeros(self.nprob)
        _check(lib().b2dev_problem_free_energy(self.ctx, fe.ctypes.data_as(C.c_void_p)), 'b2dev_problem_free_energy')
        return fe

    def tile_rows(self):
        return int(lib().b2dev_tile_rows(self.ctx))

    def close(self):
        self.ldy.close()
