"""Benchmark of the B200 contact-solve path (one JSON line on rank 0).

Workload: the 100,000-body perturbed-hexahedra scene (rigid convex hexahedra,
side 0.04 m, vertices +-10%, density 2000, friction 0.4, h = 5e-4) in a time
loop from rest under gravity, all on the device: every step is
BODY_Dynamic_Step_Begin, LOCDYN_Update_Begin on the device bodies (W_ii, rho,
A, B, V, W_ij, colouring reused while the contact graph is unchanged,
colour-sorted layout), GAUSS_SEIDEL_Solve to merit 1e-4 (meritval 1e-4 with
the relative-error test non-binding, epsilon = 1; maxiter 1000,
SEMISMOOTH_NEWTON) warm-started from the previous step's reactions, and
BODY_Dynamic_Step_End. W steps run untimed, then K consecutive steps are
timed (each a different step of the run).

`value` is the per-step time of the mixed-precision mode (FP32 off-diagonal
sweeps, FP64 diagonal solves / merit / closing refinement) with the learned
warm start (BF16 network on the tensor cores, kept only when its merit is
below the previous-step start's), inputs resident in HBM; the plain FP64 and
plain mixed modes, and both with the reference's own stopping rule
(epsilon = meritval = 1e-4), are reported beside it, with the iterations of
every timed step. `e2e` replays the same steps through the C ABI from pinned
host buffers: each step's bodies and contacts and the previous result
uploaded, assembly, learned warm start, solve, and the read-back of R, U and
the per-contact merit. `mixed_vs_fp64_converged` compares mixed precision and
FP64 run to merit 1e-7 on the last step's local dynamics. The configs key
(single-GPU runs) carries per-step times of configs 1 and 2 (device time
loops of the settled sphere packings) and the batched config 4, whose scenes
a spawned process generates on the host meanwhile.

--workload batched runs the batched workload instead: 256 independent uneven
sphere scenes (bodies log-uniform in [50, 2000], radius U[0.02, 0.05],
friction U[0.2, 0.6], h = 1e-3, epsilon = meritval = 1e-4) solved by one
persistent launch replayed from a CUDA graph, launch shape autotuned; it
reports contacts solved per second and the per-scene time to the final
decision (p50, p99).

--workload detect times the sphere contact update and detection alone on a
grid of --detect-grid^3 overlapping spheres (the `detect` key of the default
line, on 100^3 spheres).

With --gpus N > 1 (torchrun), every rank solves its own replica scene (the
path has no exchange step for independent scenes): per-step time is the max
over ranks.

--impl reference times the reference's own serial GAUSS_SEIDEL_Solve
(compiled from its sources into oracle/_ref) on the same local dynamics
(assembled by the C restatement of LOCDYN_Update_Begin) on one host core, on
a bounded sample of iterations scaled to the step (see cpu_reference_step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, 'solfec-1.0_b200'))

METRIC = 'per-step contact-solve time to merit 1e-4 (GPU plain vs mixed+NN) and sweep HBM GB/s'
# time to merit 1e-4: the merit test decides (the relative-error test is made
# non-binding with epsilon = 1; diagepsilon keeps its default 0.01 * 1e-4)
SOLVE = dict(epsilon=1.0, maxiter=1000, meritval=1e-4)
SCENE = dict(nx=100, ny=100, nz=10)
WORKLOAD = 'hexahedra-100k: 100x100x10 perturbed rigid hexahedra (side 0.04 m, +-10% vertices), friction 0.4, h=5e-4'

# algorithmic bytes of one fused sweep+merit pass (per off-diagonal block, per row)
BYTES_BLOCK = {'fp64': 100, 'mixed': 52}
BYTES_ROW = {'fp64': 316, 'mixed': 328}
# DRAM bytes (read + write) per algorithmic byte of k_solve, measured by ncu on the 100x100x6 lattice
# (one --set full capture per precision); DRAM traffic grows in proportion to blocks, rows and passes
TRAFFIC_RATIO = {'fp64': 1184.6 / 1363.6, 'mixed': 646.5 / 739.2}


def _dist():
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return ws, rank, local


def replica_seed(rank: int) -> int:
    """Scene seed of a rank's replica (independent scenes, no exchange step)."""
    return 3 + rank


def max_over_ranks(value: float, device=None) -> float:
    """Per-step time of the slowest rank (all ranks take this collective in
    the same order); identity without a process group."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, device):
        self.device = device
        self.proc = None
        # the raw samples go to B2_CLOCKS_CSV when set (the JSON line carries their summary)
        self.path = os.environ.get('B2_CLOCKS_CSV') or os.path.join(
            os.environ.get('TMPDIR', '/tmp'), 'b2_clocks_%d.csv' % os.getpid())

    def __enter__(self):
        try:
            self.fh = open(self.path, 'w')
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.device), '--query-gpu=' + self.Q,
                                          '--format=csv,noheader,nounits', '-lms', '200'], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(',')]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1])); mx = max(mx, float(f[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, f[5:9]):
                    if v.lower() == 'active':
                        reasons.add(nm)
        except Exception:
            pass
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': mx or None,
                'reasons': sorted(reasons), 'samples': len(sm)}


# the time loop of the bench: gravity on every body, the scene's contacts kept
# (referential points, frames, gaps, materials), the reactions of each step
# the warm start of the next, as in a time-stepping run of the reference
STEP_GRAVITY = (0.0, 0.0, -9.81)
# the reference's own stopping rule at the metric's tolerance (reported beside the merit-decided modes)
SOLVE_REF_RULE = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
# the mode `value` reports: mixed precision from the previous step's reactions
# (the learned start is measured beside it: in the time loop it is never
# accepted, so the plain start is the headline)
HEADLINE = 'mixed'
# converged comparison of the mixed precision with FP64 (the stack stalls near merit 4e-8)
CONVERGED_MERIT = 1e-7
CONVERGED_SEED = 12345   # seeded colouring: another valid row order for the FP64 spread


def body_resultants(rot, x, sc, R):
    """Force and torque of the contact reactions on every moving body (global
    frame), as rig_constraints_force (bod.c:390-439) sums them."""
    base = sc.base.reshape(-1, 3, 3)
    f = np.einsum('kji,kj->ki', base, R)
    M = rot.reshape(-1, 3, 3).transpose(0, 2, 1)
    m, s = sc.master, sc.slave
    p = x[m] + np.einsum('kij,kj->ki', M[m], sc.mpnt - sc.x0[m])
    F = np.zeros((sc.nbod, 3)); T = np.zeros((sc.nbod, 3))
    np.add.at(F, m, f); np.add.at(T, m, np.cross(p - x[m], f))
    ok = s >= 0
    np.add.at(F, s[ok], -f[ok]); np.add.at(T, s[ok], -np.cross(p[ok] - x[s[ok]], f[ok]))
    mov = sc.obstacle == 0
    return F[mov], T[mov]


def _rel2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


ALL_MODES = ('fp64', 'mixed', 'mixed_nn', 'fp64_ref_rule', 'mixed_nn_ref_rule')


def bench_product(args, ws, rank, local, scene=None, modes=ALL_MODES, full=True):
    """Time loop of the hexahedra scene on the device, one run per mode from
    the same initial state (bodies at rest, zero reactions). Every step is
    BODY_Dynamic_Step_Begin (device) -> LOCDYN_Update_Begin on the device
    bodies -> warm start from the previous step's R, U (device) [-> learned
    warm start] -> GAUSS_SEIDEL_Solve -> R, U kept on the device ->
    BODY_Dynamic_Step_End (device): no host round trip of bodies or state.
    W untimed steps, then K timed steps, each a different step of the run.
    scene replaces the hexahedra scene; modes picks the runs; full = False
    leaves out the end-to-end replay and the rigid-step timing."""
    import torch
    import ctypes as C
    from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, learn, scenes
    from solfec_b200._lib import b2gs_bodies, b2gs_contacts, lib
    from solfec_b200.dynamics import RIGID_DYNAMICS

    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    sc = scene if scene is not None else scenes.hexahedra_lattice(seed=replica_seed(rank), **SCENE)
    J, mass = _rigid_inertia(sc)
    h, dflag = float(sc.step), int(sc.dynamic)
    stream = torch.cuda.current_stream()
    n, nb = sc.ncon, sc.nbod

    def tens(a, dtype):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=dtype))

    host = [tens(sc.rot, np.float64), tens(sc.x0, np.float64), tens(sc.jinv, np.float64), tens(sc.minv, np.float64),
            tens(sc.velo, np.float64), tens(sc.velo0, np.float64), tens(sc.obstacle, np.int32),
            tens(sc.master, np.int32), tens(sc.slave, np.int32), tens(sc.mpnt, np.float64), tens(sc.spnt, np.float64),
            tens(sc.base, np.float64), tens(sc.gap, np.float64), tens(sc.friction, np.float64),
            tens(sc.restitution, np.float64), tens(sc.cohesion, np.float64)]
    devt = [t.to(dev) for t in host]   # the initial scene, kept on the device for each mode's start
    pinned = [t.pin_memory() for t in host]

    def structs(ts, on_device):
        p = [C.c_void_p(t.data_ptr()) for t in ts]
        return (b2gs_bodies(nb, *p[:7], on_device), b2gs_contacts(n, *p[7:], on_device))

    bd, cd = structs(devt, 1)
    bh, ch = structs(pinned, 0)
    ldy = LOCDYN(device=local, stream=stream.cuda_stream)
    ctx = ldy.device_context
    net = learn.WarmStartNet.load(device=local)
    Rd = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    Ud = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    rot_d = torch.empty(9 * nb, dtype=torch.float64, device=dev)
    x_d = torch.empty(3 * nb, dtype=torch.float64, device=dev)
    vel_d = torch.empty(6 * nb, dtype=torch.float64, device=dev)
    vel0_d = torch.empty(6 * nb, dtype=torch.float64, device=dev)

    def check(rc, what):
        if rc != 0:
            from solfec_b200._lib import last_error
            raise RuntimeError('%s failed: %s' % (what, last_error()))

    def reset():
        ldy.update_begin_arrays(bd, cd, h, dflag)
        Rd.zero_(); Ud.zero_()
        return RIGID_DYNAMICS(ldy, J, mass, sc.x)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    snaps = []   # per timed step of the mixed+NN run: the bodies the assembly read and the warm start

    def run(solve_kw, precision, nn, record=False):
        dyn = reset()
        gs = GAUSS_SEIDEL_SOLVER(**solve_kw)
        gs.precision = precision
        nn_reps, reps, its, its_all = [], [], [], []

        def step(timed):
            dyn.step_begin(h, STEP_GRAVITY)
            check(lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, dflag), 'LOCDYN update on the device bodies')
            if record and timed:
                check(lib().b2dev_rigid_get(ctx, C.c_void_p(rot_d.data_ptr()), None, C.c_void_p(vel_d.data_ptr()),
                                            C.c_void_p(vel0_d.data_ptr()), 1), 'b2dev_rigid_get')
                snaps.append([t.clone() for t in (rot_d, vel_d, vel0_d, Rd, Ud)])
            ldy.set_state_ptr(C.c_void_p(Rd.data_ptr()), C.c_void_p(Ud.data_ptr()), 1)
            if nn:
                nn_reps.append(learn.warm_start(ldy, net))
            gs.solve(ldy)
            ldy.get_state_ptr(C.c_void_p(Rd.data_ptr()), C.c_void_p(Ud.data_ptr()), None, 1)
            dyn.step_end(h)
            its_all.append(gs.iters)
            if timed:
                reps.append(gs.report)
                its.append(gs.iters)

        for _ in range(args.warmup):
            step(False)
        barrier()
        l0 = lib().b2dev_launch_count(ctx)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step(True)
        ev1.record(stream)
        barrier()
        ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dev)
        check(lib().b2dev_rigid_get(ctx, C.c_void_p(rot_d.data_ptr()), C.c_void_p(x_d.data_ptr()), None, None, 1),
              'b2dev_rigid_get')
        return dict(ms=ms, iters=its, iters_all=its_all, reps=reps, nn=nn_reps, launches=lib().b2dev_launch_count(ctx) - l0,
                    R=Rd.cpu().numpy().reshape(-1, 3).copy(), merit=ldy.merit, error=gs.error,
                    assemble_ms=ldy.assemble_ms,
                    rot=rot_d.cpu().numpy().reshape(-1, 9).copy(), x=x_d.cpu().numpy().reshape(-1, 3).copy())

    results = {}
    mode_args = dict(fp64=(SOLVE, 'FP64', False), mixed=(SOLVE, 'MIXED', False), mixed_nn=(SOLVE, 'MIXED', True),
                     fp64_ref_rule=(SOLVE_REF_RULE, 'FP64', False), mixed_nn_ref_rule=(SOLVE_REF_RULE, 'MIXED', True))
    with ClockSampler(local) as clk:
        for m in modes:
            results[m] = run(*mode_args[m])
        if not full:
            nrows, K, ncol, fe = ldy.sizes()
            conv = converged_comparison(ldy, results[HEADLINE], sc, dev)
            net.close()
            ldy.close()
            return dict(results=results, n=nrows, K=K, ncolours=ncol, clocks=clk.summary(), nbod=sc.nbod,
                        scene=sc, converged=conv)
        head_nn = HEADLINE == 'mixed_nn'
        run(SOLVE, 'MIXED', head_nn, record=True)   # untimed: the headline steps' inputs for the end-to-end leg
        # end to end through the C ABI from pinned host buffers: the headline
        # run's timed steps replayed (each step's bodies and the previous step's
        # result uploaded, the step's R, U and per-contact merit read back)
        Rh = torch.empty(3 * n, dtype=torch.float64).pin_memory()
        Uh = torch.empty(3 * n, dtype=torch.float64).pin_memory()
        Ch = torch.empty(n, dtype=torch.float64).pin_memory()
        snaps_h = [[t.cpu().pin_memory() for t in sn] for sn in snaps]
        # each step's host bodies: its rotations and velocities, the fixed arrays of the scene
        step_bodies = [structs([sn[0], pinned[1], pinned[2], pinned[3], sn[1], sn[2], pinned[6]] + pinned[7:], 0)[0]
                       for sn in snaps_h]
        gs = GAUSS_SEIDEL_SOLVER(**SOLVE)
        gs.precision = 'MIXED'
        Rh.copy_(snaps_h[0][3]); Uh.copy_(snaps_h[0][4])

        def e2e_step(k):
            ldy.update_begin_arrays(step_bodies[k], ch, h, dflag)
            ldy.set_state_ptr(C.c_void_p(Rh.data_ptr()), C.c_void_p(Uh.data_ptr()), 0)
            if head_nn:
                learn.warm_start(ldy, net)
            gs.solve(ldy)
            ldy.get_state_ptr(C.c_void_p(Rh.data_ptr()), C.c_void_p(Uh.data_ptr()), C.c_void_p(Ch.data_ptr()), 0)

        for k in range(min(args.warmup, len(snaps_h))):
            e2e_step(k)
        Rh.copy_(snaps_h[0][3]); Uh.copy_(snaps_h[0][4])
        barrier()
        t0 = time.perf_counter()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for k in range(len(snaps_h)):
            e2e_step(k)
        ev1.record(stream)
        barrier()
        e2e_ms = max_over_ranks(max(ev0.elapsed_time(ev1), 1e3 * (time.perf_counter() - t0)) / len(snaps_h), dev)
    h2d = sum(t.numel() * t.element_size() for t in host) + 2 * 3 * n * 8
    d2h = (2 * 3 * n + n) * 8
    nrows, K, ncol, fe = ldy.sizes()
    conv = converged_comparison(ldy, results[HEADLINE], sc, dev)
    rigid = rigid_step_timing(ldy, sc, bd, cd, stream, barrier, dev)
    net.close()
    ldy.close()
    return dict(results=results, e2e_ms=e2e_ms, h2d=h2d, d2h=d2h, n=nrows, K=K, ncolours=ncol,
                clocks=clk.summary(), nbod=sc.nbod, scene=sc, rigid=rigid, converged=conv)


def bench_detected_hexahedra(args, ws, rank, local):
    """Config 3 with the contacts the reference's own contact model makes: the
    bodies of the bench scene (the same seeded perturbed cubes and walls), their
    contacts detected once on the device as detect_convex_convex makes them
    (the k_cc_* kernels, bitwise with the reference's gobjcontact), then the
    bench's time loop in FP64 and mixed precision. The headline keeps the
    scene generator's face-pair contacts, whose iteration counts the reference
    arm scales to."""
    import torch
    from solfec_b200 import scenes
    from solfec_b200.detect import detected_scene
    sc = scenes.hexahedra_lattice(seed=replica_seed(rank), **SCENE)
    cv = scenes.hexahedra_geometry(seed=replica_seed(rank), nx=SCENE['nx'], ny=SCENE['ny'], nz=SCENE['nz'])
    J, mass = _rigid_inertia(sc)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    det, con = detected_scene(sc, cv, J, mass, material=(0.4, 0.0))
    detect_s = time.perf_counter() - t0
    out = bench_product(args, ws, rank, local, scene=det, modes=('fp64', 'mixed'), full=False)
    res = out['results']
    face = np.abs(np.asarray(con['base'])[:, 6:9]).max(axis=1) > 0.999   # normal along a lattice axis
    return {'workload': 'the bench scene\'s %d bodies with the contacts of the convex detection (goc.c '
                        'detect_convex_convex restated on the device)' % sc.nbod,
            'contacts': int(det.ncon), 'contacts_generator': int(sc.ncon), 'blocks': int(out['K']),
            'colours': int(out['ncolours']), 'axis_normals': int(face.sum()),
            'gap_median': float(np.median(det.gap)), 'gap_min': float(det.gap.min()),
            'detect_call_s': round(detect_s, 3),
            'modes': {m: {'ms_per_step': round(r['ms'], 4), 'iters_per_step': r['iters'],
                          'iters_mean': round(float(np.mean(r['iters'])), 2)} for m, r in res.items()},
            'speedup_mixed_vs_fp64': round(res['fp64']['ms'] / res['mixed']['ms'], 3),
            'mixed_vs_fp64_converged': out['converged'], 'clocks': out['clocks']}


def converged_comparison(ldy, last, sc, dev):
    """The last timed step's local dynamics (still in the context) solved to
    merit 1e-7 from zero reactions by FP64 and by mixed precision in the same
    row order, and by FP64 in another valid row order (seeded colouring):
    relative 2-norm differences of the reactions, of the relative velocities
    and of the per-body force and torque resultants. On this hyperstatic stack
    the contact reactions are not unique; the resultants are what moves the
    bodies."""
    from types import SimpleNamespace
    from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN
    d = ldy.download()
    ld = SimpleNamespace(W=d['W'], A=d['A'], rho=d['rho'], B=d['B'], V=d['V'], gap=sc.gap, friction=sc.friction,
                         restitution=sc.restitution, cohesion=sc.cohesion, adjptr=d['adjptr'], adjcol=d['adjcol'],
                         Woff=d['Woff'], free_energy=d['free_energy'], step=sc.step, dynamic=sc.dynamic)
    kw = dict(epsilon=1.0, maxiter=20000, meritval=CONVERGED_MERIT)
    out = {}
    for key, prec, seed in (('fp64', 'FP64', None), ('mixed', 'MIXED', None), ('fp64_other_order', 'FP64',
                                                                               CONVERGED_SEED)):
        l2 = LOCDYN(device=dev.index)
        if seed is not None:
            l2.set_colour_seed(seed)
        l2.set(ld)
        gs = GAUSS_SEIDEL_SOLVER(**kw)
        gs.precision = prec
        gs.solve(l2)
        R, U, _ = l2.get_state()
        out[key] = dict(R=R, U=U, iters=gs.iters, merit=l2.merit)
        l2.close()
    F0, T0 = body_resultants(last['rot'], last['x'], sc, out['fp64']['R'])
    res = dict(merit_target=CONVERGED_MERIT, fp64_iters=out['fp64']['iters'], fp64_merit=out['fp64']['merit'],
               note='relative 2-norm differences from the FP64 solve in the same row order')
    for key in ('mixed', 'fp64_other_order'):
        F, T = body_resultants(last['rot'], last['x'], sc, out[key]['R'])
        res[key] = dict(iters=out[key]['iters'], merit=out[key]['merit'],
                        reactions=_rel2(out[key]['R'], out['fp64']['R']),
                        velocities=_rel2(out[key]['U'], out['fp64']['U']),
                        body_forces=_rel2(F, F0), body_torques=_rel2(T, T0))
    return res


# Algorithmic bytes of the rigid time integration kernels (csrc/b2_rigid.cuh),
# each datum counted once. Per body: begin reads velo, rot, x, J, jinv, mass,
# minv, scheme, obstacle (312 B) and writes velo0, rot, x, aux, fext, velo
# (264 B); end reads rot, x0, x, velo, jinv, minv, scheme, obstacle, aux, bptr
# (280 B) and writes velo, x, rot, aux (168 B). End also reads per contact its
# frame, reaction (double4), master index and sorted position (112 B) and per
# contact side of a moving body the row index and referential point (28 B).
RIGID_BYTES_BEGIN = 576
RIGID_BYTES_END_BODY = 448
RIGID_BYTES_END_CONTACT = 112
RIGID_BYTES_END_SIDE = 28
RIGID_REPS = 20
GRAVITY_VEC = (0.0, 0.0, -9.81)
RIGID_CPU_SAMPLE = 2000


# Sphere contact detection (csrc/b2_detect.cuh) on a grid of DETECT_GRID^3
# overlapping spheres. Algorithmic bytes, each datum of a kernel counted once:
# per sphere 520 B (current centre from the body: body index, referential
# centre, radius, rotation, mass centres, written centre; grid cell and bucket;
# one radix-sort pass over key and index; the sphere's own data in the count
# and write passes; pair count and offset), per contact 512 B (pair indices
# written, ordered and read; the matched previous contact with its R and U; the
# two spheres' centres, radii, bodies and surfaces; the 272-byte contact record
# written once; the sparsification's reads of bodies, flag and point; the body
# lists). A compaction copy, needed only when the sparsification removes
# contacts, is not counted.
DETECT_GRID = 100
DETECT_BYTES_SPHERE = 520
DETECT_BYTES_CONTACT = 512
DETECT_REPS = 10


DETECT_CPU_GRID = 60


def detect_cpu_baseline():
    """The reference's own CPU detection (oracle/_ref/libref_geo.so: the hyb.c
    hybrid broad phase over the eps-inflated sphere boxes and goc.c's
    detect_sphere_sphere per overlap, one host core) on a DETECT_CPU_GRID^3
    sample of the same grid, as contacts per second. Insertion into the domain
    and the sparsification are not timed, so the figure favours the reference."""
    import time
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle as O
    from solfec_b200 import scenes
    sc = scenes.spheres_grid(DETECT_CPU_GRID)
    sp = scenes.sphere_shapes(sc, friction=0.3)
    t0 = time.perf_counter()
    n = O.ref_detect_spheres_hybrid(sc.x, sp['radius'], sp['body'])
    dt = time.perf_counter() - t0
    return {'value': round(n / dt, 1), 'unit': 'contacts/s', 'cores': 1, 'kind': 'reference',
            'sample': 'spheres-grid %d^3 (%d spheres, %d contacts): hyb.c hybrid + detect_sphere_sphere, %.2f s'
                      % (DETECT_CPU_GRID, sc.nbod, n, dt)}


def detect_timing(grid=DETECT_GRID):
    """Host call time of b2dev_detect_spheres (SPHERES.detect) on grid^3 spheres:
    the first call detects every contact, the timed calls (after 3 warm-up
    calls) update them all (same bodies); each call includes its three host
    synchronisations (pair count, contact count, completion)."""
    import time
    import torch
    from solfec_b200 import LOCDYN, scenes
    from solfec_b200.detect import SPHERES, bodies_only
    from solfec_b200.dynamics import RIGID_DYNAMICS
    sc = scenes.spheres_grid(grid)
    sp = scenes.sphere_shapes(sc, friction=0.3)
    J, mass = scenes.sphere_inertia(sc)
    ldy = LOCDYN()
    try:
        ldy.update_begin(bodies_only(sc))
        RIGID_DYNAMICS(ldy, J, mass, sc.x)
        s = SPHERES(ldy, **sp)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        nc, nn = s.detect()
        first = time.perf_counter() - t0
        for _ in range(3):
            s.detect()
        ts = []
        for _ in range(DETECT_REPS):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.detect()
            ts.append(time.perf_counter() - t0)
        ms = float(np.median(ts)) * 1e3
        nb = DETECT_BYTES_SPHERE * s.nsph + DETECT_BYTES_CONTACT * s.ncon
        peak = _peaks()[0]
        try:
            cpu = detect_cpu_baseline()
        except Exception as e:  # the reference build is test infrastructure: its absence costs only this figure
            cpu = {'error': str(e)[:200]}
        return {'workload': 'spheres-grid-%d: %d^3 spheres, pitch 0.0999, radius 0.05' % (s.nsph, grid),
                'spheres': s.nsph, 'contacts': int(s.ncon), 'new_first_call': int(nn),
                'first_call_ms': round(first * 1e3, 3), 'update_call_ms': round(ms, 3),
                'contacts_per_s': round(s.ncon / (ms * 1e-3), 1), 'bytes_per_call': int(nb),
                'achieved_gbs': round(nb / (ms * 1e-3) / 1e9, 1), 'peak_gbs': peak,
                'frac': round(nb / (ms * 1e-3) / 1e9 / peak, 3), 'timing': 'host call time, median of %d' % DETECT_REPS,
                'cpu_baseline': cpu}
    finally:
        ldy.close()


CONVEX_LATTICE = dict(nx=50, ny=50, nz=10)
CONVEX_CPU_PAIRS = 1500


def detect_convex_timing():
    """Host call time of the convex-convex contact update and detection
    (b2dev_detect_spheres with convexes only: k_cvx_update, the sweep over the
    inflated boxes, k_cc_contacts, sparsification) on a lattice of boxes with
    exact, jittered and turned members on a floor obstacle: the first call
    detects every contact, the timed calls (after 3 warm-up calls) update them
    all. CPU baseline: the reference's own gobjcontact (detect_convex_convex,
    oracle/_ref) on a sample of the contact pairs, one host core; its broad
    phase and the domain insertion are not timed, which favours it."""
    import time
    import torch
    from solfec_b200 import LOCDYN, scenes
    from solfec_b200.detect import CONVEXES, bodies_only
    from solfec_b200.dynamics import RIGID_DYNAMICS
    sc, cv = scenes.convex_lattice(**CONVEX_LATTICE)
    J = np.tile(np.eye(3).reshape(9), (sc.nbod, 1))
    ldy = LOCDYN()
    try:
        ldy.update_begin(bodies_only(sc))
        RIGID_DYNAMICS(ldy, J, np.ones(sc.nbod), sc.x)
        nsurf = int(cv['surf'].max()) + 1
        mat = np.zeros((nsurf, nsurf, 2))
        mat[..., 0] = 0.5
        det = CONVEXES(ldy, cv, mat)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        nc, nn = det.detect()
        first = time.perf_counter() - t0
        for _ in range(3):
            det.detect()
        ts = []
        for _ in range(DETECT_REPS):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            det.detect()
            ts.append(time.perf_counter() - t0)
        ms = float(np.median(ts)) * 1e3
        keys = det.contacts()['key']
        out = {'workload': 'convex-lattice-%d: %dx%dx%d unit boxes (a third exact, a third jittered, a third '
                           'also turned) on a floor' % (sc.nbod - 1, CONVEX_LATTICE['nx'], CONVEX_LATTICE['ny'],
                                                      CONVEX_LATTICE['nz']),
               'convexes': int(sc.nbod), 'contacts': int(nc), 'new_first_call': int(nn),
               'first_call_ms': round(first * 1e3, 3), 'update_call_ms': round(ms, 3),
               'contacts_per_s': round(nc / (ms * 1e-3), 1),
               'timing': 'host call time, median of %d' % DETECT_REPS}
        try:
            sys.path.insert(0, os.path.join(ROOT, 'oracle'))
            import oracle as O
            if not O.geo_available():
                raise RuntimeError('reference geometry build unavailable')
            conv = scenes.convex_list(cv)
            rng = np.random.default_rng(0)
            sample = keys[rng.choice(keys.shape[0], min(CONVEX_CPU_PAIRS, keys.shape[0]), replace=False)]
            args = [(conv[int(k >> 32)], conv[int(k & 0xFFFFFFFF)]) for k in sample]
            t0 = time.perf_counter()
            for a, b in args:
                O.ref_gobj_convex_convex(*a, *b)
            dt = time.perf_counter() - t0
            out['cpu_baseline'] = {'value': round(len(args) / dt, 1), 'unit': 'contacts/s', 'cores': 1,
                                   'kind': 'reference',
                                   'sample': '%d contact pairs of the same lattice through the reference gobjcontact '
                                             '(detect_convex_convex), %.2f s; broad phase and insertion untimed'
                                             % (len(args), dt)}
        except Exception as e:  # the reference build is test infrastructure: its absence costs only this figure
            out['cpu_baseline'] = {'error': str(e)[:200]}
        return out
    finally:
        ldy.close()


def _rigid_inertia(sc, k=None):
    k = sc.nbod if k is None else k
    ob = sc.obstacle[:k] != 0  # walls: zero inverse inertia and mass (never accelerated)
    J = np.stack([np.eye(3).reshape(9) if o else np.linalg.inv(j.reshape(3, 3).T).T.reshape(9)
                  for j, o in zip(sc.jinv[:k], ob)])
    mass = np.where(ob, 1.0, 1.0 / np.where(ob, 1.0, sc.minv[:k]))
    return J, mass


def rigid_step_timing(ldy, sc, bd, cd, stream, barrier, dev):
    """Device time of BODY_Dynamic_Step_Begin / End (k_rigid_begin,
    k_rigid_end) for every body of the bench scene, measured inside the step
    they belong to: each repetition is begin, assembly on the device bodies,
    a 5-sweep FP64 solve, end, with CUDA events on the library's stream around
    begin and around end. The solve streams the W planes (far beyond L2)
    between the two, so the body arrays come from DRAM as in a time loop (a
    plain buffer write between back-to-back launches left them in L2).
    Averaged over RIGID_REPS repetitions, outside the timed solve region."""
    import ctypes as C
    import torch
    from solfec_b200 import GAUSS_SEIDEL_SOLVER
    from solfec_b200.dynamics import RIGID_DYNAMICS
    from solfec_b200._lib import lib
    J, mass = _rigid_inertia(sc)
    ldy.update_begin_arrays(bd, cd, sc.step, sc.dynamic)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    gs = GAUSS_SEIDEL_SOLVER(epsilon=1e-12, maxiter=5, meritval=1e-12, diagepsilon=1e-6, diagmaxiter=100)
    n = sc.ncon
    Rz = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    Uz = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    pairs = []
    for rep in range(3 + RIGID_REPS):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        dyn.step_begin(sc.step, GRAVITY_VEC)
        ev[1].record(stream)
        if lib().b2gs_locdyn_update_begin_resident(ldy.handle, sc.step, sc.dynamic) != 0:
            raise RuntimeError('LOCDYN update on the device bodies failed')
        ldy.set_state_ptr(C.c_void_p(Rz.data_ptr()), C.c_void_p(Uz.data_ptr()), 1)
        gs.solve(ldy)
        ev[2].record(stream)
        dyn.step_end(sc.step)
        ev[3].record(stream)
        if rep >= 3:
            pairs.append(ev)
    barrier()
    tb = max_over_ranks(sum(e[0].elapsed_time(e[1]) for e in pairs) / RIGID_REPS, dev)
    te = max_over_ranks(sum(e[2].elapsed_time(e[3]) for e in pairs) / RIGID_REPS, dev)
    ob = sc.obstacle != 0
    inc = int(np.sum(~ob[sc.master]) + np.sum((sc.slave >= 0) & ~ob[np.maximum(sc.slave, 0)]))
    nb = sc.nbod
    return dict(bodies=nb, contact_sides=inc, begin_ms=tb, end_ms=te, begin_bytes=nb * RIGID_BYTES_BEGIN,
                end_bytes=nb * RIGID_BYTES_END_BODY + sc.ncon * RIGID_BYTES_END_CONTACT + inc * RIGID_BYTES_END_SIDE)


def rigid_cpu_sample(sc, nsample=RIGID_CPU_SAMPLE):
    """Host time of the restated BODY_Dynamic_Step_Begin (oracle/rigid_oracle.py,
    one core, scalar Python) on the first `nsample` bodies of the scene, per
    1000 bodies."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import rigid_oracle as ro
    k = min(nsample, sc.nbod)
    J, mass = _rigid_inertia(sc, k)
    bd = ro.Bodies(sc.rot[:k], sc.x[:k], sc.velo[:k], J, sc.jinv[:k], mass, sc.minv[:k], sc.x0[:k], sc.obstacle[:k])
    t0 = time.perf_counter()
    ro.step_begin(bd, sc.step, GRAVITY_VEC)
    return 1e3 * (time.perf_counter() - t0) * 1000.0 / k


BATCH = dict(seed=4, count=256, nmin=50, nmax=2000, settle_iters=300)
BATCH_SOLVE = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
BATCH_METRIC = 'batched contact solve: contacts solved per second (256 uneven sphere scenes, one persistent launch)'


def bench_batched(args, ws, rank, local, scs=None):
    """Config of the batched workload: every rank solves its own batch."""
    import ctypes as C
    import torch
    from solfec_b200 import GAUSS_SEIDEL_SOLVER, scenes
    from solfec_b200.batch import BatchSolver, concat_scenes
    from solfec_b200._lib import lib
    kw = dict(BATCH)
    kw['seed'] = BATCH['seed'] + 1000 * rank
    t0 = time.perf_counter()
    if scs is None:
        scs = scenes.batched_scenes(workers=min(32, os.cpu_count() or 1), **kw)
    gen_s = time.perf_counter() - t0
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    bs = BatchSolver(scs, device=local)
    gs = GAUSS_SEIDEL_SOLVER(**BATCH_SOLVE)
    bs.solve(gs, use_graph=False)                  # the previous step, from rest
    R0, U0, _ = bs.state()
    off = bs.offsets
    nxt = [scenes.advance_velocities(sc, R0[off[k]:off[k + 1]]) for k, sc in enumerate(scs)]
    bs.update(nxt)
    bs.set_state(R0, U0)
    tune = bs.autotune(gs)
    n = int(off[-1])
    Rd = torch.from_numpy(np.ascontiguousarray(R0.ravel())).to(dev)
    Ud = torch.from_numpy(np.ascontiguousarray(U0.ravel())).to(dev)

    def step():
        bs.ldy.set_state_ptr(C.c_void_p(Rd.data_ptr()), C.c_void_p(Ud.data_ptr()), 1)
        return bs.solve(gs, use_graph=True)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if ws > 1:
        torch.distributed.barrier()
    l0 = lib().b2dev_launch_count(bs.ctx)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    outs = []
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            outs.append(step())
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dev)
    launches = lib().b2dev_launch_count(bs.ctx) - l0
    # end to end: host scene arrays in, assembly and layout, warm start from the host, solve, results out
    u, _ = concat_scenes(nxt)
    h2d = sum(getattr(u, f).nbytes for f in ('rot', 'x0', 'jinv', 'minv', 'velo', 'velo0', 'obstacle', 'master',
                                             'slave', 'mpnt', 'spnt', 'base', 'gap', 'friction', 'restitution',
                                             'cohesion')) + 2 * R0.nbytes
    d2h = 2 * R0.nbytes + n * 8
    te = []
    for _ in range(max(1, args.steps)):
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        bs.update(nxt)
        bs.set_state(R0, U0)
        bs.solve(gs, use_graph=True)
        bs.state()
        te.append(1e3 * (time.perf_counter() - t1))
    last = outs[-1]
    td = last.ms_to_decision
    res = dict(ms=ms, contacts=n, scenes=len(scs), iters=last.iters, td=td, tune=tune, launches=launches,
               clocks=clk.summary(), gen_s=gen_s, e2e_ms=max_over_ranks(statistics.median(te), dev), h2d=h2d,
               d2h=d2h, grid=last.grid, sweeps=last.sweeps, ms_device=last.ms_device,
               merit_max=float(last.merit.max()), thrown=int(last.thrown.sum()))
    bs.close()
    return res


def batched_line(args, ws, out):
    td, it = out['td'], out['iters']
    cps = out['contacts'] * ws / (out['ms'] * 1e-3)
    return {
        'metric': BATCH_METRIC, 'value': round(cps, 1), 'unit': 'contacts/s', 'n_gpus': ws, 'steps': args.steps,
        'warmup': args.warmup, 'ms_per_step': round(out['ms'], 4), 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded scene generator)',
        'config': {'workload': 'batched: %d independent sphere scenes, bodies log-uniform in [%d, %d], radius '
                               'U[0.02, 0.05], friction U[0.2, 0.6], h=1e-3' % (out['scenes'], BATCH['nmin'],
                                                                                  BATCH['nmax']),
                   'contacts': out['contacts'], 'solver': 'GAUSS_SEIDEL_SOLVER(epsilon=1e-4, maxiter=1000, '
                                                          'meritval=1e-4), warm start from the previous step',
                   'launch': 'one persistent cooperative launch per step, replayed from a CUDA graph',
                   'autotuned': {k: out['tune'][k] for k in ('tile_rows', 'grid', 'stage_blocks', 'ms')},
                   'autotune_trials': len(out['tune']['trials']),
                   'l2': 'working set < 126 MB L2 (no flush between steps)',
                   'parallelism': 'replicas' if ws > 1 else 'single GPU'},
        'per_scene_ms_to_decision': {'p50': round(float(np.percentile(td, 50)), 4),
                                     'p99': round(float(np.percentile(td, 99)), 4),
                                     'max': round(float(td.max()), 4)},
        'per_scene_iters': {'p50': int(np.percentile(it, 50)), 'p99': int(np.percentile(it, 99)),
                            'max': int(it.max())},
        'merit_max': out['merit_max'], 'thrown': out['thrown'],
        'e2e': {'value': round(out['contacts'] * ws / (out['e2e_ms'] * 1e-3), 1), 'unit': 'contacts/s',
                'ms_per_step': round(out['e2e_ms'], 3), 'h2d_bytes_per_step': int(out['h2d']),
                'd2h_bytes_per_step': int(out['d2h'])},
        'gpu_launches': int(out['launches']), 'clocks': out['clocks'],
        'scene_generation_s': round(out['gen_s'], 1),
    }


CONFIG_SOLVE = {'config1': dict(epsilon=1e-4, maxiter=1000, meritval=1e-4),
                'config2': dict(epsilon=1e-6, maxiter=1000, meritval=1e-6)}


def _generate_config_scenes(queue, batch_seed, workers):
    """Host generation of the scenes of configs 1, 2 and 4 (runs in a spawned
    process while the GPU runs the headline workload)."""
    sys.path.insert(0, os.path.join(ROOT, 'solfec-1.0_b200'))
    from solfec_b200 import scenes
    t0 = time.perf_counter()
    c1 = scenes.spheres_lattice()
    c2 = scenes.spheres_polydisperse(seed=2, n=20000)
    kw = dict(BATCH)
    kw['seed'] = batch_seed
    c4 = scenes.batched_scenes(workers=workers, **kw)
    queue.put((c1, c2, c4, time.perf_counter() - t0))


class _ConfigScenes:
    """Scenes of configs 1, 2 and 4, generated by a spawned process."""

    def __init__(self, batch_seed):
        import multiprocessing as mp
        ctx = mp.get_context('spawn')
        self.q = ctx.Queue()
        self.p = ctx.Process(target=_generate_config_scenes,
                             args=(self.q, batch_seed, max(1, min(16, (os.cpu_count() or 2) - 1))))
        self.p.start()

    def result(self, timeout=900):
        try:
            out = self.q.get(timeout=timeout)   # read before joining: the child flushes its result into the pipe
        finally:
            self.close()
        return out

    def close(self):
        """Ends the generator (it may still be writing when the run fails early)."""
        if self.p.is_alive():
            self.p.terminate()
        self.p.join(timeout=30)


def start_scene_generation(args):
    """Configs 1, 2 and 4 ride along the default run (rank 0 only)."""
    ws, rank, _ = _dist()
    if ws > 1 or args.no_configs or args.scene:  # single-GPU runs only (the legs take no collective)
        return None
    return _ConfigScenes(BATCH['seed'])


def sphere_time_loop(sc, solve_kw, args, dev, precision='FP64'):
    """Device time loop of a sphere scene with the scene's contacts kept
    (gravity, warm start from the previous step, bodies and state on the
    device): W untimed steps, then K timed steps; per-step time by CUDA events."""
    import torch
    import ctypes as C
    from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN
    from solfec_b200._lib import lib
    from solfec_b200.dynamics import RIGID_DYNAMICS
    stream = torch.cuda.current_stream()
    J, mass = _rigid_inertia(sc)
    ldy = LOCDYN(device=dev.index, stream=stream.cuda_stream)
    ldy.update_begin(sc)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    n = sc.ncon
    Rd = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    Ud = torch.zeros(3 * n, dtype=torch.float64, device=dev)
    gs = GAUSS_SEIDEL_SOLVER(**solve_kw)
    gs.precision = precision
    h, dflag = float(sc.step), int(sc.dynamic)
    its, kms = [], []

    def step(timed):
        dyn.step_begin(h, STEP_GRAVITY)
        if lib().b2gs_locdyn_update_begin_resident(ldy.handle, h, dflag) != 0:
            raise RuntimeError('LOCDYN update failed')
        ldy.set_state_ptr(C.c_void_p(Rd.data_ptr()), C.c_void_p(Ud.data_ptr()), 1)
        gs.solve(ldy)
        ldy.get_state_ptr(C.c_void_p(Rd.data_ptr()), C.c_void_p(Ud.data_ptr()), None, 1)
        dyn.step_end(h)
        if timed:
            its.append(gs.iters)
            r = gs.report
            kms.append(r['ms_kernel'][0] + r['ms_kernel'][1])

    for _ in range(args.warmup):
        step(False)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step(True)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / args.steps
    nrows, K, ncol, _ = ldy.sizes()
    out = {'ms_per_step': round(ms, 4), 'contacts': nrows, 'blocks': K, 'colours': ncol, 'bodies': sc.nbod,
           'iters_per_step': its, 'solve_kernel_ms_mean': round(float(np.mean(kms)), 4),
           'us_per_sweep': round(1e3 * float(np.sum(kms)) / max(1, sum(its) + len(its)), 2),
           'precision': precision,
           'last_merit': ldy.merit, 'last_error': gs.error,
           'solver': 'GAUSS_SEIDEL_SOLVER(epsilon=%g, maxiter=%d, meritval=%g)' % (
               solve_kw['epsilon'], solve_kw['maxiter'], solve_kw['meritval'])}
    ldy.close()
    return out


def run_config_legs(args, ws, rank, local, extra):
    """Per-step times of configs 1 and 2 (device time loops of the settled
    sphere packings) and the batched config 4, for the default line."""
    if extra is None:
        return None
    import torch
    dev = torch.device('cuda', local)
    try:
        c1, c2, c4, gen_s = extra.result()
    except Exception as e:
        return {'error': 'scene generation: %s' % str(e)[:200]}
    out = {'scene_generation_s': round(gen_s, 1)}
    for key, sc, name in (('config1', c1, '1000 spheres r=0.05 on a 10^3 lattice, settled, friction 0.3, h=1e-3'),
                          ('config2', c2, '20000 polydisperse spheres r~U[0.03,0.06], settled, friction 0.5, '
                                          'h=5e-4')):
        try:
            out[key] = dict(sphere_time_loop(sc, CONFIG_SOLVE[key], args, dev), workload=name)
        except Exception as e:
            out[key] = {'error': str(e)[:300]}
    try:
        b = bench_batched(args, 1, 0, local, scs=c4)
        line = batched_line(args, 1, b)
        out['config4'] = {k: line[k] for k in ('value', 'unit', 'ms_per_step', 'per_scene_ms_to_decision',
                                                'per_scene_iters', 'e2e', 'gpu_launches')}
        out['config4']['metric'] = BATCH_METRIC
        out['config4']['contacts'] = b['contacts']
        out['config4']['autotuned'] = line['config']['autotuned']
    except Exception as e:
        out['config4'] = {'error': str(e)[:300]}
    return out


def roofline(mode, reps, n, K, peak):
    """Achieved bandwidth of the dominant kernel (the solve launch of the FP32
    sweeps in mixed precision, the FP64 solve launch otherwise) over the timed
    steps: algorithmic bytes of all its fused passes / its CUDA-event time."""
    sweeps = sum(r['sweeps_launch'][0] for r in reps)
    ms = sum(r['ms_kernel'][0] for r in reps)
    bytes_all = sweeps * (K * BYTES_BLOCK[mode] + n * BYTES_ROW[mode])
    gbs = bytes_all / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
    nl = max(len(reps), 1)
    return dict(bound='hbm', achieved=round(gbs, 1), peak=peak, unit='GB/s', frac=round(gbs / peak, 3),
                traffic=int(bytes_all / nl * TRAFFIC_RATIO[mode]), traffic_source='ncu, 100x100x6 lattice, scaled',
                kernel='k_solve_fp32' if mode == 'mixed' else 'k_solve<false>',
                bytes_per_launch=int(bytes_all / nl), sweeps_per_launch=round(sweeps / nl, 2),
                kernel_ms_per_launch=round(ms / nl, 4), launches=len(reps))


# FP64 iterations of steps 1 .. 60 of the bench's time loop from rest (seed of
# rank 0), as the product arm measures them (its line's fp64_iters_from_rest).
# The FP64 GPU path reproduces, bit for bit, the reference solver run on the
# same rows in the GPU's colour order, so these are also that run's counts; the
# reference's per-iteration cost does not depend on the row order or the
# state, so the reference arm runs these counts for the product arm's timed
# steps (or, when they add up to many iterations, scales a sample to their
# mean). Past step 60 the loop has settled at one iteration per step.
FP64_ITERS_FROM_REST = [45, 196, 173, 76, 48, 30, 20, 14, 11, 8, 7, 5, 5, 3, 4, 3, 3, 4, 2, 3, 2, 3, 2, 2, 3, 2, 1,
                        3, 1, 2, 2, 1, 1, 2, 1, 1, 2, 1, 1, 2, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                        1, 1, 1]


def step_iters(warmup, steps):
    """FP64 iterations of each timed step warmup+1 .. warmup+steps."""
    seq = FP64_ITERS_FROM_REST
    return [seq[k] if k < len(seq) else 1 for k in range(warmup, warmup + steps)]


def workload_iters(warmup, steps):
    """Mean FP64 iterations of the timed steps warmup+1 .. warmup+steps."""
    return float(np.mean(step_iters(warmup, steps)))


# the reference arm runs every timed step's own iteration count in full when
# the timed steps add up to at most this many iterations (about 0.27 s each on
# one host core); past it, it times a sample per step and scales it
REF_EXACT_MAX_ITERS = 600


CPU_SAMPLE_ITERS = 10


def cpu_reference_step(sc, R0, U0, iters_full, sample_iters=CPU_SAMPLE_ITERS, seed=0x5EEDC0105):
    """One step on the host: the restated LOCDYN_Update_Begin (oracle_ldy.c,
    timed in full) and the reference's own serial GAUSS_SEIDEL_Solve
    (oracle/_ref, compiled from bgs.c etc.) timed over `sample_iters`
    iterations from the step's warm start (R0/U0 may be None: cold start) and
    scaled to `iters_full` iterations; the reference spends the same work on
    every iteration (one sweep plus one merit pass). With sample_iters equal
    to iters_full nothing is scaled: the step is measured in full."""
    sys.path.insert(0, os.path.join(ROOT, 'oracle'))
    import oracle as O
    t0 = time.perf_counter()
    ld = O.assemble(sc)
    t1 = time.perf_counter()
    nc, col = O.colour(ld, seed)
    order = O.colour_order(col)
    lp = ld.permuted(order)
    Rp = None if R0 is None else np.asarray(R0).reshape(-1, 3)[order].ravel()
    Up = None if U0 is None else np.asarray(U0).reshape(-1, 3)[order].ravel()
    impl = 'ref' if O.ref_available() else 'oracle'
    kw = dict(SOLVE)
    kw['maxiter'] = sample_iters
    kw['meritval'] = 1e-300  # run the whole sample
    t2 = time.perf_counter()
    res = O.solve(lp, R=Rp, U=Up, impl=impl, **kw)
    t3 = time.perf_counter()
    per_iter = (t3 - t2) / max(res['iters'], 1)
    return dict(ms=1e3 * ((t1 - t0) + per_iter * iters_full), assemble_ms=1e3 * (t1 - t0),
                per_iter_ms=1e3 * per_iter, sample_iters=res['iters'], impl=impl, n=ld.n, K=ld.nblocks)


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from solfec_b200 import scenes
    sc = scenes.hexahedra_lattice(seed=replica_seed(0), **SCENE)
    iters = workload_iters(args.warmup, args.steps)
    per_step = step_iters(args.warmup, args.steps)
    exact = sum(per_step) <= REF_EXACT_MAX_ITERS
    for _ in range(args.warmup):  # untimed: the assembly and one iteration
        cpu_reference_step(sc, None, None, 1, sample_iters=1)
    if exact:  # every timed step runs its own iteration count in full
        times = [cpu_reference_step(sc, None, None, k, sample_iters=k) for k in per_step]
    else:
        times = [cpu_reference_step(sc, None, None, iters) for _ in range(args.steps)]
    ms = statistics.mean(t['ms'] for t in times)
    kind = 'reference' if times[-1]['impl'] == 'ref' else 'port'
    if exact:
        sample = ('per step: the restated assembly of all %d contacts (oracle/oracle_ldy.c) and the reference serial '
                  'GAUSS_SEIDEL_Solve (bgs.c, compiled unmodified) run for the FP64 iteration count of that '
                  'time-loop step from rest (steps %d .. %d, the product arm\'s timed steps; %d iterations in all, '
                  'mean %.2f), both timed in full from the scene at rest (the work of an iteration does not depend '
                  'on the state); the rigid integrator is not timed'
                  % (times[-1]['n'], args.warmup + 1, args.warmup + args.steps, sum(per_step), iters))
    else:
        sample = ('per step: the restated assembly of all %d contacts (oracle/oracle_ldy.c) timed in full, plus %d '
                  'iterations of the reference serial GAUSS_SEIDEL_Solve (bgs.c, compiled unmodified) timed and '
                  'scaled to %.2f iterations, the mean FP64 count of time-loop steps %d .. %d from rest (the product '
                  'arm\'s timed steps); the rigid integrator is not timed'
                  % (times[-1]['n'], CPU_SAMPLE_ITERS, iters, args.warmup + 1, args.warmup + args.steps))
    line = {'metric': METRIC, 'value': round(ms, 3), 'unit': 'ms', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': round(ms, 3), 'higher_is_better': False, 'scaling': 'weak',
            'vs_baseline': None, 'dtype': 'f64', 'data': 'synthetic (seeded scene generator)',
            'config': {'workload': WORKLOAD, 'contacts': times[-1]['n'], 'blocks': times[-1]['K'],
                       'mode': 'reference FP64, serial', 'parallelism': 'replicas'},
            'impl': 'reference',
            'cpu_baseline': {'value': round(ms, 3), 'unit': 'ms', 'cores': 1, 'kind': kind, 'sample': sample,
                             'assemble_ms': round(statistics.mean(t['assemble_ms'] for t in times), 3),
                             'per_iteration_ms': round(statistics.mean(t['per_iter_ms'] for t in times), 3)},
            'e2e': {'value': round(ms, 3), 'unit': 'ms', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='product', choices=['product', 'reference'])
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-configs', action='store_true', help='skip the configs 1, 2 and 4 legs of the default line')
    ap.add_argument('--scene', default=None, help='NXxNYxNZ lattice of a smaller case (profiling)')
    ap.add_argument('--maxiter', type=int, default=None, help='iteration cap of a smaller case (profiling)')
    ap.add_argument('--workload', default='hexahedra', choices=['hexahedra', 'batched', 'detect', 'detect-convex'])
    ap.add_argument('--convex-lattice', default=None, help='NXxNYxNZ boxes of the convex detection case')
    ap.add_argument('--detect-grid', type=int, default=DETECT_GRID, help='spheres per grid side (--workload detect)')
    args = ap.parse_args()
    global WORKLOAD
    if args.scene:
        nx, ny, nz = (int(v) for v in args.scene.lower().split('x'))
        SCENE.update(nx=nx, ny=ny, nz=nz)
        WORKLOAD = 'hexahedra %dx%dx%d (profiling case)' % (nx, ny, nz)
    if args.maxiter:
        SOLVE['maxiter'] = args.maxiter
    args.warmup = max(args.warmup, 3)
    ws, rank, local = _dist()
    if args.impl == 'reference':
        run_reference(args, ws, rank)
        return
    import torch
    if ws > 1:
        import datetime
        torch.cuda.set_device(local)
        torch.distributed.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
    if args.workload == 'detect':  # sphere contact detection alone (profiling)
        torch.cuda.set_device(local)
        d = detect_timing(args.detect_grid)
        if rank == 0:
            print(json.dumps(dict(d, metric='sphere contact update call time', impl='product')), flush=True)
        if ws > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    if args.workload == 'detect-convex':  # convex-convex contact detection alone (profiling)
        torch.cuda.set_device(local)
        if args.convex_lattice:
            CONVEX_LATTICE.update(zip(('nx', 'ny', 'nz'), (int(v) for v in args.convex_lattice.lower().split('x'))))
        d = detect_convex_timing()
        if rank == 0:
            print(json.dumps(dict(d, metric='convex contact update call time', impl='product')), flush=True)
        if ws > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    if args.workload == 'batched':
        out = bench_batched(args, ws, rank, local)
        if rank == 0:
            print(json.dumps(batched_line(args, ws, out)), flush=True)
        if ws > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    extra = start_scene_generation(args)          # configs 1, 2 and 4 are generated on the host meanwhile
    try:
        out = bench_product(args, ws, rank, local)
        configs = run_config_legs(args, ws, rank, local, extra)
        detected = None if args.no_configs else bench_detected_hexahedra(args, ws, rank, local)
    finally:
        if extra is not None:
            extra.close()
    peak, peak_kind = _peaks()
    if rank == 0:
        res = out['results']
        mixed, fp64, mnn = res['mixed'], res['fp64'], res['mixed_nn']
        head = res[HEADLINE]
        roof = roofline('mixed', head['reps'], out['n'], out['K'], peak)
        roof64 = roofline('fp64', fp64['reps'], out['n'], out['K'], peak)
        roof['peak_kind'] = peak_kind
        fp64_iters = float(np.mean(fp64['iters']))
        cpu = None
        if not args.no_cpu_baseline:
            t = cpu_reference_step(out['scene'], None, None, fp64_iters)
            cpu = {'value': round(t['ms'], 3), 'unit': 'ms', 'cores': 1,
                   'kind': 'reference' if t['impl'] == 'ref' else 'port',
                   'sample': 'a step of the bench scene (%d contacts): restated assembly timed in full + %d '
                             'iterations of the reference serial GAUSS_SEIDEL_Solve, scaled to the %.1f iterations '
                             'a timed step takes on average (the FP64 GPU path takes the same iterates)'
                             % (out['n'], t['sample_iters'], fp64_iters),
                   'assemble_ms': round(t['assemble_ms'], 3), 'per_iteration_ms': round(t['per_iter_ms'], 3)}
        rg = out['rigid']
        gb = rg['begin_bytes'] / (rg['begin_ms'] * 1e-3) / 1e9
        ge = rg['end_bytes'] / (rg['end_ms'] * 1e-3) / 1e9
        rigid = {'bodies': rg['bodies'], 'contact_sides': rg['contact_sides'],
                 'kernels': 'k_rigid_begin / k_rigid_end (BODY_Dynamic_Step_Begin / End of every body)',
                 'begin_ms': round(rg['begin_ms'], 5), 'end_ms': round(rg['end_ms'], 5),
                 'begin_bytes': rg['begin_bytes'], 'end_bytes': rg['end_bytes'],
                 'begin_gbs': round(gb, 1), 'end_gbs': round(ge, 1), 'peak_gbs': peak,
                 'begin_frac': round(gb / peak, 3), 'end_frac': round(ge / peak, 3),
                 'timing': 'inside the step: begin after the previous step\'s solve, end right after a 5-sweep '
                           'solve whose reactions and layout it reads back from L2 (end_frac > 1 reflects that)',
                 'cpu_port_ms_per_1k_bodies': None if args.no_cpu_baseline
                 else round(rigid_cpu_sample(out['scene']), 3)}

        def mode_summary(r):
            reps = r['reps']
            return {'ms_per_step': round(r['ms'], 4), 'iters_per_step': r['iters'],
                    'iters_mean': round(float(np.mean(r['iters'])), 2),
                    'iters_fp32_per_step': [x['iters_mixed'] for x in reps],
                    'solve_kernel_ms_mean': [round(float(np.mean([x['ms_kernel'][j] for x in reps])), 4)
                                             for j in (0, 1)],
                    'sweeps_per_step': [x['sweeps_launch'] for x in reps], 'grid': reps[-1]['grid'],
                    'last_merit': r['merit'], 'last_error': r['error'],
                    'assemble_ms_last': round(r['assemble_ms'], 4),
                    'reaction_rel_diff_vs_fp64_last_step': _rel2(r['R'], fp64['R'])}
        nn = mnn['nn']
        line = {
            'metric': METRIC, 'value': round(head['ms'], 4), 'unit': 'ms', 'n_gpus': ws, 'steps': args.steps,
            'warmup': args.warmup, 'ms_per_step': round(head['ms'], 4), 'higher_is_better': False,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'f64+f32 (mixed)',
            'data': 'synthetic (seeded scene generator)',
            'config': {'workload': WORKLOAD, 'contacts': out['n'], 'blocks': out['K'], 'bodies': out['nbod'],
                       'colours': out['ncolours'],
                       'run': 'time loop from rest under gravity: %d untimed steps, then %d timed consecutive steps; '
                              'each step = BODY_Dynamic_Step_Begin + LOCDYN_Update_Begin + solve + '
                              'BODY_Dynamic_Step_End on the device, warm start = the previous step\'s R, U'
                              % (args.warmup, args.steps),
                       'mode': '%s: FP32 off-diagonal sweeps, FP64 diagonal solves, merit and closing refinement%s'
                               % (HEADLINE, ', learned warm start kept when its merit is lower'
                                  if HEADLINE == 'mixed_nn' else ', warm start from the previous step (the '
                                  'learned start, never accepted in the time loop, is the mixed_nn mode)'),
                       'solver': 'GAUSS_SEIDEL_SOLVER(epsilon=%g, maxiter=%d, meritval=%g, SEMISMOOTH_NEWTON): '
                                 'the merit test decides (time to merit 1e-4); the modes *_ref_rule use the '
                                 'reference\'s epsilon = meritval = 1e-4' % (SOLVE['epsilon'], SOLVE['maxiter'],
                                                                          SOLVE['meritval']),
                       'l2': 'sweep working set > 126 MB L2 (W planes %.0f MB FP64 / %.0f MB FP32)'
                             % (out['K'] * 72 / 1e6, out['K'] * 36 / 1e6),
                       'parallelism': 'replicas' if ws > 1 else 'single GPU'},
            'modes': {m: mode_summary(r) for m, r in res.items()},
            'fp64_iters_from_rest': fp64['iters_all'],
            'speedup_mixed_vs_fp64': round(fp64['ms'] / mixed['ms'], 3),
            'speedup_mixed_nn_vs_fp64': round(fp64['ms'] / mnn['ms'], 3),
            'mixed_vs_fp64_converged': out['converged'],
            'warm_start': None if not nn else {
                'network_start_used_steps': sum(1 for q in nn if q['used_nn']), 'steps': len(nn),
                'merit_network_start': [q['merit_nn'] for q in nn],
                'merit_previous_step_start': [q['merit_plain'] for q in nn],
                'network_and_merit_ms_mean': round(float(np.mean([q['ms'] for q in nn])), 4)},
            'roofline': roof, 'roofline_fp64': roof64,
            'cpu_baseline': cpu,
            'e2e': {'value': round(out['e2e_ms'], 4), 'unit': 'ms', 'h2d_bytes_per_step': out['h2d'],
                    'd2h_bytes_per_step': out['d2h'],
                    'what': 'the timed steps of the %s run replayed through the C ABI from pinned host '
                            'buffers: bodies, contacts and the previous result up, assembly, %ssolve, R, U and '
                            'per-contact merit down' % (HEADLINE, 'learned warm start, ' if HEADLINE == 'mixed_nn'
                                                        else '')},
            'gpu_launches': int(head['launches']),
            'clocks': out['clocks'],
            'rigid_step': rigid,
            'configs': configs,
            'config3_detected': detected,
        }
        try:
            line['detect'] = detect_timing()
        except Exception as e:  # the headline line is printed whatever happens here
            line['detect'] = {'error': str(e)[:300]}
        try:
            line['detect_convex'] = detect_convex_timing()
        except Exception as e:
            line['detect_convex'] = {'error': str(e)[:300]}
        print(json.dumps(line), flush=True)
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == '__main__':
    main()
