"""Parity at the sizes of the stated configurations.

- Config 2 at full size (20,000 polydisperse spheres, friction 0.5,
  h = 5e-4, epsilon = meritval = 1e-6): the FP64 GPU solve against the
  reference's own GAUSS_SEIDEL_Solve (oracle/_ref, compiled from its sources;
  the C oracle where that build is absent) on identical W and B in the GPU's
  row order, bit for bit; and the mixed-precision solve run to a tight
  tolerance against the converged FP64 oracle within 1e-4 relative.
- The bench step (100 x 100 x 10 hexahedra, 302,000 contacts): a bounded
  FP64 solve (5 iterations) equals the oracle's bit for bit.
- A hexahedra lattice (40 x 40 x 8): mixed precision against FP64 from the
  same start in the same row order, both to merit 1e-6.

Tolerances: FP64 is bitwise (the path reproduces the reference arithmetic
operation for operation); the mixed precision's bar is 1e-4 relative.
"""
import numpy as np
import pytest

import oracle as O
from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, scenes

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4


def rel2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / max(np.linalg.norm(np.ravel(b)), 1e-300))


def same_bits(a, b):
    a = np.asarray(a, float).ravel(); b = np.asarray(b, float).ravel()
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def device_solve(src, precision='FP64', **kw):
    ldy = LOCDYN()
    if isinstance(src, scenes.Scene):
        ldy.update_begin(src)
    else:
        ldy.set(src)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    gs.precision = precision
    gs.solve(ldy)
    R, U, _ = ldy.get_state()
    out = dict(R=R, U=U, iters=gs.iters, iters_mixed=gs.iters_mixed, merit=ldy.merit, order=ldy.order(),
               error=gs.error)
    ldy.close()
    return out


def reference_in_order(ld, order, impl, **kw):
    res = O.solve(ld.permuted(order), impl=impl, **kw)
    n = ld.n
    R = np.empty((n, 3)); U = np.empty((n, 3))
    R[order] = res['R'].reshape(-1, 3); U[order] = res['U'].reshape(-1, 3)
    return dict(res, R=R, U=U)


def body_resultants(sc, R):
    """Force and torque of the contact reactions on every moving body (global
    frame): what the reactions do to the bodies (rig_constraints_force,
    bod.c:390-439). Reactions that differ by a self-equilibrated set of
    contact forces (the null space of a hyperstatic contact network) give the
    same resultants."""
    base = sc.base.reshape(-1, 3, 3)                     # column-major frames [t1 t2 n]
    f = np.einsum('kji,kj->ki', base, R)
    rot = sc.rot.reshape(-1, 3, 3).transpose(0, 2, 1)
    m, s = sc.master, sc.slave
    p = sc.x[m] + np.einsum('kij,kj->ki', rot[m], sc.mpnt - sc.x0[m])
    F = np.zeros((sc.nbod, 3)); T = np.zeros((sc.nbod, 3))
    np.add.at(F, m, f); np.add.at(T, m, np.cross(p - sc.x[m], f))
    ok = s >= 0
    np.add.at(F, s[ok], -f[ok]); np.add.at(T, s[ok], -np.cross(p[ok] - sc.x[s[ok]], f[ok]))
    mov = sc.obstacle == 0
    return F[mov], T[mov]


@pytest.fixture(scope='module')
def pile20k(scene_cache):
    return scene_cache('spheres_polydisperse', seed=2, n=20000)


def test_config2_fp64_full_size_against_reference(pile20k):
    ld = O.assemble(pile20k)
    kw = dict(epsilon=1e-6, maxiter=1000, meritval=1e-6)
    g = device_solve(ld, **kw)
    impl = 'ref' if O.ref_available() else 'oracle'
    r = reference_in_order(ld, g['order'], impl, **kw)
    assert ld.n > 10000
    assert g['iters'] == r['iters'] and r['error'] == 0
    assert same_bits(g['R'], r['R']) and same_bits(g['U'], r['U'])
    assert g['merit'] <= 1e-6


def test_config2_mixed_converged_against_fp64_oracle(pile20k):
    """Mixed precision (FP32 sweeps, FP64 diagonal solves, merit and closing
    refinement) run to epsilon 1e-10 / merit 1e-12 from the same start, in
    the same row order, as the FP64 oracle: converged reactions within 1e-4."""
    ld = O.assemble(pile20k)
    kw = dict(epsilon=1e-10, maxiter=6000, meritval=1e-12)
    g = device_solve(ld, precision='MIXED', **kw)
    o = reference_in_order(ld, g['order'], 'oracle', **kw)
    assert o['error'] == 0 and g['error'] == 'OK'
    assert g['merit'] <= 1e-12 and o['merit'] <= 1e-12
    assert 0 < g['iters_mixed'] < g['iters']          # FP32 sweeps first, FP64 to finish
    assert rel2(g['R'], o['R']) <= MIXED_TOL, rel2(g['R'], o['R'])
    assert rel2(g['U'], o['U']) <= MIXED_TOL, rel2(g['U'], o['U'])


def test_bench_step_bounded_fp64_bitwise():
    """The 302,000-contact bench scene: five FP64 sweeps equal the oracle's."""
    sc = scenes.hexahedra_lattice(seed=3, nx=100, ny=100, nz=10)
    ld = O.assemble(sc)
    kw = dict(epsilon=1.0, maxiter=5, meritval=1e-300)
    g = device_solve(sc, **kw)
    o = reference_in_order(ld, g['order'], 'oracle', **kw)
    assert ld.n == 302000 and g['iters'] == o['iters'] == 5
    assert same_bits(g['R'], o['R']) and same_bits(g['U'], o['U'])


def test_hexahedra_lattice_mixed_against_fp64_oracle():
    """A 40 x 40 x 8 hexahedra lattice settled by a 20-step device time loop
    (gravity, warm starts, the device integrator); the last step's local
    dynamics solved from zero reactions to merit 1e-7 (the stack's merit
    stalls near 4e-8) by mixed precision on the GPU and by the FP64 oracle in
    the same row order: reactions and per-body resultants within 1e-4."""
    from types import SimpleNamespace
    import ctypes as C
    import bench
    from solfec_b200._lib import lib
    from solfec_b200.dynamics import RIGID_DYNAMICS
    sc = scenes.hexahedra_lattice(seed=5, nx=40, ny=40, nz=8)
    J, mass = bench._rigid_inertia(sc)
    ldy = LOCDYN()
    ldy.update_begin(sc)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    gs = GAUSS_SEIDEL_SOLVER(epsilon=1.0, maxiter=1000, meritval=1e-4)
    R = np.zeros((sc.ncon, 3)); U = np.zeros((sc.ncon, 3))
    for _ in range(20):
        dyn.step_begin(sc.step, (0.0, 0.0, -9.81))
        assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, sc.step, 1) == 0
        ldy.set_state(R, U)
        gs.solve(ldy)
        R, U, _ = ldy.get_state()
        dyn.step_end(sc.step)
    dyn.step_begin(sc.step, (0.0, 0.0, -9.81))
    assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, sc.step, 1) == 0
    st = dyn.state()
    d = ldy.download()
    ldy.close()
    ld = SimpleNamespace(W=d['W'], A=d['A'], rho=d['rho'], B=d['B'], V=d['V'], gap=sc.gap, friction=sc.friction,
                         restitution=sc.restitution, cohesion=sc.cohesion, adjptr=d['adjptr'], adjcol=d['adjcol'],
                         Woff=d['Woff'], free_energy=d['free_energy'], step=sc.step, dynamic=sc.dynamic)
    ldo = O.LocalDynamics(ld.W, ld.A, ld.rho, ld.B, ld.V, ld.gap, ld.friction, ld.restitution, ld.cohesion, ld.adjptr,
                          ld.adjcol, ld.Woff, ld.free_energy, ld.step, ld.dynamic)
    kw = dict(epsilon=1.0, maxiter=20000, meritval=1e-7)
    g = device_solve(ldo, precision='MIXED', **kw)
    o = reference_in_order(ldo, g['order'], 'oracle', **kw)
    assert o['error'] == 0 and g['error'] == 'OK' and g['merit'] <= 1e-7 and o['merit'] <= 1e-7
    assert rel2(g['R'], o['R']) <= MIXED_TOL, rel2(g['R'], o['R'])
    rs = SimpleNamespace(base=sc.base, rot=st['rot'], x=st['x'], master=sc.master, slave=sc.slave, mpnt=sc.mpnt,
                         x0=sc.x0, nbod=sc.nbod, obstacle=sc.obstacle)
    Fg, Tg = body_resultants(rs, g['R'])
    Fo, To = body_resultants(rs, o['R'])
    assert rel2(Fg, Fo) <= MIXED_TOL and rel2(Tg, To) <= 10 * MIXED_TOL, (rel2(Fg, Fo), rel2(Tg, To))
