"""GPU parity of the B200 contact-solve path against the CPU oracle.

Every test here calls the sm_100a library through its C ABI
(include/solfec_b200.h via solfec_b200.solver) and checks the result against
the C restatement of the reference solver (oracle/), itself pinned bit for bit
to the reference's compiled GAUSS_SEIDEL_Solve by tests/test_oracle.py.

Tolerances. The FP64 path reproduces the reference arithmetic operation for
operation (no multiply-add contraction, off-diagonal products added in list
order), so with the oracle run on the same colour-sorted row order the
reactions and velocities are bitwise equal and the iteration counts equal;
only the error and merit sums (parallel reductions) differ in the last bits,
checked to 1e-13 relative. The acceptance bar of 1e-6 relative is therefore
met with room. Mixed precision is checked against a converged FP64 solution
on a well-posed (diagonally dominant) problem to 1e-6 after its closing FP64
refinement, and to merit <= epsilon on the settled pile. Assembly: bitwise.
"""
import numpy as np
import pytest

import oracle as O
from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, SolfecError, scenes
from solfec_b200.solver import DeviceError

pytestmark = pytest.mark.gpu

SEED = 0xC0FFEE


def rel(a, b):
    """max |a - b| / max |b| over finite entries; NaN where one side is NaN
    and the other is not."""
    a = np.asarray(a, float).ravel(); b = np.asarray(b, float).ravel()
    na, nb = np.isnan(a), np.isnan(b)
    if np.any(na != nb):
        return float('nan')
    a, b = a[~na], b[~nb]
    den = max(np.abs(b).max(initial=0.0), 1e-300)
    return float(np.abs(a - b).max(initial=0.0) / den)


def same_bits(a, b):
    a = np.asarray(a, float).ravel(); b = np.asarray(b, float).ravel()
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def gpu_solve(ld, R0=None, U0=None, precision='FP64', reverse=False, nomerit=False, stage_blocks=0, **kw):
    ldy = LOCDYN()
    ldy.set_colour_seed(SEED)
    ldy.set(ld)
    if R0 is not None or U0 is not None:
        ldy.set_state(R0, U0)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    gs.precision = precision
    if reverse:
        gs.reverse = 'ON'
    if nomerit:
        gs.nomerit = True
    if stage_blocks:
        gs.set_stage_blocks(stage_blocks)
    exc = None
    try:
        gs.solve(ldy)
    except SolfecError as e:
        exc = e
    R, U, cm = ldy.get_state()
    return dict(gs=gs, ldy=ldy, R=R, U=U, cm=cm, order=ldy.order(), colours=ldy.colours(), exc=exc,
                merit=ldy.merit)


def oracle_in_order(ld, order, R0=None, U0=None, **kw):
    n = ld.n
    R0 = np.zeros((n, 3)) if R0 is None else np.asarray(R0).reshape(n, 3)
    U0 = np.zeros((n, 3)) if U0 is None else np.asarray(U0).reshape(n, 3)
    res = O.solve(ld.permuted(order), R=R0[order].ravel(), U=U0[order].ravel(), **kw)
    R = np.empty((n, 3)); U = np.empty((n, 3)); cm = np.empty(n)
    R[order] = res['R'].reshape(-1, 3); U[order] = res['U'].reshape(-1, 3); cm[order] = res['conmerit']
    res.update(R=R, U=U, conmerit=cm)
    return res


@pytest.fixture(scope='module')
def ld1k(scene_cache):
    return O.assemble(scene_cache('spheres_lattice'))


def test_colouring_bit_exact(ld1k):
    g = gpu_solve(ld1k, epsilon=1e-4, maxiter=1)
    nc, col = O.colour(ld1k, SEED)
    assert np.array_equal(g['colours'], col)
    assert np.array_equal(g['order'], O.colour_order(col))
    # no two adjacent rows share a colour
    rows = np.repeat(np.arange(ld1k.n), np.diff(ld1k.adjptr))
    assert not np.any(col[rows] == col[ld1k.adjcol])


def test_fp64_parity_merit(ld1k):
    kw = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
    g = gpu_solve(ld1k, **kw)
    o = oracle_in_order(ld1k, g['order'], **kw)
    assert g['gs'].error == 'OK' and o['error'] == 0
    assert g['gs'].iters == o['iters'], (g['gs'].iters, o['iters'])
    assert same_bits(g['R'], o['R']) and same_bits(g['U'], o['U'])
    assert g['merit'] <= 1e-4 and o['merit'] <= 1e-4
    np.testing.assert_allclose(g['gs'].rerhist, o['rerhist'], rtol=1e-13, atol=0)
    np.testing.assert_allclose(g['gs'].merhist, o['merhist'], rtol=1e-13, atol=0)
    np.testing.assert_allclose(g['merit'], o['merit'], rtol=1e-13)
    np.testing.assert_allclose(g['cm'], o['conmerit'], rtol=1e-13, atol=1e-300)


def test_fp64_parity_nomerit_reverse(ld1k):
    kw = dict(epsilon=1e-6, maxiter=400)
    g = gpu_solve(ld1k, reverse=True, **kw)
    o = oracle_in_order(ld1k, g['order'], reverse=True, **kw)
    assert g['gs'].iters == o['iters']
    assert same_bits(g['R'], o['R']) and same_bits(g['U'], o['U'])
    assert g['merit'] == 0.0


@pytest.mark.parametrize('precision', ['FP64', 'MIXED'])
def test_staging_windows_parity(ld1k, precision):
    # a 64-block staging window splits every tile of the pile (up to ~270
    # blocks) into several windows; the result must not change
    kw = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
    g = gpu_solve(ld1k, precision=precision, stage_blocks=64, **kw)
    h = gpu_solve(ld1k, precision=precision, **kw)
    assert g['gs'].iters == h['gs'].iters
    assert same_bits(g['R'], h['R']) and same_bits(g['U'], h['U'])
    if precision == 'FP64':
        o = oracle_in_order(ld1k, g['order'], **kw)
        assert same_bits(g['R'], o['R']) and same_bits(g['U'], o['U'])
    kw = dict(epsilon=1e-6, maxiter=300)
    g = gpu_solve(ld1k, precision=precision, stage_blocks=64, reverse=True, **kw)
    h = gpu_solve(ld1k, precision=precision, reverse=True, **kw)
    assert g['gs'].iters == h['gs'].iters and same_bits(g['R'], h['R'])


def test_warm_start_parity(ld1k, scene_cache):
    kw = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
    first = gpu_solve(ld1k, **kw)
    sc = scenes.advance_velocities(scene_cache('spheres_lattice'), first['R'])
    ld2 = O.assemble(sc)
    g = gpu_solve(ld2, R0=first['R'], U0=first['U'], **kw)
    o = oracle_in_order(ld2, g['order'], R0=first['R'], U0=first['U'], **kw)
    assert g['gs'].iters == o['iters']
    assert g['gs'].iters < first['gs'].iters
    assert same_bits(g['R'], o['R']) and same_bits(g['U'], o['U'])


@pytest.mark.parametrize('diagsolver', ['PROJECTED_GRADIENT', 'DE_SAXCE_FENG', 'PROJECTED_NEWTON'])
def test_other_diagonal_solvers(ld1k, diagsolver):
    kw = dict(epsilon=1e-4, maxiter=60, meritval=1e-4, diagsolver=diagsolver)
    g = gpu_solve(ld1k, **kw)
    o = oracle_in_order(ld1k, g['order'], **kw)
    assert g['gs'].iters == o['iters']
    assert same_bits(g['R'], o['R']) and same_bits(g['U'], o['U'])  # NaN patterns included (PROJECTED_NEWTON from U = 0)
    assert g['gs'].error == ('OK', 'DIVERGED', 'DIAGONAL_DIVERGED', 'DIAGONAL_FAILED')[o['error']]


def test_mixed_precision_pile(ld1k):
    """Settled pile: the mixed solve (FP32 off-diagonal sweeps, FP64 diagonal
    solves and merit, closing FP64 refinement) meets the FP64-evaluated merit
    bar in about as many iterations as the FP64 solve."""
    kw = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
    g = gpu_solve(ld1k, precision='MIXED', **kw)
    f = gpu_solve(ld1k, **kw)
    assert g['gs'].error == 'OK' and g['merit'] <= 1e-4
    assert 1 <= g['gs'].iters_mixed < g['gs'].iters
    assert g['gs'].iters <= 1.25 * f['gs'].iters + 5
    # the pile is hyperstatic: both are 1e-4-accurate members of a family of solutions
    assert rel(g['R'], f['R']) < 5e-2


def test_mixed_precision_converged():
    """Well-posed problem (the pile's local dynamics with off-diagonal blocks
    scaled by 0.25, so the solution is unique): converged mixed-precision
    reactions agree with the converged FP64 oracle within 1e-6 relative."""
    ld = O.assemble(scenes.spheres_lattice())
    ld.Woff = ld.Woff * 0.25
    kw = dict(epsilon=1e-10, maxiter=2000, meritval=1e-14)
    g = gpu_solve(ld, precision='MIXED', **kw)
    o = oracle_in_order(ld, g['order'], **kw)
    assert o['error'] == 0 and g['gs'].error == 'OK'
    assert rel(g['R'], o['R']) < 1e-6, rel(g['R'], o['R'])
    assert g['merit'] <= 1e-14


def test_failure_exit_diverged(ld1k):
    g = gpu_solve(ld1k, epsilon=1e-10, maxiter=5, meritval=1e-12, failure='EXIT')
    o = oracle_in_order(ld1k, g['order'], epsilon=1e-10, maxiter=5, meritval=1e-12, failure='EXIT')
    assert g['exc'] is not None and g['exc'].code == 45 and o['thrown'] == 45
    assert g['gs'].iters == 5 and g['gs'].error == 'DIVERGED'
    assert same_bits(g['R'], o['R'])


def test_failure_callback_counts(ld1k):
    calls = []
    g = gpu_solve(ld1k, epsilon=1e-10, maxiter=3, meritval=1e-12, failure='CALLBACK',
                  callback=lambda d: calls.append(d), data='x')
    o = oracle_in_order(ld1k, g['order'], epsilon=1e-10, maxiter=3, meritval=1e-12, failure='CALLBACK')
    assert len(calls) == o['ncallbacks'] == 1 and calls[0] == 'x'


def test_diagonal_failure_exit():
    """A row whose diagonal block is singular (W = 0) makes the semismooth
    Newton step fail (dgesv info > 0): FAILURE_EXIT raises the diagonal code."""
    n = 2
    W = np.tile(np.eye(3).ravel(), n); W[0:9] = 0.0
    A = np.tile(np.eye(3).ravel(), n)
    ld = O.LocalDynamics(W, A, np.ones(n), np.tile([0.1, 0.0, -1.0], n), np.zeros(3 * n), -np.ones(n) * 1e-3,
                         np.full(n, 0.3), np.zeros(n), np.zeros(n), np.zeros(n + 1, np.int32), np.zeros(0, np.int32),
                         np.zeros(0), 1.0, 1e-3, 1)
    g = gpu_solve(ld, epsilon=1e-4, maxiter=10, failure='EXIT')
    o = oracle_in_order(ld, g['order'], epsilon=1e-4, maxiter=10, failure='EXIT')
    assert o['thrown'] == 44 and g['exc'] is not None and g['exc'].code == 44
    assert g['gs'].error == ('OK', 'DIVERGED', 'DIAGONAL_DIVERGED', 'DIAGONAL_FAILED')[o['error']]
    c = gpu_solve(ld, epsilon=1e-4, maxiter=10)
    oc = oracle_in_order(ld, c['order'], epsilon=1e-4, maxiter=10)
    assert c['gs'].error == ('OK', 'DIVERGED', 'DIAGONAL_DIVERGED', 'DIAGONAL_FAILED')[oc['error']]
    assert same_bits(c['R'], oc['R'])


def test_diagonal_failure_mixed_precision():
    """The same singular row in mixed precision: the FP32 sweeps' Newton step
    (Cramer's rule) meets a zero determinant, the failure is reported as in
    FP64 (FAILURE_EXIT raises the diagonal code; CONTINUE runs the fallback
    chain and ends with the same error code and reactions within 1e-6)."""
    n = 2
    W = np.tile(np.eye(3).ravel(), n); W[0:9] = 0.0
    A = np.tile(np.eye(3).ravel(), n)
    ld = O.LocalDynamics(W, A, np.ones(n), np.tile([0.1, 0.0, -1.0], n), np.zeros(3 * n), -np.ones(n) * 1e-3,
                         np.full(n, 0.3), np.zeros(n), np.zeros(n), np.zeros(n + 1, np.int32), np.zeros(0, np.int32),
                         np.zeros(0), 1.0, 1e-3, 1)
    g = gpu_solve(ld, epsilon=1e-4, maxiter=10, failure='EXIT', precision='MIXED')
    assert g['exc'] is not None and g['exc'].code == 44
    m = gpu_solve(ld, epsilon=1e-4, maxiter=10, precision='MIXED')
    f = gpu_solve(ld, epsilon=1e-4, maxiter=10)
    assert m['gs'].error == f['gs'].error
    assert np.all(np.isfinite(m['R'])) and np.abs(m['R'] - f['R']).max() <= 1e-6 * max(1.0, np.abs(f['R']).max())


def test_empty_and_single():
    ld0 = O.LocalDynamics(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0),
                          np.zeros(0), np.zeros(0), np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0), 0.0,
                          1e-3, 1)
    g = gpu_solve(ld0, epsilon=1e-4, maxiter=10, meritval=1e-4)
    o = O.solve(ld0, epsilon=1e-4, maxiter=10, meritval=1e-4)
    assert g['gs'].iters == o['iters'] == 1 and g['gs'].error == 'OK'
    W = np.array([2.0, 0.1, 0.0, 0.1, 2.0, 0.0, 0.0, 0.0, 3.0])
    ld1 = O.LocalDynamics(W, np.linalg.inv(W.reshape(3, 3).T).T.ravel(), [0.3], [0.05, -0.02, -1.0], [0, 0, -0.5],
                          [-1e-4], [0.3], [0.0], [0.0], np.array([0, 0], np.int32), np.zeros(0, np.int32),
                          np.zeros(0), 0.5, 1e-3, 1)
    g = gpu_solve(ld1, epsilon=1e-8, maxiter=50, meritval=1e-10)
    o = O.solve(ld1, epsilon=1e-8, maxiter=50, meritval=1e-10)
    assert g['gs'].iters == o['iters']
    assert same_bits(g['R'], o['R'].reshape(-1, 3))


def test_assembly_parity(scene_cache):
    sc = scene_cache('spheres_lattice')
    ld = O.assemble(sc)
    ldy = LOCDYN()
    ldy.set_colour_seed(SEED)
    ldy.update_begin(sc)
    d = ldy.download()
    assert np.array_equal(d['adjptr'], ld.adjptr) and np.array_equal(d['adjcol'], ld.adjcol)
    for k in ('W', 'A', 'rho', 'B', 'V', 'Woff'):
        assert same_bits(d[k], getattr(ld, k)), (k, rel(d[k], getattr(ld, k)))
    assert abs(d['free_energy'] - ld.free_energy) <= 1e-13 * abs(ld.free_energy)  # parallel sum
    nc, col = O.colour(ld, SEED)
    assert np.array_equal(ldy.colours(), col)


@pytest.mark.parametrize('scene', ['spheres_lattice', 'hexahedra_small'])
def test_assembly_parity_on_a_kept_layout(scene_cache, scene):
    """Assemblies after the first on an unchanged contact topology (the
    second builds the body-pair table, later ones reuse it) write W_ij from
    the body pairs instead of per block: bitwise the oracle's blocks, on moved
    bodies too."""
    import dataclasses
    from solfec_b200._lib import lib
    from solfec_b200.dynamics import RIGID_DYNAMICS
    sc = scene_cache('spheres_lattice') if scene == 'spheres_lattice' else \
        scene_cache('hexahedra_lattice', nx=12, ny=12, nz=4)
    J = np.stack([np.eye(3).reshape(9) if o else np.linalg.inv(j.reshape(3, 3).T).T.reshape(9)
                  for j, o in zip(sc.jinv, sc.obstacle != 0)])
    mass = np.where(sc.obstacle != 0, 1.0, 1.0 / np.where(sc.obstacle != 0, 1.0, sc.minv))
    ldy = LOCDYN()
    ldy.update_begin(sc)
    dyn = RIGID_DYNAMICS(ldy, J, mass, sc.x)
    for step in range(3):
        dyn.step_begin(sc.step, (0.0, 0.0, -9.81))
        assert lib().b2gs_locdyn_update_begin_resident(ldy.handle, sc.step, int(sc.dynamic)) == 0
        st = dyn.state()
        cur = dataclasses.replace(sc, rot=st['rot'], x=st['x'], velo=st['velo'], velo0=st['velo0'])
        ld = O.assemble(cur)
        d = ldy.download()
        assert np.array_equal(d['adjcol'], ld.adjcol)
        for k in ('W', 'Woff', 'B', 'V'):
            assert same_bits(d[k], getattr(ld, k)), (step, k, rel(d[k], getattr(ld, k)))
        ldy.set_state(np.zeros((sc.ncon, 3)), np.zeros((sc.ncon, 3)))
        gs = GAUSS_SEIDEL_SOLVER(1e-4, 5)
        gs.solve(ldy)
        dyn.step_end(sc.step)
    # another topology of the same sizes (roles swapped where both bodies move):
    # the row pass expected the pair kernel, the per-block kernel runs instead
    swap = (sc.slave >= 0) & (sc.obstacle[np.maximum(sc.slave, 0)] == 0)
    sc2 = dataclasses.replace(sc, master=np.where(swap, sc.slave, sc.master).astype(np.int32),
                              slave=np.where(swap, sc.master, sc.slave).astype(np.int32),
                              mpnt=np.where(swap[:, None], sc.spnt, sc.mpnt),
                              spnt=np.where(swap[:, None], sc.mpnt, sc.spnt))
    assert swap.any()
    ldy.update_begin(sc2)
    ld = O.assemble(sc2)
    d = ldy.download()
    for k in ('W', 'Woff', 'B', 'V'):
        assert same_bits(d[k], getattr(ld, k)), ('swapped', k, rel(d[k], getattr(ld, k)))
    ldy.close()


def test_hexahedra_assembly_and_solve(scene_cache):
    sc = scene_cache('hexahedra_lattice', nx=12, ny=12, nz=4)
    ld = O.assemble(sc)
    ldy = LOCDYN()
    ldy.set_colour_seed(SEED)
    ldy.update_begin(sc)
    d = ldy.download()
    for k in ('W', 'A', 'rho', 'B', 'V', 'Woff'):
        assert same_bits(d[k], getattr(ld, k)), (k, rel(d[k], getattr(ld, k)))
    gs = GAUSS_SEIDEL_SOLVER(1e-4, 1000, 1e-4)
    gs.solve(ldy)
    R, U, _ = ldy.get_state()
    o = oracle_in_order(ld, ldy.order(), epsilon=1e-4, maxiter=1000, meritval=1e-4)
    assert gs.iters == o['iters']
    assert same_bits(R, o['R']) and same_bits(U, o['U'])


def test_list_order_colouring_and_reuse(scene_cache):
    # default mode: greedy colouring in list order, bit-exact against the host
    for sc in (scene_cache('spheres_lattice'), scene_cache('hexahedra_lattice', nx=20, ny=20, nz=6)):
        ld = O.assemble(sc)
        ldy = LOCDYN()
        ldy.update_begin(sc)
        nc, col = O.colour(ld, None)
        assert np.array_equal(ldy.colours(), col)
        assert ldy.sizes()[2] == nc
        order0 = ldy.order()
        # same contact graph: the colouring is reused, the layout is the same
        reuse0 = ldy.colour_reuse_count()
        ldy.update_begin(scenes.advance_velocities(sc, np.zeros((sc.ncon, 3))))
        assert ldy.colour_reuse_count() == reuse0 + 1
        assert np.array_equal(ldy.order(), order0) and np.array_equal(ldy.colours(), col)
        # and the solve is the oracle's in that order
        gs = GAUSS_SEIDEL_SOLVER(1e-4, 1000, 1e-4)
        gs.solve(ldy)
        R, U, _ = ldy.get_state()
        ld2 = O.assemble(scenes.advance_velocities(sc, np.zeros((sc.ncon, 3))))
        o = oracle_in_order(ld2, ldy.order(), epsilon=1e-4, maxiter=1000, meritval=1e-4)
        assert gs.iters == o['iters'] and same_bits(R, o['R']) and same_bits(U, o['U'])
        ldy.close()
    # the lattice's contact graph is the line graph of a degree-6 bipartite graph: 6 colours in list order
    ld = O.assemble(scene_cache('hexahedra_lattice', nx=20, ny=20, nz=6))
    assert O.colour(ld, None)[0] == 6
    # another graph is coloured again
    ldy = LOCDYN()
    ldy.update_begin(scene_cache('spheres_lattice'))
    ldy.update_begin(scene_cache('hexahedra_lattice', nx=20, ny=20, nz=6))
    assert ldy.colour_reuse_count() == 0
    ldy.close()


def test_polydisperse_pile_against_compiled_reference():
    """Config 2 shape (polydisperse spheres, friction 0.5, h = 5e-4, epsilon =
    meritval = 1e-6), scaled to 4,000 bodies: the FP64 GPU solve against the
    reference's own GAUSS_SEIDEL_Solve (oracle/_ref, compiled from its sources)
    on identical W and B in the GPU's row order; falls back to the oracle where
    the compiled reference is absent."""
    sc = scenes.spheres_polydisperse(seed=2, n=4000)
    ld = O.assemble(sc)
    kw = dict(epsilon=1e-6, maxiter=1000, meritval=1e-6)
    ldy = LOCDYN()
    ldy.set(ld)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    gs.solve(ldy)
    R, U, _ = ldy.get_state()
    impl = 'ref' if O.ref_available() else 'oracle'
    order = ldy.order()
    res = O.solve(ld.permuted(order), impl=impl, **kw)
    Rr = np.empty((ld.n, 3)); Ur = np.empty((ld.n, 3))
    Rr[order] = res['R'].reshape(-1, 3); Ur[order] = res['U'].reshape(-1, 3)
    assert gs.iters == res['iters']
    assert same_bits(R, Rr) and same_bits(U, Ur)
    assert ldy.merit <= 1e-6 or gs.iters == 1000
    ldy.close()


def test_layout_reuse_follows_tile_rows(scene_cache):
    """An unchanged contact graph reuses the colouring and the colour-sorted
    layout with its tile table; a change of rows per tile in between rebuilds
    the tile table. Every solve equals a fresh context's bitwise (rows per tile
    never change results)."""
    from solfec_b200._lib import lib
    sc = scene_cache('hexahedra_lattice', nx=20, ny=20, nz=6)
    nxt = scenes.advance_velocities(sc, np.zeros((sc.ncon, 3)))

    def solve(ldy):
        gs = GAUSS_SEIDEL_SOLVER(1e-4, 1000, 1e-4)
        gs.solve(ldy)
        R, U, _ = ldy.get_state()
        return gs.iters, R, U

    fresh = LOCDYN()
    fresh.update_begin(nxt)
    ref = solve(fresh)
    fresh.close()
    ldy = LOCDYN()
    ldy.update_begin(sc)
    for rows in (8, 8, 32, 16):
        assert lib().b2dev_set_tile_rows(ldy.device_context, rows) == 0
        reuse0 = ldy.colour_reuse_count()
        ldy.update_begin(nxt)
        assert ldy.colour_reuse_count() == reuse0 + 1
        assert lib().b2dev_tile_rows(ldy.device_context) == rows
        it, R, U = solve(ldy)
        assert it == ref[0] and same_bits(R, ref[1]) and same_bits(U, ref[2])
    ldy.close()


@pytest.mark.parametrize('dynamic', [1, 0])
def test_bilateral_constraints_parity(ld1k, scene_cache, dynamic):
    """FIXPNT, FIXDIR, VELODIR, VELODIR3 and RIGLNK rows among the pile's
    contacts (b2dev_set_kinds; the KINDS solve kernels): FP64 bitwise with the
    oracle in the GPU's row order (which equals the compiled reference, tests/
    test_oracle.py), iterations and merit included; mixed precision reaches
    merit 1e-4 too, its reactions within 1e-2 of FP64's at that merit."""
    from kinds_data import bilateral_kinds, riglnk_gap
    sc = scene_cache('spheres_lattice')
    ld = ld1k.permuted(np.arange(ld1k.n))
    ld.dynamic = dynamic
    kinds, Z = bilateral_kinds(ld.n, bodies=(sc.master, sc.slave, sc.obstacle))
    ld.gap = riglnk_gap(kinds, Z, ld.gap)
    kw = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
    out = {}
    for precision in ('FP64', 'MIXED'):
        ldy = LOCDYN()
        ldy.set_colour_seed(SEED)
        ldy.set(ld)
        ldy.set_kinds(kinds, Z)
        gs = GAUSS_SEIDEL_SOLVER(**kw)
        gs.precision = precision
        gs.solve(ldy)
        R, U, cm = ldy.get_state()
        out[precision] = dict(R=R, U=U, cm=cm, iters=gs.iters, merit=ldy.merit, order=ldy.order(), error=gs.error)
        ldy.close()
    g = out['FP64']
    order = g['order']
    res = O.solve(ld.permuted(order), kinds=kinds[order], Z=Z[order], **kw)
    R = np.empty((ld.n, 3)); U = np.empty((ld.n, 3))
    R[order] = res['R'].reshape(-1, 3); U[order] = res['U'].reshape(-1, 3)
    assert g["iters"] == res["iters"] < 1000, (g["iters"], res["iters"])
    assert same_bits(g['R'], R) and same_bits(g['U'], U)
    np.testing.assert_allclose(g['merit'], res['merit'], rtol=1e-13)
    m = out['MIXED']
    assert m['merit'] <= 1e-4 and g['merit'] <= 1e-4
    assert rel(m['R'], g['R']) < 1e-2
    # every row kind present, and a kinds-free solve is a different problem
    assert set(np.unique(kinds)) == {0, 1, 2, 3, 4, 5}
    assert not same_bits(gpu_solve(ld, **kw)['R'], g['R'])


def test_spring_kind_rejected(ld1k):
    """SPRING rows (kind 6) and kinds outside dom.h:98 are refused; kinds of a
    wrong length too; None makes every row a contact again."""
    ldy = LOCDYN()
    ldy.set_colour_seed(SEED)
    ldy.set(ld1k)
    for bad in (np.full(ld1k.n, 6), np.full(ld1k.n, -1), np.zeros(ld1k.n - 1)):
        with pytest.raises(DeviceError):
            ldy.set_kinds(bad)
    ldy.set_kinds(None)
    gs = GAUSS_SEIDEL_SOLVER(1e-4, 1000, 1e-4)
    gs.solve(ldy)
    R, _, _ = ldy.get_state()
    assert same_bits(R, gpu_solve(ld1k, epsilon=1e-4, maxiter=1000, meritval=1e-4)['R'])
    ldy.close()
