"""GPU tests of the batched solve (many independent scenes, one persistent
launch, per-scene stopping decisions).

Every scene of the batch must come out exactly as the reference solver
(the oracle, itself pinned to the compiled reference) solves that scene alone
in the same row order: reactions and velocities bitwise, the same iteration
count. The device sums the free energy of each scene in its own order, so
the oracle is given the device's value. The CUDA graph replay and the
autotuned launch shapes must not change any result.
"""
import numpy as np
import pytest

import oracle as O
from solfec_b200 import GAUSS_SEIDEL_SOLVER, scenes
from solfec_b200.batch import BatchSolver

pytestmark = pytest.mark.gpu

KW = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)


def same_bits(a, b):
    a = np.asarray(a, float).ravel(); b = np.asarray(b, float).ravel()
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.fixture(scope='module')
def batch():
    rng = np.random.default_rng(5)
    sizes = [50, 80, 120, 200, 320, 60, 500, 90, 150, 700, 75, 260]
    sc = [scenes.spheres_small(900 + k, n, friction=float(rng.uniform(0.2, 0.6)), settle_iters=300)
          for k, n in enumerate(sizes)]
    return sc


def per_problem_order(bs, k):
    order = bs.ldy.order()
    lo, hi = bs.offsets[k], bs.offsets[k + 1]
    sel = order[(order >= lo) & (order < hi)]
    return sel - lo


def test_batch_matches_oracle_per_scene(batch):
    bs = BatchSolver(batch)
    gs = GAUSS_SEIDEL_SOLVER(**KW)
    res = bs.solve(gs, use_graph=False, histories=True)
    R, U, _ = bs.state()
    fe = bs.free_energy()
    assert np.all(res.iters >= 1) and len(set(res.iters.tolist())) > 1  # scenes stop at different sweeps
    for k, sc in enumerate(batch):
        lo, hi = bs.offsets[k], bs.offsets[k + 1]
        ld = O.assemble(sc)
        ld.free_energy = float(fe[k])
        order = per_problem_order(bs, k)
        o = O.solve(ld.permuted(order), **KW)
        Rk = np.empty((ld.n, 3)); Uk = np.empty((ld.n, 3))
        Rk[order] = o['R'].reshape(-1, 3); Uk[order] = o['U'].reshape(-1, 3)
        assert res.iters[k] == o['iters'], (k, res.iters[k], o['iters'])
        assert same_bits(R[lo:hi], Rk) and same_bits(U[lo:hi], Uk), k
        np.testing.assert_allclose(res.merit[k], o['merit'], rtol=1e-12)
        np.testing.assert_allclose(res.rerhist[k, :res.iters[k]], o['rerhist'], rtol=1e-12)
        assert res.ms_to_decision[k] > 0.0
    assert res.ms_to_decision.max() <= res.ms_device * 1.01
    bs.close()


def test_graph_replay_and_autotune_do_not_change_results(batch):
    bs = BatchSolver(batch)
    gs = GAUSS_SEIDEL_SOLVER(**KW)
    R0, U0, _ = bs.state()
    ref = bs.solve(gs, use_graph=False)
    Rref, Uref, _ = bs.state()
    for _ in range(2):  # capture, then replay
        bs.set_state(R0, U0)
        g = bs.solve(gs, use_graph=True)
        R, U, _ = bs.state()
        assert np.array_equal(g.iters, ref.iters)
        assert same_bits(R, Rref) and same_bits(U, Uref)
    bs.set_state(R0, U0)
    tune = bs.autotune(gs)
    assert tune['tile_rows'] in (8, 16, 32) and tune['grid'] > 0 and len(tune['trials']) >= 6
    bs.set_state(R0, U0)
    t = bs.solve(gs, use_graph=True)
    R, U, _ = bs.state()
    assert np.array_equal(t.iters, ref.iters)
    assert same_bits(R, Rref) and same_bits(U, Uref)
    bs.close()
