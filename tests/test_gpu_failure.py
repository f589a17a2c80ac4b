"""Failure paths of the device solve, made on the host side of the data (no
GPU fault): a bounded wait that runs out, and FAILURE_EXIT in the middle of
a sweep.

- Timeout. With a 1 ns limit on the solver's waits, any dependency not yet
  met at its first check gives up: the launch ends, the solve returns
  B2DEV_ETIMEOUT, and the context keeps its state; with the default limit
  back the next solve equals a fresh context's bit for bit.
- FAILURE_EXIT. The reference THROWs at the first failing diagonal solve
  (bgs.c:1005-1006), so the rows after it in the sweep keep their previous
  reactions; the device finishes the sweep (its rows of one colour run in
  parallel). Rows up to the failing one are bitwise the reference's; the
  later rows are the documented difference.
"""
import numpy as np
import pytest

import oracle as O
from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, DeviceError, SolfecError, scenes

pytestmark = pytest.mark.gpu


def same_bits(a, b):
    a = np.asarray(a, float).ravel(); b = np.asarray(b, float).ravel()
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_wait_timeout_reported_and_context_usable(scene_cache):
    sc = scene_cache('hexahedra_lattice', nx=40, ny=40, nz=8)
    ldy = LOCDYN()
    ldy.update_begin(sc)
    ldy.set_wait_limit(1e-9)
    gs = GAUSS_SEIDEL_SOLVER(epsilon=1.0, maxiter=200, meritval=1e-12)
    with pytest.raises(DeviceError, match='timed out'):
        gs.solve(ldy)
    ldy.set_wait_limit(0.0)
    kw = dict(epsilon=1.0, maxiter=20, meritval=1e-12)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    gs.solve(ldy)
    R, U, _ = ldy.get_state()
    fresh = LOCDYN()
    fresh.update_begin(sc)
    gf = GAUSS_SEIDEL_SOLVER(**kw)
    gf.solve(fresh)
    Rf, Uf, _ = fresh.get_state()
    assert gs.iters == gf.iters == 20
    assert same_bits(R, Rf) and same_bits(U, Uf)
    with pytest.raises(DeviceError):
        ldy.set_wait_limit(-1.0)
    ldy.close()
    fresh.close()


def test_failure_exit_mid_sweep(scene_cache):
    ld = O.assemble(scene_cache('spheres_lattice'))
    probe = LOCDYN()
    probe.set(ld)
    order = probe.order()
    probe.close()
    n = ld.n
    pos = n // 2
    m = int(order[pos])          # the row swept in the middle of the first sweep
    W = ld.W.copy()
    W[9 * m:9 * m + 9] = 0.0     # singular diagonal block: the semismooth Newton step fails there
    bad = O.LocalDynamics(W, ld.A, ld.rho, ld.B, ld.V, ld.gap, ld.friction, ld.restitution, ld.cohesion, ld.adjptr,
                          ld.adjcol, ld.Woff, ld.free_energy, ld.step, ld.dynamic)
    kw = dict(epsilon=1e-4, maxiter=10, meritval=1e-4, failure='EXIT')
    ldy = LOCDYN()
    ldy.set(bad)
    assert np.array_equal(ldy.order(), order)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    with pytest.raises(SolfecError) as e:
        gs.solve(ldy)
    assert e.value.code == 44 and gs.error == 'DIAGONAL_FAILED' and gs.iters == 0
    R, _, _ = ldy.get_state()
    ldy.close()
    res = O.solve(bad.permuted(order), **kw)
    assert res['thrown'] == 44
    Ro = np.empty((n, 3)); Ro[order] = res['R'].reshape(-1, 3)
    before = order[:pos + 1]     # swept up to and including the failing row: the reference's reactions
    after = order[pos + 1:]
    assert same_bits(R[before], Ro[before])
    # the reference left the later rows at their input (zero); the device updated them
    assert np.all(Ro[after] == 0.0)
    assert np.count_nonzero(R[after]) > 0
