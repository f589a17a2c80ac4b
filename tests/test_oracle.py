"""CPU tests of the oracle: the C restatement of the reference contact solve.

* Against the golden vectors that the reference's own GAUSS_SEIDEL_Solve
  produced (tests/golden/make_golden.py): every output bitwise.
* Against the reference compiled from its sources (oracle/_ref), where that
  build is present: every output bitwise, on the settled 1000-sphere pile in
  colour order and in a natural list order, for all diagonal solvers and
  failure actions.
* The restated assembly against an independent numpy computation of
  W = h H M^-1 H^T, and the symmetry W_ji = W_ij^T (ldy.c:829-844).
* The host colouring: a proper colouring, identical to a round-by-round
  Jones-Plassmann run in numpy with the same priorities.
"""
import glob
import os

import numpy as np
import pytest

import oracle as O
from kinds_data import bilateral_kinds, riglnk_gap
from solfec_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = sorted(glob.glob(os.path.join(HERE, 'golden', '*.npz')))


def bits(a):
    return np.ascontiguousarray(np.asarray(a, float)).view(np.uint64)


def same_bits(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return a.shape == b.shape and np.array_equal(bits(a), bits(b))


def load_fixture(path):
    z = np.load(path)
    fe, step, dyn = z['scalars']
    ld = O.LocalDynamics(z['W'], z['A'], z['rho'], z['B'], z['V'], z['gap'], z['friction'], z['restitution'],
                         z['cohesion'], z['adjptr'], z['adjcol'], z['Woff'], fe, step, int(dyn))
    kw = eval(str(z['options']), {})
    return ld, kw, z


def test_golden_fixtures_exist():
    assert len(GOLDEN) >= 8


@pytest.mark.parametrize('path', GOLDEN, ids=[os.path.basename(p)[:-4] for p in GOLDEN])
def test_oracle_reproduces_reference_golden_vectors(path):
    ld, kw, z = load_fixture(path)
    res = O.solve(ld, R=z['R0'], U=z['U0'], **kw)
    iters, error, merit, thrown, ncb = z['out']
    assert res['iters'] == int(iters) and res['error'] == int(error)
    assert res['thrown'] == int(thrown) and res['ncallbacks'] == int(ncb)
    assert same_bits(res['R'], z['R']) and same_bits(res['U'], z['U'])
    assert same_bits(res['conmerit'], z['conmerit'])
    assert same_bits([res['merit']], [merit])
    assert same_bits(res['rerhist'], z['rerhist']) and same_bits(res['merhist'], z['merhist'])


@pytest.fixture(scope='module')
def pile(scene_cache):
    sc = scene_cache('spheres_lattice')
    ld = O.assemble(sc)
    nc, col = O.colour(ld, 12345)
    return sc, ld, O.colour_order(col)


REF_CASES = [
    dict(epsilon=1e-4, maxiter=1000, meritval=1e-4),
    dict(epsilon=1e-5, maxiter=200, reverse=True),
    dict(epsilon=1e-4, maxiter=40, meritval=1e-4, diagsolver='PROJECTED_GRADIENT'),
    dict(epsilon=1e-4, maxiter=40, meritval=1e-4, diagsolver='DE_SAXCE_FENG'),
    dict(epsilon=1e-4, maxiter=10, meritval=1e-4, diagsolver='PROJECTED_NEWTON'),
    dict(epsilon=1e-10, maxiter=5, meritval=1e-12, failure='EXIT'),
    dict(epsilon=1e-10, maxiter=5, meritval=1e-12, failure='CALLBACK'),
]


@pytest.mark.skipif(not O.ref_available(), reason='reference solver build (oracle/_ref) not present')
@pytest.mark.parametrize('kw', REF_CASES, ids=lambda k: '-'.join('%s=%s' % it for it in sorted(k.items())))
@pytest.mark.parametrize('order_kind', ['colour', 'natural'])
def test_oracle_matches_compiled_reference(pile, kw, order_kind):
    sc, ld, corder = pile
    lp = ld.permuted(corder) if order_kind == 'colour' else ld
    a = O.solve(lp, impl='oracle', **kw)
    b = O.solve(lp, impl='ref', **kw)
    for k in ('iters', 'error', 'thrown', 'ncallbacks'):
        assert a[k] == b[k], k
    for k in ('R', 'U', 'conmerit', 'rerhist', 'merhist'):
        assert same_bits(a[k], b[k]), k
    assert same_bits([a['merit']], [b['merit']])


def _rot(v):
    return v.reshape(3, 3).T  # column-major storage -> matrix


def test_assembly_against_numpy(scene_cache):
    sc = scene_cache('hexahedra_lattice', nx=6, ny=5, nz=3)
    ld = O.assemble(sc)
    n = sc.ncon
    h = sc.step

    def Hmat(b, X, base):  # H = base^T [R skew(X - X0)^T | I] (bod.c:216-229)
        A = X - sc.x0[b]
        S = np.array([[0, -A[2], A[1]], [A[2], 0, -A[0]], [-A[1], A[0], 0]])
        return _rot(base).T @ np.hstack([_rot(sc.rot[b]) @ S.T, np.eye(3)])

    def Minv(b):
        M = np.zeros((6, 6)); M[:3, :3] = _rot(sc.jinv[b]); M[3:, 3:] = sc.minv[b] * np.eye(3)
        return M

    Hs = []
    for i in range(n):
        m, s = sc.master[i], sc.slave[i]
        Hm = Hmat(m, sc.mpnt[i], sc.base[i]); Hsl = Hmat(s, sc.spnt[i], sc.base[i])
        Hs.append((None if sc.obstacle[m] else Hm, None if (s < 0 or sc.obstacle[s]) else -Hsl))
        W = np.zeros((3, 3))
        for H, b in ((Hs[i][0], m), (Hs[i][1], s)):
            if H is not None:
                W += H @ Minv(b) @ H.T
        W *= h
        np.testing.assert_allclose(_rot(ld.W[9 * i:9 * i + 9]), W, rtol=1e-12, atol=1e-12 * np.abs(W).max())
        np.testing.assert_allclose(1.0 / ld.rho[i], np.linalg.eigvalsh(W).max(), rtol=1e-12)
        np.testing.assert_allclose(_rot(ld.A[9 * i:9 * i + 9]) @ W, np.eye(3), atol=1e-9)
        Bv = Hm @ sc.velo[m] - Hsl @ sc.velo[s]
        np.testing.assert_allclose(ld.B[3 * i:3 * i + 3], Bv, rtol=1e-12, atol=1e-14)
    for i in range(n):
        for k in range(ld.adjptr[i], ld.adjptr[i + 1]):
            j, b = ld.adjcol[k], ld.adjbod[k]
            Hi = Hs[i][0] if sc.master[i] == b else Hs[i][1]
            Hj = Hs[j][0] if sc.master[j] == b else Hs[j][1]
            Wij = h * Hi @ Minv(b) @ Hj.T
            np.testing.assert_allclose(_rot(ld.Woff[9 * k:9 * k + 9]), Wij, rtol=1e-10, atol=1e-12 * np.abs(Wij).max())
            # the transposed partner block is stored bitwise (ldy.c:829-844)
            q = [q for q in range(ld.adjptr[j], ld.adjptr[j + 1]) if ld.adjcol[q] == i and ld.adjbod[q] == b][0]
            assert same_bits(_rot(ld.Woff[9 * k:9 * k + 9]), _rot(ld.Woff[9 * q:9 * q + 9]).T)


def test_colouring_matches_numpy_jones_plassmann(pile):
    sc, ld, _ = pile
    seed = 987654321
    nc, col = O.colour(ld, seed)
    lib = O._load('oracle')
    prio = np.array([lib.orc_jp_priority(seed, i) for i in range(ld.n)], dtype=np.uint64)
    jp = -np.ones(ld.n, int)
    rows = np.repeat(np.arange(ld.n), np.diff(ld.adjptr))
    while np.any(jp < 0):
        unc = jp < 0
        beaten = np.zeros(ld.n, bool)
        both = unc[rows] & unc[ld.adjcol]
        beaten[rows[both & (prio[ld.adjcol] > prio[rows])]] = True
        sel = np.nonzero(unc & ~beaten)[0]
        new = {}
        for i in sel:
            used = set(jp[ld.adjcol[ld.adjptr[i]:ld.adjptr[i + 1]]].tolist())
            c = 0
            while c in used:
                c += 1
            new[i] = c
        for i, c in new.items():
            jp[i] = c
    assert np.array_equal(jp, col)
    assert not np.any(col[rows] == col[ld.adjcol])
    assert nc == col.max() + 1


def test_scene_generators_are_seeded():
    a = scenes.spheres_small(5, 60)
    b = scenes.spheres_small(5, 60)
    assert np.array_equal(a.mpnt, b.mpnt) and np.array_equal(a.velo, b.velo)
    h = scenes.hexahedra_lattice(nx=4, ny=4, nz=2)
    assert np.all(h.gap < 0) and h.ncon == 3 * 4 * 4 * 2 - 4 * 2 - 4 * 2 - 4 * 4 + 4 * 4 + 2 * 2 * 4 * 2


def test_lu_small_against_lapack():
    scipy_lapack = pytest.importorskip('scipy.linalg.lapack')
    import ctypes as C
    rng = np.random.default_rng(0)
    lib = O._load('oracle')
    for _ in range(200):
        A = rng.normal(size=(3, 3)); b = rng.normal(size=3)
        a = np.ascontiguousarray(A.T.ravel()); x = b.copy(); ipiv = np.zeros(3, np.int32)
        lib.orc_dgesv.restype = C.c_int
        info = lib.orc_dgesv(3, a.ctypes.data_as(C.c_void_p), ipiv.ctypes.data_as(C.c_void_p),
                             x.ctypes.data_as(C.c_void_p))
        lu, piv, y, info2 = scipy_lapack.dgesv(A, b)
        assert info == info2 == 0
        np.testing.assert_array_equal(ipiv, piv + 1)
        np.testing.assert_allclose(x, y, rtol=1e-12, atol=1e-13)


def test_list_order_colouring_is_greedy_in_list_order(pile):
    sc, ld, _ = pile
    nc, col = O.colour(ld, None)
    ref = -np.ones(ld.n, int)
    for i in range(ld.n):
        used = set(ref[ld.adjcol[ld.adjptr[i]:ld.adjptr[i + 1]]].tolist())
        c = 0
        while c in used:
            c += 1
        ref[i] = c
    assert np.array_equal(col, ref) and nc == ref.max() + 1


@pytest.mark.skipif(not O.ref_available(), reason='reference solver build (oracle/_ref) not present')
@pytest.mark.parametrize('kw', [REF_CASES[0], REF_CASES[1], REF_CASES[2], REF_CASES[5]],
                         ids=lambda k: '-'.join('%s=%s' % it for it in sorted(k.items())))
@pytest.mark.parametrize('dynamic', [1, 0])
def test_oracle_matches_compiled_reference_with_bilateral_constraints(pile, kw, dynamic):
    """FIXPNT, FIXDIR, VELODIR, VELODIR3 and RIGLNK rows among the contacts
    of the sphere pile (dbs.c:328-550, mrf.c:88-137): the restatement equals
    the compiled reference bit for bit, dynamic and static."""
    sc, ld, corder = pile
    lp = ld.permuted(corder)
    lp.dynamic = dynamic
    kinds, Z = bilateral_kinds(lp.n, bodies=(sc.master[corder], sc.slave[corder], sc.obstacle))
    lp.gap = riglnk_gap(kinds, Z, lp.gap)
    a = O.solve(lp, impl='oracle', kinds=kinds, Z=Z, **kw)
    b = O.solve(lp, impl='ref', kinds=kinds, Z=Z, **kw)
    for k in ('iters', 'error', 'thrown', 'ncallbacks'):
        assert a[k] == b[k], k
    for k in ('R', 'U', 'conmerit', 'rerhist', 'merhist'):
        assert same_bits(a[k], b[k]), k
    # the bilateral rows are solved: e.g. a FIXDIR row's normal velocity vanishes (dynamic: U_N = -V_N) to the
    # solver's tolerance (the final U holds the neighbours' later reactions)
    fd = np.nonzero(kinds == 2)[0]
    U = a['U'].reshape(-1, 3)
    if kw.get('maxiter', 0) >= 200:
        assert np.abs(U[fd, 2] + (lp.V.reshape(-1, 3)[fd, 2] if dynamic else 0.0)).max() < 1e-3
    c = O.solve(lp, impl='oracle', **kw)   # without kinds: a different problem
    assert not same_bits(a['R'], c['R'])
