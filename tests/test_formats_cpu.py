"""CPU tests of the interchange formats of the local dynamics (host/b2io.c:
LOCDYN_W_MatrixMarket ldy.c:1005-1052 and LOCDYN_Dump ldy.c:892-1002) through
the library's host writers, against the restatement oracle/ldy_formats.py on
oracle-assembled data, character for character."""
import dataclasses
import os

import numpy as np
import scipy.io

import oracle
import ldy_formats
from solfec_b200 import scenes
from solfec_b200._lib import lib, ptr


def spatial_points(sc):
    R = sc.rot[sc.master].reshape(-1, 3, 3).transpose(0, 2, 1)  # row-major
    return np.einsum('nij,nj->ni', R, sc.mpnt - sc.x0[sc.master]) + sc.x[sc.master]


def two_free_bodies():
    """The block-sliding scene with the table free: its four contacts join two
    moving bodies, so every row has each neighbour through two bodies (two
    blocks, which the dump sums)."""
    sc, _, _ = scenes.block_sliding()
    return dataclasses.replace(sc, obstacle=np.zeros(2, dtype=np.int32))


def cases():
    return [scenes.spheres_small(3, 40), two_free_bodies(), scenes.hexahedra_lattice(seed=2, nx=4, ny=3, nz=2)]


def _arr(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def test_formats_match_restatement(tmp_path):
    rng = np.random.default_rng(1)
    for k, sc in enumerate(cases()):
        ld = oracle.assemble(sc)
        n = ld.n
        R, U = rng.normal(size=(n, 3)), rng.normal(size=(n, 3))
        W, adjptr, adjcol, Woff = _arr(ld.W, np.float64), _arr(ld.adjptr, np.int32), _arr(ld.adjcol, np.int32), \
            _arr(ld.Woff, np.float64)
        path = str(tmp_path / ('w%d.mtx' % k))
        assert lib().b2gs_write_w_matrix_market(os.fsencode(path), n, ptr(W), ptr(adjptr), ptr(adjcol), ptr(Woff)) == 0
        text = open(path).read()
        assert text == ldy_formats.matrix_market(n, W, adjptr, adjcol, Woff)
        # the matrix reads back as W
        M = scipy.io.mmread(path, spmatrix=False).toarray()  # duplicate entries (two shared bodies) add up
        D = np.zeros((3 * n, 3 * n))
        for r in range(n):
            D[3 * r:3 * r + 3, 3 * r:3 * r + 3] += W[9 * r:9 * r + 9].reshape(3, 3).T
            for q in range(adjptr[r], adjptr[r + 1]):
                c = adjcol[q]
                D[3 * r:3 * r + 3, 3 * c:3 * c + 3] += Woff[9 * q:9 * q + 9].reshape(3, 3).T
        assert np.allclose(M, D, rtol=1e-14, atol=1e-14 * np.abs(D).max())

        pts = _arr(spatial_points(sc), np.float64)
        mid, sid = _arr(sc.master, np.int32), _arr(sc.slave, np.int32)
        base = _arr(sc.base, np.float64)
        B, V = _arr(ld.B, np.float64), _arr(ld.V, np.float64)
        Rc, Uc = _arr(R, np.float64), _arr(U, np.float64)
        path = str(tmp_path / ('d%d.txt' % k))
        assert lib().b2gs_write_locdyn_dump(os.fsencode(path), n, ptr(pts), ptr(mid), ptr(sid), ptr(base), ptr(W),
                                            ptr(B), ptr(V), ptr(Uc), ptr(Rc), ptr(adjptr), ptr(adjcol), ptr(Woff)) == 0
        text = open(path).read()
        assert text == ldy_formats.dump(n, pts, mid, sid, base, W, B, V, Uc, Rc, adjptr, adjcol, Woff)
        assert text.count('\n') == n
        if k == 1:  # two blocks per neighbour, summed: three neighbours per row, not six
            assert all(line.count(' => ') == 3 for line in text.splitlines())
            assert all(adjptr[r + 1] - adjptr[r] == 6 for r in range(n))


def test_writers_reject_bad_arguments(tmp_path):
    path = os.fsencode(str(tmp_path / 'x'))
    assert lib().b2gs_write_w_matrix_market(path, -1, None, None, None, None) != 0
    assert lib().b2gs_write_locdyn_dump(path, 2, *([None] * 12)) != 0
