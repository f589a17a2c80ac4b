"""ldy_formats.py -- TEST INFRASTRUCTURE. Not part of the product.

Python restatement of the reference's text formats of a local dynamics, the
checker of host/b2io.c:

- LOCDYN_W_MatrixMarket, ldy.c:1005-1052: header, then per row of the list
  (con->num = 3 * position + 1) the diagonal block and the row's off-diagonal
  blocks in list order, each as nine "%d  %d  %.15g" lines (row i, column j,
  W[3j+i]);
- LOCDYN_Dump, ldy.c:892-1002: per row "CONTACT (point) (master, slave)
  [base] [W] (B) (V) (U) (R)", then " => CONTACT (point) (ids) [base] [W]" per
  neighbour constraint, the neighbour's blocks summed (NNADD onto a zeroed
  block, in the list order of the blocks) and the neighbours ordered by the
  map's comparison dumpcmp (ldy.c:330-361: point, sorted id pair, kind,
  normal).

Python's "%g" formatting of finite doubles is the C library's, so the text is
comparable character for character. Parity with the reference itself is not
pinned by a fixture: its own test of the dump (tests/locdyn-test.sh) compares
two runs of the reference with each other.
"""
from __future__ import annotations

import functools

import numpy as np


def matrix_market(n, W, adjptr, adjcol, Woff):
    W = np.asarray(W, dtype=np.float64).reshape(-1)
    Woff = np.asarray(Woff, dtype=np.float64).reshape(-1)
    adjptr = np.asarray(adjptr).reshape(-1)
    adjcol = np.asarray(adjcol).reshape(-1)
    nnz = 9 * n + 9 * (int(adjptr[n]) if n > 0 else 0)
    out = ['%%MatrixMarket matrix coordinate real general\n', '%d  %d  %d\n' % (3 * n, 3 * n, nnz)]
    for r in range(n):
        row = 3 * r + 1
        for i in range(3):
            for j in range(3):
                out.append('%d  %d  %.15g\n' % (row + i, row + j, W[9 * r + 3 * j + i]))
        for k in range(int(adjptr[r]), int(adjptr[r + 1])):
            col = 3 * int(adjcol[k]) + 1
            for i in range(3):
                for j in range(3):
                    out.append('%d  %d  %.15g\n' % (row + i, col + j, Woff[9 * k + 3 * j + i]))
    return ''.join(out)


def _head(lead, p, mid, sid, base, W):
    return ('%sCONTACT (%.6g, %.6g, %.6g) (%d, %d) [%s] [%s]'
            % (lead, p[0], p[1], p[2], mid, sid, ', '.join('%.6g' % v for v in base), ', '.join('%.6g' % v for v in W)))


def dump(n, point, master_id, slave_id, base, W, B, V, U, R, adjptr, adjcol, Woff):
    point = np.asarray(point, dtype=np.float64).reshape(-1, 3)
    base = np.asarray(base, dtype=np.float64).reshape(-1, 9)
    W = np.asarray(W, dtype=np.float64).reshape(-1, 9)
    B, V, U, R = (np.asarray(a, dtype=np.float64).reshape(-1, 3) for a in (B, V, U, R))
    Woff = np.asarray(Woff, dtype=np.float64).reshape(-1, 9)
    mid = [int(v) for v in master_id]
    sid = [int(v) for v in slave_id]

    def cmp(a, b):
        for i in range(3):
            if point[a, i] < point[b, i]:
                return -1
            if point[a, i] > point[b, i]:
                return 1
        ia, ib = sorted((mid[a], sid[a])), sorted((mid[b], sid[b]))
        for i in range(2):
            if ia[i] < ib[i]:
                return -1
            if ia[i] > ib[i]:
                return 1
        for i in range(6, 9):
            if base[a, i] < base[b, i]:
                return -1
            if base[a, i] > base[b, i]:
                return 1
        return 0

    lines = []
    for r in range(n):
        s = _head('', point[r], mid[r], sid[r], base[r], W[r])
        s += ' (%s) (%s) (%s) (%s)' % tuple(', '.join('%.6g' % v for v in a[r]) for a in (B, V, U, R))
        nbrs, sums = [], []
        for k in range(int(adjptr[r]), int(adjptr[r + 1])):
            c = int(adjcol[k])
            q = next((t for t, x in enumerate(nbrs) if cmp(x, c) == 0), None)
            if q is None:
                nbrs.append(c)
                sums.append([0.0] * 9)
                q = len(nbrs) - 1
            sums[q] = [sums[q][e] + float(Woff[k, e]) for e in range(9)]
        order = sorted(range(len(nbrs)), key=functools.cmp_to_key(lambda a, b: cmp(nbrs[a], nbrs[b])))
        for q in order:
            c = nbrs[q]
            s += _head(' => ', point[c], mid[c], sid[c], base[c], sums[q])
        lines.append(s + '\n')
    return ''.join(lines)
