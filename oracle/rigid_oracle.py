"""rigid_oracle.py -- TEST INFRASTRUCTURE. Not part of the product.

CPU restatement of the rigid-body time step around the contact solve, the
checker of the device integrator (csrc/b2_rigid.cuh):

- BODY_Dynamic_Step_Begin for RIG/OBS bodies, bod.c:1316-1370;
- BODY_Dynamic_Step_End for RIG/OBS bodies, bod.c:1428-1485;
- rig_force, bod.c:327-352 (point loads given as summed triples, gravity);
- rig_constraints_force, bod.c:419-439, with rig_operator_H, bod.c:216-228;
- the exponential map of alg.h:1138-1200 (EXPMAP);
- u += h M^-1 f as MX_Matvec on the block-diagonal inverse, mtx.c:2297-2307,
  in the netlib dgemv order;
- the bilateral constraints' update of DOM_Update_Begin (update_riglnk,
  update_fixdir; dom.c:487-550), BODY_Cur_Point and BODY_Ref_Point.

The arithmetic is written in scalar Python floats (IEEE double, no fused
multiply-add) in the operation order of the reference's algebra macros, so it
is bitwise comparable with the device kernels, which are built without
multiply-add contraction, wherever the exponential map takes its small-angle
branch. Schemes: 0 = RIG_POS (NEW1), 1 = RIG_NEG (NEW2, the default), 2 = RIG_IMP (NEW3).

Parity of this restatement with the reference itself is not pinned bitwise:
the reference's point-force callbacks and BLAS are site-specific. It is pinned
end to end by the trajectory values of the reference's own test
tests/block-sliding.py:64-80 (tests/test_gpu_rigid.py), and by the
conservation properties of the schemes (tests/test_rigid_cpu.py).
"""
from __future__ import annotations

import math

import numpy as np

SCH_RIG_POS, SCH_RIG_NEG, SCH_RIG_IMP = 0, 1, 2
BODY_DISABLE_ROTATION = 0x0004  # bod.h:144
DEG_10_SQ = 3.0461741978671E-02


def expmap(w):
    """Rotation matrix (column-major list of 9) of the rotation vector w."""
    a2 = w[0] * w[0] + w[1] * w[1] + w[2] * w[2]
    if a2 < DEG_10_SQ:
        s = 1.0 + (-1.666666666666667E-1 + (8.333333333333333E-3 + (-1.984126984126984E-4 + (
            2.755731922398589E-6 + (-2.505210838544172E-8 + 1.605904383682161E-10 * a2) * a2) * a2) * a2) * a2) * a2
        c = 0.5 + (-4.166666666666667E-2 + (1.388888888888889E-3 + (-2.480158730158730E-5 + (
            2.755731922398589E-7 + (-2.087675698786810E-9 + 1.147074559772972E-11 * a2) * a2) * a2) * a2) * a2) * a2
    else:
        a = math.sqrt(a2)
        s = math.sin(a) / a
        c = (1.0 - math.cos(a)) / a2
    q0, q1, q2 = w[0] * w[0], w[1] * w[1], w[2] * w[2]
    p01, p02, p12 = w[0] * w[1], w[0] * w[2], w[1] * w[2]
    s0, s1, s2 = s * w[0], s * w[1], s * w[2]
    c01, c02, c12 = c * p01, c * p02, c * p12
    R = [0.0] * 9
    R[0] = -c * (q2 + q1) + 1.0
    R[4] = -c * (q2 + q0) + 1.0
    R[8] = -c * (q1 + q0) + 1.0
    R[1] = c01 + s2
    R[3] = c01 - s2
    R[2] = c02 - s1
    R[6] = c02 + s1
    R[5] = c12 + s0
    R[7] = c12 - s0
    return R


def expmap123(w):
    """EXPMAP123 (alg.h:1280-1382): the derivatives of exp[w] with respect to
    w[0], w[1], w[2], column-major lists of 9."""
    x = w[0] * w[0] + w[1] * w[1] + w[2] * w[2]
    if x < 1E-16 * DEG_10_SQ:
        R0, R1, R2 = [0.0] * 9, [0.0] * 9, [0.0] * 9
        R0[5], R0[7] = 1.0, -1.0
        R1[2], R1[6] = -1.0, 1.0
        R2[1], R2[3] = 1.0, -1.0
        return R0, R1, R2
    c = 1.0 / x
    if x < DEG_10_SQ:
        a = 1.0 + (-1.666666666666667E-1 + (8.333333333333333E-3 + (-1.984126984126984E-4 + (
            2.755731922398589E-6 + (-2.505210838544172E-8 + 1.605904383682161E-10 * x) * x) * x) * x) * x) * x
        b = c - 0.5 + (4.166666666666667E-2 + (-1.388888888888889E-3 + (2.480158730158730E-5 + (
            -2.755731922398589E-7 + (2.087675698786810E-9 - 1.147074559772972E-11 * x) * x) * x) * x) * x) * x
    else:
        x = math.sqrt(x)
        a = math.sin(x) / x
        b = c * math.cos(x)
    b_ac = b - a * c
    ac_2cc_2bc = (a - 2.0 * (c - b)) * c
    c_b = c - b
    aux = [w[i] * w[j] for j in range(3) for i in range(3)]
    aux = [v * ac_2cc_2bc for v in aux]
    t = [w[0] * b_ac, w[1] * b_ac, w[2] * b_ac]
    aux[0] -= a; aux[1] += t[2]; aux[2] -= t[1]
    aux[3] -= t[2]; aux[4] -= a; aux[5] += t[0]
    aux[6] += t[1]; aux[7] -= t[0]; aux[8] -= a
    t = [w[0] * c_b, w[1] * c_b, w[2] * c_b]
    R0 = [aux[0] * w[0] + 2.0 * t[0], aux[1] * w[0] + t[1], aux[2] * w[0] + t[2],
          aux[3] * w[0] + t[1], aux[4] * w[0], aux[5] * w[0] + a,
          aux[6] * w[0] + t[2], aux[7] * w[0] - a, aux[8] * w[0]]
    R1 = [aux[0] * w[1], aux[1] * w[1] + t[0], aux[2] * w[1] - a,
          aux[3] * w[1] + t[0], aux[4] * w[1] + 2.0 * t[1], aux[5] * w[1] + t[2],
          aux[6] * w[1] + a, aux[7] * w[1] + t[2], aux[8] * w[1]]
    R2 = [aux[0] * w[2], aux[1] * w[2] + a, aux[2] * w[2] + t[0],
          aux[3] * w[2] - a, aux[4] * w[2], aux[5] * w[2] + t[1],
          aux[6] * w[2] + t[0], aux[7] * w[2] + t[1], aux[8] * w[2] + 2.0 * t[2]]
    return R0, R1, R2


def dgesv3(a, b):
    """Solve a x = b in place (a column-major list of 9, b a list of 3) in
    the arithmetic of LAPACK dgetf2 / dgetrs (as oracle/lu_small.c); returns
    LAPACK's info (0, or k > 0 for an exactly zero U(k,k))."""
    n, info, ipiv = 3, 0, [0, 0, 0]
    for j in range(n):
        p, amax = j, abs(a[j + j * n])
        for i in range(j + 1, n):
            if abs(a[i + j * n]) > amax:
                amax, p = abs(a[i + j * n]), i
        ipiv[j] = p
        if a[p + j * n] != 0.0:
            if p != j:
                for c in range(n):
                    a[j + c * n], a[p + c * n] = a[p + c * n], a[j + c * n]
            piv = a[j + j * n]
            if abs(piv) >= 2.2250738585072014e-308:
                r = 1.0 / piv
                for i in range(j + 1, n):
                    a[i + j * n] *= r
            else:
                for i in range(j + 1, n):
                    a[i + j * n] /= piv
        elif info == 0:
            info = j + 1
        for c in range(j + 1, n):
            u = a[j + c * n]
            if u != 0.0:
                t = -u
                for i in range(j + 1, n):
                    a[i + c * n] += a[i + j * n] * t
    if info:
        return info
    for i in range(n):
        p = ipiv[i]
        if p != i:
            b[i], b[p] = b[p], b[i]
    for k in range(n):
        if b[k] != 0.0:
            for i in range(k + 1, n):
                b[i] -= b[k] * a[i + k * n]
    for k in range(n - 1, -1, -1):
        if b[k] != 0.0:
            b[k] /= a[k + k * n]
            for i in range(k):
                b[i] -= b[k] * a[i + k * n]
    return 0


def new3_solve(h, J, W, G):
    """SOLVE (bod.c:163-209, NEW3): W with exp[hW] J W = G by Newton's method
    from W; returns (W, A = exp[hW], code), code 1 for a singular Jacobian, 2
    after 50 Newton steps (the reference stops there), else 0."""
    W = list(W)
    O = [W[0] * h, W[1] * h, W[2] * h]
    A = expmap(O)
    B = mat_mul(A, J)
    R = mat_vec(B, W)
    R = [R[i] - G[i] for i in range(3)]
    level = 1E-12 * h
    error = max(abs(R[0]), abs(R[1]), abs(R[2]))
    i = 0
    while error > level:
        JW = mat_vec(J, W)
        Z0, Z1, Z2 = expmap123(O)
        Z = mat_vec(Z0, JW) + mat_vec(Z1, JW) + mat_vec(Z2, JW)
        Z = [v * h for v in Z]
        Z = [Z[q] + B[q] for q in range(9)]
        if dgesv3(Z, R):
            return W, A, 1
        W = [W[k] - R[k] for k in range(3)]
        O = [W[0] * h, W[1] * h, W[2] * h]
        A = expmap(O)
        B = mat_mul(A, J)
        R = mat_vec(B, W)
        R = [R[k] - G[k] for k in range(3)]
        error = max(abs(R[0]), abs(R[1]), abs(R[2]))
        i += 1
        if not i < 50:
            return W, A, 2
    return W, A, 0


def mat_mul(A, B):  # NNMUL
    return [A[i] * B[3 * j] + A[3 + i] * B[3 * j + 1] + A[6 + i] * B[3 * j + 2] for j in range(3) for i in range(3)]


def mat_vec(A, x):  # NVMUL
    return [A[i] * x[0] + A[3 + i] * x[1] + A[6 + i] * x[2] for i in range(3)]


def matt_vec(A, x):  # TVMUL
    return [A[3 * i] * x[0] + A[3 * i + 1] * x[1] + A[3 * i + 2] * x[2] for i in range(3)]


def add_minv_force(jinv, minv, step, f, u):
    """u += step * blockdiag(J^-1, minv I) f (netlib dgemv 'N', beta = 1)."""
    for j in range(3):
        t = step * f[j]
        u[0] = u[0] + t * jinv[3 * j]
        u[1] = u[1] + t * jinv[3 * j + 1]
        u[2] = u[2] + t * jinv[3 * j + 2]
    for i in range(3):
        u[3 + i] = u[3 + i] + (step * f[3 + i]) * minv


def operator_H(R, X0, base, X):
    """rig_operator_H (bod.c:216-228): H (3x6, column-major list of 18)."""
    A0, A1, A2 = X[0] - X0[0], X[1] - X0[1], X[2] - X0[2]
    S = [0.0, A2, -A1, -A2, 0.0, A0, A1, -A0, 0.0]
    T = [R[i] * S[j] + R[3 + i] * S[3 + j] + R[6 + i] * S[6 + j] for j in range(3) for i in range(3)]
    H = [0.0] * 18
    for j in range(3):
        for i in range(3):
            H[3 * j + i] = base[3 * i] * T[3 * j] + base[3 * i + 1] * T[3 * j + 1] + base[3 * i + 2] * T[3 * j + 2]
    for j in range(3):
        for i in range(3):
            H[9 + 3 * j + i] = base[3 * i + j]
    return H


class Bodies:
    """Rigid body state as plain lists (per body): rot[9], x[3], velo[6],
    velo0[6], J[9], jinv[9], mass, minv, scheme, obstacle, x0[3] (referential
    mass centre), fext[6], aux[3]."""

    def __init__(self, rot, x, velo, J, jinv, mass, minv, x0, obstacle, scheme=None, flags=None):
        nb = len(mass)
        f = lambda a, k: [list(map(float, np.asarray(a, dtype=np.float64).reshape(nb, k)[b])) for b in range(nb)]
        self.rot, self.x, self.velo = f(rot, 9), f(x, 3), f(velo, 6)
        self.velo0 = [list(v) for v in self.velo]
        self.J, self.jinv, self.x0 = f(J, 9), f(jinv, 9), f(x0, 3)
        self.mass = [float(v) for v in np.asarray(mass, dtype=np.float64)]
        self.minv = [float(v) for v in np.asarray(minv, dtype=np.float64)]
        self.obstacle = [int(v) for v in obstacle]
        self.scheme = [SCH_RIG_NEG] * nb if scheme is None else [int(v) for v in scheme]
        self.flags = [0] * nb if flags is None else [int(v) for v in flags]
        self.failures = 0
        self.fext = [[0.0] * 6 for _ in range(nb)]
        self.aux = [[0.0] * 3 for _ in range(nb)]

    @property
    def nbod(self):
        return len(self.mass)


def step_begin(bd: Bodies, step, gravity=(0.0, 0.0, 0.0), loads=None):
    """BODY_Dynamic_Step_Begin (bod.c:1316-1370) for every body."""
    half = 0.5 * step
    for b in range(bd.nbod):
        u = bd.velo[b]
        if bd.flags[b] & BODY_DISABLE_ROTATION:
            u[0] = u[1] = u[2] = 0.0
        bd.velo0[b] = list(u)
        J, I, Rold = bd.J[b], bd.jinv[b], bd.rot[b]
        W = u[0:3]
        DR = expmap([W[0] * half, W[1] * half, W[2] * half])
        Rn = mat_mul(Rold, DR)
        bd.rot[b] = Rn
        x = bd.x[b]
        for i in range(3):
            x[i] = x[i] + half * u[3 + i]
        lin, spat, ref = [0.0] * 3, [0.0] * 3, [0.0] * 3
        if not bd.obstacle[b]:
            if loads is not None:
                L = [float(v) for v in np.asarray(loads, dtype=np.float64).reshape(bd.nbod, 9)[b]]
                for i in range(3):
                    lin[i] = L[i] + lin[i]
                    spat[i] = L[3 + i] + spat[i]
                    ref[i] = L[6 + i] + ref[i]
            m = bd.mass[b]
            for i in range(3):
                lin[i] = lin[i] + m * float(gravity[i])
        t = matt_vec(Rn, spat)
        f = [ref[0] + t[0], ref[1] + t[1], ref[2] + t[2], lin[0], lin[1], lin[2]]
        if bd.scheme[b] > SCH_RIG_POS:
            A = matt_vec(DR, mat_vec(J, W))
            bd.aux[b] = [A[i] + step * f[i] for i in range(3)]
        P = [f[0] * half, f[1] * half, f[2] * half]
        W05 = mat_vec(J, W)
        t = matt_vec(DR, W05)
        P = [P[0] + t[0], P[1] + t[1], P[2] + t[2]]
        W05 = mat_vec(I, P)
        P = mat_vec(J, W05)
        f[0] -= W05[1] * P[2] - W05[2] * P[1]
        f[1] -= W05[2] * P[0] - W05[0] * P[2]
        f[2] -= W05[0] * P[1] - W05[1] * P[0]
        bd.fext[b] = list(f)
        add_minv_force(I, bd.minv[b], step, f, u)


def step_end(bd: Bodies, step, master, slave, mpnt, spnt, base, R):
    """BODY_Dynamic_Step_End (bod.c:1428-1485) for every body, with the
    contact reactions R[ncon][3] (local frames)."""
    half = 0.5 * step
    master = [int(v) for v in master]
    slave = [int(v) for v in slave]
    ncon = len(master)
    mpnt = np.asarray(mpnt, dtype=np.float64).reshape(ncon, 3)
    spnt = np.asarray(spnt, dtype=np.float64).reshape(ncon, 3)
    base = np.asarray(base, dtype=np.float64).reshape(ncon, 9)
    R = np.asarray(R, dtype=np.float64).reshape(ncon, 3)
    contacts_of = [[] for _ in range(bd.nbod)]
    for i in range(ncon):
        contacts_of[master[i]].append(i)
        if slave[i] >= 0:
            contacts_of[slave[i]].append(i)
    for b in range(bd.nbod):
        u = bd.velo[b]
        Rb = list(bd.rot[b])
        f = [0.0] * 6
        if not bd.obstacle[b]:
            for i in sorted(contacts_of[b]):
                isma = master[i] == b
                X = [float(v) for v in (mpnt[i] if isma else spnt[i])]
                H = operator_H(Rb, bd.x0[b], [float(v) for v in base[i]], X)
                rc = [float(v) for v in R[i]]
                r = [H[3 * j] * rc[0] + H[3 * j + 1] * rc[1] + H[3 * j + 2] * rc[2] for j in range(6)]
                for j in range(6):
                    f[j] = f[j] + r[j] if isma else f[j] - r[j]
        I = bd.jinv[b]
        add_minv_force(I, bd.minv[b], step, f, u)
        x = bd.x[b]
        for i in range(3):
            x[i] = x[i] + half * u[3 + i]
        if bd.flags[b] & BODY_DISABLE_ROTATION:
            u[0] = u[1] = u[2] = 0.0
        sch = bd.scheme[b]
        DR = None
        if sch <= SCH_RIG_NEG:
            DR = expmap([u[0] * half, u[1] * half, u[2] * half])
            bd.rot[b] = mat_mul(Rb, DR)
        if sch > SCH_RIG_POS:
            A = [bd.aux[b][i] + step * f[i] for i in range(3)]
            bd.aux[b] = A
            if sch == SCH_RIG_NEG:
                W = mat_vec(I, matt_vec(DR, A))
                u[0], u[1], u[2] = W[0], W[1], W[2]
            else:  # NEW3
                W, DR, code = new3_solve(half, bd.J[b], u[0:3], A)
                bd.failures |= code
                u[0], u[1], u[2] = W[0], W[1], W[2]
                bd.rot[b] = mat_mul(Rb, DR)


def cur_point(bd: Bodies, b, X):
    """BODY_Cur_Point of a rigid body or obstacle (bod.c:1702-1716, NVADDMUL)."""
    R, c, C = bd.rot[b], bd.x[b], bd.x0[b]
    A = [X[0] - C[0], X[1] - C[1], X[2] - C[2]]
    return [c[i] + (R[i] * A[0] + R[3 + i] * A[1] + R[6 + i] * A[2]) for i in range(3)]


def ref_point(bd: Bodies, b, x):
    """BODY_Ref_Point of a rigid body or obstacle (bod.c:1736-1750, TVADDMUL)."""
    R, c, C = bd.rot[b], bd.x[b], bd.x0[b]
    a = [x[0] - c[0], x[1] - c[1], x[2] - c[2]]
    return [C[i] + (R[3 * i] * a[0] + R[3 * i + 1] * a[1] + R[3 * i + 2] * a[2]) for i in range(3)]


CON_FIXDIR, CON_RIGLNK = 2, 5  # dom.h:98


def update_constraints(bd: Bodies, kinds, master, slave, mpnt, spnt, base, gap, Z):
    """The bilateral constraints' part of DOM_Update_Begin (dom.c:3716-3732)
    on the bodies at t + h/2, in place on the row arrays: RIGLNK as
    update_riglnk (dom.c:524-550), with Z[i][0..2] the link vector in the new
    base (the diagonal solver's TVMUL, dbs.c:409) and Z[i][3] the length;
    FIXDIR with a slave body as update_fixdir (dom.c:487-500), the master's
    referential direction in Z[i][0..2]. spnt is the spatial point of a row
    without a slave."""
    import oracle  # localbase restated in C (oracle_detect.c)
    for i, k in enumerate(kinds):
        m, s = int(master[i]), int(slave[i])
        if k == CON_RIGLNK:
            pm = cur_point(bd, m, [float(v) for v in mpnt[i]])
            ps = cur_point(bd, s, [float(v) for v in spnt[i]]) if s >= 0 else [float(v) for v in spnt[i]]
            v = [pm[0] - ps[0], pm[1] - ps[1], pm[2] - ps[2]]
            ln = math.sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2])
            gap[i] = ln - float(Z[i][3])
            ln = 1.0 / ln
            b = oracle.localbase(np.array([v[0] * ln, v[1] * ln, v[2] * ln]))
            base[i] = b
            Z[i][:3] = matt_vec([float(q) for q in b], v)
        elif k == CON_FIXDIR and s >= 0:
            p = cur_point(bd, s, [float(v) for v in spnt[i]])
            mpnt[i] = ref_point(bd, m, p)
            base[i] = oracle.localbase(np.array(mat_vec(bd.rot[m], [float(q) for q in Z[i][:3]])))


def kinetic_energy(bd: Bodies, b):
    """1/2 (Omega^T J Omega + m v.v) of body b (referential angular velocity)."""
    u = bd.velo[b]
    JW = mat_vec(bd.J[b], u[0:3])
    return 0.5 * (u[0] * JW[0] + u[1] * JW[1] + u[2] * JW[2]) + 0.5 * bd.mass[b] * (u[3] ** 2 + u[4] ** 2 + u[5] ** 2)


def spatial_angular_momentum(bd: Bodies, b):
    """R J Omega of body b."""
    return mat_vec(bd.rot[b], mat_vec(bd.J[b], bd.velo[b][0:3]))
