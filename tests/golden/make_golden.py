"""Generate the golden vectors of the contact solve from the reference itself.

Each fixture is a small local-dynamics problem (a seeded settled sphere pile)
in colour-sorted row order, together with the result of the reference's own
GAUSS_SEIDEL_Solve (bgs.c:913-1069, compiled unmodified from the reference
sources into oracle/_ref by oracle/Makefile) for one solver configuration:
R, U, per-constraint merit, iterations, error code, merit, relative-error and
merit histories, THROW code and callback count.

Run from the repository root in an environment holding the reference tree:
    python tests/golden/make_golden.py
The fixtures are checked by tests/test_oracle.py against the C restatement.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, 'solfec-1.0_b200'))
sys.path.insert(0, os.path.join(ROOT, 'oracle'))

import oracle as O  # noqa: E402
from solfec_b200 import scenes  # noqa: E402

SEED = 0xC0FFEE

CASES = {
    'ssn_merit': dict(epsilon=1e-4, maxiter=1000, meritval=1e-4),
    'ssn_nomerit_reverse': dict(epsilon=1e-6, maxiter=300, reverse=True),
    'pg': dict(epsilon=1e-4, maxiter=60, meritval=1e-4, diagsolver='PROJECTED_GRADIENT'),
    'dsf': dict(epsilon=1e-4, maxiter=60, meritval=1e-4, diagsolver='DE_SAXCE_FENG'),
    'pn_from_zero': dict(epsilon=1e-4, maxiter=20, meritval=1e-4, diagsolver='PROJECTED_NEWTON'),
    'exit_diverged': dict(epsilon=1e-10, maxiter=7, meritval=1e-12, failure='EXIT'),
    'callback_diverged': dict(epsilon=1e-10, maxiter=4, meritval=1e-12, failure='CALLBACK'),
}


def problem(seed=11, n=400):
    sc = scenes.spheres_small(seed, n)
    ld = O.assemble(sc)
    nc, col = O.colour(ld, SEED)
    order = O.colour_order(col)
    return sc, ld.permuted(order)


def save(name, lp, res, kw, R0=None, U0=None):
    arrays = dict(W=lp.W, A=lp.A, rho=lp.rho, B=lp.B, V=lp.V, gap=lp.gap, friction=lp.friction,
                  restitution=lp.restitution, cohesion=lp.cohesion, adjptr=lp.adjptr, adjcol=lp.adjcol, Woff=lp.Woff,
                  scalars=np.array([lp.free_energy, lp.step, lp.dynamic]),
                  R0=np.zeros(3 * lp.n) if R0 is None else R0, U0=np.zeros(3 * lp.n) if U0 is None else U0,
                  R=res['R'], U=res['U'], conmerit=res['conmerit'], rerhist=res['rerhist'], merhist=res['merhist'],
                  out=np.array([res['iters'], res['error'], res['merit'], res['thrown'], res['ncallbacks']]))
    np.savez_compressed(os.path.join(HERE, name + '.npz'), options=repr(kw), **arrays)


def main():
    if not O.ref_available():
        raise SystemExit('the reference solver (oracle/_ref) is not available here')
    sc, lp = problem()
    first = None
    for name, kw in CASES.items():
        res = O.solve(lp, impl='ref', **kw)
        save(name, lp, res, kw)
        if name == 'ssn_merit':
            first = res
        print(name, lp.n, 'rows', lp.nblocks, 'blocks', 'iters', res['iters'], 'error', res['error'],
              'thrown', res['thrown'])
    # a warm-started next step: bodies advanced with the solved reactions
    ld0 = O.assemble(sc)
    nc, col = O.colour(ld0, SEED)
    corder = O.colour_order(col)
    R = np.empty((lp.n, 3)); R[corder] = first['R'].reshape(-1, 3)
    U = np.empty((lp.n, 3)); U[corder] = first['U'].reshape(-1, 3)
    sc1 = scenes.advance_velocities(sc, R)
    lp1 = O.assemble(sc1).permuted(corder)
    kw = dict(epsilon=1e-4, maxiter=1000, meritval=1e-4)
    R0, U0 = R[corder].ravel(), U[corder].ravel()
    res = O.solve(lp1, R=R0, U=U0, impl='ref', **kw)
    save('ssn_warm_start', lp1, res, kw, R0, U0)
    print('ssn_warm_start iters', res['iters'])


if __name__ == '__main__':
    main()
