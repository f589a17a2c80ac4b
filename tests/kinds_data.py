"""Constraint kinds for the bilateral-constraint tests (shared by the CPU and
GPU tests)."""
import numpy as np


def _forest(kinds, master, slave, obstacle):
    """Kinds with the bilateral rows that would close a loop of bilateral
    constraints among the bodies (obstacles one ground node) turned back into
    contacts: prescribed velocities on a loop need not be compatible, and then
    no reaction solves every row."""
    nb = int(max(master.max(), slave.max())) + 2
    ground = nb - 1
    par = np.arange(nb)

    def find(x):
        while par[x] != x:
            par[x] = par[par[x]]
            x = par[x]
        return x
    out = kinds.copy()
    for i in np.nonzero(kinds)[0]:
        a = ground if obstacle[master[i]] else master[i]
        b = ground if (slave[i] < 0 or obstacle[slave[i]]) else slave[i]
        ra, rb = find(a), find(b)
        if ra == rb:
            out[i] = 0
        else:
            par[ra] = rb
    return out


def bilateral_kinds(n, seed=4, bodies=None):
    """Constraint kinds (dom.h:98) on strides of the rows and their Z: VELODIR
    and VELODIR3 small prescribed velocities; RIGLNK a link vector along the
    row's normal (the local form of update_riglnk's Z, dom.c:524-550: the base
    is built from the link direction) of length D in [0.3, 0.6] and a link
    length within 1e-6 D of it. With bodies = (master, slave, obstacle) of the
    rows, the bilateral rows are thinned to a forest (_forest) so that the
    problem has a solution."""
    kinds = np.zeros(n, np.int32)
    kinds[3::7] = 1
    kinds[5::11] = 2
    kinds[6::13] = 3
    kinds[8::17] = 4
    kinds[9::19] = 5
    if bodies is not None:
        kinds = _forest(kinds, *(np.asarray(b) for b in bodies))
    rng = np.random.default_rng(seed)
    Z = np.zeros((n, 4))
    Z[kinds == 3, 0] = rng.normal(size=int((kinds == 3).sum())) * 0.01
    Z[kinds == 4, :3] = rng.normal(size=(int((kinds == 4).sum()), 3)) * 0.01
    r = kinds == 5
    D = rng.uniform(0.3, 0.6, int(r.sum()))
    Z[r, 2] = D
    Z[r, 3] = D * (1 + rng.uniform(-1e-6, 1e-6, int(r.sum())))
    return kinds, Z


def riglnk_gap(kinds, Z, gap):
    """Row gaps with those of the RIGLNK rows set as update_riglnk sets them
    (dom.c:546): link distance minus link length."""
    g = np.array(gap, dtype=np.float64, copy=True)
    r = kinds == 5
    g[r] = Z[r, 2] - Z[r, 3]
    return g
