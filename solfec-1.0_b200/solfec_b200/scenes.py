"""Seeded synthetic rigid-body contact scenes.

The reference builds its contact problems inside a full simulation
(SOLFEC_Run, sol.c:665-842: body time stepping, contact detection in goc.c and
LOCDYN_Insert). That pipeline is outside the solver path, so the scenes here
are generated directly in the form the solver path consumes:

* rigid bodies: rotation R (3x3, column-major), referential mass centre X0,
  inverse referential inertia J^-1, 1/mass, velocity [Omega (body frame); v]
  at time t (``velo0``) and after the free step t+h (``velo``), obstacle flag
  (bod.c:53-74 layout);
* contacts: master/slave body, referential points on both bodies, local frame
  ``base`` (column-major, normal = third column, pointing from slave to
  master), gap, Coulomb friction, restitution and cohesion (dom.h:77-129).

Every generator is deterministic for a given seed. Contact detection follows
the reference threshold: a pair is a contact when gap < GEOMETRIC_EPSILON
(alg.c:24, goc.c:431).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

GEOMETRIC_EPSILON = 1e-6  # alg.c:24
GRAVITY = np.array([0.0, 0.0, -9.81])


@dataclasses.dataclass
class Scene:
    name: str
    step: float
    dynamic: int
    # bodies
    rot: np.ndarray        # (nb, 9) column-major rotation
    x: np.ndarray          # (nb, 3) current mass centre
    x0: np.ndarray         # (nb, 3) referential mass centre
    jinv: np.ndarray       # (nb, 9) inverse referential inertia, column-major
    minv: np.ndarray       # (nb,)
    velo: np.ndarray       # (nb, 6) [Omega; v] after the free step (t+h)
    velo0: np.ndarray      # (nb, 6) [Omega; v] at t
    obstacle: np.ndarray   # (nb,) int32, 1 for obstacles (walls)
    # contacts
    master: np.ndarray     # (nc,) int32
    slave: np.ndarray      # (nc,) int32, -1 for none
    mpnt: np.ndarray       # (nc, 3) master referential point
    spnt: np.ndarray       # (nc, 3) slave referential point
    base: np.ndarray       # (nc, 9) column-major [t1 t2 n]
    gap: np.ndarray        # (nc,)
    friction: np.ndarray   # (nc,)
    restitution: np.ndarray
    cohesion: np.ndarray   # (nc,) cohesion * area, as dbs.c:500 forms it
    mass: np.ndarray = None  # (nb,) for diagnostics
    radius: np.ndarray = None  # (nb,) sphere radius of sphere bodies, 0 for the others

    @property
    def nbod(self) -> int:
        return int(self.rot.shape[0])

    @property
    def ncon(self) -> int:
        return int(self.master.shape[0])

    def body_arrays(self):
        return dict(rot=self.rot, x0=self.x0, jinv=self.jinv, minv=self.minv,
                    velo=self.velo, velo0=self.velo0, obstacle=self.obstacle)

    def contact_arrays(self):
        return dict(master=self.master, slave=self.slave, mpnt=self.mpnt, spnt=self.spnt,
                    base=self.base, gap=self.gap, friction=self.friction,
                    restitution=self.restitution, cohesion=self.cohesion)


# ----------------------------------------------------------------------------- helpers

def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotations (Shoemake quaternions), column-major (n, 9)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    x, y, z, w = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R.transpose(0, 2, 1).reshape(n, 9)  # column-major flattening


def _colmajor(M: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(M.transpose(0, 2, 1).reshape(M.shape[0], 9))


def local_base(normal: np.ndarray) -> np.ndarray:
    """Right-handed frame [t1 t2 n] per normal, column-major (nc, 9)."""
    n = normal / np.linalg.norm(normal, axis=1, keepdims=True)
    e = np.zeros_like(n)
    idx = np.argmin(np.abs(n), axis=1)
    e[np.arange(n.shape[0]), idx] = 1.0
    t1 = np.cross(n, e)
    t1 /= np.linalg.norm(t1, axis=1, keepdims=True)
    t2 = np.cross(n, t1)
    return np.ascontiguousarray(np.concatenate([t1, t2, n], axis=1))


def _referential(rot: np.ndarray, x: np.ndarray, x0: np.ndarray, p: np.ndarray) -> np.ndarray:
    """Referential point X with R (X - X0) = p - x."""
    R = rot.reshape(-1, 3, 3).transpose(0, 2, 1)  # row-major view of column-major storage
    return x0 + np.einsum('nji,nj->ni', R, p - x)


def _walls(lo, hi):
    """Six obstacle walls of an axis-aligned box: (outward-into-box normal, plane point)."""
    lo = np.asarray(lo, float); hi = np.asarray(hi, float)
    normals = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], float)
    points = np.array([lo, hi, lo, hi, lo, hi], float)
    return normals, points


def _settle_spheres(x, r, lo, hi, iters, drop, overlap, rng, relax=200, shake=0.15):
    """Gravity compaction by position projection: every iteration lowers all
    spheres by a drop that decays to zero and then pushes overlapping pairs
    apart until they interpenetrate by at most ``overlap``, with a decaying
    lateral shake (a fraction ``shake`` of the radius) that lets spheres roll
    off unstable columns into the hollows below; a final run of
    projection passes without drop relaxes the packing. Produces a dense
    resting packing in which touching spheres overlap slightly (so they are
    detected contacts)."""
    from scipy.spatial import cKDTree
    rmax = float(r.max())
    skin = 4 * drop + 0.1 * rmax
    pairs = None
    total = iters + relax
    for it in range(total):
        if it % 5 == 0:
            pairs = cKDTree(x).query_pairs(2 * rmax + skin, output_type='ndarray')
        if it < iters:
            decay = (1.0 - it / float(iters)) ** 2
            x[:, 2] -= drop * decay
            x[:, 0:2] += rng.uniform(-shake, shake, (x.shape[0], 2)) * decay * r[:, None]
        for _ in range(4):
            if pairs.shape[0]:
                i, j = pairs[:, 0], pairs[:, 1]
                d = x[i] - x[j]
                dist = np.sqrt(np.einsum('ij,ij->i', d, d))
                pen = (r[i] + r[j] - overlap) - dist
                m = pen > 0
                if np.any(m):
                    dd = d[m] / np.maximum(dist[m], 1e-12)[:, None]
                    corr = 0.5 * pen[m][:, None] * dd
                    np.add.at(x, i[m], corr)
                    np.add.at(x, j[m], -corr)
            x[:] = np.clip(x, lo + r[:, None] - overlap, hi - r[:, None] + overlap)
    return x


def _sphere_contacts(x, r, walls_n, walls_p, nsph, threshold=0.0):
    """Sphere-sphere and sphere-wall contacts with gap < threshold.

    The reference detects contacts at gap < GEOMETRIC_EPSILON (goc.c:431), but
    the diagonal solvers force R = 0 on rows with gap > 0 (dbs.c:43-48,149-154)
    while the merit function still counts their approach velocity (mrf.c:84),
    which puts a floor under the merit that no sweep removes. The settled
    scenes therefore keep touching pairs only (threshold 0)."""
    from scipy.spatial import cKDTree
    pairs = cKDTree(x).query_pairs(2 * float(r.max()) + GEOMETRIC_EPSILON, output_type='ndarray')
    masters, slaves, points, normals, gaps = [], [], [], [], []
    if pairs.shape[0]:
        a, b = pairs[:, 0], pairs[:, 1]   # master a, slave b; normal from b to a
        d = x[a] - x[b]
        dist = np.linalg.norm(d, axis=1)
        g = dist - r[a] - r[b]
        m = g < threshold
        a, b, d, dist, g = a[m], b[m], d[m], dist[m], g[m]
        n = d / dist[:, None]
        p = x[b] + n * (r[b] + 0.5 * g)[:, None]
        masters.append(a); slaves.append(b); points.append(p); normals.append(n); gaps.append(g)
    for w in range(walls_n.shape[0]):   # sphere is master, wall obstacle is slave
        n = walls_n[w]
        dist = (x - walls_p[w]) @ n
        g = dist - r
        idx = np.nonzero(g < threshold)[0]
        if idx.size:
            nn = np.repeat(n[None], idx.size, axis=0)
            p = x[idx] - nn * (r[idx] + 0.5 * g[idx])[:, None]
            masters.append(idx); slaves.append(np.full(idx.size, nsph + w)); points.append(p)
            normals.append(nn); gaps.append(g[idx])
    cat = lambda L, shape: np.concatenate(L) if L else np.zeros(shape)
    return (cat(masters, (0,)).astype(np.int32), cat(slaves, (0,)).astype(np.int32),
            cat(points, (0, 3)), cat(normals, (0, 3)), cat(gaps, (0,)))


def _assemble_scene(name, step, x_b, rot, x0, jinv, minv, mass, velo0, obstacle, master, slave, points, normals,
                    gaps, friction, restitution, cohesion, gravity=GRAVITY):
    velo = velo0.copy()
    movable = obstacle == 0
    velo[movable, 3:6] += step * gravity  # free step: u_free = u + h M^-1 f_ext (gravity on v)
    base = local_base(normals)
    mpnt = _referential(rot[master], x_b[master], x0[master], points)
    spnt = _referential(rot[slave], x_b[slave], x0[slave], points)
    nc = master.shape[0]
    full = lambda v: np.ascontiguousarray(np.broadcast_to(np.asarray(v, float), (nc,)).copy())
    return Scene(name=name, step=step, dynamic=1, rot=np.ascontiguousarray(rot), x=np.ascontiguousarray(x_b),
                 x0=np.ascontiguousarray(x0), jinv=np.ascontiguousarray(jinv), minv=np.ascontiguousarray(minv),
                 velo=np.ascontiguousarray(velo), velo0=np.ascontiguousarray(velo0),
                 obstacle=np.ascontiguousarray(obstacle.astype(np.int32)),
                 master=np.ascontiguousarray(master.astype(np.int32)), slave=np.ascontiguousarray(slave.astype(np.int32)),
                 mpnt=np.ascontiguousarray(mpnt), spnt=np.ascontiguousarray(spnt), base=base,
                 gap=np.ascontiguousarray(gaps.astype(float)), friction=full(friction), restitution=full(restitution),
                 cohesion=full(cohesion), mass=mass)


def _sphere_scene(name, rng, x, r, density, lo, hi, step, friction, restitution, vel_sigma, settle_iters,
                  drop, overlap):
    n = x.shape[0]
    x = _settle_spheres(x, r, np.asarray(lo, float), np.asarray(hi, float), settle_iters, drop, overlap, rng)
    walls_n, walls_p = _walls(lo, hi)
    master, slave, points, normals, gaps = _sphere_contacts(x, r, walls_n, walls_p, n)
    nb = n + 6
    mass = np.empty(nb); mass[:n] = density * 4.0 / 3.0 * math.pi * r ** 3; mass[n:] = 1.0
    J = 0.4 * mass[:n] * r ** 2                      # solid sphere inertia
    jinv = np.zeros((nb, 9)); jinv[:n, 0] = jinv[:n, 4] = jinv[:n, 8] = 1.0 / J
    minv = np.zeros(nb); minv[:n] = 1.0 / mass[:n]
    rot = np.zeros((nb, 9)); rot[:, 0] = rot[:, 4] = rot[:, 8] = 1.0
    rot[:n] = _random_rotations(rng, n)
    xb = np.concatenate([x, walls_p], axis=0)
    x0 = xb.copy()
    velo0 = np.zeros((nb, 6))
    if vel_sigma > 0:
        velo0[:n, 3:6] = rng.normal(0.0, vel_sigma, (n, 3))
        velo0[:n, 0:3] = rng.normal(0.0, vel_sigma, (n, 3)) / r[:, None]
    obstacle = np.zeros(nb, np.int32); obstacle[n:] = 1
    fr = friction(master.shape[0]) if callable(friction) else friction
    sc = _assemble_scene(name, step, xb, rot, x0, jinv, minv, mass, velo0, obstacle, master, slave, points,
                         normals, gaps, fr, restitution, 0.0)
    rad = np.zeros(nb); rad[:n] = r
    return dataclasses.replace(sc, radius=rad)


# ----------------------------------------------------------------------------- configurations

def spheres_lattice(seed: int = 1, n_side: int = 10, radius: float = 0.05, pitch: float = 0.11,
                    jitter: float = 0.005, density: float = 2000.0, box: float = 1.2, friction: float = 0.3,
                    step: float = 1e-3, settle_iters: int = 200) -> Scene:
    """1000 spheres of radius 0.05 m on a 10^3 lattice (0.11 m pitch, +-0.005 m
    jitter) in a 1.2 m box, settled under gravity; friction 0.3, e = 0, h = 1e-3."""
    rng = np.random.default_rng(seed)
    g = (np.arange(n_side) - (n_side - 1) / 2.0) * pitch
    X, Y, Z = np.meshgrid(g, g, g + box / 2.0, indexing='ij')
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    x += rng.uniform(-jitter, jitter, x.shape)
    r = np.full(x.shape[0], radius)
    lo = [-box / 2, -box / 2, 0.0]; hi = [box / 2, box / 2, box]
    return _sphere_scene('spheres-lattice-%d' % x.shape[0], rng, x, r, density, lo, hi, step, friction, 0.0, 0.0,
                         settle_iters, 0.01, 1e-5)


def spheres_polydisperse(seed: int = 2, n: int = 20000, rmin: float = 0.03, rmax: float = 0.06,
                         density: float = 2500.0, box=(2.0, 2.0, 4.0), friction: float = 0.5, step: float = 5e-4,
                         vel_sigma: float = 0.1, settle_iters: int = 200) -> Scene:
    """Polydisperse packing: radius U[rmin, rmax], density 2500, footprint 2x2 m,
    friction 0.5, h = 5e-4, initial velocities N(0, 0.1) m/s. Initial positions
    by seeded random sequential addition in a column twice the box height (at
    the box height the solid fraction would be ~0.53, beyond the jamming limit
    of sequential addition), then settled under gravity into the 2x2x4 box."""
    from scipy.spatial import cKDTree
    rng = np.random.default_rng(seed)
    r = np.sort(rng.uniform(rmin, rmax, n))[::-1].copy()   # large first
    lo = np.array([-box[0] / 2, -box[1] / 2, 0.0]); hi = np.array([box[0] / 2, box[1] / 2, 2.0 * box[2]])
    placed = np.zeros((0, 3)); pr = np.zeros(0)
    k = 0
    while k < n:
        m = min(4096, n - k)
        cand_r = r[k:k + m]
        cand = rng.uniform(lo + rmax, hi - rmax, (4 * m, 3))
        cr = np.resize(cand_r, 4 * m)
        ok = np.ones(4 * m, bool)
        if placed.shape[0]:
            d, _ = cKDTree(placed).query(cand, k=1)
            ok &= d > cr + rmax
        acc_idx = []
        tree_new = []
        for c in np.nonzero(ok)[0]:
            if len(acc_idx) >= m:
                break
            p = cand[c]
            if tree_new:
                q = np.asarray(tree_new)
                if np.any(np.linalg.norm(q - p, axis=1) < 2 * rmax):
                    continue
            tree_new.append(p); acc_idx.append(c)
        if acc_idx:
            placed = np.concatenate([placed, cand[acc_idx]], axis=0)
            pr = np.concatenate([pr, r[k:k + len(acc_idx)]])
            k += len(acc_idx)
    hi_box = np.array([box[0] / 2, box[1] / 2, 2.0 * box[2]])
    return _sphere_scene('spheres-polydisperse-%d' % n, rng, placed, pr, density, lo, hi_box, step, friction, 0.0,
                         vel_sigma, settle_iters, 0.02, 1e-5)


def spheres_small(seed: int, n: int, rmin: float = 0.02, rmax: float = 0.05, friction: float = 0.4,
                  step: float = 1e-3, density: float = 2000.0, settle_iters: int = 80) -> Scene:
    """A small uneven sphere scene (batched-solve workload): n spheres on a
    jittered lattice in a square column, settled under gravity."""
    rng = np.random.default_rng(seed)
    r = rng.uniform(rmin, rmax, n)
    side = max(2, int(round((n / 2.0) ** (1.0 / 3.0))))
    layers = int(math.ceil(n / float(side * side)))
    pitch = 2.2 * rmax
    g = (np.arange(side) - (side - 1) / 2.0) * pitch
    X, Y, Z = np.meshgrid(g, g, (np.arange(layers) + 0.5) * pitch, indexing='ij')
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)[:n]
    x += rng.uniform(-0.1 * rmax, 0.1 * rmax, x.shape)
    half = side * pitch / 2.0 + rmax
    lo = [-half, -half, 0.0]; hi = [half, half, layers * pitch + 2 * rmax]
    return _sphere_scene('spheres-small-%d' % n, rng, x, r, density, lo, hi, step, friction, 0.0, 0.0,
                         settle_iters, 0.004, 1e-5)


def _hexahedron_mass(verts: np.ndarray, density: float):
    """Volume, mass centre and inertia (about the centre) of hexahedra given by
    8 vertices each, by tetrahedra from the vertex mean over the 12 surface
    triangles. verts: (n, 8, 3) ordered as the unit-cube corners (x fastest)."""
    faces = np.array([[0, 2, 3, 1], [4, 5, 7, 6], [0, 1, 5, 4], [2, 6, 7, 3], [0, 4, 6, 2], [1, 3, 7, 5]])
    tris = np.concatenate([faces[:, [0, 1, 2]], faces[:, [0, 2, 3]]], axis=0)
    o = verts.mean(axis=1)
    vol = np.zeros(verts.shape[0]); first = np.zeros((verts.shape[0], 3)); second = np.zeros((verts.shape[0], 3, 3))
    for t in tris:
        a, b, c = verts[:, t[0]] - o, verts[:, t[1]] - o, verts[:, t[2]] - o
        v = np.einsum('ij,ij->i', a, np.cross(b, c)) / 6.0
        s = a + b + c
        vol += v
        first += v[:, None] * s / 4.0
        second += (v / 20.0)[:, None, None] * (np.einsum('ni,nj->nij', a, a) + np.einsum('ni,nj->nij', b, b)
                                               + np.einsum('ni,nj->nij', c, c) + np.einsum('ni,nj->nij', s, s))
    c_rel = first / vol[:, None]
    cov = second - vol[:, None, None] * np.einsum('ni,nj->nij', c_rel, c_rel)
    J = density * (np.trace(cov, axis1=1, axis2=2)[:, None, None] * np.eye(3)[None] - cov)
    return vol, o + c_rel, J, density * vol


def _hexahedra_vertices(rng, nx, ny, nz, side, perturb):
    """Lattice indices (n, 3) and vertices (n, 8, 3) of the perturbed cubes of
    hexahedra_lattice (vertex v = i + 2 j + 4 k at corner (x_i, y_j, z_k))."""
    n = nx * ny * nz
    corners = np.array([[i, j, k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], float) - 0.5
    I, J_, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing='ij')
    idx = np.stack([I.ravel(), J_.ravel(), K.ravel()], axis=1)
    lat = np.stack([(idx[:, 0] - (nx - 1) / 2.0) * side, (idx[:, 1] - (ny - 1) / 2.0) * side,
                    (idx[:, 2] + 0.5) * side], axis=1)
    return idx, lat[:, None, :] + side * (corners[None] + rng.uniform(-perturb, perturb, (n, 8, 3)))


def hexahedra_geometry(seed: int = 3, nx: int = 100, ny: int = 100, nz: int = 10, side: float = 0.04,
                       perturb: float = 0.1, nsurf: int = 1):
    """The bodies of hexahedra_lattice as convexes for contact detection: per
    hexahedron its 8 perturbed vertices (the same seeded values) with the
    faces of HEX_FACES, and the floor and four side walls as obstacle boxes
    0.1 m thick whose inner faces are the walls' planes. Referential vertices
    are spatial ones (rotations identity, mass centres as in the scene).

    Returns set_convexes arguments."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    _, verts = _hexahedra_vertices(rng, nx, ny, nz, side, perturb)
    halfx, halfy = nx * side / 2.0 + 0.5 * side * perturb, ny * side / 2.0 + 0.5 * side * perturb
    t, top = 0.1, (nz + 2) * side
    walls = [([-halfx - t, -halfy - t, -t], [halfx + t, halfy + t, 0.0]),     # floor
             ([-halfx - t, -halfy - t, 0.0], [-halfx, halfy + t, top]),      # -x
             ([halfx, -halfy - t, 0.0], [halfx + t, halfy + t, top]),        # +x
             ([-halfx, -halfy - t, 0.0], [halfx, -halfy, top]),              # -y
             ([-halfx, halfy, 0.0], [halfx, halfy + t, top])]                # +y
    convexes = [(v, HEX_FACES, np.zeros(6, np.int32)) for v in verts]
    for lo, hi in walls:
        v, _ = box_convex(lo, hi)
        convexes.append((v, HEX_FACES, np.zeros(6, np.int32)))
    return _convex_arrays(convexes, np.arange(n + len(walls)))


def hexahedra_lattice(seed: int = 3, nx: int = 100, ny: int = 100, nz: int = 10, side: float = 0.04,
                      perturb: float = 0.1, density: float = 2000.0, friction: float = 0.4, step: float = 5e-4,
                      vel_sigma: float = 0.02) -> Scene:
    """Rigid convex hexahedra: unit cubes of side 0.04 m whose 8 vertices get
    seeded uniform perturbations of +-10% of the side, density 2000, stacked
    face to face on a jittered nx x ny x nz lattice resting on the floor of a
    4x4x3 m box; friction 0.4, h = 5e-4.

    Contacts (a simplified convex-convex generator; the reference uses the
    polyhedral intersection of cvi.c): one contact per face-adjacent pair and
    per face resting on a wall, at the mid-point of the two facing face
    centroids, with the normal the normalised mean of the two facing face
    normals and a settled interpenetration gap drawn from -|N(0, 2e-5)| m."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    idx, verts = _hexahedra_vertices(rng, nx, ny, nz, side, perturb)
    vol, xc, Jt, mass_b = _hexahedron_mass(verts, density)
    # face vertex sets (outward): -x, +x, -y, +y, -z, +z
    fv = {0: [0, 2, 6, 4], 1: [1, 5, 7, 3], 2: [0, 4, 5, 1], 3: [2, 3, 7, 6], 4: [0, 1, 3, 2], 5: [4, 6, 7, 5]}

    def face(f):
        q = verts[:, fv[f]]
        cen = q.mean(axis=1)
        nrm = np.cross(q[:, 2] - q[:, 0], q[:, 3] - q[:, 1])
        nrm *= np.sign(np.einsum('ij,ij->i', nrm, cen - xc))[:, None]   # orient outward
        return cen, nrm / np.linalg.norm(nrm, axis=1, keepdims=True)

    F = [face(f) for f in range(6)]
    body_of = np.empty((nx, ny, nz), np.int64)
    body_of[idx[:, 0], idx[:, 1], idx[:, 2]] = np.arange(n)
    masters, slaves, points, normals = [], [], [], []
    for axis, (fneg, fpos) in enumerate(((0, 1), (2, 3), (4, 5))):
        sl_lo = [slice(None)] * 3; sl_hi = [slice(None)] * 3
        sl_lo[axis] = slice(0, -1); sl_hi[axis] = slice(1, None)
        a = body_of[tuple(sl_lo)].ravel(); b = body_of[tuple(sl_hi)].ravel()   # a below/left, b above/right
        nrm = F[fpos][1][a] - F[fneg][1][b]
        nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
        p = 0.5 * (F[fpos][0][a] + F[fneg][0][b])
        masters.append(b); slaves.append(a); points.append(p); normals.append(nrm)   # normal from slave a to master b
    # walls: floor and four sides of the box around the lattice
    halfx, halfy = nx * side / 2.0 + 0.5 * side * perturb, ny * side / 2.0 + 0.5 * side * perturb
    walls_n = np.array([[0, 0, 1], [1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0]], float)
    walls_p = np.array([[0, 0, 0], [-halfx, 0, 0], [halfx, 0, 0], [0, -halfy, 0], [0, halfy, 0]], float)
    wall_faces = [(4, body_of[:, :, 0].ravel()), (0, body_of[0, :, :].ravel()), (1, body_of[-1, :, :].ravel()),
                  (2, body_of[:, 0, :].ravel()), (3, body_of[:, -1, :].ravel())]
    for w, (f, bodies) in enumerate(wall_faces):
        cen = F[f][0][bodies]
        nn = np.repeat(walls_n[w][None], bodies.size, axis=0)
        p = cen.copy()
        p -= nn * ((cen - walls_p[w]) @ walls_n[w])[:, None] * 0.5
        masters.append(bodies); slaves.append(np.full(bodies.size, n + w)); points.append(p); normals.append(nn)
    master = np.concatenate(masters).astype(np.int32); slave = np.concatenate(slaves).astype(np.int32)
    points = np.concatenate(points); normals = np.concatenate(normals)
    gaps = -np.abs(rng.normal(0.0, 2e-5, master.shape[0]))
    nb = n + walls_n.shape[0]
    xb = np.concatenate([xc, walls_p], axis=0)
    rot = np.zeros((nb, 9)); rot[:, 0] = rot[:, 4] = rot[:, 8] = 1.0
    x0 = xb.copy()
    jinv = np.zeros((nb, 9)); jinv[:n] = _colmajor(np.linalg.inv(Jt))
    minv = np.zeros(nb); minv[:n] = 1.0 / mass_b
    mass = np.ones(nb); mass[:n] = mass_b
    velo0 = np.zeros((nb, 6))
    if vel_sigma > 0:
        velo0[:n, 3:6] = rng.normal(0.0, vel_sigma, (n, 3))
        velo0[:n, 0:3] = rng.normal(0.0, vel_sigma / side, (n, 3))
    obstacle = np.zeros(nb, np.int32); obstacle[n:] = 1
    return _assemble_scene('hexahedra-lattice-%d' % n, step, xb, rot, x0, jinv, minv, mass, velo0, obstacle,
                           master, slave, points, normals, gaps, friction, 0.0, 0.0)


def batched_scene_specs(seed: int = 4, count: int = 256, nmin: int = 50, nmax: int = 2000, settle_iters: int = 300):
    """Arguments of spheres_small for each scene of the batched workload: body
    count log-uniform in [nmin, nmax], radius U[0.02, 0.05], friction
    U[0.2, 0.6], h = 1e-3."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(nmin), math.log(nmax), count)).astype(int)
    fr = rng.uniform(0.2, 0.6, count)
    return [(seed * 100003 + s, int(sizes[s]), float(fr[s]), settle_iters) for s in range(count)]


def batched_scene(spec) -> Scene:
    seed, n, friction, settle_iters = spec
    return spheres_small(seed, n, friction=friction, settle_iters=settle_iters)


def batched_scenes(seed: int = 4, count: int = 256, nmin: int = 50, nmax: int = 2000, settle_iters: int = 300,
                   workers: int = 1):
    """Uneven independent sphere scenes (see batched_scene_specs); with
    workers > 1 they are generated by a spawned process pool."""
    specs = batched_scene_specs(seed, count, nmin, nmax, settle_iters)
    if workers > 1:
        import multiprocessing as mp
        with mp.get_context('spawn').Pool(workers) as pool:
            return pool.map(batched_scene, specs, chunksize=1)
    return [batched_scene(sp) for sp in specs]


def box_inertia(mass: float, a: float, b: float, c: float) -> np.ndarray:
    """Referential inertia (column-major 9) of a solid a x b x c box about its
    mass centre."""
    return np.diag([mass * (b * b + c * c) / 12.0, mass * (a * a + c * c) / 12.0,
                    mass * (a * a + b * b) / 12.0]).reshape(9)


def block_sliding(step: float = 1e-3, friction: float = 0.8, density: float = 111.11111111111111111):
    """The scene of the reference's tests/block-sliding.py as a fixed contact
    set: a 0.3 x 0.3 x 0.1 block (mass 1) resting on a 1 x 0.3 x 0.1 table
    (an obstacle), both translated by (3, 0, 0). The block touches the table
    with its bottom face, split 2 x 2 as the test's HEX (cube, 2, 2, 1) mesh
    splits it: one contact at the centre of each quarter, normal +z (from the
    table to the block), gap 0, friction 0.8, no restitution or cohesion.
    Returns (scene, J, mass): the inertia and masses for RIGID_DYNAMICS."""
    xt = np.array([3.0, 0.0, -0.05])   # table centre
    xb = np.array([3.0, 0.0, 0.05])    # block centre
    mt = density * (1.0 * 0.3 * 0.1)
    mb = density * (0.3 * 0.3 * 0.1)
    J = np.stack([box_inertia(mt, 1.0, 0.3, 0.1), box_inertia(mb, 0.3, 0.3, 0.1)])
    jinv = np.stack([np.linalg.inv(Ji.reshape(3, 3)).T.reshape(9) for Ji in J])
    mass = np.array([mt, mb])
    pts = np.array([[3.0 + dx, dy, 0.0] for dx in (-0.075, 0.075) for dy in (-0.075, 0.075)])
    nc = pts.shape[0]
    base = np.tile(np.eye(3).T.reshape(9), (nc, 1))  # columns t1 = x, t2 = y, n = z
    scene = Scene(name='block-sliding', step=step, dynamic=1,
                  rot=np.tile(np.eye(3).reshape(9), (2, 1)), x=np.stack([xt, xb]), x0=np.stack([xt, xb]),
                  jinv=jinv, minv=1.0 / mass, velo=np.zeros((2, 6)), velo0=np.zeros((2, 6)),
                  obstacle=np.array([1, 0], dtype=np.int32),
                  master=np.full(nc, 1, dtype=np.int32), slave=np.zeros(nc, dtype=np.int32),
                  mpnt=pts.copy(), spnt=pts.copy(), base=base, gap=np.zeros(nc), friction=np.full(nc, friction),
                  restitution=np.zeros(nc), cohesion=np.zeros(nc), mass=mass)
    return scene, J, mass


def masonry_arch(ratio: float, step: float = 1e-3, friction: float = 0.5, density: float = 1.0, n: int = 27,
                 radius: float = 10.0, width: float = 5.0):
    """The scene of the reference's tests/arch.py as a fixed contact set: a
    semicircular arch of n voussoirs (angle pi/n each, radius 10, thickness
    ratio * radius, width 5, density 1) between two obstacle bases of one
    voussoir each. The test meshes every voussoir 3 x 2 x 1, with radial cells
    of relative sizes 0.05, 1.9, 0.05 (from the extrados) and two equal cells
    across the width, so two touching voussoirs meet face to face on six cell
    faces; the reference's convex-convex contact of two touching cells sits at
    the centre of their common face. Each interface therefore carries six
    contacts, at the cell-face centres, with the interface's normal (from the
    voussoir at the lower angle to the one at the higher), gap 0, friction
    0.5, no restitution or cohesion. Angles are measured from the vertical
    (x = r sin a, z = r cos a). Returns (scene, J, mass)."""
    dalpha = math.pi / n
    t = ratio * radius

    def hexahedron(alpha):  # the test's node order: far/near at the lower angle, then at the upper angle
        out = []
        for a in (alpha, alpha + dalpha):
            for rr, y in ((radius + t / 2, -width / 2), (radius - t / 2, -width / 2), (radius - t / 2, width / 2),
                          (radius + t / 2, width / 2)):
                out.append([rr * math.sin(a), y, rr * math.cos(a)])
        return np.array(out)

    lows = [-0.5 * math.pi - dalpha, 0.5 * math.pi] + [-0.5 * math.pi + i * dalpha for i in range(n)]
    nodes = np.stack([hexahedron(a) for a in lows])
    corners = nodes[:, [0, 1, 3, 2, 4, 5, 7, 6]]          # unit-cube corner order (radial, width, angle)
    vol, xc, Jc, mass = _hexahedron_mass(corners, density)
    if np.any(vol <= 0):
        vol, xc, Jc, mass = _hexahedron_mass(corners[:, [1, 0, 3, 2, 5, 4, 7, 6]], density)
    nb = n + 2
    obstacle = np.zeros(nb, dtype=np.int32); obstacle[:2] = 1
    J = Jc.reshape(nb, 9)
    jinv = np.stack([np.linalg.inv(Ji.reshape(3, 3)).T.reshape(9) for Ji in J])
    jinv[obstacle != 0] = 0.0
    minv = np.where(obstacle != 0, 0.0, 1.0 / mass)
    # interfaces k = 0 .. n at angle -pi/2 + k dalpha: slave = the body below, master = the body above
    below = [0] + [2 + i for i in range(n)]
    above = [2 + i for i in range(n)] + [1]
    fr = [0.0125, 0.5, 0.9875]                            # cell-face centres, fraction of t from the extrados
    pts, nrm, master, slave = [], [], [], []
    for k in range(n + 1):
        a = -0.5 * math.pi + k * dalpha
        for f in fr:
            rr = radius + t / 2 - f * t
            for y in (-width / 4, width / 4):
                pts.append([rr * math.sin(a), y, rr * math.cos(a)])
                nrm.append([math.cos(a), 0.0, -math.sin(a)])
                master.append(above[k]); slave.append(below[k])
    pts = np.array(pts); nc = pts.shape[0]
    scene = Scene(name='masonry-arch-%g' % ratio, step=step, dynamic=1, rot=np.tile(np.eye(3).reshape(9), (nb, 1)),
                  x=xc.copy(), x0=xc.copy(), jinv=jinv, minv=minv, velo=np.zeros((nb, 6)), velo0=np.zeros((nb, 6)),
                  obstacle=obstacle, master=np.array(master, dtype=np.int32), slave=np.array(slave, dtype=np.int32),
                  mpnt=pts.copy(), spnt=pts.copy(), base=local_base(np.array(nrm)), gap=np.zeros(nc),
                  friction=np.full(nc, friction), restitution=np.zeros(nc), cohesion=np.zeros(nc), mass=mass)
    Jr = J.copy(); Jr[obstacle != 0] = np.eye(3).reshape(9)
    massr = np.where(obstacle != 0, 1.0, mass)
    return scene, Jr, massr


def block_sliding_loads(t: float) -> np.ndarray:
    """The test's block_force callback, 8 cos(t) along x on the block, as the
    (nbod, 9) load triples RIGID_DYNAMICS.step_begin takes."""
    L = np.zeros((2, 9))
    L[1, 0] = 8.0 * np.cos(t)
    return L


def projectile():
    """The scene of the reference's tests/projectile.py: one rigid body of mass
    0.45359237 kg and unit inertia at the origin, launched at (2.54, 0, 12.7)
    m/s under gravity 9.81456 m/s^2, with a drag load -m v evaluated from the
    velocity at the start of each step (projectile_loads); no contacts. Step
    1.976 / 1024 s. Returns (scene, J, mass)."""
    m = 0.45359237
    z3, z9 = np.zeros((0, 3)), np.zeros((0, 9))
    zi, zd = np.zeros(0, dtype=np.int32), np.zeros(0)
    velo = np.array([[0.0, 0.0, 0.0, 2.54, 0.0, 12.7]])
    scene = Scene(name='projectile', step=1.976 / 1024.0, dynamic=1, rot=np.eye(3).reshape(1, 9),
                  x=np.zeros((1, 3)), x0=np.zeros((1, 3)), jinv=np.eye(3).reshape(1, 9), minv=np.array([1.0 / m]),
                  velo=velo, velo0=velo.copy(), obstacle=np.zeros(1, dtype=np.int32), master=zi, slave=zi,
                  mpnt=z3, spnt=z3, base=z9, gap=zd, friction=zd, restitution=zd, cohesion=zd, mass=np.array([m]))
    return scene, np.eye(3).reshape(1, 9), np.array([m])


def projectile_loads(mass: float, velo: np.ndarray) -> np.ndarray:
    """The test's projectile_force callback, (-m v, 0, 0), from the body's
    velocity [Omega; v] at the start of the step."""
    L = np.zeros((1, 9))
    L[0, 0:3] = [-mass * velo[3], -mass * velo[4], -mass * velo[5]]
    return L


PROJECTILE_GRAVITY = 9.81456


def _one_body_rows(name, step, x, J, mass, kinds, mpnt, spnt, base, gap, Z):
    """A scene of one rigid body (index 0) whose rows are bilateral
    constraints without a slave body (slave -1, spnt the spatial point)."""
    nc = len(kinds)
    jinv = np.linalg.inv(J.reshape(3, 3).T).T.reshape(1, 9)
    scene = Scene(name=name, step=step, dynamic=1, rot=np.eye(3).reshape(1, 9), x=x.reshape(1, 3).copy(),
                  x0=x.reshape(1, 3).copy(), jinv=jinv, minv=np.array([1.0 / mass]), velo=np.zeros((1, 6)),
                  velo0=np.zeros((1, 6)), obstacle=np.zeros(1, dtype=np.int32),
                  master=np.zeros(nc, dtype=np.int32), slave=np.full(nc, -1, dtype=np.int32),
                  mpnt=np.asarray(mpnt, float).reshape(nc, 3), spnt=np.asarray(spnt, float).reshape(nc, 3),
                  base=np.asarray(base, float).reshape(nc, 9), gap=np.asarray(gap, float).reshape(nc),
                  friction=np.zeros(nc), restitution=np.zeros(nc), cohesion=np.zeros(nc), mass=np.array([mass]))
    return (scene, J.reshape(1, 9).copy(), np.array([mass]), np.asarray(kinds, dtype=np.int32),
            np.asarray(Z, float).reshape(nc, 4))


MATH_PENDULUM_GRAVITY = math.pi * math.pi


def math_pendulum(step: float = 1e-3):
    """The scene of the reference's tests/math-pendulum.py: a rigid ball of
    mass 1 and unit inertia centred at (1, 0, 1) on a rigid link
    (PUT_RIGID_LINK, dom.c:3379-3427) of length 1 to the fixed point (0, 0, 1),
    at rest on the horizontal, under gravity pi^2 (MATH_PENDULUM_GRAVITY), so
    that the period from the horizontal is 2.36 s. One RIGLNK row: master the
    ball at its centre, no slave, spnt the fixed point; a frame with the link
    direction as its normal, gap 0 and Z = (the link in that frame, length 1)
    until the first step's update_riglnk (dom.c:524-550) replaces them.
    Returns (scene, J, mass, kinds, Z)."""
    n = np.array([[1.0, 0.0, 0.0]])
    base = local_base(n)
    link = base.reshape(3, 3, order='F').T @ n[0]
    return _one_body_rows('math-pendulum', step, np.array([1.0, 0.0, 1.0]), np.eye(3).reshape(9), 1.0, [5],
                          [[1.0, 0.0, 1.0]], [[0.0, 0.0, 1.0]], base, [0.0], [[link[0], link[1], link[2], 1.0]])


DOUBLE_PENDULUM_GRAVITY = 9.81


def _length(v) -> float:
    """LEN of alg.h: sqrt of the dot product summed left to right."""
    return math.sqrt(float(v[0]) * float(v[0]) + float(v[1]) * float(v[1]) + float(v[2]) * float(v[2]))


def double_pendulum(step: float = 1e-3):
    """The scene of the reference's tests/double-pendulum.py: two rigid balls
    (SPHERE radius 0.05, surface 1, mass 1, unit inertia) hanging from the
    fixed point a = (0, 0, 2) by two rigid links of length 1: ball 1 at
    b = a + (sin 60, 0, -cos 60) linked to a, ball 2 at c = b + (sin 36, 0,
    -cos 36) linked to ball 1 (PUT_RIGID_LINK (bod2, bod1, c, b)); a fixed
    0.05 x 0.4 x 2 box (HEX obstacle, surfaces 0) at x in [-0.1, -0.05] that
    the balls strike; SIGNORINI_COULOMB with restitution 0.1, no friction;
    gravity 9.81 (DOUBLE_PENDULUM_GRAVITY). The test sets GEOMETRIC_EPSILON to
    1e-5; the device detection keeps the default 1e-6.
    Returns (scene without contacts, SPHERES arguments with the box as
    `convex`, SPHERES.set_constraints arguments, J, mass)."""
    x1, z1 = math.sin(math.pi / 3.0), -math.cos(math.pi / 3.0)
    x2, z2 = x1 + math.sin(math.pi / 5.0), z1 - math.cos(math.pi / 5.0)
    a = np.array([0.0, 0.0, 2.0])
    b = np.array([x1, 0.0, 2.0 + z1])
    c = np.array([x2, 0.0, 2.0 + z2])
    lo, hi = np.array([-0.10, -0.2, 0.0]), np.array([-0.05, 0.2, 2.0])
    x = np.stack([b, c, 0.5 * (lo + hi)])
    nb = 3
    jinv = np.zeros((nb, 9)); jinv[:2] = np.eye(3).reshape(9)
    mass = np.ones(nb)
    z = np.zeros((nb, 6)); e = np.zeros(0)
    sc = Scene(name='double-pendulum', step=step, dynamic=1, rot=np.tile(np.eye(3).reshape(9), (nb, 1)), x=x.copy(),
               x0=x.copy(), jinv=jinv, minv=np.array([1.0, 1.0, 0.0]), velo=z.copy(), velo0=z.copy(),
               obstacle=np.array([0, 0, 1], np.int32), master=np.zeros(0, np.int32), slave=np.zeros(0, np.int32),
               mpnt=np.zeros((0, 3)), spnt=np.zeros((0, 3)), base=np.zeros((0, 9)), gap=e, friction=e,
               restitution=e, cohesion=e, mass=mass, radius=np.array([0.05, 0.05, 0.0]))
    v, f = box_convex(lo, hi)
    convex = dict(body=np.array([2], np.int32), vptr=np.array([0, 8], np.int32), vert=v,
                  fptr=np.array([0, f.shape[0]], np.int32), fac=f, sptr=np.array([0, 6], np.int32),
                  surf=np.zeros(6, np.int32))
    mat = np.zeros((2, 2, 2)); mat[:, :, 1] = 0.1
    spheres = dict(body=np.array([0, 1], np.int32), centre=np.stack([b, c]), radius=np.array([0.05, 0.05]),
                   surface=np.array([1, 1], np.int32), material=mat, convex=convex)
    base = np.tile(np.eye(3).reshape(9), (2, 1))  # replaced by the first update_riglnk
    constraints = dict(kinds=np.array([5, 5], np.int32), master=np.array([0, 1], np.int32),
                       slave=np.array([-1, 0], np.int32), mpnt=np.stack([b, c]), spnt=np.stack([a, b]), base=base,
                       Z=np.array([[0.0, 0.0, 1.0, _length(b - a)], [0.0, 0.0, 1.0, _length(c - b)]]))
    J = np.tile(np.eye(3).reshape(9), (nb, 1))
    return sc, spheres, constraints, J, mass


PINNED_BAR_GRAVITY = 9.8


def pinned_bar(step: float = 1e-3):
    """The scene of the reference's tests/pinned-bar.py: a rigid 0.1 x 0.1 x 1
    bar of density 1 (its mesh from z = 0 to 1, centred on the z axis),
    turned by -30 degrees about the y axis through (0, 0, 0.75), with two
    FIX_POINT constraints (DOM_Fix_Point, dom.c:3272-3292: identity base) at
    (0, -0.05, 0.75) and (0, 0.05, 0.75), which make a hinge about y; gravity
    9.8 (PINNED_BAR_GRAVITY). Released at rest, the bar swings about the
    hinge; the test reads its angular velocity about y when the mass centre
    passes x = 0 (2.121 rad/s). Returns (scene, J, mass, kinds, Z)."""
    mass = 0.1 * 0.1 * 1.0
    a = -math.radians(30.0)  # right-handed turn about +y
    Ry = np.array([[math.cos(a), 0.0, math.sin(a)], [0.0, 1.0, 0.0], [-math.sin(a), 0.0, math.cos(a)]])
    pivot = np.array([0.0, 0.0, 0.75])
    x = pivot + Ry @ (np.array([0.0, 0.0, 0.5]) - pivot)
    J = Ry @ box_inertia(mass, 0.1, 0.1, 1.0).reshape(3, 3) @ Ry.T
    pts = [[0.0, -0.05, 0.75], [0.0, 0.05, 0.75]]
    return _one_body_rows('pinned-bar', step, x, J.T.reshape(9), mass, [1, 1], pts, pts,
                          np.tile(np.eye(3).reshape(9), (2, 1)), [0.0, 0.0], np.zeros((2, 4)))


def advance_velocities(scene: Scene, R: np.ndarray) -> Scene:
    """One velocity step of the rigid bodies with the solved reactions: the new
    velocity at t is u = u_free + h M^-1 sum H^T R (bod.c:418-439 force
    accumulation, bod.c:1425-1493 second half step), then a new free velocity
    u_free' = u + h M^-1 f_ext. Geometry is kept (a one-step snapshot), so the
    returned scene is the next solve of the same contact set, warm-started by R."""
    nb = scene.nbod
    imp = np.zeros((nb, 6))
    Rw = np.einsum('nij,nj->ni', scene.base.reshape(-1, 3, 3).transpose(0, 2, 1), R)
    for side, pnt, sign in ((scene.master, scene.mpnt, 1.0), (scene.slave, scene.spnt, -1.0)):
        ok = side >= 0
        b = side[ok]
        rot = scene.rot[b].reshape(-1, 3, 3).transpose(0, 2, 1)
        lever = np.einsum('nij,nj->ni', rot, pnt[ok] - scene.x0[b])          # spatial lever arm
        f = sign * Rw[ok]
        torque_w = np.cross(lever, f)
        torque_b = np.einsum('nji,nj->ni', rot, torque_w)                  # body-frame torque
        np.add.at(imp, b, np.concatenate([torque_b, f], axis=1))
    J = scene.jinv.reshape(-1, 3, 3).transpose(0, 2, 1)
    du = np.zeros((nb, 6))
    du[:, 0:3] = np.einsum('nij,nj->ni', J, imp[:, 0:3])
    du[:, 3:6] = scene.minv[:, None] * imp[:, 3:6]
    movable = scene.obstacle == 0
    u = scene.velo.copy()
    u[movable] += scene.step * du[movable]
    nxt = dataclasses.replace(scene)
    nxt.velo0 = np.ascontiguousarray(u)
    uf = u.copy()
    uf[movable, 3:6] += scene.step * GRAVITY
    nxt.velo = np.ascontiguousarray(uf)
    return nxt


CONFIGS = {
    'spheres1k': spheres_lattice,
    'spheres20k': spheres_polydisperse,
    'hexahedra100k': hexahedra_lattice,
}


# ----------------------------------------------------------------------------- sphere shapes for detection

def sphere_shapes(scene: Scene, friction: float = None, restitution: float = 0.0) -> dict:
    """SPHERES arguments for the sphere bodies of a scene (radius > 0): one
    sphere per body, centred on its referential mass centre, one surface, and
    the scene's friction (its first contact's) unless given."""
    if scene.radius is None:
        raise ValueError('scene %s has no sphere bodies' % scene.name)
    body = np.nonzero(scene.radius > 0)[0].astype(np.int32)
    if friction is None:
        friction = float(scene.friction[0]) if scene.ncon else 0.0
    return dict(body=body, centre=scene.x0[body].copy(), radius=scene.radius[body].copy(),
                surface=np.zeros(body.shape[0], np.int32), material=(float(friction), float(restitution)))


def sphere_inertia(scene: Scene):
    """(J, mass) of a sphere scene for RIGID_DYNAMICS: J = 0.4 m r^2 I for the
    spheres, the identity and mass 1 for the other (obstacle) bodies."""
    nb = scene.nbod
    mass = np.ones(nb) if scene.mass is None else np.asarray(scene.mass, float).copy()
    J = np.zeros((nb, 9))
    r = np.zeros(nb) if scene.radius is None else scene.radius
    for k in (0, 4, 8):
        J[:, k] = np.where(r > 0, 0.4 * mass * r ** 2, 1.0)
    return J, mass


def spheres_on_bed(seed: int = 5, n_side: int = 6, layers: int = 3, radius: float = 0.05, pitch: float = 0.11,
                   bed_radius: float = 0.1, bed_pitch: float = 0.2, density: float = 2000.0, friction: float = 0.3,
                   step: float = 1e-3, drop: float = 0.002):
    """Spheres falling onto a bed of fixed spheres: an n_side x n_side x layers
    jittered lattice of spheres (radius, pitch) above a square grid of obstacle
    spheres (bed_radius, bed_pitch) covering the lattice's footprint. The lowest
    layer starts ``drop`` above the bed. Every body is one sphere, so the
    contacts come from sphere detection alone.

    Returns (scene without contacts, SPHERES arguments, J, mass)."""
    rng = np.random.default_rng(seed)
    half = (n_side - 1) / 2.0 * pitch + radius
    nbed = int(np.ceil(2 * half / bed_pitch)) + 1
    gb = (np.arange(nbed) - (nbed - 1) / 2.0) * bed_pitch
    BX, BY = np.meshgrid(gb, gb, indexing='ij')
    bed = np.stack([BX.ravel(), BY.ravel(), np.zeros(BX.size)], axis=1)
    g = (np.arange(n_side) - (n_side - 1) / 2.0) * pitch
    z0 = bed_radius + radius + drop
    X, Y, Z = np.meshgrid(g, g, z0 + np.arange(layers) * pitch, indexing='ij')
    xs = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    xs[:, :2] += rng.uniform(-0.1 * (pitch - 2 * radius), 0.1 * (pitch - 2 * radius), (xs.shape[0], 2))
    n = xs.shape[0]
    nb = n + bed.shape[0]
    x = np.concatenate([xs, bed], axis=0)
    r = np.concatenate([np.full(n, radius), np.full(bed.shape[0], bed_radius)])
    mass = np.ones(nb); mass[:n] = density * 4.0 / 3.0 * math.pi * radius ** 3
    jinv = np.zeros((nb, 9)); jinv[:n, 0] = jinv[:n, 4] = jinv[:n, 8] = 1.0 / (0.4 * mass[:n] * radius ** 2)
    minv = np.zeros(nb); minv[:n] = 1.0 / mass[:n]
    rot = np.zeros((nb, 9)); rot[:, 0] = rot[:, 4] = rot[:, 8] = 1.0
    rot[:n] = _random_rotations(rng, n)
    obstacle = np.zeros(nb, np.int32); obstacle[n:] = 1
    z = np.zeros((nb, 6))
    e = np.zeros(0)
    sc = Scene(name='spheres-on-bed-%d' % n, step=step, dynamic=1, rot=rot, x=x.copy(), x0=x.copy(), jinv=jinv,
               minv=minv, velo=z.copy(), velo0=z.copy(), obstacle=obstacle, master=np.zeros(0, np.int32),
               slave=np.zeros(0, np.int32), mpnt=np.zeros((0, 3)), spnt=np.zeros((0, 3)), base=np.zeros((0, 9)),
               gap=e, friction=e, restitution=e, cohesion=e, mass=mass, radius=r)
    J, mass = sphere_inertia(sc)
    sph = dict(body=np.arange(nb, dtype=np.int32), centre=x.copy(), radius=r.copy(),
               surface=np.zeros(nb, np.int32), material=(friction, 0.0))
    return sc, sph, J, mass


def spheres_grid(n_side: int = 100, radius: float = 0.05, pitch: float = 0.0999, jitter: float = 1e-5,
                 density: float = 2000.0, seed: int = 8, step: float = 1e-3) -> Scene:
    """n_side^3 spheres on a cubic grid whose face neighbours overlap by
    2 radius - pitch (jittered by +-jitter per coordinate), no obstacles and no
    contacts: a detection workload with six contacts per interior sphere."""
    rng = np.random.default_rng(seed)
    g = np.arange(n_side) * pitch
    X, Y, Z = np.meshgrid(g, g, g, indexing='ij')
    x = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1) + rng.uniform(-jitter, jitter, (n_side ** 3, 3))
    n = x.shape[0]
    m = density * 4.0 / 3.0 * math.pi * radius ** 3
    eye = np.tile(np.eye(3).reshape(9), (n, 1))
    e = np.zeros(0)
    return Scene(name='spheres-grid-%d' % n, step=step, dynamic=1, rot=eye.copy(), x=x, x0=x.copy(),
                 jinv=eye / (0.4 * m * radius ** 2), minv=np.full(n, 1.0 / m), velo=np.zeros((n, 6)),
                 velo0=np.zeros((n, 6)), obstacle=np.zeros(n, np.int32), master=np.zeros(0, np.int32),
                 slave=np.zeros(0, np.int32), mpnt=np.zeros((0, 3)), spnt=np.zeros((0, 3)), base=np.zeros((0, 9)),
                 gap=e, friction=e, restitution=e, cohesion=e, mass=np.full(n, m), radius=np.full(n, radius))


# faces of a hexahedron whose vertex v = i + 2 j + 4 k sits at corner (x_i, y_j, z_k):
# counter-clockwise seen from outside, so (b - a) x (c - b) points out
HEX_FACES = ((0, 4, 6, 2), (1, 3, 7, 5), (0, 1, 5, 4), (2, 6, 7, 3), (0, 2, 3, 1), (4, 5, 7, 6))


def box_convex(lo, hi):
    """Vertices (8, 3) and faces (reference fac layout: count, then indices) of
    the axis-aligned box [lo, hi]."""
    lo = np.asarray(lo, float); hi = np.asarray(hi, float)
    v = np.array([[(lo, hi)[i][0], (lo, hi)[j][1], (lo, hi)[k][2]] for k in (0, 1) for j in (0, 1) for i in (0, 1)])
    fac = []
    for f in HEX_FACES:
        fac += [4] + list(f)
    return v, np.array(fac, np.int32)


def _convex_arrays(convexes, bodies):
    """set_convexes arguments from a list of (vertices (nv, 3), faces as vertex
    index lists, surface id per face) and a body per convex."""
    vptr, fptr, sptr, vert, fac, surf = [0], [0], [0], [], [], []
    for (v, faces, sids) in convexes:
        vert.append(np.asarray(v, float))
        for f in faces:
            fac += [len(f)] + list(f)
        surf += list(sids)
        vptr.append(vptr[-1] + len(v)); fptr.append(len(fac)); sptr.append(len(surf))
    return dict(body=np.asarray(bodies, np.int32), vptr=np.array(vptr, np.int32), vert=np.concatenate(vert),
                fptr=np.array(fptr, np.int32), fac=np.array(fac, np.int32), sptr=np.array(sptr, np.int32),
                surf=np.array(surf, np.int32))


def convex_list(cv):
    """Per convex of set_convexes arguments: (vertices (nv, 3), reference face
    layout (count, then indices), surface ids)."""
    out = []
    for c in range(cv['body'].shape[0]):
        out.append((cv['vert'][cv['vptr'][c]:cv['vptr'][c + 1]], cv['fac'][cv['fptr'][c]:cv['fptr'][c + 1]],
                    cv['surf'][cv['sptr'][c]:cv['sptr'][c + 1]]))
    return out


def hull_faces(points):
    """Triangles of the convex hull of points, counter-clockwise seen from
    outside: (vertices used, faces as index triples)."""
    from scipy.spatial import ConvexHull
    P = np.asarray(points, float)
    H = ConvexHull(P)
    used = sorted(set(H.simplices.ravel()))
    remap = {u: i for i, u in enumerate(used)}
    V = P[used]
    cen = V.mean(axis=0)
    faces = []
    for s in H.simplices:
        a, b, c = (remap[i] for i in s)
        if np.dot(np.cross(V[b] - V[a], V[c] - V[b]), V[a] - cen) < 0:
            b, c = c, b
        faces.append((a, b, c))
    return V, faces


def convex_pile(seed: int = 1, nx: int = 5, ny: int = 4, nz: int = 3, hulls: int = 20, nsurf: int = 7):
    """Convex bodies for contact detection checks, every body at the origin
    with the identity rotation (its convex's vertices are its current ones):
    an nx x ny x nz lattice of unit boxes on a floor obstacle, a third of them
    exact (faces touching exactly), the rest with sizes and positions jittered
    by a few thousandths (touching, slightly overlapping or slightly apart),
    some of those turned by up to 3 degrees; `hulls` random convex hulls of 6 to
    8 points dropped over the top layer and among the boxes. Surface ids are
    seeded per face in 0 .. nsurf - 1.

    Returns (scene without contacts, set_convexes arguments)."""
    rng = np.random.default_rng(seed)
    convexes, kinds = [], []

    def box(c, h, R=None):
        v = np.array([[(-h[0], h[0])[i], (-h[1], h[1])[j], (-h[2], h[2])[k]] for k in (0, 1) for j in (0, 1)
                      for i in (0, 1)])
        if R is not None:
            v = v @ R.T
        return v + c

    def turn(angle):
        w = rng.normal(size=3)
        w *= angle / np.linalg.norm(w)
        K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
        a = np.linalg.norm(w)
        return np.eye(3) + np.sin(a) / a * K + (1 - np.cos(a)) / a ** 2 * K @ K

    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                c = np.array([i, j, k + 0.5], float)
                t = rng.integers(3)
                if t == 0:
                    v = box(c, np.full(3, 0.5))
                elif t == 1:
                    v = box(c + rng.uniform(-2e-3, 2e-3, 3), 0.5 * (1 + rng.uniform(-3e-3, 3e-3, 3)))
                else:
                    v = box(c + rng.uniform(-2e-3, 2e-3, 3), 0.5 * (1 + rng.uniform(-3e-3, 3e-3, 3)),
                            turn(rng.uniform(0, np.radians(3))))
                convexes.append((v, HEX_FACES, rng.integers(nsurf, size=6)))
    for _ in range(hulls):
        c = np.array([rng.uniform(0, nx - 1), rng.uniform(0, ny - 1), rng.uniform(nz - 0.6, nz + 0.3)])
        V, faces = hull_faces(c + rng.normal(size=(int(rng.integers(6, 9)), 3)) * 0.3)
        convexes.append((V, faces, rng.integers(nsurf, size=len(faces))))
    floor = box(np.array([(nx - 1) / 2, (ny - 1) / 2, -0.25]), np.array([nx / 2 + 1, ny / 2 + 1, 0.25]))
    convexes.append((floor, HEX_FACES, rng.integers(nsurf, size=6)))
    nb = len(convexes)
    obstacle = np.zeros(nb, np.int32); obstacle[-1] = 1
    e = np.zeros(0)
    eye = np.tile(np.eye(3).reshape(9), (nb, 1))
    sc = Scene(name='convex-pile-%d' % nb, step=1e-3, dynamic=1, rot=eye.copy(), x=np.zeros((nb, 3)),
               x0=np.zeros((nb, 3)), jinv=np.where(obstacle[:, None] != 0, 0.0, eye), minv=1.0 - obstacle,
               velo=np.zeros((nb, 6)), velo0=np.zeros((nb, 6)), obstacle=obstacle, master=np.zeros(0, np.int32),
               slave=np.zeros(0, np.int32), mpnt=np.zeros((0, 3)), spnt=np.zeros((0, 3)), base=np.zeros((0, 9)),
               gap=e, friction=e, restitution=e, cohesion=e, mass=np.ones(nb))
    return sc, _convex_arrays(convexes, np.arange(nb))


def convex_lattice(seed: int = 11, nx: int = 50, ny: int = 50, nz: int = 10, nsurf: int = 4):
    """Convex bodies for detection timing, as convex_pile without hulls: an
    nx x ny x nz lattice of unit boxes on a floor obstacle, a third exact
    (faces, edges and corners of exact neighbours touching), a third with
    sizes and positions jittered by a few thousandths, a third also turned by
    up to 3 degrees; every body at the origin with the identity rotation.

    Returns (scene without contacts, set_convexes arguments)."""
    rng = np.random.default_rng(seed)
    n = nx * ny * nz
    I, J_, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing='ij')
    c = np.stack([I.ravel(), J_.ravel(), K.ravel() + 0.5], axis=1).astype(float)
    kind = rng.integers(3, size=n)
    h = np.full((n, 3), 0.5)
    jit = kind > 0
    h[jit] = 0.5 * (1 + rng.uniform(-3e-3, 3e-3, (int(jit.sum()), 3)))
    c[jit] += rng.uniform(-2e-3, 2e-3, (int(jit.sum()), 3))
    corners = np.array([[i, j, k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], float) * 2 - 1
    v = corners[None] * h[:, None, :]
    rot = kind == 2
    if rot.any():
        m = int(rot.sum())
        w = rng.normal(size=(m, 3))
        w *= (rng.uniform(0, np.radians(3), m) / np.linalg.norm(w, axis=1))[:, None]
        a = np.linalg.norm(w, axis=1)
        Kx = np.zeros((m, 3, 3))
        Kx[:, 0, 1], Kx[:, 0, 2], Kx[:, 1, 2] = -w[:, 2], w[:, 1], -w[:, 0]
        Kx[:, 1, 0], Kx[:, 2, 0], Kx[:, 2, 1] = w[:, 2], -w[:, 1], w[:, 0]
        R = np.eye(3)[None] + (np.sin(a) / a)[:, None, None] * Kx + ((1 - np.cos(a)) / a ** 2)[:, None, None] * (Kx @ Kx)
        v[rot] = np.einsum('nij,nkj->nki', R, v[rot])
    v += c[:, None, :]
    fh = np.array([nx / 2 + 1, ny / 2 + 1, 0.25])
    floor = corners * fh + np.array([(nx - 1) / 2, (ny - 1) / 2, -0.25])
    vert = np.concatenate([v.reshape(-1, 3), floor])
    nb = n + 1
    fac1 = np.array(sum(([4] + list(f) for f in HEX_FACES), []), np.int32)
    cv = dict(body=np.arange(nb, dtype=np.int32), vptr=np.arange(nb + 1, dtype=np.int32) * 8, vert=vert,
              fptr=np.arange(nb + 1, dtype=np.int32) * fac1.shape[0], fac=np.tile(fac1, nb),
              sptr=np.arange(nb + 1, dtype=np.int32) * 6, surf=rng.integers(nsurf, size=6 * nb).astype(np.int32))
    obstacle = np.zeros(nb, np.int32); obstacle[-1] = 1
    e = np.zeros(0)
    eye = np.tile(np.eye(3).reshape(9), (nb, 1))
    sc = Scene(name='convex-lattice-%d' % n, step=1e-3, dynamic=1, rot=eye.copy(), x=np.zeros((nb, 3)),
               x0=np.zeros((nb, 3)), jinv=np.where(obstacle[:, None] != 0, 0.0, eye), minv=1.0 - obstacle,
               velo=np.zeros((nb, 6)), velo0=np.zeros((nb, 6)), obstacle=obstacle, master=np.zeros(0, np.int32),
               slave=np.zeros(0, np.int32), mpnt=np.zeros((0, 3)), spnt=np.zeros((0, 3)), base=np.zeros((0, 9)),
               gap=e, friction=e, restitution=e, cohesion=e, mass=np.ones(nb))
    return sc, cv


def convex_drop(seed: int = 5, nx: int = 3, ny: int = 2, nz: int = 2, hulls: int = 2, gap: float = 1.5e-3,
                density: float = 1000.0, nsurf: int = 3, step: float = 1e-3):
    """Convex bodies dropped onto a floor obstacle: an nx x ny x nz stack of
    boxes of side about 1, 1 cm apart sideways (sizes and positions jittered
    by a few thousandths, turned by up to 0.3 degrees), each layer `gap` above
    the highest vertex of the one below it, and
    `hulls` random hulls of 7 points above the stack; every body's mass centre
    at its vertices' mean, inertia that of its bounding box. Surface ids are
    seeded per face.

    Returns (scene without contacts, set_convexes arguments, J, mass)."""
    rng = np.random.default_rng(seed)
    convexes = []

    def turn(angle):
        w = rng.normal(size=3)
        w *= angle / np.linalg.norm(w)
        K = np.array([[0, -w[2], w[1]], [w[2], 0, -w[0]], [-w[1], w[0], 0]])
        a = np.linalg.norm(w)
        return np.eye(3) + np.sin(a) / a * K + (1 - np.cos(a)) / a ** 2 * K @ K

    top = 0.0
    for k in range(nz):
        layer = []
        for j in range(ny):
            for i in range(nx):
                h = 0.5 * (1 + rng.uniform(-3e-3, 3e-3, 3))
                v = np.array([[(-h[0], h[0])[a], (-h[1], h[1])[b], (-h[2], h[2])[c]] for c in (0, 1)
                              for b in (0, 1) for a in (0, 1)]) @ turn(rng.uniform(0, np.radians(0.3))).T
                v += np.array([i * 1.01, j * 1.01, 0.0]) + rng.uniform(-1e-3, 1e-3, 3)
                v[:, 2] += top + gap - v[:, 2].min()
                layer.append(v)
                convexes.append((v, HEX_FACES, rng.integers(nsurf, size=6)))
        top = max(v[:, 2].max() for v in layer)
    for _ in range(hulls):
        P = rng.normal(size=(7, 3)) * 0.3
        V, faces = hull_faces(P)
        V = V + np.array([rng.uniform(0, nx - 1), rng.uniform(0, ny - 1), 0.0])
        V[:, 2] += top + gap - V[:, 2].min()
        convexes.append((V, faces, rng.integers(nsurf, size=len(faces))))
    floor_h = np.array([nx / 2 + 1, ny / 2 + 1, 0.25])
    floor_c = np.array([(nx - 1) / 2, (ny - 1) / 2, -0.25])
    floor = np.array([[(-floor_h[0], floor_h[0])[a], (-floor_h[1], floor_h[1])[b], (-floor_h[2], floor_h[2])[c]]
                      for c in (0, 1) for b in (0, 1) for a in (0, 1)]) + floor_c
    convexes.append((floor, HEX_FACES, rng.integers(nsurf, size=6)))
    nb = len(convexes)
    obstacle = np.zeros(nb, np.int32); obstacle[-1] = 1
    x = np.array([v.mean(axis=0) for v, _, _ in convexes])
    ext = np.array([v.max(axis=0) - v.min(axis=0) for v, _, _ in convexes])
    mass = density * ext.prod(axis=1)
    J = np.zeros((nb, 9))
    J[:, 0] = mass * (ext[:, 1] ** 2 + ext[:, 2] ** 2) / 12
    J[:, 4] = mass * (ext[:, 0] ** 2 + ext[:, 2] ** 2) / 12
    J[:, 8] = mass * (ext[:, 0] ** 2 + ext[:, 1] ** 2) / 12
    jinv = np.zeros((nb, 9))
    jinv[:, 0], jinv[:, 4], jinv[:, 8] = 1 / J[:, 0], 1 / J[:, 4], 1 / J[:, 8]
    jinv[obstacle != 0] = 0.0
    minv = np.where(obstacle != 0, 0.0, 1.0 / mass)
    J[obstacle != 0] = np.eye(3).reshape(9)
    mass = np.where(obstacle != 0, 1.0, mass)
    e = np.zeros(0)
    eye = np.tile(np.eye(3).reshape(9), (nb, 1))
    sc = Scene(name='convex-drop-%d' % nb, step=step, dynamic=1, rot=eye, x=x.copy(), x0=x.copy(), jinv=jinv,
               minv=minv, velo=np.zeros((nb, 6)), velo0=np.zeros((nb, 6)), obstacle=obstacle,
               master=np.zeros(0, np.int32), slave=np.zeros(0, np.int32), mpnt=np.zeros((0, 3)),
               spnt=np.zeros((0, 3)), base=np.zeros((0, 9)), gap=e, friction=e, restitution=e, cohesion=e,
               mass=mass)
    return sc, _convex_arrays(convexes, np.arange(nb)), J, mass


def spheres_in_box(seed: int = 9, n_side: int = 5, layers: int = 3, radius: float = 0.05, pitch: float = 0.11,
                   wall: float = 0.05, clearance: float = 0.002, density: float = 2000.0, friction: float = 0.3,
                   step: float = 1e-3):
    """A jittered lattice of spheres in an open-topped box of five fixed
    hexahedral walls (floor and four sides, each `wall` thick), the lowest
    layer `clearance` above the floor and the outer columns `clearance` from
    the sides. Walls are convex obstacles; every sphere is its own body.

    Returns (scene without contacts, SPHERES arguments with `convex`, J, mass)."""
    rng = np.random.default_rng(seed)
    half = (n_side - 1) / 2.0 * pitch + radius + clearance
    top = clearance + radius + (layers - 1) * pitch + radius + pitch
    g = (np.arange(n_side) - (n_side - 1) / 2.0) * pitch
    X, Y, Z = np.meshgrid(g, g, clearance + radius + np.arange(layers) * pitch, indexing='ij')
    xs = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    xs[:, :2] += rng.uniform(-0.1 * (pitch - 2 * radius), 0.1 * (pitch - 2 * radius), (xs.shape[0], 2))
    n = xs.shape[0]
    walls = [([-half - wall, -half - wall, -wall], [half + wall, half + wall, 0.0]),       # floor
             ([-half - wall, -half - wall, 0.0], [-half, half + wall, top]),               # -x
             ([half, -half - wall, 0.0], [half + wall, half + wall, top]),                 # +x
             ([-half, -half - wall, 0.0], [half, -half, top]),                             # -y
             ([-half, half, 0.0], [half, half + wall, top])]                               # +y
    nw = len(walls)
    nb = n + nw
    centres = np.array([0.5 * (np.asarray(a) + np.asarray(b)) for a, b in walls])
    x = np.concatenate([xs, centres], axis=0)
    mass = np.ones(nb); mass[:n] = density * 4.0 / 3.0 * math.pi * radius ** 3
    jinv = np.zeros((nb, 9)); jinv[:n, 0] = jinv[:n, 4] = jinv[:n, 8] = 1.0 / (0.4 * mass[:n] * radius ** 2)
    minv = np.zeros(nb); minv[:n] = 1.0 / mass[:n]
    rot = np.zeros((nb, 9)); rot[:, 0] = rot[:, 4] = rot[:, 8] = 1.0
    rot[:n] = _random_rotations(rng, n)
    obstacle = np.zeros(nb, np.int32); obstacle[n:] = 1
    r = np.zeros(nb); r[:n] = radius
    z = np.zeros((nb, 6)); e = np.zeros(0)
    sc = Scene(name='spheres-in-box-%d' % n, step=step, dynamic=1, rot=rot, x=x.copy(), x0=x.copy(), jinv=jinv,
               minv=minv, velo=z.copy(), velo0=z.copy(), obstacle=obstacle, master=np.zeros(0, np.int32),
               slave=np.zeros(0, np.int32), mpnt=np.zeros((0, 3)), spnt=np.zeros((0, 3)), base=np.zeros((0, 9)),
               gap=e, friction=e, restitution=e, cohesion=e, mass=mass, radius=r)
    J, mass = sphere_inertia(sc)
    verts, facs = [], []
    for lo, hi in walls:
        v, f = box_convex(lo, hi)
        verts.append(v); facs.append(f)
    convex = dict(body=np.arange(n, nb, dtype=np.int32), vptr=np.arange(nw + 1, dtype=np.int32) * 8,
                  vert=np.concatenate(verts), fptr=np.arange(nw + 1, dtype=np.int32) * 30, fac=np.concatenate(facs),
                  sptr=np.arange(nw + 1, dtype=np.int32) * 6, surf=np.zeros(6 * nw, np.int32))
    sph = dict(body=np.arange(n, dtype=np.int32), centre=xs.copy(), radius=np.full(n, radius),
               surface=np.zeros(n, np.int32), material=(friction, 0.0), convex=convex)
    return sc, sph, J, mass
