"""Learned warm start of the contact solve.

A BF16 MLP (32 -> 128 -> 128 -> 16, GELU, FP32 accumulation; 25 per-contact
features plus a constant input, 3 outputs used) predicts, for every contact,
the change of its reaction from the previous step. Training and inference run
in libsolfec_b200.so on sm_100a tensor cores (tcgen05.mma, TMEM accumulators);
this module drives them through the C ABI of include/b2_device.h:

* ``WarmStartNet`` -- the network on one GPU: parameters, gradient, Adam
  training, forward, save/load.
* ``features(ldy)`` -- the network's inputs for a LOCDYN's current problem,
  with its current reactions as the previous-step reactions.
* ``warm_start(ldy, net)`` -- replace the LOCDYN's initial reactions by the
  prediction when, and only when, its merit (mrf.c:35-185) is lower than that
  of the plain previous-step start; the plain start is the fallback.
* ``training_set(...)`` / ``train(...)`` -- reactions produced by the plain
  solver on seeded scenes, and the training run that produced the weights
  shipped in ``data/warm_start_mlp.npz``.

The reference has no learned component: it starts each solve from con->R of
the previous step (zero for new contacts, mem.c:64-86), which is exactly what
the network reproduces with its last layer at zero.
"""
from __future__ import annotations

import ctypes as C
import os
import time

import numpy as np

from ._lib import last_error, lib

IN, HID, OUT, USED_OUT, BIAS_COL = 32, 128, 16, 3, 25
PW1 = 0
PW2 = PW1 + HID * IN
PB2 = PW2 + HID * HID
PW3 = PB2 + HID
PB3 = PW3 + OUT * HID
NPARAMS = PB3 + OUT
TARGET_CLIP = 50.0  # |y| bound of the training targets (samples in units of rho v_s)

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'data', 'warm_start_mlp.npz')


class b2dev_nn_report(C.Structure):
    _fields_ = [('merit_nn', C.c_double), ('merit_plain', C.c_double), ('used_nn', C.c_int), ('ms', C.c_float)]


def _check(rc, what):
    if rc != 0:
        raise RuntimeError('%s failed (status %d): %s' % (what, rc, last_error()))


def init_params(seed: int = 0) -> np.ndarray:
    """Initial parameters: Gaussian hidden layers (variance 1/fan-in), zero
    biases and a zero last layer, so the untrained network predicts no change
    (the plain previous-step start)."""
    rng = np.random.default_rng(seed)
    P = np.zeros(NPARAMS, dtype=np.float32)
    W1 = rng.normal(0.0, 1.0 / np.sqrt(BIAS_COL + 1), size=(HID, IN)).astype(np.float32)
    W1[:, BIAS_COL:] = 0.0
    P[PW1:PW2] = W1.ravel()
    P[PW2:PB2] = rng.normal(0.0, 1.0 / np.sqrt(HID), size=HID * HID).astype(np.float32)
    return P


def _dptr(t):
    return C.c_void_p(t.data_ptr())


class WarmStartNet:
    """The warm-start network resident on one CUDA device."""

    def __init__(self, device: int = 0, params=None, seed: int = 0):
        L = lib()
        assert L.b2dev_mlp_nparams() == NPARAMS
        h = C.c_void_p()
        _check(L.b2dev_mlp_create(int(device), None, C.byref(h)), 'b2dev_mlp_create')
        self._h = h
        self.device = int(device)
        self.meta = {}
        self.set_params(init_params(seed) if params is None else params)

    def close(self):
        if getattr(self, '_h', None):
            lib().b2dev_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def set_params(self, P):
        P = np.ascontiguousarray(P, dtype=np.float32)
        assert P.shape == (NPARAMS,)
        _check(lib().b2dev_mlp_set_params(self._h, P.ctypes.data_as(C.c_void_p)), 'b2dev_mlp_set_params')

    def params(self) -> np.ndarray:
        P = np.zeros(NPARAMS, dtype=np.float32)
        _check(lib().b2dev_mlp_get_params(self._h, P.ctypes.data_as(C.c_void_p)), 'b2dev_mlp_get_params')
        return P

    def grad(self, feat, target):
        """(loss, gradient) over all samples; feat [n, 32], target [n, 3]
        float32 CUDA tensors."""
        feat, target = feat.contiguous(), target.contiguous()
        g = np.zeros(NPARAMS, dtype=np.float32)
        loss = C.c_double()
        _check(lib().b2dev_mlp_grad(self._h, int(feat.shape[0]), _dptr(feat), _dptr(target),
                                    g.ctypes.data_as(C.c_void_p), C.byref(loss)), 'b2dev_mlp_grad')
        return loss.value, g

    def train(self, feat, target, epochs=10, batch_tiles=64, lr=1e-3, seed=0):
        """Adam over `epochs` passes; returns the mean loss of every epoch."""
        feat, target = feat.contiguous(), target.contiguous()
        out = np.zeros(max(int(epochs), 1))
        _check(lib().b2dev_mlp_train(self._h, int(feat.shape[0]), _dptr(feat), _dptr(target), int(epochs),
                                     int(batch_tiles), float(lr), int(seed) & 0xFFFFFFFFFFFFFFFF,
                                     out.ctypes.data_as(C.c_void_p)), 'b2dev_mlp_train')
        return out[:epochs]

    def forward(self, feat):
        import torch
        feat = feat.contiguous()
        out = torch.empty((feat.shape[0], USED_OUT), dtype=torch.float32, device=feat.device)
        _check(lib().b2dev_mlp_forward(self._h, int(feat.shape[0]), _dptr(feat), _dptr(out)), 'b2dev_mlp_forward')
        return out

    def save(self, path):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        np.savez_compressed(path, params=self.params(), meta=repr(self.meta))

    @classmethod
    def load(cls, path=WEIGHTS, device: int = 0):
        z = np.load(path, allow_pickle=False)
        net = cls(device, params=z['params'])
        net.meta = eval(str(z['meta']), {}) if 'meta' in z.files else {}
        return net


def features(ldy):
    """(feat [n, 32] float32, scale [n] float64, rprev [n, 3] float64) CUDA
    tensors for the LOCDYN's problem in caller row order."""
    import torch
    n = ldy.sizes()[0]
    dev = torch.device('cuda', ldy.device)
    feat = torch.empty((max(n, 1), IN), dtype=torch.float32, device=dev)
    scale = torch.empty(max(n, 1), dtype=torch.float64, device=dev)
    rprev = torch.empty((max(n, 1), 3), dtype=torch.float64, device=dev)
    _check(lib().b2dev_nn_features(ldy.device_context, _dptr(feat), _dptr(scale), _dptr(rprev)), 'b2dev_nn_features')
    return feat[:n], scale[:n], rprev[:n]


ACCEPT_RATIO = 0.5  # the network start must at least halve the merit of the plain start


def warm_start(ldy, net: WarmStartNet, accept_ratio: float = ACCEPT_RATIO) -> dict:
    """Network start with the plain start as the fallback, by merit: the
    prediction replaces the previous-step reactions only when its merit is
    below accept_ratio times theirs. A start with a somewhat lower merit can
    still need more iterations (the network corrects local residuals, while
    the iteration count follows the slowly converging global modes), hence
    the margin."""
    rep = b2dev_nn_report()
    _check(lib().b2dev_nn_warm_start(ldy.device_context, net.handle, float(accept_ratio), C.addressof(rep)),
           'b2dev_nn_warm_start')
    return dict(merit_nn=rep.merit_nn, merit_plain=rep.merit_plain, used_nn=bool(rep.used_nn), ms=rep.ms)


# ---- training data and the shipped weights ----------------------------------------------------

def training_scenes(seed0: int = 100):
    """Seeded scene variants of the three rigid configurations (sphere lattice,
    polydisperse spheres, perturbed hexahedra), disjoint in seed from the
    benchmark and test scenes. Yields (name, scene)."""
    from . import scenes
    for k in range(8):
        yield 'spheres_lattice', scenes.spheres_lattice(seed=seed0 + k)
    yield 'spheres_polydisperse', scenes.spheres_polydisperse(seed=seed0, n=8000)
    for k, (nx, ny, nz) in enumerate([(40, 40, 10), (60, 40, 10), (50, 50, 8), (80, 60, 10), (100, 100, 10),
                                      (70, 70, 10), (100, 60, 10), (100, 100, 10)]):
        yield 'hexahedra_lattice', scenes.hexahedra_lattice(seed=seed0 + 10 + k, nx=nx, ny=ny, nz=nz)


def training_set(scene_iter, steps: int = 4, solver=None, log=print):
    """Features and targets from the plain FP64 solver: every scene is stepped
    `steps` times from rest (zero reactions), each step warm-started from the
    previous one as the benchmark does; each solved step contributes one
    sample per contact. Returns CUDA tensors feat [N, 32], target [N, 3]."""
    import torch
    from .solver import GAUSS_SEIDEL_SOLVER, LOCDYN
    from . import scenes as S
    solver = solver or dict(epsilon=1.0, maxiter=1000, meritval=1e-4)
    feats, targets = [], []
    for name, sc in scene_iter:
        ldy = LOCDYN()
        R = U = None
        for step in range(steps):
            ldy.update_begin(sc)
            ldy.set_state(R, U)
            f, scale, rprev = features(ldy)
            gs = GAUSS_SEIDEL_SOLVER(**solver)
            gs.solve(ldy)
            R, U, _ = ldy.get_state()
            Rt = torch.from_numpy(R.reshape(-1, 3)).to(f.device)
            y = ((Rt - rprev) / scale[:, None]).clamp_(-TARGET_CLIP, TARGET_CLIP).float()
            ok = torch.isfinite(y).all(dim=1) & torch.isfinite(f).all(dim=1)
            feats.append(f[ok].clone())
            targets.append(y[ok].clone())
            log('  %-22s step %d: %6d contacts, %4d iterations, merit %.2e' % (name, step, sc.ncon, gs.iters,
                                                                                ldy.merit))
            sc = S.advance_velocities(sc, R.reshape(-1, 3))
        ldy.close()
    return torch.cat(feats), torch.cat(targets)


def train(out=WEIGHTS, epochs=30, batch_tiles=64, lr=2e-3, seed=0, steps=4, log=print):
    """Generate the training set on the GPU and train the shipped network."""
    t0 = time.time()
    feat, target = training_set(training_scenes(), steps=steps, log=log)
    t1 = time.time()
    log('training set: %d samples in %.0f s' % (feat.shape[0], t1 - t0))
    net = WarmStartNet(params=init_params(seed))
    hist = []
    for e in range(epochs):
        lr_e = lr * 0.5 * (1.0 + np.cos(np.pi * e / epochs))  # cosine schedule
        hist.append(float(net.train(feat, target, epochs=1, batch_tiles=batch_tiles, lr=lr_e, seed=seed + e)[0]))
        log('epoch %2d  lr %.2e  loss %.5f' % (e, lr_e, hist[-1]))
    base = float((target.double() ** 2).sum(dim=1).mean())
    net.meta = dict(samples=int(feat.shape[0]), epochs=epochs, batch=batch_tiles * 128, lr=lr, seed=seed,
                    steps=steps, loss_history=hist, loss_zero_prediction=base,
                    train_seconds=time.time() - t1, data_seconds=t1 - t0)
    if out:
        net.save(out)
    return net


if __name__ == '__main__':
    import argparse
    ap = argparse.ArgumentParser(description='Train the warm-start network on solver output (one GPU).')
    ap.add_argument('--out', default=WEIGHTS)
    ap.add_argument('--epochs', type=int, default=60)
    ap.add_argument('--batch-tiles', type=int, default=64)
    ap.add_argument('--lr', type=float, default=2e-3)
    ap.add_argument('--steps', type=int, default=4)
    ap.add_argument('--seed', type=int, default=0)
    a = ap.parse_args()
    net = train(out=a.out, epochs=a.epochs, batch_tiles=a.batch_tiles, lr=a.lr, seed=a.seed, steps=a.steps)
    print('meta', net.meta)
