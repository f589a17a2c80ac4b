"""GPU tests of the learned warm start (tcgen05 network kernels).

* Forward: the device network against the numpy restatement
  (oracle/mlp_oracle.py) on random parameters and features.
* Gradient: every parameter block of the device gradient (k_mlp_grad) against
  the restatement's backward pass, same BF16 rounding points. Tolerance:
  relative 2e-2 per block (FP32 accumulation order differs between the
  tensor cores and numpy, and a value on a BF16 rounding boundary may round
  the other way).
* Training: Adam on a smooth synthetic regression lowers the loss.
* Warm start: on a seeded scene, the network's start is taken only when its
  merit is lower than the plain previous-step start, and the solve from the
  chosen start converges to the requested merit; with the shipped weights the
  gain over the plain start is measured.
"""
import numpy as np
import pytest

import mlp_oracle as M
from solfec_b200 import learn

pytestmark = pytest.mark.gpu
torch = pytest.importorskip('torch')


def _params(seed):
    rng = np.random.default_rng(seed)
    P = M.init_params(seed)
    P[M.PW3:M.PW3 + 3 * M.HID] = rng.normal(0, 0.15, size=3 * M.HID)
    P[M.PB2:M.PW3] = rng.normal(0, 0.1, size=M.HID)
    P[M.PB3:M.PB3 + 3] = rng.normal(0, 0.1, size=3)
    W1 = P[M.PW1:M.PW2].reshape(M.HID, M.IN)
    W1[:, M.BIAS_COL] = rng.normal(0, 0.1, size=M.HID)
    return P.astype(np.float32)


def _features(seed, n):
    rng = np.random.default_rng(seed)
    X = rng.normal(0, 1, size=(n, M.IN)).astype(np.float32)
    X[:, M.BIAS_COL] = 1.0
    X[:, M.BIAS_COL + 1:] = 0.0
    return X


@pytest.fixture(scope='module')
def net():
    n = learn.WarmStartNet()
    yield n
    n.close()


@pytest.mark.parametrize('n', [1, 200, 1000])
def test_forward_matches_oracle(net, n):
    P, X = _params(1), _features(2, n)
    net.set_params(P)
    y = net.forward(torch.from_numpy(X).cuda()).cpu().numpy()
    yr, _ = M.forward(P, X)
    err = np.abs(y - yr).max() / (np.abs(yr).max() + 1e-6)
    assert err < 2e-2, err


def test_untrained_network_predicts_no_change(net):
    net.set_params(learn.init_params(0))
    y = net.forward(torch.from_numpy(_features(3, 300)).cuda()).cpu().numpy()
    assert np.all(y == 0.0)


@pytest.mark.parametrize('n', [128, 1000])
def test_gradient_matches_oracle(net, n):
    P, X = _params(4), _features(5, n)
    T = np.random.default_rng(6).normal(0, 1, size=(n, 3)).astype(np.float32)
    net.set_params(P)
    loss, g = net.grad(torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda())
    lr, gr = M.loss_and_grad(P, X, T)
    assert abs(loss - lr) <= 1e-2 * lr
    blocks = dict(W1=(M.PW1, M.PW2), W2=(M.PW2, M.PB2), b2=(M.PB2, M.PW3), W3=(M.PW3, M.PB3), b3=(M.PB3, M.NPARAMS))
    for name, (a, b) in blocks.items():
        rel = np.linalg.norm(g[a:b] - gr[a:b]) / (np.linalg.norm(gr[a:b]) + 1e-12)
        assert rel < 2e-2, (name, rel)
    # padding rows of W3 / b3 get no gradient
    assert np.all(g[M.PW3 + 3 * M.HID:M.PB3] == 0.0) and np.all(g[M.PB3 + 3:] == 0.0)


def test_training_lowers_the_loss(net):
    rng = np.random.default_rng(7)
    n = 20000
    X = _features(8, n)
    A = rng.normal(0, 0.3, size=(M.BIAS_COL, 3))
    T = np.tanh(X[:, :M.BIAS_COL] @ A).astype(np.float32)
    net.set_params(learn.init_params(1))
    Xt, Tt = torch.from_numpy(X).cuda(), torch.from_numpy(T).cuda()
    l0, _ = net.grad(Xt, Tt)
    hist = net.train(Xt, Tt, epochs=8, batch_tiles=16, lr=3e-3, seed=1)
    l1, _ = net.grad(Xt, Tt)
    assert np.all(np.isfinite(hist))
    assert l1 < 0.1 * l0, (l0, hist, l1)


def test_warm_start_fallback_and_convergence():
    from solfec_b200 import GAUSS_SEIDEL_SOLVER, LOCDYN, scenes
    sc0 = scenes.hexahedra_lattice(seed=31, nx=30, ny=30, nz=6)
    ldy = LOCDYN()
    ldy.update_begin(sc0)
    kw = dict(epsilon=1.0, maxiter=1000, meritval=1e-4)
    gs = GAUSS_SEIDEL_SOLVER(**kw)
    gs.solve(ldy)
    R0, U0, _ = ldy.get_state()
    sc1 = scenes.advance_velocities(sc0, R0)
    ldy.update_begin(sc1)
    # plain previous-step start
    ldy.set_state(R0, U0)
    gs_plain = GAUSS_SEIDEL_SOLVER(**kw)
    gs_plain.solve(ldy)
    # an untrained network predicts no change: equal merits, the plain start is kept
    net0 = learn.WarmStartNet(params=learn.init_params(0))
    ldy.set_state(R0, U0)
    rep = learn.warm_start(ldy, net0)
    assert not rep['used_nn'] and rep['merit_nn'] == rep['merit_plain']
    # a network with large random outputs has a higher merit: the plain start is kept
    netr = learn.WarmStartNet(params=_params(9) * np.float32(3.0))
    ldy.set_state(R0, U0)
    rep = learn.warm_start(ldy, netr)
    assert not rep['used_nn'] and rep['merit_nn'] > rep['merit_plain']
    gs_r = GAUSS_SEIDEL_SOLVER(**kw)
    gs_r.solve(ldy)
    assert gs_r.iters == gs_plain.iters        # untouched plain start
    # the shipped network: whichever start is chosen, the solve converges
    import os
    if os.path.exists(learn.WEIGHTS):
        net = learn.WarmStartNet.load()
        ldy.set_state(R0, U0)
        rep = learn.warm_start(ldy, net)
        assert rep['used_nn'] == (rep['merit_nn'] < learn.ACCEPT_RATIO * rep['merit_plain'])
        # with the bare fallback rule (any lower merit) the network start is taken whenever it is better
        ldy.set_state(R0, U0)
        rep1 = learn.warm_start(ldy, net, accept_ratio=1.0)
        assert rep1['used_nn'] == (rep1['merit_nn'] < rep1['merit_plain'])
        ldy.set_state(R0, U0)
        rep = learn.warm_start(ldy, net)
        gs_nn = GAUSS_SEIDEL_SOLVER(**kw)
        gs_nn.solve(ldy)
        assert ldy.merit <= 1e-4
        print('warm start: plain %d iterations (start merit %.3g), network %d iterations (start merit %.3g, used %s)'
              % (gs_plain.iters, rep['merit_plain'], gs_nn.iters, rep['merit_nn'], rep['used_nn']))
    ldy.close()
