"""The oracle's FP64 restatement of the surrogate network (oracle/sma_mlp.c):
its analytic backpropagation against central finite differences of its own
loss, the padding of the parameter layout, and a hand-computed forward pass.
It is the checker of the library's tensor-core training kernel, so its
gradient is pinned here first."""
import numpy as np
import pytest

NIN, NOUT, H = 14, 13, 64
OFF = dict(W1=0, b1=1024, W2=1088, b2=5184, W3=5248, b3=9344, W4=9408, b4=13504, W5=13568, b5=14592)


def _params(rng, scale=0.3):
    p = np.zeros(14608)
    p[OFF["W1"]:OFF["b1"]] = (rng.normal(size=(64, 16)) * np.r_[np.ones(14), 0, 0] * scale).ravel()
    for l in (2, 3, 4):
        p[OFF[f"W{l}"]:OFF[f"b{l}"]] = rng.normal(size=64 * 64) * scale / 2
    for l in (1, 2, 3, 4):
        p[OFF[f"b{l}"]:OFF[f"b{l}"] + 64] = rng.normal(size=64) * 0.1
    p[OFF["W5"]:OFF["b5"]] = (rng.normal(size=(16, 64)) * (np.arange(16) < 13)[:, None] * scale / 2).ravel()
    p[OFF["b5"]:OFF["b5"] + 13] = rng.normal(size=13) * 0.1
    return p


def _stats(rng):
    return np.concatenate([rng.normal(size=NIN), rng.uniform(0.5, 2.0, NIN),
                           rng.normal(size=NOUT), rng.uniform(0.5, 2.0, NOUT)])


def test_layout_size(oracle):
    assert oracle.mlp_nparam() == 14608


def test_forward_by_hand(oracle):
    """A network whose only nonzero path is input 3 -> hidden unit 5 in every
    layer -> output 2 computes silu^4 of the normalised input, scaled."""
    p = np.zeros(14608)
    p[OFF["W1"] + 5 * 16 + 3] = 1.0
    for l in (2, 3, 4):
        p[OFF[f"W{l}"] + 5 * 64 + 5] = 1.0
    p[OFF["W5"] + 2 * 64 + 5] = 2.0
    stats = np.concatenate([np.zeros(NIN), np.ones(NIN), np.zeros(NOUT), np.ones(NOUT)])
    x = np.zeros((1, NIN))
    x[0, 3] = 0.7
    silu = lambda v: v / (1.0 + np.exp(-v))
    y = oracle.mlp_forward(p, stats, x)
    assert abs(y[0, 2] - 2.0 * silu(silu(silu(silu(0.7))))) < 1e-15
    assert np.count_nonzero(y) == 1


def test_backprop_matches_finite_differences(oracle):
    rng = np.random.default_rng(11)
    p, stats = _params(rng), _stats(rng)
    x = rng.normal(size=(16, NIN)) * 1.5 + stats[:NIN]
    y = rng.normal(size=(16, NOUT)) * 2.0
    loss, g = oracle.mlp_loss_grad(p, stats, x, y)
    assert loss > 0
    # every parameter block, biases included
    idx = np.concatenate([rng.choice(np.arange(a, b), 40, replace=False)
                          for a, b in zip(list(OFF.values()), list(OFF.values())[1:] + [14608])
                          if b - a >= 40] +
                         [np.arange(OFF["b5"], OFF["b5"] + 13)])
    h = 1e-6
    for k in idx:
        if g[k] == 0.0 and p[k] == 0.0:
            continue                                        # padding (checked below)
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        fd = (oracle.mlp_loss_grad(pp, stats, x, y, grad=False)[0] -
              oracle.mlp_loss_grad(pm, stats, x, y, grad=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 1e-5 * max(abs(fd), 1e-3 * np.abs(g).max()), (k, fd, g[k])


def test_padding_has_no_gradient(oracle):
    rng = np.random.default_rng(12)
    p, stats = _params(rng), _stats(rng)
    x = rng.normal(size=(8, NIN))
    y = rng.normal(size=(8, NOUT))
    _, g = oracle.mlp_loss_grad(p, stats, x, y)
    W1 = g[OFF["W1"]:OFF["b1"]].reshape(64, 16)
    W5 = g[OFF["W5"]:OFF["b5"]].reshape(16, 64)
    assert not W1[:, 14:].any() and not W5[13:].any() and not g[OFF["b5"] + 13:].any()
