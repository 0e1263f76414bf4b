"""The CPU restatement of the closure network (oracle/cnn_oracle.cpp), which
the GPU tensor-core kernels are checked against: its convolution against a
direct numpy evaluation, and its back-propagated gradient against central
finite differences of the loss (FP64, no BF16 rounding)."""
import numpy as np
import pytest

from oracle import pycnn


def np_conv(x, w, H, W, px):
    """x [n][H][W][cin], w [9][nout][cin] -> [n][H][W][nout], 'same' 3x3."""
    n = x.shape[0]
    out = np.zeros((n, H, W, w.shape[1]))
    for t in range(9):
        dy, dx = t // 3 - 1, t % 3 - 1
        src = np.zeros_like(x)
        ys = slice(max(0, -dy), H - max(0, dy))
        yd = slice(max(0, dy), H - max(0, -dy))
        if px:
            rolled = np.roll(x, -dx, axis=2)
            src[:, ys] = rolled[:, yd]
        else:
            xs = slice(max(0, -dx), W - max(0, dx))
            xd = slice(max(0, dx), W - max(0, -dx))
            src[:, ys, xs] = x[:, yd, xd]
        out += np.einsum("nyxc,oc->nyxo", src, w[t])
    return out


@pytest.mark.parametrize("px", [0, 1])
def test_oracle_conv_matches_numpy(px):
    rng = np.random.default_rng(3)
    H, W, cin, nout = 5, 7, 16, 64
    x = rng.standard_normal((2, H, W, cin)).astype(np.float32)
    w = rng.standard_normal((9, nout, cin)).astype(np.float32)
    b = np.zeros(nout, np.float32)
    ref = np_conv(x.astype(np.float64), w.astype(np.float64), H, W, px).reshape(-1, nout)
    got = pycnn.conv(cin, nout, x.reshape(-1, cin), w, b, None, H, W, px, 1, nstore=nout)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def _problem(seed, H=4, W=5, nimg=2):
    rng = np.random.default_rng(seed)
    npar = pycnn.param_count()
    par = (rng.standard_normal(npar) * 0.1).astype(np.float32)
    npix = H * W * nimg
    x = np.zeros((npix, 16), np.float32)
    x[:, :5] = rng.standard_normal((npix, 5))
    t = rng.standard_normal((npix, 4)).astype(np.float32)
    m = (rng.random((npix, 4)) > 0.2).astype(np.float32)
    return par, x, t, m


@pytest.mark.parametrize("px", [0, 1])
def test_oracle_gradient_finite_differences(px):
    H, W = 4, 5
    par, x, t, m = _problem(7)
    loss, g = pycnn.loss_grad(par, x, t, m, H, W, px, 0)
    assert np.isfinite(loss)
    rng = np.random.default_rng(11)
    # a sample of parameters from every layer (weights of real channels and biases)
    offs, o = [], 0
    for k, n in ((16, 64), (64, 64), (64, 64), (64, 64), (64, 16)):
        offs.append((o, 9 * n * k, n))
        o += 9 * n * k + n
    idx = []
    for (wo, ws, nb) in offs:
        idx += list(wo + rng.choice(ws, 12, replace=False))
        idx += list(wo + ws + rng.choice(nb, 3, replace=False))
    fails = 0
    for i in idx:
        h = 1e-3 * max(abs(float(par[i])), 1e-2)
        lp, xp = _loss_at(par, i, h, x, t, m, H, W, px)
        lm, xm = _loss_at(par, i, -h, x, t, m, H, W, px)
        fd = (lp - lm) / (xp - xm)
        if abs(fd - g[i]) > 1e-6 + 2e-3 * abs(g[i]):
            fails += 1
    assert fails <= 2, f"{fails} of {len(idx)} parameters disagree with finite differences"


def _loss_at(par, i, h, x, t, m, H, W, px):
    """Loss with parameter i moved by about h; the oracle takes FP32
    parameters, so the realised (FP32-rounded) value is returned with it."""
    p = par.copy()
    p[i] = np.float32(float(par[i]) + h)
    lo, _ = pycnn.loss_grad(p, x, t, m, H, W, px, 0)
    return lo, float(p[i])


def test_oracle_bf16_mode_close_to_fp64():
    H, W = 4, 5
    par, x, t, m = _problem(5)
    l0, g0 = pycnn.loss_grad(par, x, t, m, H, W, 1, 0)
    l1, g1 = pycnn.loss_grad(par, x, t, m, H, W, 1, 1)
    assert abs(l1 - l0) <= 2e-2 * abs(l0)
    assert np.abs(g1 - g0).max() <= 5e-2 * np.abs(g0).max()
