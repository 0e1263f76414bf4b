"""The closure network's tcgen05 kernels against the CPU restatement
(oracle/cnn_oracle.cpp): each convolution form, the weight gradient, the
full network's loss gradient at BF16 rounding, and a short training run."""
import ctypes as C

import numpy as np
import pytest

from oracle import pycnn
from pcom_b200 import _lib as L

pytestmark = pytest.mark.gpu


def cnn_check(rc, what):
    if rc != 0:
        buf = C.create_string_buffer(512)
        L.load().pcom_cnn_last_error(buf, 512)
        raise RuntimeError(f"{what}: rc {rc}: {buf.value.decode()}")


def bf16(a):
    """(device BF16 tensor, float32 numpy array of the same values)"""
    import torch

    t = torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda().to(torch.bfloat16)
    return t, t.float().cpu().numpy()


H, W, NIMG = 10, 13, 3  # 390 pixels: a partial last tile of 128


@pytest.mark.parametrize("px", [0, 1])
@pytest.mark.parametrize("cin,nout", [(16, 64), (64, 64), (64, 16), (16, 16)])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_conv_layer(cin, nout, mode, px):
    import torch

    rng = np.random.default_rng(cin * 7 + nout + mode)
    npix = H * W * NIMG
    xd, x = bf16(rng.standard_normal((npix, cin)))
    wd, w = bf16(rng.standard_normal((9, nout, cin)) / np.sqrt(9 * cin))
    b = rng.standard_normal(nout).astype(np.float32)
    bd = torch.from_numpy(b).cuda()
    auxd, aux = bf16(rng.standard_normal((npix, nout)))
    nstore = 4 if mode == 1 else 0
    if mode == 1:
        outd = torch.zeros((npix, nstore), dtype=torch.float32, device="cuda")
    else:
        outd = torch.zeros((npix, nout), dtype=torch.bfloat16, device="cuda")
    rc = L.load().pcom_cnn_conv_layer(cin, nout, xd.data_ptr(), wd.data_ptr(), bd.data_ptr(),
                                      auxd.data_ptr() if mode == 2 else None, outd.data_ptr(), npix, H, W, px, mode,
                                      nstore, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    cnn_check(rc, "conv")
    ref = pycnn.conv(cin, nout, x, w, b, aux if mode == 2 else None, H, W, px, mode, nstore)
    got = outd.float().cpu().numpy()
    scale = np.abs(ref).max()
    if mode == 1:  # FP32 output: accumulation-order differences only
        assert np.abs(got - ref).max() <= 1e-5 * scale
    else:  # BF16 output: one rounding of the FP32 result
        assert np.abs(got - ref).max() <= 2 ** -8 * scale + 1e-6


def _conv_case(cin, nout, mode, px, h, w, nimg, seed):
    """One convolution through the C ABI against the CPU restatement; the
    largest error over the scale of the reference."""
    import torch

    rng = np.random.default_rng(seed)
    npix = h * w * nimg
    xd, x = bf16(rng.standard_normal((npix, cin)))
    wd, wt = bf16(rng.standard_normal((9, nout, cin)) / np.sqrt(9 * cin))
    b = rng.standard_normal(nout).astype(np.float32)
    bd = torch.from_numpy(b).cuda()
    auxd, aux = bf16(rng.standard_normal((npix, nout)))
    nstore = 4 if mode == 1 else 0
    if mode == 1:
        outd = torch.zeros((npix, nstore), dtype=torch.float32, device="cuda")
    else:
        outd = torch.zeros((npix, nout), dtype=torch.bfloat16, device="cuda")
    rc = L.load().pcom_cnn_conv_layer(cin, nout, xd.data_ptr(), wd.data_ptr(), bd.data_ptr(),
                                      auxd.data_ptr() if mode == 2 else None, outd.data_ptr(), npix, h, w, px, mode,
                                      nstore, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    cnn_check(rc, "conv")
    ref = pycnn.conv(cin, nout, x, wt, b, aux if mode == 2 else None, h, w, px, mode, nstore)
    got = outd.float().cpu().numpy()
    return np.abs(got - ref).max() / np.abs(ref).max()


# Image shapes at the edges of the row kernel's bookkeeping: one-row and
# two-row images (every input row starts or ends an image), widths of
# exactly one and two 128-pixel tiles (the wrapped right-halo pixel is the
# slot's last row), one pixel over a tile, and a ragged second tile column.
@pytest.mark.parametrize("h,w,nimg", [(1, 130, 4), (2, 128, 3), (5, 256, 2), (3, 200, 2), (7, 129, 2)])
@pytest.mark.parametrize("px", [0, 1])
@pytest.mark.parametrize("cin,nout,mode", [(64, 64, 0), (16, 64, 0), (64, 16, 1), (64, 64, 2)])
def test_conv_layer_edge_shapes(cin, nout, mode, px, h, w, nimg):
    rel = _conv_case(cin, nout, mode, px, h, w, nimg, seed=h * 1000 + w + 7 * cin + nout + mode)
    if mode == 1:
        assert rel <= 1e-5
    else:
        assert rel <= 2 ** -8 + 1e-6


@pytest.mark.parametrize("cin,nout", [(16, 64), (64, 64), (64, 16)])
def test_conv_partial_image(cin, nout):
    """A pixel count that is not whole images takes the per-tap tile form."""
    import torch

    rng = np.random.default_rng(5)
    npix = H * W * NIMG - 37
    xd, x = bf16(rng.standard_normal((npix, cin)))
    wd, w = bf16(rng.standard_normal((9, nout, cin)) / np.sqrt(9 * cin))
    b = rng.standard_normal(nout).astype(np.float32)
    bd = torch.from_numpy(b).cuda()
    outd = torch.zeros((npix, 4), dtype=torch.float32, device="cuda")
    rc = L.load().pcom_cnn_conv_layer(cin, nout, xd.data_ptr(), wd.data_ptr(), bd.data_ptr(), None, outd.data_ptr(),
                                      npix, H, W, 1, 1, 4, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    cnn_check(rc, "conv")
    # the oracle on whole images, restricted to the pixels computed (the last
    # image is partial: its missing pixels are zero input)
    full = np.zeros((H * W * NIMG, cin), np.float32)
    full[:npix] = x
    ref = pycnn.conv(cin, nout, full, w, b, None, H, W, 1, 1, 4)[:npix]
    assert np.abs(outd.cpu().numpy() - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("px", [0, 1])
@pytest.mark.parametrize("cin,nout", [(16, 64), (64, 64), (64, 16)])
def test_wgrad(cin, nout, px):
    import torch

    rng = np.random.default_rng(cin + 3 * nout + px)
    npix = H * W * NIMG
    xd, x = bf16(rng.standard_normal((npix, cin)))
    gd, g = bf16(rng.standard_normal((npix, nout)))
    dw = torch.zeros(9 * nout * cin, dtype=torch.float32, device="cuda")
    rc = L.load().pcom_cnn_wgrad_layer(cin, nout, xd.data_ptr(), gd.data_ptr(), dw.data_ptr(), npix, H, W, px,
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
    cnn_check(rc, "wgrad")
    ref = pycnn.wgrad(cin, nout, x, g, H, W, px)
    got = dw.cpu().numpy().reshape(9, nout, cin)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


# the 1-degree closure's images: one 160 x 360 level image per model level,
# periodic in x (the production row walk of the persistent kernel)
HF, WF, NF = 160, 360, 2


@pytest.mark.parametrize("cin,nout,mode", [(16, 64, 0), (64, 64, 0), (64, 64, 2), (64, 16, 1), (64, 16, 2)])
def test_conv_layer_full_shape(cin, nout, mode):
    """Every convolution form the network uses, on two full 1-degree level
    images (160 x 360, periodic in x), against the CPU restatement."""
    import torch

    rng = np.random.default_rng(100 + cin + nout + mode)
    npix = HF * WF * NF
    xd, x = bf16(rng.standard_normal((npix, cin)))
    wd, w = bf16(rng.standard_normal((9, nout, cin)) / np.sqrt(9 * cin))
    b = rng.standard_normal(nout).astype(np.float32)
    bd = torch.from_numpy(b).cuda()
    auxd, aux = bf16(rng.standard_normal((npix, nout)))
    nstore = 4 if mode == 1 else 0
    if mode == 1:
        outd = torch.zeros((npix, nstore), dtype=torch.float32, device="cuda")
    else:
        outd = torch.zeros((npix, nout), dtype=torch.bfloat16, device="cuda")
    rc = L.load().pcom_cnn_conv_layer(cin, nout, xd.data_ptr(), wd.data_ptr(), bd.data_ptr(),
                                      auxd.data_ptr() if mode == 2 else None, outd.data_ptr(), npix, HF, WF, 1, mode,
                                      nstore, C.c_void_p(torch.cuda.current_stream().cuda_stream))
    cnn_check(rc, "conv")
    torch.cuda.synchronize()
    ref = pycnn.conv(cin, nout, x, w, b, aux if mode == 2 else None, HF, WF, 1, mode, nstore)
    got = outd.float().cpu().numpy()
    scale = np.abs(ref).max()
    if mode == 1:
        assert np.abs(got - ref).max() <= 1e-5 * scale
    else:
        assert np.abs(got - ref).max() <= 2 ** -8 * scale + 1e-6
    # every pixel was written (the row walk covers the whole image)
    assert np.count_nonzero(np.abs(got - ref) > 2 ** -8 * scale + 1e-6) == 0


@pytest.mark.parametrize("cin,nout", [(16, 64), (64, 64), (64, 16)])
def test_wgrad_full_shape(cin, nout):
    """The weight gradient over two full 1-degree level images."""
    import torch

    rng = np.random.default_rng(200 + cin + nout)
    npix = HF * WF * NF
    xd, x = bf16(rng.standard_normal((npix, cin)))
    gd, g = bf16(rng.standard_normal((npix, nout)))
    dw = torch.zeros(9 * nout * cin, dtype=torch.float32, device="cuda")
    rc = L.load().pcom_cnn_wgrad_layer(cin, nout, xd.data_ptr(), gd.data_ptr(), dw.data_ptr(), npix, HF, WF, 1,
                                       C.c_void_p(torch.cuda.current_stream().cuda_stream))
    cnn_check(rc, "wgrad")
    ref = pycnn.wgrad(cin, nout, x, g, HF, WF, 1)
    got = dw.cpu().numpy().reshape(9, nout, cin)
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


def _net(lib, nimg, H_, W_):
    h = C.c_void_p()
    cnn_check(lib.pcom_cnn_create(H_, W_, nimg, 1, C.byref(h)), "create")
    return h


def _problem(seed, nimg, H_, W_, scale=0.1):
    rng = np.random.default_rng(seed)
    npar = pycnn.param_count()
    par = (rng.standard_normal(npar) * scale).astype(np.float32)
    npix = H_ * W_ * nimg
    x = np.zeros((npix, 16), np.float32)
    x[:, :5] = rng.standard_normal((npix, 5))
    t = rng.standard_normal((npix, 4)).astype(np.float32)
    m = (rng.random((npix, 4)) > 0.2).astype(np.float32)
    return par, x, t, m


def test_network_gradient_matches_oracle():
    """Loss and every parameter's gradient against the oracle run with the
    device path's BF16 rounding points (same inputs)."""
    import torch

    lib = L.load()
    Hs, Ws, nimg = 6, 9, 2
    par, x, t, m = _problem(4, nimg, Hs, Ws)
    h = _net(lib, nimg, Hs, Ws)
    cnn_check(lib.pcom_cnn_set_params(h, par.ctypes.data, par.size), "set_params")
    xd, x16 = bf16(x)
    td = torch.from_numpy(t).cuda()
    md = torch.from_numpy(m).cuda()
    g = np.zeros(par.size, np.float32)
    loss = C.c_double()
    cnn_check(lib.pcom_cnn_gradient(h, xd.data_ptr(), td.data_ptr(), md.data_ptr(), nimg, g.ctypes.data,
                                    C.byref(loss)), "gradient")
    lref, gref = pycnn.loss_grad(par, x16, t, m, Hs, Ws, 1, 1)
    assert abs(loss.value - lref) <= 1e-3 * abs(lref)
    rel = np.linalg.norm(g - gref) / np.linalg.norm(gref)
    assert rel <= 2e-2, f"gradient relative error {rel:.3e}"
    lib.pcom_cnn_destroy(h)


def test_training_reduces_loss():
    """Fit a smooth synthetic target (a fixed local function of the inputs):
    Adam with the tensor-core backward pass must cut the loss by 5x."""
    import torch

    lib = L.load()
    Hs, Ws, nimg = 16, 24, 4
    rng = np.random.default_rng(9)
    npix = Hs * Ws * nimg
    x = np.zeros((npix, 16), np.float32)
    x[:, :5] = rng.standard_normal((npix, 5))
    xi = x[:, :5].reshape(nimg, Hs, Ws, 5)
    t = np.stack([0.5 * xi[..., 0] - 0.3 * np.roll(xi[..., 1], 1, axis=2),
                  np.tanh(xi[..., 2]),
                  0.2 * xi[..., 3] * xi[..., 4],
                  0.1 * (np.roll(xi[..., 0], -1, axis=1) + xi[..., 0])], axis=-1).reshape(npix, 4).astype(np.float32)
    m = np.ones((npix, 4), np.float32)
    npar = pycnn.param_count()
    par = np.zeros(npar, np.float32)
    o = 0
    for k, n in ((16, 64), (64, 64), (64, 64), (64, 64), (64, 16)):
        par[o:o + 9 * n * k] = rng.standard_normal(9 * n * k) * np.sqrt(2.0 / (9 * k))
        o += 9 * n * k + n
    h = _net(lib, nimg, Hs, Ws)
    cnn_check(lib.pcom_cnn_set_params(h, par.ctypes.data, npar), "set_params")
    xd, _ = bf16(x)
    td = torch.from_numpy(t).cuda()
    md = torch.from_numpy(m).cuda()
    loss = C.c_double()
    losses = []
    for it in range(300):
        cnn_check(lib.pcom_cnn_train_step(h, xd.data_ptr(), td.data_ptr(), md.data_ptr(), nimg, C.c_float(2e-3),
                                          C.byref(loss)), "train_step")
        losses.append(loss.value)
    print(f"\nloss {losses[0]:.4f} -> {losses[-1]:.4f}")
    assert np.isfinite(losses[-1]) and losses[-1] < losses[0] / 5
    lib.pcom_cnn_destroy(h)
