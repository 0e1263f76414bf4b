"""Closure coupling and the closure's gain over the plain coarse model.

A fine 360x160x30 run is coarse-grained 4x4 onto the nested 90x40 grid;
the network is trained on the one-step tendency residual of the coarse
model and must predict it better than the plain coarse model does (which
is the zero prediction) on held-out samples."""
import ctypes as C

import numpy as np
import pytest

from pcom_b200 import _lib as L
from pcom_b200.closure import Experiment, Network, coarse_case, evaluate, train
from pcom_b200.model import Model
from pcom_b200.synth import make_case

pytestmark = pytest.mark.gpu


def test_coarsen_is_block_mean_over_wet_cells():
    fc = make_case("global1")
    f = Model(fc)
    f.run(3)
    cc = coarse_case(fc, 4)
    c = Model(cc)
    L.check(L.load().pcom_gpu_coarsen(f.handle, c.handle, 4), "coarsen")
    lev = f.static()["lev_t"][1:-1, 1:-1]
    tf = f.field("tc")[:, 1:-1, 1:-1]
    got = c.field("tc")[:, 1:-1, 1:-1]
    nk, nj, ni = got.shape
    for k in (0, 10, 25):
        w = (lev >= k + 1).reshape(nj, 4, ni, 4)
        v = tf[k].reshape(nj, 4, ni, 4)
        num, den = (v * w).sum(axis=(1, 3)), w.sum(axis=(1, 3))
        ref = np.where(den > 0, num / np.maximum(den, 1), v.mean(axis=(1, 3)))
        assert np.abs(got[k] - ref).max() <= 1e-12 * np.abs(ref).max()
    # velocities vanish at the coarse grid's land U points
    k = np.arange(1, nk + 1)[:, None, None]
    land_u = (c.static()["lev_u"][None] < k)[:, 1:-1, 1:-1]
    assert np.all(c.field("uc")[:, 1:-1, 1:-1][land_u] == 0.0)
    # halo twins of the periodic coarse grid
    full = c.field("tc")
    assert np.array_equal(full[:, :, 0], full[:, :, -2]) and np.array_equal(full[:, :, -1], full[:, :, 1])
    f.close()
    c.close()


def test_closure_beats_plain_coarse_model():
    exp = Experiment(make_case("global1"), 4)
    exp.fine.run(24)
    exp.compute_stats()
    xs, ts, mask = exp.generate(40, 1)
    net = Network(exp.H, exp.W, exp.nk, seed=1)
    res = train(net, xs, ts, mask, epochs=12, lr=1e-3, val_frac=0.25)
    val = res["history"][-1][1]
    print(f"\nvalidation loss {val:.4f} vs zero-output (plain model) {res['val_zero_baseline']:.4f}")
    assert np.isfinite(val) and val < 0.8 * res["val_zero_baseline"]
    net.close()


def test_closure_free_run_beats_plain():
    """Free runs, not offline loss: from CG(fine(t0)) the coarse model runs
    a day beside the fine run, with and without the trained network's T and
    S tendencies at half strength after every step; the closure run's
    temperature error against CG(fine), averaged over the day, is lower
    than the plain coarse model's."""
    exp = Experiment(make_case("global1"), 4)
    exp.fine.run(48)
    exp.compute_stats()
    xs, ts, mask = exp.generate(48, 1)
    net = Network(exp.H, exp.W, exp.nk, seed=1)
    train(net, xs, ts, mask, epochs=12, lr=1e-3, val_frac=0.25, log=lambda *a: None)
    del xs, ts
    res = evaluate(exp, net, 24, {"tracers-half": ([0.0, 0.0, 0.5, 0.5], 3.0, 1)}, record_every=6)
    plain = res["plain"]["plain"]["rms_mean"]["tc"]
    form = res["forms"]["tracers-half"]
    print(f"\nT RMS vs CG(fine) over a day: plain {plain:.4e}, closure {form['rms_mean']['tc']:.4e}")
    assert form["fell_back_at_step"] is None
    assert form["rms_mean"]["tc"] < plain
    net.close()


def _f32(x):
    return np.float64(np.float32(x))


@pytest.mark.parametrize("flags", [L.PCOM_PREC_FP64, L.PCOM_PREC_MIXED], ids=["fp64", "mixed"])
def test_features_and_apply_match_numpy(flags):
    """The network's input features and the tendency application, bit for
    bit against a numpy restatement of their arithmetic: (x - mean) / std in
    FP64 (alpha as stored plus the reference profile on the mixed path),
    rounded to FP32 then BF16 (round to nearest even), zero on land and in
    channels 5..15; and x += dt gain std clip(y) in FP64 on the wet U (u, v)
    and T (T, S) points of the current and previous levels, rounded to the
    handle's storage."""
    import torch

    from pcom_b200.closure import _stats_struct

    c = make_case("global1")
    m = Model(c, flags=flags)
    store = np.float32 if flags == L.PCOM_PREC_MIXED else np.float64
    m.run(3)
    H, W, nk = c["glo_nj"], c["glo_ni"], c["nk"]
    rng = np.random.default_rng(4)
    st = dict(in_mean=[0.003, -0.002, 12.5, 34.8, 1.3e-5], in_std=[0.07, 0.05, 6.3, 0.41, 7e-5],
              out_std=[2e-6, 3e-6, 4e-5, 1e-6], out_gain=[0.5, 1.0, 0.75, 0.25], out_clip=2.5,
              alpha_ref=list(rng.normal(0.0, 1e-5, nk)))
    s = _stats_struct(st)
    lib = L.load()
    x = torch.full((nk * H * W, 16), 7.0, dtype=torch.bfloat16, device="cuda")
    L.check(lib.pcom_gpu_cnn_features(m.handle, C.c_void_p(x.data_ptr()), C.byref(s)), "features")
    torch.cuda.synchronize()
    got = x.view(torch.int16).cpu().numpy().reshape(nk, H, W, 16)
    sta = m.static()
    k = np.arange(1, nk + 1)[:, None, None]
    wu = sta["lev_u"][None, 1:-1, 1:-1] >= k
    wt = sta["lev_t"][None, 1:-1, 1:-1] >= k
    f = {n: m.field(n)[:, 1:-1, 1:-1] for n in ("uc", "vc", "tc", "sc", "alpha")}
    mean, std = [_f32(v) for v in st["in_mean"]], [_f32(v) for v in st["in_std"]]
    aref = np.asarray(st["alpha_ref"])[:, None, None]
    ref = np.zeros((nk, H, W, 16), dtype=np.float32)
    for ch, (name, w) in enumerate((("uc", wu), ("vc", wu), ("tc", wt), ("sc", wt))):
        ref[..., ch] = np.where(w, ((f[name] - mean[ch]) / std[ch]), 0.0).astype(np.float32)
    ref[..., 4] = np.where(wt, ((f["alpha"] - aref - mean[4]) / std[4]), 0.0).astype(np.float32)
    want = torch.from_numpy(ref).to(torch.bfloat16).view(torch.int16).numpy()
    assert np.array_equal(got, want), f"{np.count_nonzero(got != want)} features differ"

    y = torch.from_numpy(rng.normal(0.0, 2.0, (nk * H * W, 4)).astype(np.float32)).cuda()
    names = ("uc", "up", "vc", "vp", "tc", "tp", "sc", "sp")
    before = {n: m.field(n)[:, 1:-1, 1:-1] for n in names}
    dt = 3600.0
    L.check(lib.pcom_gpu_cnn_apply(m.handle, C.c_void_p(y.data_ptr()), C.byref(s), C.c_double(dt)), "apply")
    torch.cuda.synchronize()
    yv = y.cpu().numpy().reshape(nk, H, W, 4)
    clip = np.float32(st["out_clip"])
    for ch, (a, b, w) in enumerate((("uc", "up", wu), ("vc", "vp", wu), ("tc", "tp", wt), ("sc", "sp", wt))):
        yc = np.minimum(np.maximum(yv[..., ch], -clip), clip).astype(np.float64)
        d = dt * _f32(st["out_gain"][ch]) * _f32(st["out_std"][ch]) * yc
        for n in (a, b):
            after = m.field(n)[:, 1:-1, 1:-1]
            want = np.where(w, (before[n] + d).astype(store).astype(np.float64), before[n])
            assert np.array_equal(after, want), f"{n}: {np.count_nonzero(after != want)} points differ"
    m.close()
