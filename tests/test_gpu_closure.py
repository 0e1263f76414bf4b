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
