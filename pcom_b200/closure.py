"""The learned subgrid closure: data from a fine run coarse-grained onto a
nested coarse grid, training of the tensor-core network (include/pcom_cnn.h)
and coarse runs with and without it.

Target.  For a sample time t the coarse model is started from the
coarse-grained fine state CG(fine(t)) and stepped k times (dt = the coarse
baroclinic step); the target is the per-level tendency residual
    (CG(fine(t + k dt)) - coarse_steps(CG(fine(t)))) / (k dt)
for u, v, T and S, the part of the fine model's evolution the coarse model
misses.  Inputs: u, v, T, S and the specific-volume anomaly per level, as
5 channels of one image per level.  Closure run: every `cadence` coarse
steps the network's output (scaled back) is added as a tendency over
cadence x dt.

Windows.  The fine run goes on through four consecutive windows: spin-up;
training (samples every `every` coarse steps); validation (coarse runs with
each output variant of VARIANTS, which picks the one applied); test (coarse
runs of the chosen variant at each cadence, in the closure form's precision,
beside the plain coarse model in FP64 and in that precision), evaluated by
the RMS error against CG(fine) averaged over the window.  The SYPD of each
form comes from CUDA-event timings of its step and of the network.

Usage (configuration 5: a year of 0.25-degree training data, a year of
coarse runs):
    python -m pcom_b200.closure --fine global025 --spinup-days 10 \
        --train-days 365 --every 24 --target-steps 3 --val-days 30 \
        --test-days 365 --form-flags mixed --cadences 1,4,8 --epochs 15 \
        --out closure_year.json
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time

import numpy as np

from . import _lib as L
from .model import Model
from .synth import make_case

STEP = 3600  # coarse baroclinic step (s)


def _check_cnn(rc, what):
    if rc != 0:
        buf = C.create_string_buffer(512)
        L.load().pcom_cnn_last_error(buf, 512)
        raise L.PcomError(f"{what}: {buf.value.decode(errors='replace')}")


def coarse_case(fine: dict, factor: int = 4) -> dict:
    """The nested coarse grid of a fine case: lon block means, every
    factor-th north edge in lat, each coarse column as deep as the
    shallowest fine column of its block, block-mean initial state and
    forcing; dtbt 60 s, dtbc 3600 s."""
    f = factor
    ni, nj, nk = fine["glo_ni"] // f, fine["glo_nj"] // f, fine["nk"]
    blk = lambda a: a.reshape(a.shape[:-2] + (nj, f, ni, f)).mean(axis=(-3, -1))
    itn = fine["itn"].reshape(nj, f, ni, f).min(axis=(1, 3)).astype(np.int32)
    c = dict(fine)
    c.update(name=fine["name"] + f"_c{f}", glo_ni=ni, glo_nj=nj, dtbt=60, dtbc=STEP,
             lon=fine["lon"].reshape(ni, f).mean(axis=1), lat=fine["lat"][f - 1::f].copy(), itn=itn,
             pt=blk(fine["pt"]), sa=blk(fine["sa"]))
    for k in ("taux", "tauy", "bct", "bcs", "pa", "fw"):
        c[k] = blk(fine[k])
    return c


class Network:
    """The tensor-core network on device buffers for `nimg` images of H x W."""

    def __init__(self, H: int, W: int, nimg: int, periodic_x: bool = True, seed: int = 0):
        self.lib = L.load()
        self.H, self.W, self.nimg = H, W, nimg
        self.h = C.c_void_p()
        _check_cnn(self.lib.pcom_cnn_create(H, W, nimg, 1 if periodic_x else 0, C.byref(self.h)), "pcom_cnn_create")
        self.nparam = int(self.lib.pcom_cnn_param_count())
        rng = np.random.default_rng(seed)
        par = np.zeros(self.nparam, np.float32)
        o = 0
        for li, (k, n) in enumerate(((16, 64), (64, 64), (64, 64), (64, 64), (64, 16))):
            std = np.sqrt(2.0 / (9 * (5 if li == 0 else k)))
            if li == 4:
                std *= 0.1  # start close to the plain model (zero tendency)
            par[o:o + 9 * n * k] = rng.standard_normal(9 * n * k) * std
            o += 9 * n * k + n
        self.set_params(par)

    def set_params(self, par):
        par = np.ascontiguousarray(par, np.float32)
        _check_cnn(self.lib.pcom_cnn_set_params(self.h, par.ctypes.data, par.size), "set_params")

    def params(self):
        out = np.zeros(self.nparam, np.float32)
        _check_cnn(self.lib.pcom_cnn_get_params(self.h, out.ctypes.data, out.size), "get_params")
        return out

    def set_stream(self, ptr: int):
        _check_cnn(self.lib.pcom_cnn_set_stream(self.h, C.c_void_p(ptr)), "set_stream")

    def train_step(self, x, target, mask, lr) -> float:
        loss = C.c_double()
        _check_cnn(self.lib.pcom_cnn_train_step(self.h, x.data_ptr(), target.data_ptr(), mask.data_ptr(), self.nimg,
                                                C.c_float(lr), C.byref(loss)), "train_step")
        return loss.value

    def loss(self, x, target, mask) -> float:
        loss = C.c_double()
        _check_cnn(self.lib.pcom_cnn_gradient(self.h, x.data_ptr(), target.data_ptr(), mask.data_ptr(), self.nimg,
                                              None, C.byref(loss)), "gradient")
        return loss.value

    def forward(self, x, y):
        _check_cnn(self.lib.pcom_cnn_forward(self.h, x.data_ptr(), y.data_ptr(), self.nimg), "forward")

    def close(self):
        if self.h and self.h.value:
            self.lib.pcom_cnn_destroy(self.h)
            self.h = C.c_void_p()


def _stats_struct(st: dict) -> L.CnnStats:
    s = L.CnnStats()
    for q in range(5):
        s.in_mean[q] = st["in_mean"][q]
        s.in_std[q] = st["in_std"][q]
    for q in range(4):
        s.out_std[q] = st["out_std"][q]
        s.out_gain[q] = st.get("out_gain", [1.0] * 4)[q]
    s.out_clip = st.get("out_clip", 0.0)
    for k, v in enumerate(st["alpha_ref"]):
        s.alpha_ref[k] = v
    return s


class Experiment:
    """Fine model, two coarse models on the nested grid (prediction and
    coarse-grained truth) and the data they produce."""

    def __init__(self, fine_case: dict, factor: int = 4, target_steps: int = 1):
        import torch

        self.torch = torch
        self.lib = L.load()
        self.factor = factor
        self.fine = Model(fine_case)
        self.fc = fine_case
        self.cc = coarse_case(fine_case, factor)
        self.pred = Model(self.cc)
        self.truth = Model(self.cc)
        for m in (self.pred, self.truth):
            m.set_forcing(m.int_bnd())
        self.nk, self.H, self.W = self.cc["nk"], self.cc["glo_nj"], self.cc["glo_ni"]
        self.npix = self.nk * self.H * self.W
        self.fine_steps = STEP // fine_case["dtbc"]
        self.stats = None
        self.citer = 100  # coarse iteration numbers past the AB3 start-up
        self.kt = target_steps  # coarse steps the residual is accumulated over

    def coarsen(self, into: Model):
        L.check(self.lib.pcom_gpu_coarsen(self.fine.handle, into.handle, self.factor), "coarsen")

    def _features(self, m: Model, x):
        L.check(self.lib.pcom_gpu_cnn_features(m.handle, C.c_void_p(x.data_ptr()), C.byref(self.st)), "features")
        m.sync()

    def _current_alpha(self, m: Model):
        """den_alpha of the model's current T, S, ch (alpha is not carried
        over by coarse-graining)."""
        m.phase("den_alpha", self.citer)

    def compute_stats(self):
        """Input normalisation from the current coarse-grained fine state and
        output scales from one target sample."""
        torch = self.torch
        self.coarsen(self.pred)
        self._current_alpha(self.pred)
        st = self.pred.static()
        k = np.arange(1, self.nk + 1)[:, None, None]
        wt, wu = st["lev_t"][None] >= k, st["lev_u"][None] >= k
        alpha = self.pred.field("alpha")
        aref = [float(alpha[q][wt[q]].mean()) if wt[q].any() else 0.0 for q in range(self.nk)]
        an = alpha - np.array(aref)[:, None, None]
        fields = [(self.pred.field("uc"), wu), (self.pred.field("vc"), wu), (self.pred.field("tc"), wt),
                  (self.pred.field("sc"), wt), (an, wt)]
        mean = [float(f[w].mean()) for f, w in fields]
        std = [float(f[w].std()) or 1.0 for f, w in fields]
        self.stats = dict(in_mean=mean, in_std=std, out_std=[1.0] * 4, alpha_ref=aref)
        self.st = _stats_struct(self.stats)
        # output scales from one unscaled target
        t = torch.zeros((self.npix, 4), dtype=torch.float32, device="cuda")
        mk = torch.zeros((self.npix, 4), dtype=torch.float32, device="cuda")
        self._one_target(t, mk)
        tn, mn = t.cpu().numpy(), mk.cpu().numpy()
        # a residual that is identically zero (e.g. S of a case with uniform
        # salinity) gets scale 0: its target is 0 and the closure never adds it
        self.stats["out_std"] = [float(np.sqrt((tn[:, q] ** 2 * mn[:, q]).sum() / max(mn[:, q].sum(), 1)))
                                 for q in range(4)]
        self.st = _stats_struct(self.stats)

    def _one_target(self, target, mask, x=None):
        """From the fine model's current time t: features of CG(fine(t)) into
        x, kt coarse steps from it, the fine model advanced to t + kt dt, and
        the mean residual tendency into target.  The fine model ends at
        t + kt dt."""
        self.coarsen(self.pred)
        self.pred.den_prho()
        if x is not None:
            self._current_alpha(self.pred)
            self._features(self.pred, x)
        for _ in range(self.kt):
            self.citer += 1
            self.pred.step_handle(self.citer)
        self.fine.run(self.fine_steps * self.kt)
        self.coarsen(self.truth)
        L.check(self.lib.pcom_gpu_cnn_target(self.pred.handle, self.truth.handle, C.c_void_p(target.data_ptr()),
                                             C.c_void_p(mask.data_ptr()), C.byref(self.st), float(STEP * self.kt)),
                "target")
        self.pred.sync()

    def generate(self, nsamples: int, every: int = 1):
        """nsamples (x, target) pairs, one every max(every, kt) coarse steps."""
        torch = self.torch
        xs = torch.zeros((nsamples, self.npix, 16), dtype=torch.bfloat16, device="cuda")
        ts = torch.zeros((nsamples, self.npix, 4), dtype=torch.float32, device="cuda")
        mask = torch.zeros((self.npix, 4), dtype=torch.float32, device="cuda")
        for s in range(nsamples):
            for _ in range(every - self.kt):
                self.fine.run(self.fine_steps)
            self._one_target(ts[s], mask, xs[s])
        return xs, ts, mask


def train(net: Network, xs, ts, mask, epochs: int, lr: float, val_frac: float = 0.2, log=print):
    """Adam over the samples (one sample = all levels = one step); returns
    training and validation curves and the zero-prediction baseline."""
    n = xs.shape[0]
    nval = max(1, int(round(n * val_frac)))
    ntr = n - nval
    order = np.arange(ntr)
    rng = np.random.default_rng(0)
    base = [float(((ts[s] ** 2) * mask).sum() / mask.sum()) for s in range(ntr, n)]
    hist = []
    for ep in range(epochs):
        rng.shuffle(order)
        tr = [net.train_step(xs[s], ts[s], mask, lr) for s in order]
        val = [net.loss(xs[s], ts[s], mask) for s in range(ntr, n)]
        hist.append((float(np.mean(tr)), float(np.mean(val))))
        log(f"epoch {ep + 1}: train {hist[-1][0]:.4f}  val {hist[-1][1]:.4f}  (zero-output {np.mean(base):.4f})")
    return dict(history=hist, val_zero_baseline=float(np.mean(base)), ntrain=ntr, nval=nval)


def coarse_rms(exp: Experiment, m: Model) -> dict:
    """RMS difference of u, v, T, S between a coarse model and CG(fine)."""
    exp.coarsen(exp.truth)
    st = m.static()
    k = np.arange(1, exp.nk + 1)[:, None, None]
    wt, wu = st["lev_t"][None] >= k, st["lev_u"][None] >= k
    out = {}
    for f, w in (("uc", wu), ("vc", wu), ("tc", wt), ("sc", wt)):
        d = (m.field(f) - exp.truth.field(f))[w]
        out[f] = float(np.sqrt(np.mean(d * d)))
    return out


VARIANTS = {  # applied fraction of each output (du, dv, dT, dS) and the |y| clip
    "all": ([1.0, 1.0, 1.0, 1.0], 3.0),
    "tracers": ([0.0, 0.0, 1.0, 1.0], 3.0),
    "tracers+0.25uv": ([0.25, 0.25, 1.0, 1.0], 3.0),
    "tracers-half": ([0.0, 0.0, 0.5, 0.5], 3.0),
}
# state fields pcom_gpu_coarsen sets (what a coarse run starts from)
START_FIELDS = ("tc", "sc", "tp", "sp", "uc", "vc", "up", "vp", "auc", "aup", "aupp", "avc", "avp", "avpp",
                "ubc", "vbc", "ubp", "vbp", "chc", "chp", "mch", "mch2", "am")
FLAGS = {"fp64": L.PCOM_PREC_FP64, "mixed": L.PCOM_PREC_MIXED}


def coarse_run(exp: Experiment, flags: int) -> Model:
    """A coarse model started from CG(fine(now)) in the given precision."""
    m = Model(exp.cc, flags=flags)
    m.set_forcing(m.int_bnd())
    if flags & L.PCOM_PREC_MIXED:
        exp.coarsen(exp.truth)
        m.set_state(**{f: exp.truth.field(f) for f in START_FIELDS})
    else:
        exp.coarsen(m)
    return m


def evaluate(exp: Experiment, net: Network, steps: int, forms: dict, flags: int = L.PCOM_PREC_FP64,
             record_every: int = 24, plain_flags=(("plain", L.PCOM_PREC_FP64),)):
    """Coarse runs from CG(fine(t0)) beside the fine run for `steps` coarse
    steps: plain coarse models (`plain_flags`: name -> precision) and, per
    form (name -> (gain, clip, cadence)), the model in precision `flags` with
    the network's tendency applied every `cadence` steps over cadence x dt.
    A closure run whose state stops being finite falls back to the plain
    model (its state is replaced by the first plain run's and the closure is
    switched off).  RMS error of u, v, T, S against CG(fine(t)) every
    `record_every` steps and at the end."""
    torch = exp.torch
    plains = {n: coarse_run(exp, f) for n, f in plain_flags}
    runs = {v: coarse_run(exp, flags) for v in forms}
    stats = {v: _stats_struct(dict(exp.stats, out_gain=g, out_clip=c)) for v, (g, c, _) in forms.items()}
    x = torch.zeros((exp.npix, 16), dtype=torch.bfloat16, device="cuda")
    y = torch.zeros((exp.npix, 4), dtype=torch.float32, device="cuda")
    active = {v: True for v in forms}
    fallback = {v: None for v in forms}
    hist = {n: [] for n in list(plains) + list(runs)}
    first_plain = next(iter(plains.values()))
    it = 100
    for s in range(steps):
        it += 1
        day = s % 24 == 0
        for m in list(plains.values()) + list(runs.values()):
            if day:
                m.den_prho()
            m.step_handle(it)
        for v, m in runs.items():
            cad = forms[v][2]
            if active[v] and (s + 1) % cad == 0:
                exp._features(m, x)
                net.forward(x, y)
                L.check(exp.lib.pcom_gpu_cnn_apply(m.handle, C.c_void_p(y.data_ptr()), C.byref(stats[v]),
                                                   float(STEP * cad)), "apply")
        if (s + 1) % 6 == 0 or s == steps - 1:
            for v, m in runs.items():
                if not active[v]:
                    continue
                try:
                    m.check_finite()
                except L.PcomError:
                    m.set_state(**{f: first_plain.field(f) for f in L.STATE_FIELDS})
                    active[v] = False
                    fallback[v] = s + 1
        exp.fine.run(exp.fine_steps)
        if (s + 1) % record_every == 0 or s == steps - 1:
            for n, m in list(plains.items()) + list(runs.items()):
                hist[n].append(coarse_rms(exp, m))
    mean = lambda h: {f: float(np.mean([r[f] for r in h])) for f in h[0]}
    res = dict(steps=steps, record_every=record_every, plain={}, forms={})
    for n in plains:
        res["plain"][n] = dict(rms_end=hist[n][-1], rms_mean=mean(hist[n]))
    for v in runs:
        g, c, cad = forms[v]
        res["forms"][v] = dict(gain=g, clip=c, cadence=cad, rms_end=hist[v][-1], rms_mean=mean(hist[v]),
                               fell_back_at_step=fallback[v])
    for m in list(plains.values()) + list(runs.values()):
        m.close()
    return res


def form_cost(exp: Experiment, net: Network, flags: int, steps: int = 48) -> dict:
    """Device time of a coarse step in precision `flags` and of one closure
    application (features, forward, apply), CUDA events."""
    torch = exp.torch
    m = coarse_run(exp, flags)
    s = torch.cuda.current_stream()
    m.set_stream(s.cuda_stream)
    net.set_stream(s.cuda_stream)
    st = _stats_struct(dict(exp.stats, out_gain=[0.0, 0.0, 0.0, 0.0], out_clip=3.0))
    x = torch.zeros((exp.npix, 16), dtype=torch.bfloat16, device="cuda")
    y = torch.zeros((exp.npix, 4), dtype=torch.float32, device="cuda")
    lib = exp.lib

    def net_once():
        L.check(lib.pcom_gpu_cnn_features(m.handle, C.c_void_p(x.data_ptr()), C.byref(st)), "features")
        net.forward(x, y)
        L.check(lib.pcom_gpu_cnn_apply(m.handle, C.c_void_p(y.data_ptr()), C.byref(st), float(STEP)), "apply")

    it = 100
    for _ in range(3):
        it += 1
        L.check(lib.pcom_gpu_step_async(m.handle, it), "step")
        net_once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        it += 1
        L.check(lib.pcom_gpu_step_async(m.handle, it), "step")
    e1.record(s)
    torch.cuda.synchronize()
    step_ms = e0.elapsed_time(e1) / steps
    e0.record(s)
    for _ in range(steps // 4):
        net_once()
    e1.record(s)
    torch.cuda.synchronize()
    net_ms = e0.elapsed_time(e1) / (steps // 4)
    m.close()
    net.set_stream(0)
    return dict(step_ms=round(step_ms, 4), network_ms=round(net_ms, 4))


def sypd_of(ms_per_step: float) -> float:
    return (86400.0 / (ms_per_step / 1000.0)) * STEP / (365 * 86400.0)


def main():
    import torch

    p = argparse.ArgumentParser()
    p.add_argument("--fine", default="global025")
    p.add_argument("--fine-flags", default="fp64", choices=sorted(FLAGS))
    p.add_argument("--factor", type=int, default=4)
    p.add_argument("--spinup-days", type=float, default=2)
    p.add_argument("--train-days", type=float, default=8)
    p.add_argument("--every", type=int, default=2, help="coarse steps between training samples")
    p.add_argument("--target-steps", type=int, default=1,
                   help="coarse steps the training residual is accumulated over")
    p.add_argument("--val-days", type=float, default=2, help="window that picks the applied outputs and gain")
    p.add_argument("--test-days", type=float, default=2, help="window the chosen closure is evaluated on")
    p.add_argument("--form-flags", default="fp64", choices=sorted(FLAGS),
                   help="precision of the closure form's coarse model")
    p.add_argument("--cadences", default="1", help="comma-separated: apply the network every k coarse steps")
    p.add_argument("--epochs", type=int, default=8)
    p.add_argument("--lr", type=float, default=1e-3)
    p.add_argument("--out", default=None)
    a = p.parse_args()
    torch.cuda.set_device(0)
    t0 = time.time()
    fc = make_case(a.fine)
    exp = Experiment(fc, a.factor, a.target_steps)
    if FLAGS[a.fine_flags] != L.PCOM_PREC_FP64:
        exp.fine.close()
        exp.fine = Model(fc, flags=FLAGS[a.fine_flags])
    fine_spd = 86400 // exp.fc["dtbc"]
    tf = time.perf_counter()
    exp.fine.run(int(a.spinup_days * fine_spd))
    exp.fine.sync()
    fine_s_per_step = (time.perf_counter() - tf) / max(1, int(a.spinup_days * fine_spd))
    exp.compute_stats()
    nsamp = int(a.train_days * 24 / max(a.every, a.target_steps))
    xs, ts, mask = exp.generate(nsamp, a.every)
    net = Network(exp.H, exp.W, exp.nk)
    tt = time.perf_counter()
    tr = train(net, xs, ts, mask, a.epochs, a.lr)
    t_train = time.perf_counter() - tt
    del xs, ts
    torch.cuda.empty_cache()
    # validation window: which outputs, at which gain (every step, FP64)
    val = evaluate(exp, net, int(a.val_days * 24), {v: (g, c, 1) for v, (g, c) in VARIANTS.items()})
    score = lambda r: r["rms_mean"]["tc"] / max(val["plain"]["plain"]["rms_mean"]["tc"], 1e-30)
    best = min(val["forms"], key=lambda v: score(val["forms"][v]))
    g, c = VARIANTS[best]
    # test window: the chosen closure at each cadence in the form's precision,
    # beside the plain model in FP64 and in the form's precision
    cads = [int(x) for x in a.cadences.split(",")]
    forms = {f"{best}@{k}": (g, c, k) for k in cads}
    plains = (("plain", L.PCOM_PREC_FP64),) + ((("plain_" + a.form_flags, FLAGS[a.form_flags]),)
                                               if a.form_flags != "fp64" else ())
    test = evaluate(exp, net, int(a.test_days * 24), forms, FLAGS[a.form_flags], plain_flags=plains)
    cost_fp64 = form_cost(exp, net, L.PCOM_PREC_FP64)
    cost_form = form_cost(exp, net, FLAGS[a.form_flags])
    test["sypd"] = {"plain": round(sypd_of(cost_fp64["step_ms"]), 1)}
    if a.form_flags != "fp64":
        test["sypd"]["plain_" + a.form_flags] = round(sypd_of(cost_form["step_ms"]), 1)
    for k in cads:
        test["sypd"][f"{best}@{k}"] = round(sypd_of(cost_form["step_ms"] + cost_form["network_ms"] / k), 1)
    res = dict(fine=a.fine, fine_flags=a.fine_flags, coarse_grid=[exp.W, exp.H, exp.nk], samples=nsamp,
               every=a.every, epochs=a.epochs, target_steps=a.target_steps, spinup_days=a.spinup_days,
               train_days=a.train_days, val_days=a.val_days, test_days=a.test_days, form_flags=a.form_flags,
               train=tr, train_seconds=t_train, validation=val, chosen=best, test=test,
               cost={"fp64": cost_fp64, a.form_flags: cost_form}, stats=exp.stats, fine_s_per_step=fine_s_per_step,
               fine_steps_per_coarse_step=exp.fine_steps, wall_seconds=time.time() - t0)
    line = json.dumps(res)
    print(line)
    if a.out:
        with open(a.out, "w") as f:
            f.write(line + "\n")


if __name__ == "__main__":
    main()
