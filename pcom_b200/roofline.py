"""Per-kernel HBM roofline of the step, FP64 and mixed precision.

For each kernel of the step: its CUDA-event time per launch (an event pair
around every launch), the bytes it must move per launch at minimum (the
algorithmic bytes: every 3-D and 2-D field it reads or writes, once), the
achieved GB/s and the fraction of the measured HBM copy bandwidth
(MEASURED_PEAKS.json beside the repository, else the pool's earlier
measurement of 6,650 GB/s).  Optionally a run of whole model days on both
paths, with the time per step, the simulated years per wall day and the
mixed path's error against the FP64 path at the end.

    python -m pcom_b200.roofline [--case global025] [--steps 12] [--days 10]
        [--json out.json]
"""
from __future__ import annotations

import argparse
import json
import os


from . import _lib as L

HERE = os.path.dirname(os.path.abspath(__file__))

# kernel: (3-D fields read + written, 2-D fields read + written); the
# barotropic subcycle moves (ch, ub, vb) in and out once per substep plus
# its static fields once per launch
FIELDS = {
    "den_alpha+int_tobot": (4, 1),         # R tc, sc; W alpha, adp; R chc
    "int_pgra": (2, 8 + 4),                # R alpha, adp; W bphi/bgraphi (8); statics
    "readyc_2d": (0, 4 + 6),
    "upwelling": (3, 4),                   # R uc, vc; W wm
    "readyc_3d": (2 + 1 + 2 + 4 + 1, 6),   # R uc, vc, wm, am, (km); W auc, avc, fx, fy
    "int_trop": (0, 30),                   # statics once; substeps below
    "clin_2d": (0, 5 + 6),                # int_clin's 2-D prep and, in the full step, int_ts's (one launch)
    "int_clin": (12 + 7, 8),               # R adp, alpha, 6 AB3, fx, fy, uc, vc, up, vp; W uc, vc, up, vp, uu, vv, acu
    "smag": (3, 2),
    "int_ssh": (3, 3),
    "ts_2d": (0, 4),                       # its own launch only when phases run one by one
    "upwelling+acw": (6, 4),
    "int_ts": (4 + 2 + 1 + 2 + 1 + 2 + 6, 6),  # R tc, sc, tp, sp, uc, vc, wm, kh, prho(2); W tn, sn; RW act, acs, acr
    "den_prho": (4, 1),
}


def algorithmic_bytes(kernel: str, glo_ni: int, glo_nj: int, nk: int, nstep: int, mixed: bool = False) -> float:
    """Bytes a kernel must move per launch at minimum, over the interior
    points (glo_ni x glo_nj [x nk]).  FP64: 8 bytes per value.  Mixed: 3-D
    fields in FP32 (4 bytes), 2-D fields FP64, and the barotropic substep's
    ub, vb in FP32 with ch in FP64."""
    n2 = glo_ni * glo_nj
    n3 = n2 * nk
    s3 = 4.0 if mixed else 8.0
    f3, f2 = FIELDS.get(kernel, (0, 0))
    b = s3 * f3 * n3 + 8.0 * f2 * n2
    if kernel == "int_trop":
        per_point = (2 * 8 + 4 * 4) if mixed else 6 * 8  # R/W ch, ub, vb
        b += nstep * per_point * n2
    return b


def hbm_peak() -> tuple:
    for p in (os.path.join(HERE, "..", "MEASURED_PEAKS.json"),):
        try:
            with open(p) as f:
                v = json.load(f).get("hbm_gbs")
            if v:
                return float(v), "measured"
        except (OSError, ValueError):
            pass
    return 6650.0, "fallback"


def _steps(m, first: int, n: int, day_of):
    lib = m.lib
    for q in range(n):
        it = first + q
        if day_of(it) != day_of(it - 1):
            L.check(lib.pcom_gpu_den_prho(m.handle), "den_prho")
        L.check(lib.pcom_gpu_step_async(m.handle, it), "step")


def kernel_table(case: dict, mixed: bool, steps: int) -> dict:
    import torch

    from .model import Model

    m = Model(case, flags=L.PCOM_PREC_MIXED if mixed else L.PCOM_PREC_FP64)
    m.run(3)  # AB3 start-up and a warm cache of kernels
    spd = 86400 // case["dtbc"]
    day_of = lambda it: (it - 1) // spd
    it0 = m.iter + 1
    s = torch.cuda.current_stream()
    m.set_stream(s.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    _steps(m, it0, steps, day_of)
    e1.record(s)
    torch.cuda.synchronize()
    ms_step = e0.elapsed_time(e1) / steps
    m.profile(True)
    _steps(m, it0 + steps, steps, day_of)
    m.sync()
    prof = m.profile_read()
    m.profile(False)
    m.close()
    peak, src = hbm_peak()
    nstep = case["dtbc"] // case["dtbt"] * 2
    rows = {}
    for k, (n, ms) in sorted(prof.items(), key=lambda kv: -kv[1][1]):
        us = ms / n * 1000.0
        b = algorithmic_bytes(k, case["glo_ni"], case["glo_nj"], case["nk"], nstep, mixed)
        gbs = b / (us * 1e-6) / 1e9 if us > 0 else 0.0
        rows[k] = {"launches": n, "us_per_launch": round(us, 1), "algorithmic_MB": round(b / 1e6, 2),
                   "GB_s": round(gbs, 1), "frac_of_peak": round(gbs / peak, 4)}
    return {"ms_per_step": round(ms_step, 4), "peak_GB_s": peak, "peak_source": src, "kernels": rows}


def days_run(case: dict, days: float) -> dict:
    """Whole model days through the time loop (daily forcing and den_prho)
    on both paths: time per step, simulated years per wall day, finiteness,
    and the mixed path's error against the FP64 path at the end."""
    import torch

    from .model import Model
    from .precision_report import _masks, field_errors, sum_errors

    nsteps = int(round(days * 86400 / case["dtbc"]))
    out = {"days": days, "steps": nsteps}
    models = {}
    for name, flags in (("fp64", L.PCOM_PREC_FP64), ("mixed", L.PCOM_PREC_MIXED)):
        m = Model(case, flags=flags)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        m.run(nsteps)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / nsteps
        m.check_finite()
        sypd = (case["dtbc"] / (365.0 * 86400.0)) / (ms / 1000.0 / 86400.0)
        out[name] = {"ms_per_step": round(ms, 3), "sypd": round(sypd, 2)}
        models[name] = m
    masks = _masks(models["fp64"])
    out["mixed_vs_fp64"] = {"fields": field_errors(models["mixed"], models["fp64"], masks),
                            "global_sums": sum_errors(models["mixed"], models["fp64"])}
    for m in models.values():
        m.close()
    return out


def cnn_table(H: int, W: int, nimg: int, steps: int) -> dict:
    """The closure network on nimg images of H x W (one per level of a
    H x W grid): CUDA-event time of the forward pass and of a training step
    (forward, data and weight gradients, Adam) on random inputs, and their
    tensor throughput on the FLOPs the convolutions issue (padded channels)."""
    import torch

    from .closure import Network

    net = Network(H, W, nimg, seed=5)
    npix = H * W * nimg
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.zeros((npix, 16), dtype=torch.bfloat16, device="cuda")
    x[:, :5] = torch.randn((npix, 5), generator=g, device="cuda").to(torch.bfloat16)
    y = torch.zeros((npix, 4), dtype=torch.float32, device="cuda")
    t = torch.randn((npix, 4), generator=g, device="cuda")
    mk = torch.ones((npix, 4), device="cuda")
    s = torch.cuda.current_stream()
    net.set_stream(s.cuda_stream)
    flop = npix * 9 * 2 * (16 * 64 + 3 * 64 * 64 + 64 * 16)
    out = {"images": nimg, "H": H, "W": W, "flop_per_forward": flop}
    for name, fn in (("forward", lambda: net.forward(x, y)), ("train_step", lambda: net.train_step(x, t, mk, 1e-4))):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s)
        for _ in range(steps):
            fn()
        e1.record(s)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        f = flop * (3 if name == "train_step" else 1)
        out[name] = {"ms": round(ms, 4), "TFLOP_s": round(f / (ms * 1e-3) / 1e12, 1)}
    net.close()
    return out


def markdown(rep: dict) -> str:
    lines = []
    for name in ("fp64", "mixed"):
        t = rep.get(name)
        if not t:
            continue
        lines += [f"{name}: {t['ms_per_step']} ms per step (device-resident, {rep['steps']} steps), "
                  f"HBM peak {t['peak_GB_s']} GB/s ({t['peak_source']})", "",
                  "| kernel | us per launch | algorithmic MB | GB/s | of peak |", "|---|---:|---:|---:|---:|"]
        for k, r in t["kernels"].items():
            lines.append(f"| {k} | {r['us_per_launch']} | {r['algorithmic_MB']} | {r['GB_s']} | {r['frac_of_peak']:.3f} |")
        lines.append("")
    d = rep.get("days_run")
    if d:
        lines.append(f"{d['days']} model days ({d['steps']} steps): FP64 {d['fp64']['ms_per_step']} ms/step "
                     f"({d['fp64']['sypd']} SYPD), mixed {d['mixed']['ms_per_step']} ms/step ({d['mixed']['sypd']} SYPD)")
        e = d["mixed_vs_fp64"]
        lines.append("mixed vs FP64, relative RMS: " + ", ".join(f"{f} {v['rel_rms']:.1e}" for f, v in e["fields"].items())
                     + f"; heat sum {e['global_sums']['heat']:.1e}")
    return "\n".join(lines)


def main(argv=None):
    from .synth import make_case

    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--case", default="global025")
    ap.add_argument("--steps", type=int, default=12, help="steps timed per path (and again with events)")
    ap.add_argument("--days", type=float, default=0.0, help="model days of the time loop on both paths")
    ap.add_argument("--json", default=None)
    ap.add_argument("--cnn", type=int, default=0, help="also time N forward passes and training steps of the "
                                                      "closure network on the case's level images")
    a = ap.parse_args(argv)
    case = make_case(a.case)
    rep = {"case": a.case, "grid": [case["glo_ni"], case["glo_nj"], case["nk"]], "steps": a.steps,
           "fp64": kernel_table(case, False, a.steps), "mixed": kernel_table(case, True, a.steps)}
    if a.days > 0:
        rep["days_run"] = days_run(case, a.days)
    if a.cnn > 0:
        rep["cnn"] = cnn_table(case["glo_nj"], case["glo_ni"], case["nk"], a.cnn)
        print(json.dumps(rep["cnn"]))
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rep, f, indent=1)
    print(markdown(rep))


if __name__ == "__main__":
    main()
