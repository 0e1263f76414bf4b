"""Error of the mixed-precision path (PCOM_PREC_MIXED) against the FP64 path
over long integrations.

Three handles advance the same case side by side through the time loop
(pcom_model_run: daily int_bnd and den_prho, one baroclinic step per step):

- ``fp64``: the FP64 path (bit-equal to the oracle);
- ``mixed``: the mixed-precision path;
- ``control``: the FP64 path started from a temperature field that differs
  by seeded N(0, sigma) noise with sigma = 1e-10 K, some five orders of
  magnitude below the FP32 rounding of T.

At each checkpoint the relative RMS and relative max error over wet points
of the prognostic fields, and the relative error of the global volume, heat
and salt sums, are reported for ``mixed`` and ``control`` against ``fp64``.
The control separates the model's own sensitivity to perturbations of the
initial state (which grows with time in any nonlinear ocean model) from the
error the reduced precision adds.

    python -m pcom_b200.precision_report [--case global1] [--steps 1,720,8760]
        [--json out.json]
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import _lib as L
from .model import Model
from .synth import make_case, perturb

FIELDS = {"tc": "t3", "sc": "t3", "uc": "u3", "vc": "u3", "chc": "t2", "ubc": "u2", "vbc": "u2"}


def _masks(m: Model) -> dict:
    st = m.static()
    k = np.arange(1, m.nk + 1)[:, None, None]
    inner = np.zeros_like(st["lev_t"], dtype=bool)
    inner[1:-1, 1:-1] = True
    return {"t3": (st["lev_t"][None] >= k) & inner[None], "u3": (st["lev_u"][None] >= k) & inner[None],
            "t2": (st["lev_t"] >= 1) & inner, "u2": (st["lev_u"] >= 1) & inner}


def field_errors(test: Model, ref: Model, masks: dict) -> dict:
    out = {}
    for f, w in FIELDS.items():
        x, y = test.field(f)[masks[w]], ref.field(f)[masks[w]]
        d = x - y
        rms_ref = float(np.sqrt(np.mean(y * y)))
        out[f] = {"rel_rms": float(np.sqrt(np.mean(d * d))) / max(rms_ref, 1e-300),
                  "rel_max": float(np.max(np.abs(d))) / max(float(np.max(np.abs(y))), 1e-300),
                  "finite": bool(np.isfinite(x).all())}
    return out


def sum_errors(test: Model, ref: Model) -> dict:
    a, b = test.global_sums(), ref.global_sums()
    return {k: abs(x - y) / max(abs(y), 1e-300) for k, x, y in zip(("volume", "heat", "salt"), a, b)}


def run(case_name: str = "global1", checkpoints=(1, 720, 8760), sigma: float = 1e-10) -> dict:
    case = make_case(case_name)
    models = {"fp64": Model(case), "mixed": Model(case, flags=L.PCOM_PREC_MIXED),
              "control": Model(perturb(case, 0, sigma))}
    masks = _masks(models["fp64"])
    report = {"case": case_name, "grid": [case["glo_ni"], case["glo_nj"], case["nk"]],
              "control_sigma_K": sigma, "checkpoints": []}
    done = 0
    t0 = time.time()
    for n in sorted(checkpoints):
        for m in models.values():
            m.run(n - done)
        done = n
        entry = {"steps": n, "days": n * case["dtbc"] / 86400.0}
        for name in ("mixed", "control"):
            entry[name] = {"fields": field_errors(models[name], models["fp64"], masks),
                           "global_sums": sum_errors(models[name], models["fp64"])}
        report["checkpoints"].append(entry)
        print(f"[{time.time() - t0:7.1f} s] step {n}: " +
              ", ".join(f"{f} mixed {entry['mixed']['fields'][f]['rel_rms']:.2e} / control "
                        f"{entry['control']['fields'][f]['rel_rms']:.2e}" for f in FIELDS), flush=True)
    for m in models.values():
        m.close()
    return report


def markdown(report: dict) -> str:
    lines = [f"Relative RMS (max) error over wet points against the FP64 path, "
             f"{report['case']} {report['grid']}; control = FP64 with N(0, {report['control_sigma_K']:g} K) on the initial T",
             "", "| steps (days) | run | " + " | ".join(FIELDS) + " | heat sum | salt sum |",
             "|---|---|" + "---:|" * (len(FIELDS) + 2)]
    for e in report["checkpoints"]:
        for name in ("mixed", "control"):
            r = e[name]
            cells = [f"{r['fields'][f]['rel_rms']:.1e} ({r['fields'][f]['rel_max']:.1e})" for f in FIELDS]
            cells += [f"{r['global_sums']['heat']:.1e}", f"{r['global_sums']['salt']:.1e}"]
            lines.append(f"| {e['steps']} ({e['days']:g}) | {name} | " + " | ".join(cells) + " |")
    return "\n".join(lines)


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--case", default="global1")
    ap.add_argument("--steps", default="1,720,8760", help="comma-separated checkpoints (steps)")
    ap.add_argument("--sigma", type=float, default=1e-10)
    ap.add_argument("--json", default=None)
    a = ap.parse_args(argv)
    rep = run(a.case, [int(s) for s in a.steps.split(",")], a.sigma)
    if a.json:
        with open(a.json, "w") as f:
            json.dump(rep, f, indent=1)
    print(markdown(rep))


if __name__ == "__main__":
    main()
