#!/usr/bin/env python
"""Benchmark: simulated years per wall-clock day (SYPD) of the PCOM baroclinic
step at 1 degree x 30 levels (360 x 160 x 30 near-global synthetic case) on
B200, FP64 plain path.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One "step" is one baroclinic step of dtbc = 3600 s (main.f90:205-223: EOS,
pressure-gradient integrals, advection/friction, the 120-substep barotropic
subcycle, baroclinic momentum, SSH, tracers with convective adjustment), plus
the daily density derivatives when the model day changes.  SYPD =
(steps * 3600 s / 365 d) / wall days.  With N > 1 GPUs every rank advances its
own ensemble member (replicas, no data-path collective): value = the sum over
ranks, timed as the max over ranks.

--impl reference times the reference algorithm's CPU implementation (the C++
restatement in oracle/, OpenMP over all host cores) on the same case.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CASE = "global1"
STEP_SECONDS = 3600
YEAR_STEPS = 365 * 86400 / STEP_SECONDS  # 8760 steps per model year


def sypd(seconds_per_step: float, dtbc: float = STEP_SECONDS) -> float:
    """Simulated years per wall-clock day for steps of dtbc model seconds."""
    return (86400.0 / seconds_per_step) * dtbc / (365 * 86400.0)


def max_over_ranks(t_ms: float, world: int, device: str) -> float:
    """The slowest rank's time (every rank takes part in the collective)."""
    if world <= 1:
        return t_ms
    import torch
    import torch.distributed as dist

    tt = torch.tensor([t_ms], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def replica_sypd(ms_per_step: float, world: int) -> float:
    """Whole-job SYPD of `world` replicas (one member per rank), each step
    timed as the max over ranks: every rank advanced its member by one step."""
    return world * sypd(ms_per_step / 1000.0)


METRIC = "SYPD at 1deg x 30L (360x160x30 near-global), FP64 plain path"


def workload_config(case: dict, world: int) -> dict:
    """The workload both arms time (the GPU arm and --impl reference)."""
    return {
        "workload": "global1: 360x160x30 1-degree near-global ocean, dtbc 3600 s, dtbt 60 s "
                    "(120 barotropic substeps per step), one baroclinic step per step",
        "grid": [case["glo_ni"], case["glo_nj"], case["nk"]],
        "parallelism": "replicas" if world > 1 else "single GPU",
        "l2": "inputs larger than L2: ~0.9 GB of resident state vs 126 MB L2",
    }


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=48)
    p.add_argument("--warmup", type=int, default=4)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-sample-steps", type=int, default=8)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision leg")
    p.add_argument("--no-closure", action="store_true", help="skip the closure-network leg")
    p.add_argument("--no-global025", action="store_true", help="skip the 0.25-degree leg")
    p.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble leg")
    p.add_argument("--decomp", action="store_true",
                   help="one 1-degree domain split into row slabs over the N ranks (strong scaling) "
                        "instead of N replicas")
    p.add_argument("--halo", type=int, default=2, help="halo rows of the row-slab split")
    p.add_argument("--workload", default="global1", choices=["global1", "ensemble"],
                   help="ensemble: 32 perturbed 1-degree members + 16 uneven basins, batched")
    p.add_argument("--members", type=int, default=32)
    p.add_argument("--member-case", default="box", choices=["box", "global1"],
                   help="ensemble member grid: box 128x64x20 or the 1-degree 360x160x30 case")
    p.add_argument("--basins", type=int, default=16)
    return p.parse_args()


# ---------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a moment to start: begin timing once it samples
            t0 = time.time()
            while not self.lines and time.time() - t0 < 5.0 and self.proc.poll() is None:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------- roofline
def algorithmic_bytes(kernel: str, glo_ni: int, glo_nj: int, nk: int, nstep: int) -> float:
    """Bytes a kernel must move per launch at minimum on the FP64 path (the
    per-kernel field counts of pcom_b200.roofline)."""
    from pcom_b200.roofline import algorithmic_bytes as ab

    return ab(kernel, glo_ni, glo_nj, nk, nstep, mixed=False)


def run_ours(args):
    import torch
    import torch.distributed as dist

    from pcom_b200 import _lib as L
    from pcom_b200.model import Model
    from pcom_b200.synth import make_case, perturb

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    case = make_case(CASE)
    if world > 1 and rank > 0:
        case = perturb(case, rank)  # each rank integrates its own ensemble member
    m = Model(case)
    stream = torch.cuda.current_stream()
    m.set_stream(stream.cuda_stream)
    lib, h = m.lib, m.handle
    ni, nj, nk = m.ni, m.nj, m.nk
    n2 = ni * nj

    # warm-up through the host driver (includes the AB3 start-up steps)
    m.run(max(args.warmup, 3))
    it0 = m.iter

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # ------------------------------------------------ value: device-resident
    # per step: den_prho when the model day changes (every 24 steps), then the
    # step block.  The state (~0.9 GB) is far larger than L2 (126 MB).
    steps = args.steps
    day_of = lambda it: (it - 1) * STEP_SECONDS // 86400

    def device_loop(first):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for q in range(steps):
            it = first + q
            if day_of(it) != day_of(it - 1):
                L.check(lib.pcom_gpu_den_prho(h), "den_prho")
            L.check(lib.pcom_gpu_step_async(h, it), "step")
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    launches0 = m.launch_count()
    barrier()
    # clocks are sampled over every timed loop below (device-resident, with
    # kernel events, end to end): the first alone is ~60 ms
    clk = Clocks(dev).__enter__()
    t_ms = device_loop(it0 + 1)
    launches = m.launch_count() - launches0
    L.check(lib.pcom_gpu_check_finite(h), "watchdog")
    t_max = max_over_ranks(t_ms, world, "cuda")
    ms_per_step = t_max / steps
    value = replica_sypd(ms_per_step, world)
    # the same K steps again with an event pair around every kernel: the
    # per-kernel durations of the breakdown and the roofline
    m.profile(True)
    barrier()
    t_prof = max_over_ranks(device_loop(it0 + 1 + steps), world, "cuda")
    prof = m.profile_read()
    m.profile(False)
    it0 += steps

    # ------------------------------------------------ e2e: host buffers
    # per step through the reference-facing API: the day's forcing from pinned
    # host memory (int_bnd on the host; taux, tauy, t, s, pa), the step, and
    # the barotropic state (ch, ub, vb) read back into pinned host memory.
    # The headline form uses the asynchronous transfer calls (forcing staged
    # and state copied out on the handle's upload/download streams, overlapping the
    # steps; one synchronisation at the end); e2e_sync times the
    # synchronous calls (set_forcing, step, get_state) for comparison.
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True)
    frc = [pin(n2) for _ in range(6)]
    out = [pin(n2) for _ in range(3)]
    host_f = m.int_bnd()
    for t_, k_ in zip(frc, ("taux", "tauy", "t", "s", "pa", "fw")):
        t_.copy_(torch.from_numpy(host_f[k_].reshape(-1)))
    import ctypes as C
    dp = lambda t_: C.cast(t_.data_ptr(), L.dbl_p)
    fo = L.Forcing(*[dp(t_) for t_ in frc])
    st_out = L.State(*[None] * len(L.STATE_FIELDS))
    st_out.chc, st_out.ubc, st_out.vbc = dp(out[0]), dp(out[1]), dp(out[2])
    def e2e_loop(first, asynchronous):
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        barrier()
        f0.record(stream)
        for q in range(steps):
            it = first + q
            if asynchronous:
                L.check(lib.pcom_gpu_set_forcing_async(h, C.byref(fo)), "set_forcing_async")
            else:
                L.check(lib.pcom_gpu_set_forcing(h, C.byref(fo)), "set_forcing")
            if day_of(it) != day_of(it - 1):
                L.check(lib.pcom_gpu_den_prho(h), "den_prho")
            if asynchronous:
                L.check(lib.pcom_gpu_step_async(h, it), "step_async")
                L.check(lib.pcom_gpu_get_state_async(h, C.byref(st_out)), "get_state_async")
            else:
                L.check(lib.pcom_gpu_step(h, it), "step")
                L.check(lib.pcom_gpu_get_state(h, C.byref(st_out)), "get_state")
        if asynchronous:
            L.check(lib.pcom_gpu_sync(h), "sync")  # the last state is in host memory
        f1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(f0.elapsed_time(f1), world, "cuda")

    it1 = it0 + steps
    e2e_ms = e2e_loop(it1 + 1, True)
    e2e = replica_sypd(e2e_ms / steps, world)
    e2e_sync = replica_sypd(e2e_loop(it1 + 1 + steps, False) / steps, world)
    clk.__exit__(None, None, None)

    # the barotropic subcycle's latency floor: its synchronisation skeleton
    # (same grid, block, barriers, ring reload and stores; no arithmetic),
    # the median of 3 launches after 2; None where the handle does not run
    # the resident FP64 kernel
    floor_ms = None
    t_ = C.c_double(0.0)
    vals = []
    for r in range(5):
        if lib.pcom_gpu_trop_floor(h, C.byref(t_)) != 0:
            vals = []
            break
        if r >= 2:
            vals.append(t_.value)
    if vals:
        floor_ms = statistics.median(vals)

    # ------------------------------------------------ roofline of the dominant kernel
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    top = max(prof.items(), key=lambda kv: kv[1][1]) if prof else ("", (1, 0.0))
    kname, (klaunch, kms) = top
    nstep = case["dtbc"] // case["dtbt"] * 2
    kbytes = algorithmic_bytes(kname, case["glo_ni"], case["glo_nj"], nk, nstep)
    avg_s = kms / max(klaunch, 1) / 1000.0
    achieved = kbytes / avg_s / 1e9 if avg_s > 0 else 0.0
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "ncu_traffic.json")))
        traffic = tr.get(kname, {}).get("bytes_per_launch")
    except Exception:
        pass
    kernels = {k: {"launches": v[0], "ms_total": round(v[1], 4), "share": round(v[1] / max(1e-9, sum(x[1] for x in prof.values())), 4)}
               for k, v in sorted(prof.items(), key=lambda kv: -kv[1][1])}

    # ------------------------------------------------ mixed-precision path
    # the same device-resident loop on a PCOM_PREC_MIXED handle, and the
    # per-field error of a fresh pair of runs after one model day
    mixed = None
    if not args.no_mixed:
        mixed = run_mixed_leg(args, case, stream, steps)
    closure = None
    if not args.no_closure:
        closure = run_closure_leg(args, case, ms_per_step)
    # the 0.25-degree grid (bandwidth-sized) and the batched ensemble: N = 1 only
    global025 = ensemble = None
    if world == 1 and not args.no_global025:
        global025 = run_global025_leg(args)
    if world == 1 and not args.no_ensemble:
        ensemble = ensemble_measure(args, steps=min(steps, 24), print_line=False)

    # ------------------------------------------------ CPU baseline (rank 0, N = 1)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_sample_steps)

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC,
            "value": round(value, 2),
            "unit": "SYPD",
            "n_gpus": world,
            "steps": steps,
            "warmup": max(args.warmup, 3),
            "ms_per_step": round(ms_per_step, 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic (seeded k^-2 bathymetry, analytic wind and restoring)",
            "config": workload_config(case, world),
            "timing": "CUDA events on the model's stream; kernels and roofline from a second timed pass "
                      "of the same K steps with an event pair around every kernel",
            "ms_per_step_with_kernel_events": round(t_prof / steps, 4),
            "e2e": {"value": round(e2e, 2), "unit": "SYPD", "h2d_bytes_per_step": 5 * n2 * 8,
                    "d2h_bytes_per_step": 3 * n2 * 8,
                    "transfers": "pinned host memory; forcing staged and state copied out on the handle's upload/download streams "
                                 "(pcom_gpu_set_forcing_async / pcom_gpu_get_state_async), overlapping the steps",
                    "sync_calls_value": round(e2e_sync, 2)},
            "roofline": {"kernel": kname, "bound": "hbm", "achieved": round(achieved, 1),
                         "peak": hbm_peak, "peak_source": peak_src, "unit": "GB/s",
                         "frac": round(achieved / hbm_peak, 4), "traffic": traffic,
                         "algorithmic_bytes_per_launch": kbytes,
                         # the barotropic subcycle keeps its state on chip: its
                         # time is the latency of 120 dependent substeps
                         "us_per_substep": round(avg_s * 1e6 / nstep, 3) if kname == "int_trop" else None,
                         # against the latency floor: the kernel's barriers,
                         # ring reload and stores without its arithmetic
                         "latency_floor": ({"us_per_substep": round(floor_ms * 1e3 / nstep, 3),
                                            "floor_over_actual": round(floor_ms * 1e-3 / avg_s, 3),
                                            "measured": "pcom_gpu_trop_floor: the resident kernel's synchronisation "
                                                        "skeleton, same grid and barriers, no arithmetic"}
                                           if floor_ms and kname == "int_trop" and avg_s > 0 else None)},
            "kernels": kernels,
            "gpu_launches": int(launches),
            "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
            "cpu_baseline": cpu,
            "mixed": mixed,
            "closure": closure,
            "global025": global025,
            "ensemble": ensemble,
        }
        print(json.dumps(line))
    m.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_mixed_leg(args, case, stream, steps):
    import torch

    from pcom_b200 import _lib as L
    from pcom_b200.model import Model

    mm = Model(case, flags=L.PCOM_PREC_MIXED)
    mm.set_stream(stream.cuda_stream)
    mm.run(max(args.warmup, 3))
    it0 = mm.iter
    day_of = lambda it: (it - 1) * STEP_SECONDS // 86400
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for q in range(steps):
        it = it0 + 1 + q
        if day_of(it) != day_of(it - 1):
            L.check(mm.lib.pcom_gpu_den_prho(mm.handle), "den_prho")
        L.check(mm.lib.pcom_gpu_step_async(mm.handle, it), "step")
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    mm.check_finite()
    mm.close()
    # error after one model day (24 steps) against the FP64 path
    a, b = Model(case), Model(case, flags=L.PCOM_PREC_MIXED)
    a.run(24)
    b.run(24)
    st = a.static()
    k = np.arange(1, a.nk + 1)[:, None, None]
    mk = {"t3": st["lev_t"][None] >= k, "u3": st["lev_u"][None] >= k, "t2": st["lev_t"] >= 1, "u2": st["lev_u"] >= 1}
    which = {"tc": "t3", "sc": "t3", "uc": "u3", "vc": "u3", "chc": "t2", "ubc": "u2", "vbc": "u2"}
    err = {}
    for f, w in which.items():
        x, y = b.field(f)[mk[w]], a.field(f)[mk[w]]
        err[f] = float(np.sqrt(np.mean((x - y) ** 2)) / max(np.sqrt(np.mean(y * y)), 1e-30))
    a.close()
    b.close()
    return {"ms_per_step": round(ms, 4), "value": round(sypd(ms / 1000.0), 2), "unit": "SYPD", "dtype": "f32 stencils and barotropic velocities, f64 bottom pressure",
            "rel_rms_error_vs_fp64_after_24_steps": {k_: float(f"{v:.3e}") for k_, v in err.items()}}


def device_ms_per_step(m, stream, steps: int, warmup: int) -> float:
    """CUDA-event time per step of `steps` device-resident steps (den_prho on
    day change) after `warmup` steps through the host driver."""
    import torch

    from pcom_b200 import _lib as L

    m.set_stream(stream.cuda_stream)
    m.run(max(warmup, 3))
    it0 = m.iter
    day_of = lambda it: (it - 1) * STEP_SECONDS // 86400
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for q in range(steps):
        it = it0 + 1 + q
        if day_of(it) != day_of(it - 1):
            L.check(m.lib.pcom_gpu_den_prho(m.handle), "den_prho")
        L.check(m.lib.pcom_gpu_step_async(m.handle, it), "step")
    e1.record(stream)
    torch.cuda.synchronize()
    m.check_finite()
    return e0.elapsed_time(e1) / steps


CLOSURE_CADENCE = 8  # the closure form: the network every 8 coarse steps (tendency over 8 dt)


def run_closure_leg(args, case, plain_ms):
    """Cost of the closure form on the same grid: the mixed-precision model
    with the network (input features, 5 tcgen05 convolutions over the 30
    level images, the tendency applied) every k steps; each piece timed with
    CUDA events.  k = 8 is the form pcom_b200.closure's year-long run of
    configuration 5 evaluates (its errors are the same at k = 1, 4 and 8);
    the tensor throughput of the forward pass is against the measured BF16
    peak.  The weights are random here (cost does not depend on them); the
    closure's accuracy is measured by pcom_b200.closure against the
    coarse-grained 0.25-degree run."""
    import ctypes as C

    import torch

    from pcom_b200 import _lib as L
    from pcom_b200.closure import Network
    from pcom_b200.model import Model

    stream = torch.cuda.current_stream()
    m = Model(case, flags=L.PCOM_PREC_MIXED)
    mixed_ms = device_ms_per_step(m, stream, args.steps, args.warmup)
    H, W, nk = case["glo_nj"], case["glo_ni"], case["nk"]
    npix = H * W * nk
    net = Network(H, W, nk, seed=3)
    x = torch.zeros((npix, 16), dtype=torch.bfloat16, device="cuda")
    y = torch.zeros((npix, 4), dtype=torch.float32, device="cuda")
    st = L.CnnStats()
    for q in range(5):
        st.in_std[q] = 1.0
    for q in range(4):
        st.out_std[q] = 1e-9
        st.out_gain[q] = 1.0
    st.out_clip = 3.0
    net.set_stream(stream.cuda_stream)
    lib = m.lib

    def once():
        L.check(lib.pcom_gpu_cnn_features(m.handle, C.c_void_p(x.data_ptr()), C.byref(st)), "features")
        net.forward(x, y)
        L.check(lib.pcom_gpu_cnn_apply(m.handle, C.c_void_p(y.data_ptr()), C.byref(st), 3600.0), "apply")

    for _ in range(3):
        once()
    torch.cuda.synchronize()
    n = 10
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(n):
        once()
    e1.record(stream)
    torch.cuda.synchronize()
    net_ms = e0.elapsed_time(e1) / n
    # the forward alone, for the tensor-core throughput
    e0.record(stream)
    for _ in range(n):
        net.forward(x, y)
    e1.record(stream)
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / n
    flop = npix * 9 * 2 * (16 * 64 + 3 * 64 * 64 + 64 * 16)  # padded channels, as issued
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = float(peaks.get("bf16_tflops", 1590.0))
    tf = flop / (fwd_ms * 1e-3) / 1e12
    net.close()
    m.close()
    per = {k: round(sypd((mixed_ms + net_ms / k) / 1000.0), 2) for k in (1, 4, CLOSURE_CADENCE)}
    total = mixed_ms + net_ms / CLOSURE_CADENCE
    return {"form": f"mixed-precision model + network every {CLOSURE_CADENCE} steps (tendency over {CLOSURE_CADENCE} dt)",
            "ms_per_step": round(total, 4), "value": round(sypd(total / 1000.0), 2), "unit": "SYPD",
            "cadence": CLOSURE_CADENCE, "value_per_cadence": per, "plain_fp64_ms_per_step": round(plain_ms, 4),
            "mixed_ms_per_step": round(mixed_ms, 4), "network_ms": round(net_ms, 4), "forward_ms": round(fwd_ms, 4),
            "tensor": {"achieved": round(tf, 1), "peak": peak, "unit": "TFLOP/s",
                       "peak_source": "measured" if "bf16_tflops" in peaks else "fallback",
                       "frac": round(tf / peak, 4), "flop_per_forward": flop},
            "note": "cost with random weights; accuracy: pcom_b200.closure (configuration 5)"}


def run_global025_leg(args, steps: int = 8):
    """The 1440x640x30 0.25-degree case (dtbc 1200 s, dtbt 20 s), FP64 and
    mixed: time per step (CUDA events, device-resident, ~10 GB of state) and
    the per-kernel algorithmic GB/s of a second pass with kernel events."""
    from pcom_b200.roofline import kernel_table
    from pcom_b200.synth import make_case

    case = make_case("global025")
    out = {"grid": [case["glo_ni"], case["glo_nj"], case["nk"]], "dtbc": case["dtbc"], "dtbt": case["dtbt"],
           "steps": steps}
    for name, mixed in (("fp64", False), ("mixed", True)):
        t = kernel_table(case, mixed, steps)
        ms = t["ms_per_step"]
        top = dict(list(t["kernels"].items())[:6])
        out[name] = {"ms_per_step": ms, "value": round(sypd(ms / 1000.0, case["dtbc"]), 2), "unit": "SYPD",
                     "kernels": {k: {"us": v["us_per_launch"], "GB_s": v["GB_s"], "frac": v["frac_of_peak"]}
                                 for k, v in top.items()},
                     "peak_GB_s": t["peak_GB_s"], "peak_source": t["peak_source"]}
    return out


def ensemble_cases(members: int, basins: int, member_case: str = "box"):
    """Members of one case (default the 128x64x20 1-degree box) with seeded
    N(0, 0.05 K) perturbations of T (seeds 1..members), and idealized basins
    from 64x32 to 256x128 with 20 to 30 levels (all with dtbt 60 s, dtbc
    3600 s)."""
    from pcom_b200.synth import make_case, perturb

    base = make_case(member_case)
    cases = [perturb(base, m + 1, 0.05) for m in range(members)]
    for b in range(basins):
        f = b / max(basins - 1, 1)
        ni = int(round((64 + 192 * f) / 8)) * 8
        cases.append(make_case("basin", seed=100 + b, glo_ni=ni, glo_nj=ni // 2, nk=int(round(20 + 10 * f))))
    return cases


def run_ensemble(args):
    ensemble_measure(args, args.steps, print_line=True)


def ensemble_measure(args, steps: int, print_line: bool):
    """Aggregate SYPD of a batched ensemble vs the same members stepped one
    after another through the single-domain path (same stream, same models)."""
    import ctypes as C

    import torch

    from pcom_b200 import _lib as L
    from pcom_b200.model import Batch, Model

    torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    cases = ensemble_cases(args.members, args.basins, args.member_case)
    stream = torch.cuda.current_stream()
    models = []
    for c in cases:
        m = Model(c)
        m.set_stream(stream.cuda_stream)
        models.append(m)
    lib = models[0].lib
    n = len(models)
    b = Batch(models)
    warm = max(args.warmup, 3)
    b.run(warm)  # AB3 start-up steps
    tune = b.autotune()
    b.run(3)  # capture the graph of every ring phase
    it0 = models[0].iter
    day_of = lambda it: (it - 1) * STEP_SECONDS // 86400

    def timed(body):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        body()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    counts0 = b.launch_count()

    def batched(first):
        def body():
            for q in range(steps):
                it = first + q
                if day_of(it) != day_of(it - 1):
                    b.den_prho()
                b.step_async(it)
        return body

    with Clocks(dev) as clk:
        t_batch = timed(batched(it0 + 1))
    b.sync()
    launches_batched = b.launch_count() - counts0

    def sequential(first):
        def body():
            for q in range(steps):
                it = first + q
                for m in models:
                    if day_of(it) != day_of(it - 1):
                        L.check(lib.pcom_gpu_den_prho(m.handle), "den_prho")
                    L.check(lib.pcom_gpu_step_async(m.handle, it), "step")
        return body

    t_seq = timed(sequential(it0 + 1 + steps))
    for m in models:
        m.sync()

    # e2e through the public API: per step every member's forcing from pinned
    # host memory, the batched step, and every member's barotropic state back
    pin = lambda k: torch.empty(k, dtype=torch.float64, pin_memory=True)
    dp = lambda t_: C.cast(t_.data_ptr(), L.dbl_p)
    fos, sts, keep = [], [], []
    h2d = d2h = 0
    for m in models:
        n2 = m.ni * m.nj
        hf = m.int_bnd()
        frc = [pin(n2) for _ in range(6)]
        for t_, k_ in zip(frc, ("taux", "tauy", "t", "s", "pa", "fw")):
            t_.copy_(torch.from_numpy(hf[k_].reshape(-1)))
        out = [pin(n2) for _ in range(3)]
        keep += frc + out
        fos.append(L.Forcing(*[dp(t_) for t_ in frc]))
        st = L.State(*[None] * len(L.STATE_FIELDS))
        st.chc, st.ubc, st.vbc = dp(out[0]), dp(out[1]), dp(out[2])
        sts.append(st)
        h2d += 6 * n2 * 8
        d2h += 3 * n2 * 8
    first = it0 + 1 + 2 * steps

    # the asynchronous calls, as in the single-domain e2e: each member's
    # forcing staged on its upload stream, its state copied out on its
    # download stream while the next batched step runs; one sync at the end
    def e2e_body():
        for q in range(steps):
            it = first + q
            for m, fo in zip(models, fos):
                L.check(lib.pcom_gpu_set_forcing_async(m.handle, C.byref(fo)), "set_forcing_async")
            if day_of(it) != day_of(it - 1):
                b.den_prho()
            b.step_async(it)
            for m, st in zip(models, sts):
                L.check(lib.pcom_gpu_get_state_async(m.handle, C.byref(st)), "get_state_async")
        b.sync()
        for m in models:
            L.check(lib.pcom_gpu_sync(m.handle), "sync")  # the last states are in host memory

    t_e2e = timed(e2e_body)
    for m in models:
        L.check(lib.pcom_gpu_check_finite(m.handle), "watchdog")

    ms_b, ms_s, ms_e = t_batch / steps, t_seq / steps, t_e2e / steps
    member_desc = {"box": "128x64x20 1-degree box", "global1": "360x160x30 1-degree near-global"}[args.member_case]
    clocks = clk.summary()
    line = {
        "metric": "aggregate SYPD of a batched ensemble (sum over members), FP64 plain path",
        "value": round(n * sypd(ms_b / 1000.0), 2),
        "unit": "SYPD",
        "n_gpus": 1,
        "steps": steps,
        "warmup": warm + 3,
        "ms_per_step": round(ms_b, 4),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded k^-2 bathymetry, analytic wind and restoring; seeded T perturbations)",
        "config": {
            "workload": f"ensemble: {args.members} members of the {member_desc} case (T + N(0, 0.05 K), "
                        f"seeds 1..{args.members}) + {args.basins} basins 64x32..256x128 with 20-30 levels, "
                        "dtbc 3600 s, dtbt 60 s, one batched step per step",
            "members": n,
            "parallelism": "single GPU, batched (grid z = member; one persistent barotropic launch)",
            "l2": "inputs larger than L2: the members' state is tens of GB",
            "autotune": tune,
        },
        "sequential": {"ms_per_step": round(ms_s, 4), "value": round(n * sypd(ms_s / 1000.0), 2),
                       "speedup": round(ms_s / ms_b, 3)},
        "e2e": {"value": round(n * sypd(ms_e / 1000.0), 2), "unit": "SYPD", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": int(launches_batched),
        "clocks": {k: clocks[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "cpu_baseline": None,
    }
    b.close()
    for m in models:
        m.close()
    if print_line:
        print(json.dumps(line))
    return {k: line[k] for k in ("metric", "value", "unit", "steps", "ms_per_step", "config", "sequential", "e2e",
                                 "gpu_launches", "clocks")}


def cpu_baseline(nsteps: int):
    """The oracle (C++ restatement, OpenMP over all host threads) on a bounded
    sample of the same workload: nsteps steps of the 360x160x30 case."""
    from oracle import pyoracle
    from pcom_b200.synth import make_case

    threads = os.cpu_count() or 1
    o = pyoracle.Oracle(make_case(CASE), threads=threads)
    o.step(1)  # first step includes the AB3 start-up and the first den_prho
    t0 = time.perf_counter()
    o.step(nsteps)
    dt = (time.perf_counter() - t0) / nsteps
    return {"value": round(sypd(dt), 3), "unit": "SYPD", "cores": threads, "kind": "port",
            "sample": f"{nsteps} steps of the 360x160x30 case after 1 warm-up step, {dt:.3f} s/step"}


def run_reference(args):
    """The reference algorithm's CPU implementation (the oracle's C++
    restatement, OpenMP over all host threads) on the GPU arm's workload,
    --warmup and --steps: rank 0 only."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import pyoracle
    from pcom_b200.synth import make_case

    threads = os.cpu_count() or 1
    case = make_case(CASE)
    o = pyoracle.Oracle(case, threads=threads)
    warm = max(args.warmup, 3)
    o.step(warm)
    # ~0.5 s per step on a 16-core host: the default 48 steps take ~25 s
    nsteps = args.steps
    t0 = time.perf_counter()
    o.step(nsteps)
    dt = (time.perf_counter() - t0) / nsteps
    v = sypd(dt)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": round(v, 3), "unit": "SYPD", "n_gpus": world, "steps": nsteps, "warmup": warm,
        "ms_per_step": round(dt * 1000, 2), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded k^-2 bathymetry, analytic wind and restoring)",
        "config": workload_config(case, world),
        "timing": f"wall clock around {nsteps} steps of the CPU restatement on {threads} host threads",
        "cpu_baseline": {"value": round(v, 3), "unit": "SYPD", "cores": threads, "kind": "port",
                         "sample": f"{nsteps} steps of the 360x160x30 case after {warm} warm-up steps"},
        "e2e": {"value": round(v, 3), "unit": "SYPD", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_decomp(args):
    """One 1-degree domain split into row slabs, one per rank (pcom_b200.decomp:
    3-D subroutines on each rank's rows, halo rows over NCCL after each, the
    barotropic subcycle replicated from all-gathered 2-D inputs): SYPD of
    that one domain, timed on the device as the max over ranks."""
    import torch
    import torch.distributed as dist

    from pcom_b200 import decomp as D
    from pcom_b200.model import Model
    from pcom_b200.synth import make_case

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    case = make_case(CASE)
    m = Model(case)
    slab = D.slabs(case["glo_nj"], world, args.halo)[rank]
    e = D.GpuSlab(m, slab)
    links = D.DistLinks(e, world) if world > 1 else D.LocalLinks({0: e})
    drv = D.SlabDriver(links, args.halo)
    drv.run(max(args.warmup, 3))
    stream = e.stream
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = m.launch_count()
    with Clocks(local) as clk:
        e0.record(stream)
        drv.run(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    t = max_over_ranks(e0.elapsed_time(e1), world, "cuda")
    launches = m.launch_count() - launches0
    m.check_finite()
    ms = t / args.steps
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(sypd(ms / 1000.0), 2), "unit": "SYPD", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 4),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded k^-2 bathymetry, analytic wind and restoring)",
            "config": dict(workload_config(case, 1), parallelism=f"row slabs over {world} ranks, halo {args.halo}"),
            "slab_rows": [[s.lo, s.hi] for s in D.slabs(case["glo_nj"], world, args.halo)],
            "gpu_launches": int(launches),
            "clocks": {k: clk.summary()[k] for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        }
        print(json.dumps(line))
    m.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.decomp:
        run_decomp(a)
    elif a.workload == "ensemble":
        run_ensemble(a)
    else:
        run_ours(a)
