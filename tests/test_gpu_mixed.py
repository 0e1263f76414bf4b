"""The mixed-precision path (PCOM_PREC_MIXED) against the FP64 path.

The FP64 path is bit-equal to the oracle (test_gpu_parity), so it stands in
for the oracle here.  The mixed path stores 3-D fields in FP32 and computes
the stencils in FP32, so it is checked against stated error bounds per
prognostic field (relative RMS over wet points, normalised by the field's
RMS), and for exact host round trips of its conversions.
"""
import numpy as np
import pytest

from pcom_b200 import _lib as L
from pcom_b200.model import Model
from pcom_b200.synth import make_case

pytestmark = pytest.mark.gpu

FIELDS = ("tc", "sc", "uc", "vc", "chc", "ubc", "vbc")
# relative RMS error bounds after the stated number of steps
# (measured on B200: after 24 steps of the 1-degree case tc 1.6e-7, uc 3.7e-5,
# vc 3.0e-5, chc 3.0e-10, ubc 1.5e-5, vbc 1.6e-5; sc stays exact)
BOUNDS = {"tc": 2e-6, "sc": 1e-7, "uc": 5e-4, "vc": 5e-4, "chc": 1e-8, "ubc": 5e-4, "vbc": 5e-4}


def rel_rms(a, b, mask):
    d = (a - b)[mask]
    r = b[mask]
    return float(np.sqrt(np.mean(d * d)) / max(np.sqrt(np.mean(r * r)), 1e-30))


def masks(m):
    st = m.static()
    k = np.arange(1, m.nk + 1)[:, None, None]
    return {"t3": st["lev_t"][None] >= k, "u3": st["lev_u"][None] >= k,
            "t2": st["lev_t"] >= 1, "u2": st["lev_u"] >= 1}


def errors(mm, md):
    mk = masks(md)
    which = {"tc": "t3", "sc": "t3", "uc": "u3", "vc": "u3", "chc": "t2", "ubc": "u2", "vbc": "u2"}
    return {f: rel_rms(mm.field(f), md.field(f), mk[which[f]]) for f in FIELDS}


@pytest.mark.parametrize("name,steps", [("tiny_bathy", 1), ("tiny_bathy", 30), ("global1", 24)])
def test_mixed_within_bounds(name, steps):
    c = make_case(name)
    md = Model(c)
    mm = Model(c, flags=L.PCOM_PREC_MIXED)
    md.run(steps)
    mm.run(steps)
    mm.check_finite()
    err = errors(mm, md)
    print(f"\n{name} after {steps} steps, relative RMS error of the mixed path:",
          {k: f"{v:.2e}" for k, v in err.items()})
    for f, e in err.items():
        assert e <= BOUNDS[f], f"{name}: {f} rel RMS {e:.3e} > {BOUNDS[f]:.0e}"
    md.close()
    mm.close()


def test_mixed_state_round_trip():
    """set_state -> get_field gives the FP32 rounding of the input; alpha and
    adp travel as anomalies from the reference profile, so they come back to
    the FP32 precision of the anomaly, far below FP32 of the full value."""
    c = make_case("tiny_bathy")
    md = Model(c)
    md.run(2)
    mm = Model(c, flags=L.PCOM_PREC_MIXED)
    vals = {f: md.field(f) for f in ("tc", "uc", "alpha", "adp", "wm")}
    mm.set_state(**vals)
    for f, v in vals.items():
        back = mm.field(f)
        if f in ("alpha", "adp"):
            # FP32 of the anomaly (|alpha - alpha_r| < 5e-5 here, land
            # included), not of the full value (2^-23 * 1e-3 ~ 1.2e-10)
            tol = 5e-9 * np.abs(v).max()
        else:
            tol = 2 ** -23 * np.abs(v).max()
        assert np.abs(back - v).max() <= tol, f
    md.close()
    mm.close()


def test_mixed_over_30_days():
    """30 model days (720 steps, daily forcing and den_prho) of the 128x64x20
    box: the mixed path stays within its bounds (measured on B200: tc 4.3e-7,
    uc 3.7e-5, vc 2.5e-5, chc 3.4e-11, ubc 5.7e-6, vbc 2.4e-6, heat sum
    9.0e-9), while an FP64 run from a temperature perturbed by N(0, 1e-10 K)
    stays within 1e-8 of the unperturbed one, so the model does not amplify
    perturbations over this horizon and the difference is the precision's."""
    from pcom_b200.precision_report import run

    rep = run("box", [720])
    e = rep["checkpoints"][-1]
    bounds = {"tc": 2e-6, "sc": 1e-12, "uc": 2e-4, "vc": 2e-4, "chc": 1e-9, "ubc": 1e-4, "vbc": 1e-4}
    for f, b in bounds.items():
        r = e["mixed"]["fields"][f]
        assert r["finite"] and r["rel_rms"] <= b, f"mixed {f} rel RMS {r['rel_rms']:.3e} > {b:.0e}"
        assert e["control"]["fields"][f]["rel_rms"] <= 1e-8, f
    assert e["mixed"]["global_sums"]["heat"] <= 1e-7
    assert e["mixed"]["global_sums"]["volume"] == 0.0


@pytest.mark.parametrize("flags", [L.PCOM_PREC_FP64, L.PCOM_PREC_MIXED])
def test_global_sums(flags):
    c = make_case("tiny_bathy")
    m = Model(c, flags=flags)
    m.run(3)
    vol, ht, sl = m.global_sums()
    st = m.static()
    a = float(np.float32(6370e3))  # the earth radius as the model's REAL(4) literal
    area = (a * st["rh1"] * st["dx1x"]) * (a * st["dx1y"])
    k = np.arange(1, m.nk + 1)[:, None, None]
    wet = st["lev_t"][None] >= k
    wet[:, 0, :] = False
    wet[:, -1, :] = False
    wet[:, :, 0] = False
    wet[:, :, -1] = False
    dv = area[None] * st["dz2"][:, None, None] * wet
    tc, sc = m.field("tc"), m.field("sc")
    assert vol == pytest.approx(dv.sum(), rel=1e-12)
    assert ht == pytest.approx((tc * dv).sum(), rel=1e-12)
    assert sl == pytest.approx((sc * dv).sum(), rel=1e-12)
    m.close()


def test_mixed_multi_tile_within_bounds():
    """720 x 320 x 30 is too large for the resident kernel, so the mixed
    handle runs the multi-tile mixed kernel (FP32 coefficients and
    velocities between substeps); after 24 steps its error against the FP64
    path is within the mixed bounds."""
    c = make_case("global05")
    md = Model(c)
    mm = Model(c, flags=L.PCOM_PREC_MIXED)
    md.run(24)
    mm.run(24)
    mm.check_finite()
    err = errors(mm, md)
    print("\nglobal05 mixed (multi-tile) after 24 steps:", {k: f"{v:.2e}" for k, v in err.items()})
    for f, e in err.items():
        assert e <= BOUNDS[f], f"{f} rel RMS {e:.3e} > {BOUNDS[f]:.0e}"
    md.close()
    mm.close()


def test_mixed_multi_tile_matches_resident():
    """On the 1-degree domain the mixed handle's two barotropic kernels (the
    resident one and the multi-tile one, forced) do the same FP32/FP64
    arithmetic, in code compiled apart (FMA contraction may differ): after 6
    steps they agree within half the mixed bounds."""
    c = make_case("global1")
    ms = [Model(c, flags=L.PCOM_PREC_MIXED) for _ in range(2)]
    L.check(ms[1].lib.pcom_gpu_set_trop_kernel(ms[1].handle, 2), "set_trop_kernel")
    for m in ms:
        m.run(6)
    err = errors(ms[1], ms[0])
    print("\nglobal1 mixed multi-tile vs resident after 6 steps:", {k: f"{v:.2e}" for k, v in err.items()})
    for f, e in err.items():
        assert e <= 0.5 * BOUNDS[f], f"{f} rel RMS {e:.3e}"
    for m in ms:
        m.close()
