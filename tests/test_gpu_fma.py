"""Handles created with PCOM_FMA (the step kernels built with a*b+c contracted
into fused multiply-adds) against the oracle (needs a GPU).

Contraction rounds once where the reference's x86-64 build rounds twice, so
the FMA build is not bit-equal to the oracle.  The tolerance for the FP64
path is 1e-12 relative per field after one step (max |gpu - oracle| over max
|oracle|, every state field); the drift over 30 model days of the box is held
to the bounds below, and the mixed path built with FMA to the mixed path's
own error bounds against the FP64 path.
"""
import numpy as np
import pytest

from pcom_b200 import _lib as L
from pcom_b200.model import Model
from pcom_b200.synth import make_case
from parity_util import STATE_FIELDS, acr_mask, compare

pytestmark = pytest.mark.gpu
TOL_STEP = 1e-12
# 30 days (720 steps) of the 128 x 64 x 20 box: max relative difference per
# field against the oracle
TOL_30_DAYS = 1e-6


def _rel(m, o, fields, lev_t, nk):
    out = {}
    for f in fields:
        mask = acr_mask(lev_t, nk) if f == "acr" else None
        out[f] = compare(m.field(f), o.field(f), mask)["rel"]
    return out


@pytest.mark.parametrize("name", ["tiny_bathy", "box", "global1"])
def test_fma_one_step_within_tolerance(oracle_lib, name):
    c = make_case(name)
    o = oracle_lib.Oracle(c)
    m = Model(c, flags=L.PCOM_FMA)
    lev_t = m.static()["lev_t"]
    for steps in (1, 2):
        m.run(1)
        o.step(1)
        rel = _rel(m, o, STATE_FIELDS + ["acr"], lev_t, c["nk"])
        worst = max(rel, key=rel.get)
        print(f"\n{name} FMA after {steps} step(s): worst {worst} {rel[worst]:.2e}")
        if steps == 1:
            for f, r in rel.items():
                assert r <= TOL_STEP, f"{name}: {f} rel {r:.3e} after one step"
    m.close()


def test_fma_drift_over_30_days(oracle_lib):
    c = make_case("box")
    o = oracle_lib.Oracle(c)
    m = Model(c, flags=L.PCOM_FMA)
    lev_t = m.static()["lev_t"]
    m.run(720)
    o.step(720)
    rel = _rel(m, o, STATE_FIELDS + ["acr"], lev_t, c["nk"])
    print("\nbox FMA after 720 steps, max relative difference per field:",
          {k: f"{v:.1e}" for k, v in sorted(rel.items(), key=lambda kv: -kv[1])[:8]})
    for f, r in rel.items():
        assert r <= TOL_30_DAYS, f"{f} rel {r:.3e} after 720 steps"
    m.check_finite()
    m.close()


def test_fma_batch_matches_oracle(oracle_lib):
    """A batch of FMA handles (batched kernels, group barotropic launch)."""
    from pcom_b200.model import Batch

    cases = [make_case("tiny_bathy"), make_case("tiny"), make_case("box")]
    ms = [Model(c, flags=L.PCOM_FMA) for c in cases]
    b = Batch(ms)
    b.run(3)
    for c, m in zip(cases, ms):
        o = oracle_lib.Oracle(c)
        o.step(3)
        rel = _rel(m, o, STATE_FIELDS, m.static()["lev_t"], c["nk"])
        for f, r in rel.items():
            assert r <= 1e-11, f"{c['name']}: {f} rel {r:.3e} after 3 batched steps"
    b.close()
    for m in ms:
        m.close()
    # members of one batch share the build
    with pytest.raises(L.PcomError, match="PCOM_FMA"):
        Batch([Model(cases[0], flags=L.PCOM_FMA), Model(cases[1])])


def test_fma_mixed_within_bounds():
    """The mixed path built with FMA keeps its error bounds against FP64."""
    from test_gpu_mixed import BOUNDS, errors

    c = make_case("global1")
    md = Model(c)
    mm = Model(c, flags=L.PCOM_PREC_MIXED | L.PCOM_FMA)
    md.run(24)
    mm.run(24)
    mm.check_finite()
    err = errors(mm, md)
    print("\nglobal1 mixed+FMA after 24 steps:", {k: f"{v:.2e}" for k, v in err.items()})
    for f, e in err.items():
        assert e <= BOUNDS[f], f"{f} rel RMS {e:.3e} > {BOUNDS[f]:.0e}"
    md.close()
    mm.close()
