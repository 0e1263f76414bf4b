"""The oracle against the reference's own known-answer value and semantics (CPU)."""
import numpy as np
import pytest

from pcom_b200.synth import make_case

# notes.rst:20-26: Jackett & McDougall (1995) check value, and the residual
# the reference reports for its own den_rho (mod_den.f90:57-118)
KAT_T, KAT_S, KAT_P = 3.0, 35.5, 300e5
KAT_RHO = 1041.83267
KAT_RESIDUAL = 3.6e-7


def test_density_kat_r8(oracle_lib):
    # literals read as REAL(8): reproduces the documented residual
    rho = oracle_lib.den_rho(KAT_T, KAT_S, KAT_P, 1)
    assert abs(rho - KAT_RHO) <= KAT_RESIDUAL + 1e-8
    assert abs(rho - KAT_RHO) >= KAT_RESIDUAL - 1e-8


def test_density_kat_gfortran_literals(oracle_lib):
    # gfortran keeps the unsuffixed coefficients in REAL(4): a slightly
    # larger, but still small, departure from the check value
    rho = oracle_lib.den_rho(KAT_T, KAT_S, KAT_P, 0)
    assert abs(rho - KAT_RHO) < 1e-5
    assert rho != oracle_lib.den_rho(KAT_T, KAT_S, KAT_P, 1)


def test_literal_precision(oracle_lib):
    o = oracle_lib.Oracle(make_case("tiny"))
    f32 = lambda x: float(np.float32(x))
    assert o.const("g") == f32(9.8)
    assert o.const("gamma_b") == f32(0.2)
    assert o.const("c_tc") == float(np.float32(23.0) / np.float32(12))
    assert o.const("c_tp") == float(np.float32(-16.0) / np.float32(12))
    assert o.const("gamma_s") == float(np.float32(1.0) / np.float32(120 * 24 * 60 * 60))
    assert o.const("alpha_land") == float(np.float32(1.0) / np.float32(1000.0))
    r8 = dict(make_case("tiny"), r8=1)
    o8 = oracle_lib.Oracle(r8)
    assert o8.const("g") == 9.8 and o8.const("c_tc") == 23.0 / 12


def _area(o):
    a = o.const("a")
    return (a * o.field("rh1") * o.field("dx1x")) * (a * o.field("dx1y"))


@pytest.mark.parametrize("name", ["tiny", "tiny_bathy"])
def test_oracle_steps_finite_and_mass(oracle_lib, name):
    c = make_case(name)
    o = oracle_lib.Oracle(c)
    lev = o.field("lev_t")
    wet = lev > 0
    wet[:, 0] = wet[:, -1] = False  # x-halo columns are copies of interior ones
    area = _area(o)
    prh = o.field("prh_t")
    m0 = float(np.sum((o.field("chc") * prh * area)[wet]))
    o.step(4)
    for f in ("tc", "sc", "uc", "vc", "chc", "ubc", "wm", "am"):
        assert np.isfinite(o.field(f)).all(), f
    m1 = float(np.sum((o.field("chc") * prh * area)[wet]))
    # the barotropic continuity equation is in flux form: bottom-pressure mass is conserved
    assert abs(m1 - m0) <= 1e-13 * abs(m0)
    assert o.iter == 4


def test_calendar_and_daily_forcing(oracle_lib):
    c = make_case("tiny")
    o = oracle_lib.Oracle(c)
    o.step(25)  # crosses one day boundary at dtbc = 3600 s
    assert (o.const("year"), o.const("month"), o.const("day"), o.const("hour")) == (1, 1, 2, 1)


def test_oracle_threads_bit_identical(oracle_lib):
    # every parallel loop of the oracle is point-wise: one thread and four
    # threads give the same bits for every field (across a day boundary)
    c = make_case("tiny_bathy")
    names = ("tc", "sc", "tp", "sp", "uc", "vc", "up", "vp", "chc", "chp", "ubc", "vbc", "alpha", "adp", "wm",
             "am", "act", "acs", "acr", "acu", "acv", "acw", "mch", "mch2")
    out = []
    for threads in (1, 4):
        o = oracle_lib.Oracle(c, threads=threads)
        o.step(26)
        out.append({f: o.field(f).copy() for f in names})
        del o
    for f in names:
        assert out[0][f].tobytes() == out[1][f].tobytes(), f
