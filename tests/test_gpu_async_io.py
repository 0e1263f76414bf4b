"""Asynchronous host transfers (pcom_gpu_set_forcing_async,
pcom_gpu_get_state_async): a run that stages each step's forcing and copies
each step's state out on the copy stream, synchronising once at the end,
must produce the same per-step outputs and final state, bit for bit, as the
same run through the synchronous calls."""
import ctypes as C

import numpy as np
import pytest

from pcom_b200 import _lib as L
from pcom_b200.model import Model
from pcom_b200.synth import make_case
from parity_util import STATE_FIELDS, acr_mask, compare

pytestmark = pytest.mark.gpu

OUT = ("chc", "ubc", "vbc", "tc")


def _forcings(m, nsteps):
    """A different forcing per step (taux and pa scaled), as host arrays."""
    base = m.int_bnd()
    fs = []
    for q in range(nsteps):
        f = {k: np.ascontiguousarray(base[k], dtype=np.float64).copy() for k in ("taux", "tauy", "t", "s", "pa", "fw")}
        f["taux"] *= 1.0 + 0.02 * q
        f["pa"] = f["pa"] + 10.0 * q
        fs.append(f)
    return fs


def _fo(f):
    p = lambda a: a.ctypes.data_as(L.dbl_p)
    return L.Forcing(p(f["taux"]), p(f["tauy"]), p(f["t"]), p(f["s"]), p(f["pa"]), p(f["fw"]))


def _state_req(m, bufs):
    st = L.State(*[None] * len(L.STATE_FIELDS))
    for name in OUT:
        setattr(st, name, bufs[name].ctypes.data_as(L.dbl_p))
    return st


@pytest.mark.parametrize("name,mixed", [("tiny_bathy", False), ("box", False), ("tiny_bathy", True)])
def test_async_transfers_equal_sync(name, mixed):
    c = make_case(name)
    flags = L.PCOM_PREC_MIXED if mixed else L.PCOM_PREC_FP64
    a, b = Model(c, flags=flags), Model(c, flags=flags)
    lib = a.lib
    nsteps = 7
    fs = _forcings(a, nsteps)
    sizes = {k: a.field(k).size for k in OUT}
    out_sync = [{k: np.zeros(sizes[k]) for k in OUT} for _ in range(nsteps)]
    out_async = [{k: np.full(sizes[k], np.nan) for k in OUT} for _ in range(nsteps)]
    for m in (a, b):
        L.check(lib.pcom_gpu_den_prho(m.handle), "den_prho")
    fo = [_fo(f) for f in fs]
    req_s = [_state_req(a, o) for o in out_sync]
    req_a = [_state_req(b, o) for o in out_async]
    for q in range(nsteps):
        L.check(lib.pcom_gpu_set_forcing(a.handle, C.byref(fo[q])), "set_forcing")
        L.check(lib.pcom_gpu_step(a.handle, q + 1), "step")
        L.check(lib.pcom_gpu_get_state(a.handle, C.byref(req_s[q])), "get_state")
    for q in range(nsteps):
        L.check(lib.pcom_gpu_set_forcing_async(b.handle, C.byref(fo[q])), "set_forcing_async")
        L.check(lib.pcom_gpu_step_async(b.handle, q + 1), "step_async")
        L.check(lib.pcom_gpu_get_state_async(b.handle, C.byref(req_a[q])), "get_state_async")
    L.check(lib.pcom_gpu_sync(b.handle), "sync")
    for q in range(nsteps):
        for k in OUT:
            assert np.array_equal(out_sync[q][k], out_async[q][k]), f"step {q + 1}: {k} differs"
    # the steps did see different forcing
    assert not np.array_equal(out_sync[0]["ubc"], out_sync[-1]["ubc"])
    lev_t = a.static()["lev_t"]
    for f in STATE_FIELDS + ["acr"]:
        mask = acr_mask(lev_t, c["nk"]) if f == "acr" else None
        r = compare(b.field(f), a.field(f), mask)
        assert r["unequal"] == 0, f"{name}: {f} differs at {r['unequal']} points"
    a.close()
    b.close()


def test_async_forcing_requires_all_fields():
    m = Model(make_case("tiny"))
    f = _forcings(m, 1)[0]
    fo = _fo(f)
    fo.pa = None
    with pytest.raises(L.PcomError):
        L.check(m.lib.pcom_gpu_set_forcing_async(m.handle, C.byref(fo)), "set_forcing_async")
    m.close()


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_async_transfers_equal_sync(graphs):
    """The same with a batch: every member's forcing staged with
    set_forcing_async and its state copied out with get_state_async around
    each batched step (CUDA graphs on and off) equals the batch driven
    through the synchronous calls, per step and at the end."""
    from pcom_b200.model import Batch
    from pcom_b200.synth import perturb

    base = make_case("tiny_bathy")
    cases = [base, perturb(base, 1), make_case("tiny")]
    nsteps = 7
    runs = {}
    for mode in ("sync", "async"):
        ms = [Model(c) for c in cases]
        lib = ms[0].lib
        bt = Batch(ms, graphs=graphs)
        fs = [_forcings(m, nsteps) for m in ms]
        fo = [[_fo(f) for f in fm] for fm in fs]
        outs = [[{k: np.full(m.field(k).size, np.nan) for k in OUT} for _ in range(nsteps)] for m in ms]
        reqs = [[_state_req(m, o) for o in om] for m, om in zip(ms, outs)]
        bt.den_prho()
        for q in range(nsteps):
            for mi, m in enumerate(ms):
                if mode == "sync":
                    L.check(lib.pcom_gpu_set_forcing(m.handle, C.byref(fo[mi][q])), "set_forcing")
                else:
                    L.check(lib.pcom_gpu_set_forcing_async(m.handle, C.byref(fo[mi][q])), "set_forcing_async")
            bt.step_async(q + 1)
            if mode == "sync":
                bt.sync()
            for mi, m in enumerate(ms):
                if mode == "sync":
                    L.check(lib.pcom_gpu_get_state(m.handle, C.byref(reqs[mi][q])), "get_state")
                else:
                    L.check(lib.pcom_gpu_get_state_async(m.handle, C.byref(reqs[mi][q])), "get_state_async")
        bt.sync()
        for m in ms:
            L.check(lib.pcom_gpu_sync(m.handle), "sync")
        runs[mode] = (ms, outs, bt)
    (ma, oa, ba), (mb, ob, bb) = runs["sync"], runs["async"]
    for mi in range(len(cases)):
        for q in range(nsteps):
            for k in OUT:
                assert np.array_equal(oa[mi][q][k], ob[mi][q][k]), f"member {mi} step {q + 1}: {k} differs"
        for f in STATE_FIELDS:
            assert np.array_equal(ma[mi].field(f), mb[mi].field(f)), f"member {mi}: {f} differs"
    assert not np.array_equal(oa[0][0]["ubc"], oa[0][-1]["ubc"])
    for bt in (ba, bb):
        bt.close()
    for m in ma + mb:
        m.close()
