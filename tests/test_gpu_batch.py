"""Batched stepping (pcom_gpu_batch_*): ensemble members and basins of uneven
size advanced together must end bit-equal to the same cases advanced one at
a time through the single-domain path (which the oracle tests pin to the
reference).  Covers the batched kernels (grid z = member), the batched
barotropic launch over the work list of all members' tiles, CUDA-graph
replay after the AB3 start-up steps, a day change (int_bnd + den_prho), and
the tile autotuner."""
import numpy as np
import pytest

from pcom_b200.model import Batch, Model
from pcom_b200.synth import make_case, perturb
from parity_util import STATE_FIELDS, acr_mask, compare

pytestmark = pytest.mark.gpu


def _members():
    base = make_case("tiny_bathy")
    return [base, perturb(base, 1), perturb(base, 2), make_case("tiny"),
            make_case("basin", glo_ni=40, glo_nj=20, nk=8)]


def _assert_equal(mb: Model, ms: Model, label: str):
    lev_t = mb.static()["lev_t"]
    for f in STATE_FIELDS + ["acr"]:
        a, b = mb.field(f), ms.field(f)
        mask = acr_mask(lev_t, mb.nk) if f == "acr" else None
        r = compare(a, b, mask)
        assert r["unequal"] == 0, f"{label}: {f} differs at {r['unequal']} points (rel {r['rel']:.3e})"


@pytest.mark.parametrize("graphs", [True, False])
def test_batch_matches_sequential(graphs):
    cases = _members()
    steps = 26  # AB3 start-up, graph replays over every ring phase, one day change
    seq = []
    for c in cases:
        m = Model(c)
        m.run(steps)
        seq.append(m)
    bm = [Model(c) for c in cases]
    b = Batch(bm, graphs=graphs)
    b.run(steps)
    for q, (x, y) in enumerate(zip(bm, seq)):
        assert x.iter == y.iter == steps
        _assert_equal(x, y, f"member {q} ({cases[q]['name']})")
        acc = x.accum()
        assert acc["n_ts"] == acc["n_ch"] == steps
    b.close()
    for m in bm + seq:
        m.close()


def test_batch_packing_and_multitile_fallback():
    """16x8 tiles with at most 40 tiles per co-resident group: the small
    members are packed into groups (first-fit decreasing) and the box (72
    tiles) falls back to the multi-tile kernel; results stay bit-equal."""
    cases = _members() + [make_case("box")]
    steps = 5
    seq = []
    for c in cases:
        m = Model(c)
        m.run(steps)
        seq.append(m)
    bm = [Model(c) for c in cases]
    b = Batch(bm)
    b.set_tiles(16, 8, max_resident=40)
    b.run(steps)
    for q, (x, y) in enumerate(zip(bm, seq)):
        _assert_equal(x, y, f"member {q} ({cases[q]['name']}) with packed groups")
    b.set_tiles(16, 8, max_resident=1)  # every member on the multi-tile kernel
    b.run(2)
    for m in seq:
        m.run(2)
    for q, (x, y) in enumerate(zip(bm, seq)):
        _assert_equal(x, y, f"member {q} ({cases[q]['name']}) on the multi-tile kernel")
    b.close()
    for m in bm + seq:
        m.close()


def test_batch_autotune_keeps_results():
    cases = _members()[:3] + [make_case("box")]
    seq = []
    for c in cases:
        m = Model(c)
        m.run(5)
        seq.append(m)
    bm = [Model(c) for c in cases]
    b = Batch(bm)
    b.run(3)
    report = b.autotune()  # trials restore the state they change
    assert "->" in report
    b.run(2)
    for q, (x, y) in enumerate(zip(bm, seq)):
        _assert_equal(x, y, f"member {q} after autotune ({report})")
    b.close()
    for m in bm + seq:
        m.close()


def test_batch_on_caller_stream():
    """Members on the caller's (legacy default) stream: the batch captures on
    its own stream and joins the members' streams by events."""
    cases = _members()[:2]
    seq = []
    for c in cases:
        m = Model(c)
        m.run(6)
        seq.append(m)
    bm = [Model(c) for c in cases]
    for m in bm:
        m.set_stream(0)
    b = Batch(bm)
    b.run(6)
    for q, (x, y) in enumerate(zip(bm, seq)):
        _assert_equal(x, y, f"member {q} on the default stream")
    b.close()
    for m in bm + seq:
        m.close()


def test_batch_rejects_mixed_time_steps():
    from pcom_b200 import _lib as L

    a = Model(make_case("tiny"))
    c = make_case("tiny")
    c["dtbc"] = 1800
    d = Model(c)
    with pytest.raises(L.PcomError):
        Batch([a, d])
    a.close()
    d.close()
