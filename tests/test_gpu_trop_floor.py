"""The barotropic subcycle's latency floor (pcom_gpu_trop_floor): the
resident kernel's synchronisation skeleton, which the bench reports beside
int_trop's time per substep.  It must leave the model untouched (the steps
that follow are bit-equal to a handle that never ran it), take less time
than the kernel itself, and be refused where the handle runs another form
of the subcycle."""
import ctypes as C

import numpy as np
import pytest

from pcom_b200 import _lib as L
from pcom_b200.model import Model
from pcom_b200.synth import make_case
from parity_util import STATE_FIELDS

pytestmark = pytest.mark.gpu


def test_floor_leaves_state_and_bounds_int_trop():
    c = make_case("global1")
    a, b = Model(c), Model(c)
    a.run(2)
    b.run(2)
    t = C.c_double(0.0)
    for _ in range(3):
        L.check(a.lib.pcom_gpu_trop_floor(a.handle, C.byref(t)), "trop_floor")
    floor_ms = t.value
    a.run(2)
    b.run(2)
    for f in STATE_FIELDS:
        assert np.array_equal(a.field(f), b.field(f)), f
    a.profile(True)
    a.run(4)
    launches, ms = a.profile_read()["int_trop"]
    a.profile(False)
    trop_ms = ms / launches
    print(f"\nint_trop {trop_ms * 1e3:.1f} us per launch, floor {floor_ms * 1e3:.1f} us")
    assert 0.0 < floor_ms < trop_ms
    a.close()
    b.close()


def test_floor_refused_on_the_mixed_handle():
    m = Model(make_case("global1"), flags=L.PCOM_PREC_MIXED)
    t = C.c_double(0.0)
    assert m.lib.pcom_gpu_trop_floor(m.handle, C.byref(t)) == 3  # PCOM_ERR_STATE
    m.close()
