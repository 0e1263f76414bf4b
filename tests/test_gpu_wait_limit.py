"""Failure detection on the device without a fault: the barotropic kernels'
grid-barrier waits are bounded in global time (pcom_gpu_set_wait_limit).
With a 1 ns limit a real step's barrier wait runs out, the kernel returns
early, the host reads PCOM_ERR_TIMEOUT, and the context stays usable: the
same handle runs further steps, and a fresh model in the same process is
bit-equal to one that never saw a timeout."""
import pytest

from pcom_b200 import _lib as L
from pcom_b200.model import Model
from pcom_b200.synth import make_case
from parity_util import STATE_FIELDS, compare

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form,mixed", [(1, False), (2, False), (1, True)])
def test_barrier_wait_runs_out_and_handle_recovers(form, mixed):
    c = make_case("box")  # 128 x 64: many CTAs, so barrier waits happen
    flags = L.PCOM_PREC_MIXED if mixed else L.PCOM_PREC_FP64
    ref = Model(c, flags=flags)
    L.check(ref.lib.pcom_gpu_set_trop_kernel(ref.handle, form), "set_trop_kernel")
    ref.run(3)

    m = Model(c, flags=flags)
    lib = m.lib
    L.check(lib.pcom_gpu_set_trop_kernel(m.handle, form), "set_trop_kernel")
    L.check(lib.pcom_gpu_set_wait_limit(m.handle, 1e-9), "set_wait_limit")
    with pytest.raises(L.PcomError) as ei:
        m.run(1)
    assert "TIMEOUT" in str(ei.value) or "gave up" in str(ei.value)
    # the same handle keeps working once the limit is back to normal
    L.check(lib.pcom_gpu_set_wait_limit(m.handle, 2.0), "set_wait_limit")
    m.run(2)
    m.close()

    # the context is intact: a fresh model reproduces the undisturbed run
    f = Model(c, flags=flags)
    L.check(f.lib.pcom_gpu_set_trop_kernel(f.handle, form), "set_trop_kernel")
    f.run(3)
    for name in STATE_FIELDS:
        r = compare(f.field(name), ref.field(name))
        assert r["unequal"] == 0, f"{name} differs after a timeout in the same process"
    f.close()
    ref.close()


def test_wait_limit_rejects_bad_values():
    m = Model(make_case("tiny"))
    for bad in (-1.0, float("nan"), 1e7):
        with pytest.raises(L.PcomError):
            L.check(m.lib.pcom_gpu_set_wait_limit(m.handle, bad), "set_wait_limit")
    m.close()
