"""The product's host driver setup against the oracle's restatement (CPU)."""
import numpy as np
import pytest

from pcom_b200 import _lib as L
from pcom_b200.model import Model
from pcom_b200.synth import make_case


@pytest.mark.parametrize("name,r8", [("tiny", 0), ("tiny_bathy", 0), ("box", 0), ("global1", 0), ("tiny_bathy", 1)])
def test_setup_bit_exact(oracle_lib, name, r8):
    c = dict(make_case(name), r8=r8)
    m = Model(c, flags=L.PCOM_MODEL_HOST_ONLY)
    st = m.static()
    o = oracle_lib.Oracle(c)
    n = 0
    for k, v in st.items():
        try:
            ref = np.asarray(o.field(k))
        except KeyError:
            continue
        ref = ref.reshape(v.shape)
        assert np.array_equal(ref, v), k
        n += 1
    assert n >= 35
    m.close()


def test_int_bnd_matches(oracle_lib):
    c = make_case("box")
    m = Model(c, flags=L.PCOM_MODEL_HOST_ONLY)
    o = oracle_lib.Oracle(c)
    o.phase("int_bnd")
    f = m.int_bnd()
    for k, name in (("taux", "bnd_taux"), ("t", "bnd_t"), ("s", "bnd_s"), ("pa", "bnd_pa")):
        assert np.array_equal(f[k], o.field(name)), k
