"""Row-slab decomposition driving the CUDA handles (needs a GPU).

Several ranks run in this process on one GPU, one handle each, their rows
moved by copies (pcom_b200.decomp.LocalLinks); no kernel of one rank waits
for another.  Every row outside a rank's window of the fields the step
splits is set to NaN at the start (except the first level of am, which the
barotropic subcycle reads on every row) and after each subroutine, so the ranks' own rows can only match the
single-domain run if the kernels stay inside their windows and the halo
refresh and the all-gather supply every row they read.  The result is held
bit-equal to the single-domain FP64 path (itself bit-equal to the oracle).
"""
import numpy as np
import pytest

from pcom_b200 import decomp as D
from pcom_b200.model import Model
from pcom_b200.synth import make_case
from decomp_util import assemble, poison
from parity_util import STATE_FIELDS

pytestmark = pytest.mark.gpu
HALO = 2


@pytest.mark.parametrize("name,ranks,steps", [("box", 2, 26), ("box", 3, 3), ("global1", 2, 3), ("global1", 8, 2)])
def test_gpu_slabs_bit_equal(name, ranks, steps):
    c = make_case(name)
    ref = Model(c)
    ref.run(steps)
    models = [Model(c) for _ in range(ranks)]
    eng = {s.rank: D.GpuSlab(models[s.rank], s) for s in D.slabs(c["glo_nj"], ranks, HALO)}
    links = D.LocalLinks(eng)
    for e in eng.values():
        poison(e, None)
    links.gather([("am", 1)])  # the subcycle reads level 1 of the initial am on every row
    drv = D.SlabDriver(links, HALO, after_phase=lambda ph: [poison(e, ph) for e in eng.values()])
    drv.run(steps)
    for f in STATE_FIELDS + ["acr"]:
        g = assemble(eng, f)
        r = ref.field(f).reshape(g.shape)
        bad = int(np.count_nonzero((g != r) & ~(np.isnan(g) & np.isnan(r))))
        assert bad == 0, f"{name} over {ranks} ranks: {f} differs at {bad} points after {steps} steps"
    for m in models + [ref]:
        m.close()
