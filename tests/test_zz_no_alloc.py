"""pcom_gpu_trop_noalloc, the allocation-free barotropic subcycle (needs a GPU).

Callers that own all of the GPU's memory and hand it out from their own pool
(a coupled-model driver with one pre-sized pool, a serving stack with its own
caching allocator) cannot let the library cudaMalloc its scratch; this entry
point takes only the caller's inputs and outputs and keeps its scratch in a
fixed array inside the library.  The test drives it through the C ABI on
arrays the test owns and checks two calls in a row against the handle-based
int_trop (pcom_gpu_phase 3) on the same inputs, on a small domain and on the
1-degree 362 x 162 domain the fixed scratch is sized for.
"""
import ctypes as C

import numpy as np
import pytest

from pcom_b200 import _lib as L
from pcom_b200.model import Model
from pcom_b200.synth import make_case
from parity_util import compare

pytestmark = pytest.mark.gpu
TOL = 1e-12
STATE = ["chc", "chp", "mch", "mch2", "ubc", "vbc", "ubp", "vbp", "acch"]


@pytest.mark.parametrize("name", ["tiny_bathy", "global1"])
def test_trop_noalloc_matches_handle_path(name):
    import torch

    case = make_case(name)
    m = Model(case)
    m.set_forcing(m.int_bnd())
    m.den_prho()
    for ph in ("den_alpha", "int_pgra", "int_readyc"):
        m.phase(ph, 1)
    st = m.static()
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    keep = {}
    io = L.TropIO()
    io.glo_ni, io.glo_nj = case["glo_ni"], case["glo_nj"]
    io.dtbt, io.dtbc, io.flags = case["dtbt"], case["dtbc"], 0

    def put(name, arr):
        t = dev(arr)
        keep[name] = t
        return t.data_ptr()

    io.lev_t = put("lev_t", st["lev_t"].astype(np.int32))
    io.lev_u = put("lev_u", st["lev_u"].astype(np.int32))
    for f in ("prh_t", "prh_u", "cor", "graphihx", "graphihy"):
        setattr(io, f, put(f, st[f]))
    io.am1 = put("am1", m.field("am")[0])
    for g in range(4):
        io.dxx[g] = put(f"dxx{g}", st[f"dx{g + 1}x"])
        io.dxy[g] = put(f"dxy{g}", st[f"dx{g + 1}y"])
        io.rh[g] = put(f"rh{g}", st[f"rh{g + 1}"])
    io.ut = put("ut", m.field("ut"))
    io.vt = put("vt", m.field("vt"))
    for q, s in enumerate(("xn", "xs", "ye", "yw")):
        io.bphi[q] = put("bphi" + s, m.field("bphi_" + s))
        io.bgraphi[q] = put("bgraphi" + s, m.field("bgraphi_" + s))
    for f in STATE:
        setattr(io, f, put(f, m.field(f)))

    stream = torch.cuda.current_stream()
    for call in (1, 2):
        m.phase("int_trop", 1)  # the handle-based subcycle
        rc = m.lib.pcom_gpu_trop_noalloc(C.byref(io), C.c_void_p(stream.cuda_stream))
        L.check(rc, "pcom_gpu_trop_noalloc")
        torch.cuda.synchronize()
        for f in STATE:
            r = compare(keep[f].cpu().numpy(), m.field(f))
            assert r["rel"] <= TOL, f"{name} call {call}: {f} rel {r['rel']:.3e}"
    m.close()


def test_trop_noalloc_rejects_oversize():
    lib = L.load()
    io = L.TropIO()
    io.glo_ni, io.glo_nj, io.dtbt, io.dtbc = 2000, 10, 60, 3600
    rc = lib.pcom_gpu_trop_noalloc(C.byref(io), None)
    assert rc == 1
    buf = C.create_string_buffer(256)
    lib.pcom_gpu_last_error(buf, 256)
    assert b"PCOM_NOALLOC_MAX" in buf.value
