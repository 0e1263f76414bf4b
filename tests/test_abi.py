"""The C-ABI library loads and exports every symbol include/*.h declares (CPU)."""
import os
import re

from pcom_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DECL = re.compile(r"^\s*(?:int|int64_t|pcom_handle\s*\*)\s*\**\s*(pcom_\w+)\s*\(", re.M)


def declared():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", h)).read()
            names += DECL.findall(txt)
    return names


def test_every_declared_symbol_is_exported():
    lib = L.load()
    names = declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n


def test_bindings_cover_declarations():
    assert set(declared()) == set(L.SIGNATURES)


def test_errors_without_device():
    import ctypes as C
    lib = L.load()
    h = C.c_void_p()
    d = L.Dims(4, 4, 3, 99, 6, 60, 3600, 0, 0)  # ni != glo_ni + 2
    assert lib.pcom_gpu_create(C.byref(d), C.byref(h)) == 1
    buf = C.create_string_buffer(256)
    lib.pcom_gpu_last_error(buf, 256)
    assert b"glo_ni + 2" in buf.value
    assert lib.pcom_gpu_step(None, 1) == 1
