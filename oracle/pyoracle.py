"""ctypes bridge to the CPU oracle (test infrastructure only).

Used by tests/, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
bench.py to drive the C++ restatement of PCOM in oracle/pcom_oracle.cpp.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libpcom_oracle.so")
_lib = None


class _Inputs(C.Structure):
    _fields_ = [
        ("glo_ni", C.c_int32), ("glo_nj", C.c_int32), ("nk", C.c_int32),
        ("dtbt", C.c_int32), ("dtbc", C.c_int32), ("r8", C.c_int32), ("rst", C.c_int32),
        ("year", C.c_int32), ("month", C.c_int32), ("day", C.c_int32), ("hour", C.c_int32),
        ("lon", C.c_void_p), ("lat", C.c_void_p), ("z", C.c_void_p),
        ("tmn", C.c_void_p), ("smn", C.c_void_p), ("itn", C.c_void_p),
        ("pt", C.c_void_p), ("sa", C.c_void_p),
        ("taux", C.c_void_p), ("tauy", C.c_void_p), ("bct", C.c_void_p),
        ("bcs", C.c_void_p), ("pa", C.c_void_p), ("fw", C.c_void_p),
        ("vmix", C.c_void_p),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.POINTER(_Inputs)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p]
        L.orc_phase.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_iter.argtypes = [C.c_void_p, C.c_int64]
        L.orc_get_iter.argtypes = [C.c_void_p]
        L.orc_get_iter.restype = C.c_int64
        L.orc_field.restype = C.POINTER(C.c_double)
        L.orc_field.argtypes = [C.c_void_p, C.c_char_p] + [C.POINTER(C.c_int32)] * 3
        L.orc_ifield.restype = C.POINTER(C.c_int32)
        L.orc_ifield.argtypes = [C.c_void_p, C.c_char_p] + [C.POINTER(C.c_int32)] * 3
        L.orc_const.restype = C.c_double
        L.orc_const.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_den_rho.restype = C.c_double
        L.orc_den_rho.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int32]
        L.orc_set_threads.argtypes = [C.c_int]
        _lib = L
    return _lib


def den_rho(t: float, s: float, p0: float, r8: int = 0) -> float:
    return lib().orc_den_rho(t, s, p0, r8)


PHASES = {"int_bnd": 0, "den_prho": 1, "den_alpha": 2, "int_pgra": 3, "int_readyc": 4,
          "int_trop": 5, "int_clin": 6, "int_ssh": 7, "int_ts": 8, "advance": 9}


class Oracle:
    """One single-domain PCOM model instance, set up from a synthetic case."""

    def __init__(self, case: dict, threads: int | None = None):
        L = lib()
        if threads:
            L.orc_set_threads(int(threads))
        self._keep = []

        def p(a, dt=np.float64):
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a.ctypes.data

        y, m, d, h = case.get("bdate", (1, 1, 1, 0))
        inp = _Inputs(case["glo_ni"], case["glo_nj"], case["nk"], case["dtbt"], case["dtbc"],
                      case.get("r8", 0), case.get("rst", 0), y, m, d, h,
                      p(case["lon"]), p(case["lat"]), p(case["z"]), p(case["tmn"]), p(case["smn"]),
                      p(case["itn"], np.int32), p(case["pt"]), p(case["sa"]),
                      p(case["taux"]), p(case["tauy"]), p(case["bct"]), p(case["bcs"]),
                      p(case["pa"]), p(case["fw"]), p(case.get("vmix")))
        self.h = L.orc_create(C.byref(inp))
        self.ni = case["glo_ni"] + 2
        self.nj = case["glo_nj"] + 2
        self.nk = case["nk"]

    def __del__(self):
        try:
            if self.h:
                lib().orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def step(self, n: int = 1):
        for _ in range(n):
            lib().orc_step(self.h)

    def phase(self, name: str):
        lib().orc_phase(self.h, PHASES[name])

    @property
    def iter(self) -> int:
        return lib().orc_get_iter(self.h)

    @iter.setter
    def iter(self, i: int):
        lib().orc_set_iter(self.h, int(i))

    def field(self, name: str) -> np.ndarray:
        """A copy of a named array, numpy shape [n3][n2][n1] (Fortran order)."""
        n1, n2, n3 = C.c_int32(), C.c_int32(), C.c_int32()
        ptr = lib().orc_field(self.h, name.encode(), C.byref(n1), C.byref(n2), C.byref(n3))
        if not ptr:
            ip = lib().orc_ifield(self.h, name.encode(), C.byref(n1), C.byref(n2), C.byref(n3))
            if not ip:
                raise KeyError(name)
            a = np.ctypeslib.as_array(ip, shape=(n3.value, n2.value, n1.value)).copy()
        else:
            a = np.ctypeslib.as_array(ptr, shape=(n3.value, n2.value, n1.value)).copy()
        return a[0] if a.shape[0] == 1 and name not in ("z1", "pr1", "dz1", "dpr1", "z2", "pr2", "dz2", "dpr2", "lon", "lat") else a

    def view(self, name: str) -> np.ndarray:
        """The named array itself (writable, shares the oracle's memory),
        numpy shape [n3][n2][n1]."""
        n1, n2, n3 = C.c_int32(), C.c_int32(), C.c_int32()
        ptr = lib().orc_field(self.h, name.encode(), C.byref(n1), C.byref(n2), C.byref(n3))
        if not ptr:
            raise KeyError(name)
        return np.ctypeslib.as_array(ptr, shape=(n3.value, n2.value, n1.value))

    def vec(self, name: str) -> np.ndarray:
        return self.field(name).reshape(-1)

    def const(self, name: str) -> float:
        return lib().orc_const(self.h, name.encode())
