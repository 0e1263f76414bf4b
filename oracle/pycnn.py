"""ctypes bridge to the CPU restatement of the closure network in
oracle/cnn_oracle.cpp (test infrastructure only)."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import pyoracle

_f = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_d = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def _lib():
    lib = pyoracle.lib()
    if not getattr(lib, "_cnn_bound", False):
        lib.orc_cnn_conv.argtypes = [C.c_int, C.c_int, _f, _f, _f, C.c_void_p, _f, C.c_longlong, C.c_int, C.c_int,
                                     C.c_int, C.c_int, C.c_int]
        lib.orc_cnn_wgrad.argtypes = [C.c_int, C.c_int, _f, _f, _d, C.c_longlong, C.c_int, C.c_int, C.c_int]
        lib.orc_cnn_param_count.restype = C.c_longlong
        lib.orc_cnn_loss_grad.argtypes = [_f, _f, _f, _f, C.c_longlong, C.c_int, C.c_int, C.c_int, C.c_int, _d]
        lib.orc_cnn_loss_grad.restype = C.c_double
        lib._cnn_bound = True
    return lib


def param_count() -> int:
    return int(_lib().orc_cnn_param_count())


def conv(cin, nout, x, w, bias, aux, H, W, periodic_x, mode, nstore=0):
    """One layer; x [npix][cin], w [9][nout][cin] (float32 holding BF16 values)."""
    x = np.ascontiguousarray(x, np.float32)
    npix = x.shape[0]
    out = np.zeros((npix, nstore if mode == 1 else nout), np.float32)
    a = None if aux is None else np.ascontiguousarray(aux, np.float32)
    _lib().orc_cnn_conv(cin, nout, x, np.ascontiguousarray(w, np.float32), np.ascontiguousarray(bias, np.float32),
                        None if a is None else a.ctypes.data, out, npix, H, W, periodic_x, mode, nstore)
    return out


def wgrad(cin, nout, x, g, H, W, periodic_x):
    x = np.ascontiguousarray(x, np.float32)
    dw = np.zeros(9 * nout * cin)
    _lib().orc_cnn_wgrad(cin, nout, x, np.ascontiguousarray(g, np.float32), dw, x.shape[0], H, W, periodic_x)
    return dw.reshape(9, nout, cin)


def loss_grad(params, x, target, mask, H, W, periodic_x, round_bf16):
    params = np.ascontiguousarray(params, np.float32)
    g = np.zeros(param_count())
    loss = _lib().orc_cnn_loss_grad(params, np.ascontiguousarray(x, np.float32), np.ascontiguousarray(target, np.float32),
                                    np.ascontiguousarray(mask, np.float32), x.shape[0], H, W, periodic_x, round_bf16, g)
    return loss, g
