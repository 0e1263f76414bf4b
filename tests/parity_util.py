"""Helpers for comparing the CUDA path with the CPU oracle (tests only)."""
from __future__ import annotations

import numpy as np

# fields compared after each subroutine of the step (main.f90:205-223)
PHASE_FIELDS = {
    "den_alpha": ["alpha"],
    "int_pgra": ["adp", "bphi_xn", "bphi_xs", "bphi_ye", "bphi_yw",
                 "bgraphi_xn", "bgraphi_xs", "bgraphi_ye", "bgraphi_yw"],
    "int_readyc": ["pax", "pay", "wm", "auc", "avc", "aup", "avp", "aupp", "avpp", "fx", "fy", "ut", "vt"],
    "int_trop": ["ubc", "vbc", "ubp", "vbp", "chc", "chp", "mch", "mch2", "acch"],
    "int_clin": ["uc", "vc", "up", "vp", "acu", "acv", "am"],
    "int_ssh": ["alpha", "acssh"],
    "int_ts": ["wm", "acw", "tc", "sc", "tp", "sp", "act", "acs", "acr"],
}
STATE_FIELDS = ["tc", "sc", "tp", "sp", "uc", "vc", "up", "vp", "auc", "avc", "aup", "avp", "aupp", "avpp",
                "ubc", "vbc", "ubp", "vbp", "chc", "chp", "mch", "mch2", "am", "alpha", "adp", "wm",
                "act", "acs", "acu", "acv", "acw", "acch", "acssh"]


def compare(gpu: np.ndarray, ref: np.ndarray, mask: np.ndarray | None = None) -> dict:
    """max |gpu - ref| relative to max |ref|, and the count of unequal values."""
    g = np.asarray(gpu, dtype=np.float64).reshape(ref.shape)
    r = np.asarray(ref, dtype=np.float64)
    if mask is not None:
        g = g[mask]
        r = r[mask]
    scale = float(np.max(np.abs(r))) if r.size else 0.0
    diff = np.abs(g - r)
    both_nan = np.isnan(g) & np.isnan(r)
    diff = np.where(both_nan, 0.0, diff)
    mx = float(np.nanmax(diff)) if diff.size else 0.0
    if np.isnan(diff).any():
        mx = float("inf")
    rel = mx / scale if scale > 0 else mx
    return dict(rel=rel, abs=mx, scale=scale, unequal=int(np.count_nonzero((g != r) & ~both_nan)), n=int(r.size))


def acr_mask(lev_t: np.ndarray, nk: int) -> np.ndarray:
    """acr is only defined on wet points (the reference leaves land undefined)."""
    k = np.arange(1, nk + 1)[:, None, None]
    return lev_t[None, :, :] >= k
