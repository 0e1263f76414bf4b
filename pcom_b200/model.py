"""Python face of the B200 PCOM time step.

``Model`` mirrors the reference's driver (main.f90): it is created from the
input-file contents of a case (see ``pcom_b200.synth``), performs the one-time
setup on the host, uploads it, and advances the ocean with the time loop of
main.f90:158-238.  ``Model.handle`` is the underlying pcom_gpu handle for
direct C-ABI calls (phases, fields, state, accumulators).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

PHASES = ("den_alpha", "int_pgra", "int_readyc", "int_trop", "int_clin", "int_ssh", "int_ts")


def _dp(a: np.ndarray):
    return a.ctypes.data_as(L.dbl_p)


def _ip(a: np.ndarray):
    return a.ctypes.data_as(L.i32_p)


class Model:
    def __init__(self, case: dict, flags: int = L.PCOM_PREC_FP64):
        self.lib = L.load()
        self.case = case
        self.glo_ni, self.glo_nj, self.nk = case["glo_ni"], case["glo_nj"], case["nk"]
        self.ni, self.nj, self.nkp = self.glo_ni + 2, self.glo_nj + 2, self.nk + 1
        self._keep = []

        def d(name, dt=np.float64):
            a = case.get(name)
            if a is None:
                return None
            a = np.ascontiguousarray(a, dtype=dt)
            self._keep.append(a)
            return a.ctypes.data_as(L.i32_p if dt == np.int32 else L.dbl_p)

        y, mo, dd, hh = case.get("bdate", (1, 1, 1, 0))
        cs = L.Case(self.glo_ni, self.glo_nj, self.nk, case["dtbt"], case["dtbc"], case.get("r8", 0),
                    case.get("rst", 0), y, mo, dd, hh,
                    d("lon"), d("lat"), d("z"), d("tmn"), d("smn"), d("itn", np.int32), d("pt"), d("sa"),
                    d("taux"), d("tauy"), d("bct"), d("bcs"), d("pa"), d("fw"), d("vmix"))
        self._m = C.c_void_p()
        L.check(self.lib.pcom_model_create(C.byref(cs), flags, C.byref(self._m)), "pcom_model_create")
        self.handle = C.c_void_p(self.lib.pcom_model_handle(self._m))
        self.host_only = bool(flags & L.PCOM_MODEL_HOST_ONLY)

    # ------------------------------------------------------------------ life
    def close(self):
        if getattr(self, "_m", None) and self._m.value:
            self.lib.pcom_model_destroy(self._m)
            self._m = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --------------------------------------------------------------- driving
    def run(self, nsteps: int = 1):
        L.check(self.lib.pcom_model_run(self._m, int(nsteps)), "pcom_model_run")

    @property
    def iter(self) -> int:
        return int(self.lib.pcom_model_iter(self._m))

    @property
    def date(self):
        a = (C.c_int32 * 4)()
        self.lib.pcom_model_date(self._m, a)
        return tuple(a)

    def int_bnd(self) -> dict:
        n2 = self.ni * self.nj
        out = {k: np.zeros(n2) for k in ("taux", "tauy", "t", "s", "pa", "fw")}
        L.check(self.lib.pcom_model_int_bnd(self._m, *[_dp(out[k]) for k in ("taux", "tauy", "t", "s", "pa", "fw")]))
        return {k: v.reshape(self.nj, self.ni) for k, v in out.items()}

    def set_forcing(self, f: dict):
        arrs = [np.ascontiguousarray(f[k], dtype=np.float64) for k in ("taux", "tauy", "t", "s", "pa", "fw")]
        fo = L.Forcing(*[_dp(a) for a in arrs])
        L.check(self.lib.pcom_gpu_set_forcing(self.handle, C.byref(fo)), "set_forcing")

    def den_prho(self):
        L.check(self.lib.pcom_gpu_den_prho(self.handle), "den_prho")

    def phase(self, name_or_index, tctr_i: int):
        ph = PHASES.index(name_or_index) if isinstance(name_or_index, str) else int(name_or_index)
        L.check(self.lib.pcom_gpu_phase(self.handle, ph, int(tctr_i)), f"phase {ph}")

    def step_handle(self, tctr_i: int):
        L.check(self.lib.pcom_gpu_step(self.handle, int(tctr_i)), "pcom_gpu_step")

    def set_rows(self, j_lo: int, j_hi: int):
        """Rows the step's 3-D kernels compute (padded, 1-based; default all)."""
        L.check(self.lib.pcom_gpu_set_rows(self.handle, int(j_lo), int(j_hi)), "set_rows")

    def check_finite(self):
        L.check(self.lib.pcom_gpu_check_finite(self.handle), "check_finite")

    # ----------------------------------------------------------------- data
    def field(self, name: str) -> np.ndarray:
        """A named device array as numpy [n3][nj][ni] (2-D fields: [nj][ni])."""
        n = int(self.lib.pcom_gpu_field_size(self.handle, name.encode()))
        if n <= 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        L.check(self.lib.pcom_gpu_get_field(self.handle, name.encode(), _dp(out), n), f"field {name}")
        n2 = self.ni * self.nj
        if name == "prho":
            return out.reshape(self.nk, self.nj, self.ni, 2)
        if n == n2:
            return out.reshape(self.nj, self.ni)
        return out.reshape(n // n2, self.nj, self.ni)

    def static(self) -> dict:
        s = L.Static()
        L.check(self.lib.pcom_model_static(self._m, C.byref(s)))
        n2, n3, n3p = self.ni * self.nj, self.ni * self.nj * self.nk, self.ni * self.nj * self.nkp

        def cp(ptr, n, shape, dt=np.float64):
            return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dt, copy=True).reshape(shape)

        out = {}
        for g in range(4):
            out[f"rh{g + 1}"] = cp(s.rh[g], n2, (self.nj, self.ni))
            out[f"tn{g + 1}"] = cp(s.tn[g], n2, (self.nj, self.ni))
            dx = cp(s.dx[g], 2 * n2, (self.nj, self.ni, 2))
            out[f"dx{g + 1}x"], out[f"dx{g + 1}y"] = dx[..., 0].copy(), dx[..., 1].copy()
        for v, n in (("z1", self.nkp), ("pr1", self.nkp), ("dz1", self.nkp), ("dpr1", self.nkp),
                     ("z2", self.nk), ("pr2", self.nk), ("dz2", self.nk), ("dpr2", self.nk)):
            out[v] = cp(getattr(s, v), n, (n,))
        out["msk_t"] = cp(s.msk_t, n3, (self.nk, self.nj, self.ni), np.int32)
        out["msk_u"] = cp(s.msk_u, n3, (self.nk, self.nj, self.ni), np.int32)
        out["lev_t"] = cp(s.lev_t, n2, (self.nj, self.ni), np.int32)
        out["lev_u"] = cp(s.lev_u, n2, (self.nj, self.ni), np.int32)
        for v in ("phih_t", "prh_t", "phih_u", "prh_u", "cv1", "cv2", "cor", "graphihx", "graphihy"):
            out[v] = cp(getattr(s, v), n2, (self.nj, self.ni))
        out["km"] = cp(s.km, n3p, (self.nkp, self.nj, self.ni))
        out["kh"] = cp(s.kh, n3p, (self.nkp, self.nj, self.ni))
        return out

    def accum(self) -> dict:
        n2, n3 = self.ni * self.nj, self.ni * self.nj * self.nk
        bufs = {k: np.zeros(n3 if k not in ("acch", "acssh") else n2) for k in L.ACCUM_FIELDS}
        a = L.Accum(*[_dp(bufs[k]) for k in L.ACCUM_FIELDS], 0, 0, 0, 0, 0)
        L.check(self.lib.pcom_gpu_get_accum(self.handle, C.byref(a)), "get_accum")
        out = {k: (v.reshape(self.nj, self.ni) if v.size == n2 else v.reshape(self.nk, self.nj, self.ni))
               for k, v in bufs.items()}
        out.update(n_ts=a.n_ts, n_uv=a.n_uv, n_w=a.n_w, n_ch=a.n_ch, n_ssh=a.n_ssh)
        return out

    def reset_accum(self):
        L.check(self.lib.pcom_gpu_reset_accum(self.handle), "reset_accum")

    def set_state(self, **fields):
        keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in fields.items()}
        st = L.State(*[(_dp(keep[n]) if n in keep else None) for n in L.STATE_FIELDS])
        L.check(self.lib.pcom_gpu_set_state(self.handle, C.byref(st)), "set_state")

    # ------------------------------------------------------------- streams
    def set_overlap(self, enable: bool):
        """Concurrent phases in the full step (default on); results are the
        same either way."""
        L.check(self.lib.pcom_gpu_set_overlap(self.handle, int(bool(enable))), "set_overlap")

    def set_stream(self, stream_ptr: int):
        L.check(self.lib.pcom_gpu_set_stream(self.handle, C.c_void_p(stream_ptr)), "set_stream")

    def sync(self):
        L.check(self.lib.pcom_gpu_sync(self.handle), "sync")

    def profile(self, on: bool = True):
        L.check(self.lib.pcom_gpu_profile(self.handle, 1 if on else 0))

    def profile_read(self) -> dict:
        cap = 64
        names = C.create_string_buffer(64 * cap)
        launches = (C.c_int64 * cap)()
        ms = (C.c_double * cap)()
        n = self.lib.pcom_gpu_profile_read(self.handle, names, launches, ms, cap)
        out = {}
        for q in range(min(n, cap)):
            nm = names.raw[64 * q: 64 * q + 64].split(b"\0", 1)[0].decode()
            out[nm] = (int(launches[q]), float(ms[q]))
        return out

    def launch_count(self) -> int:
        return int(self.lib.pcom_gpu_launch_count(self.handle))

    def global_sums(self) -> tuple:
        """(volume m^3, sum T dV, sum S dV) over the wet interior, FP64."""
        out = np.zeros(3)
        L.check(self.lib.pcom_gpu_global_sums(self.handle, _dp(out)), "global_sums")
        return tuple(float(x) for x in out)


class Batch:
    """Several models stepped together on one device (ensemble members and
    basins of uneven size sharing dtbt, dtbc and the start date): each
    kernel of the step runs once for all members, the barotropic subcycles
    of all members are one persistent launch, and after the two start-up
    steps the batched step replays from captured CUDA graphs."""

    def __init__(self, models: list[Model], graphs: bool = True):
        self.lib = L.load()
        self.models = list(models)
        n = len(self.models)
        hs = (C.c_void_p * n)(*[m.handle.value for m in self.models])
        self._b = C.c_void_p()
        L.check(self.lib.pcom_gpu_batch_create(hs, n, C.byref(self._b)), "pcom_gpu_batch_create")
        self._ms = (C.c_void_p * n)(*[m._m.value for m in self.models])
        self.use_graphs(graphs)

    def use_graphs(self, on: bool):
        L.check(self.lib.pcom_gpu_batch_use_graphs(self._b, 1 if on else 0), "batch_use_graphs")

    def run(self, nsteps: int = 1):
        L.check(self.lib.pcom_model_run_batch(self._ms, len(self.models), self._b, int(nsteps)),
                "pcom_model_run_batch")

    def step_async(self, tctr_i: int):
        L.check(self.lib.pcom_gpu_batch_step_async(self._b, int(tctr_i)), "batch_step_async")

    def den_prho(self):
        L.check(self.lib.pcom_gpu_batch_den_prho(self._b), "batch_den_prho")

    def sync(self):
        L.check(self.lib.pcom_gpu_batch_sync(self._b), "batch_sync")

    def autotune(self) -> str:
        buf = C.create_string_buffer(1024)
        L.check(self.lib.pcom_gpu_batch_autotune(self._b, buf, 1024), "batch_autotune")
        return buf.value.decode()

    def set_tiles(self, tx: int, ty: int, max_resident: int = 0):
        L.check(self.lib.pcom_gpu_batch_set_tiles(self._b, tx, ty, max_resident), "batch_set_tiles")

    def launch_count(self) -> int:
        return int(self.lib.pcom_gpu_batch_launch_count(self._b))

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            self.lib.pcom_gpu_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
