"""Host-side output of a model run: the time means of output()
(main.f90:726-760) and the restart file (mod_mympi.f90:133-176, read back by
mod_mympi.f90:460-547), as netCDF classic files.

Time means.  One file per variable per output time, named
``<name>_<YYYY-MM-DD_HH:MM>.nc`` (mod_io.f90:332-353), dimensions lon, lat,
z, time (unlimited), FP32 values with ``_FillValue`` = -9.99999e30
(mod_param.f90:62) where the reference masks them: u, v and w on the U-grid
mask (merge_out_equvw, mod_mympi.f90:201-227, w included), rho on the T-grid
mask (merge_out_eqts, :178-199), ch and ssh on the surface T mask; ssh has
its area-weighted (rh * msk) global mean removed (merge_out_r2d_weight,
:283-312).  After writing, the accumulators are reset.

Restart.  FP64 interior arrays chc, chp, bnd_*, buc/bvc/bup/bvp, tc, sc, tp,
sp, prpt, prps, uc, vc, up, vp, auc, avc, aup, avp, aupp, avpp, am, with the
dates as global attributes cdate and pdate (mod_io.f90:59-124).
"""
from __future__ import annotations

import os

import numpy as np
from scipy.io import netcdf_file

MISSING = np.float32(-9.99999e30)

MEANS = {  # name: (accumulator, counter, long name, units, mask)
    "pt": ("act", "n_ts", "potential temperature", "degrees Celcius", None),
    "sa": ("acs", "n_ts", "salinity", "psu", None),
    "rho": ("acr", "n_ts", "sea water density", "kg/m^3", "t3"),
    "u": ("acu", "n_uv", "zonal velocity", "m/s", "u3"),
    "v": ("acv", "n_uv", "meridional velocity", "m/s", "u3"),
    "w": ("acw", "n_w", "vertical velocity", "m/s", "u3"),
    "ch": ("acch", "n_ch", "normalized sea bottom pressure", "", "t2"),
    "ssh": ("acssh", "n_ssh", "sea surface height", "m", "t2"),
}
RESTART_3D = ["tc", "sc", "tp", "sp", "uc", "vc", "up", "vp", "auc", "avc", "aup", "avp", "aupp", "avpp", "am"]
RESTART_2D = {"chc": "chc", "chp": "chp", "buc": "ubc", "bvc": "vbc", "bup": "ubp", "bvp": "vbp"}
BND = {"bnd_taux": "bnd_taux", "bnd_tauy": "bnd_tauy", "bnd_t": "bnd_t", "bnd_s": "bnd_s", "bnd_pa": "bnd_pa"}


def date_str(ymdh) -> str:
    y, m, d, h = ymdh
    return f"{y:04d}-{m:02d}-{d:02d}_{h:02d}:00"


def _dims(f, model, nk=None):
    f.createDimension("time", None)  # the record dimension comes first in netCDF classic
    f.createDimension("lon", model.glo_ni)
    f.createDimension("lat", model.glo_nj)
    if nk:
        f.createDimension("z", nk)
    for name, vals, ln, un in (("lon", model.case["lon"], "longitude", "degrees_east"),
                               ("lat", model.case["lat"], "latitude", "degrees_north")):
        v = f.createVariable(name, "f4", (name,))
        v[:] = np.asarray(vals, np.float32)
        v.long_name, v.units = ln, un
    if nk:
        v = f.createVariable("z", "f4", ("z",))
        v[:] = np.asarray(model.case["z"], np.float32)
        v.long_name, v.units = "depth", "m"


def write_means(model, outdir: str, reset: bool = True) -> list:
    """Write the time means accumulated since the last output; returns the
    files written."""
    os.makedirs(outdir, exist_ok=True)
    acc = model.accum()
    st = model.static()
    nk = model.nk
    k = np.arange(1, nk + 1)[:, None, None]
    inner = (slice(1, -1), slice(1, -1))
    masks = {"t3": (st["lev_t"][None] >= k)[(slice(None),) + inner],
             "u3": (st["lev_u"][None] >= k)[(slice(None),) + inner],
             "t2": (st["lev_t"] >= 1)[inner]}
    stamp = date_str(model.date)
    files = []
    for name, (a, n, ln, un, mk) in MEANS.items():
        cnt = acc[n]
        v = acc[a] / cnt if cnt else acc[a] * 0.0
        v = v[(slice(None),) + inner] if v.ndim == 3 else v[inner]
        v = v.astype(np.float64)
        if mk is not None:
            v = np.where(masks[mk], v, float(MISSING))
        if name == "ssh":
            w = st["rh1"][inner] * masks["t2"]
            mean = (v * w).sum() / w.sum()
            v = np.where(v != float(MISSING), v - mean, v)
        path = os.path.join(outdir, f"{name}_{stamp}.nc")
        with netcdf_file(path, "w") as f:
            _dims(f, model, nk if v.ndim == 3 else None)
            dims = ("time", "z", "lat", "lon") if v.ndim == 3 else ("time", "lat", "lon")
            var = f.createVariable(name, "f4", dims)
            var._FillValue = MISSING
            var.long_name, var.units = ln, un
            var[0] = v.astype(np.float32)
        files.append(path)
    if reset:
        model.reset_accum()
    return files


def write_restart(model, path: str, pdate=None):
    """The restart file of mod_mympi.f90:133-176 for the model's state."""
    nk = model.nk
    inner = (slice(1, -1), slice(1, -1))
    with netcdf_file(path, "w") as f:
        _dims(f, model, nk)
        y, m, d, h = model.date
        f.cdate = f"{y:04d}-{m:02d}-{d:02d} {h:02d}:00:00"
        if pdate is not None:
            f.pdate = pdate
        for name in RESTART_3D:
            v = f.createVariable(name, "f8", ("time", "z", "lat", "lon"))
            v[0] = model.field(name)[(slice(None),) + inner]
        pr = model.field("prho")
        for q, name in enumerate(("prpt", "prps")):
            v = f.createVariable(name, "f8", ("time", "z", "lat", "lon"))
            v[0] = pr[..., q][(slice(None),) + inner]
        for name, fld in list(RESTART_2D.items()) + list(BND.items()):
            v = f.createVariable(name, "f8", ("time", "lat", "lon"))
            v[0] = model.field(fld)[inner]


def read_restart(model, path: str):
    """Load a restart file into a model created with rst = 1 at the file's
    date: interior values from the file, x-halo columns as the periodic
    copies the reference's exchange makes, y-halo rows kept as they are."""
    def pad(interior, cur):
        out = cur.copy()
        out[..., 1:-1, 1:-1] = interior
        out[..., :, 0] = out[..., :, -2]
        out[..., :, -1] = out[..., :, 1]
        return out

    fields = {}
    with netcdf_file(path, "r", mmap=False) as f:
        for name in RESTART_3D:
            fields[name] = pad(f.variables[name][0], model.field(name))
        pr = model.field("prho")
        for q, name in enumerate(("prpt", "prps")):
            pr[..., q] = pad(f.variables[name][0], pr[..., q])
        fields["prho"] = pr
        for name, fld in RESTART_2D.items():
            fields[fld] = pad(f.variables[name][0], model.field(fld))
    model.set_state(**fields)
