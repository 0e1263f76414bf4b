"""Seeded synthetic PCOM input cases.

The reference reads its grid, initial state and forcing from netCDF files
(main.f90:292-298, 499-512, 585-599, 675-697; mod_mympi.f90:493-560).  No
input data ships with it (its ``input`` link dangles), so these generators
stand in for those files.  Each case returns the *file contents* for a
single-domain run: global interior arrays with numpy shape ``[k][j][i]``
(= Fortran ``(glo_ni, glo_nj, nk)`` order, i fastest).

Cases
-----
``box``       128 x 64 x 20 flat-bottom basin, 1 deg, 10-74N, walls on the
              outer ring, zonal wind 0.1 cos(2 pi (lat-10)/64), SST restored to
              a linear 28->2 degC profile, T = 2 + 23 exp(-z/800 m) + N(0, 0.01).
``global1``   360 x 160 x 30, 1 deg, 78S-80N, zonally periodic, bathymetry
              from a seeded Gaussian random field with a k^-2 power spectrum
              mapped to 0-5500 m (land where the field is negative), wind
              0.1 sin(3 lat), SST/SSS restoring.
``global05``  720 x 320 x 30, the same generator at 0.5 deg with dtbt = 30 s,
              dtbc = 1800 s (too many barotropic tiles for one per SM).
``global025`` 1440 x 640 x 30, the same generator at 0.25 deg with
              dtbt = 20 s, dtbc = 1200 s.
``basin``     glo_ni x glo_nj x nk (default 64 x 32 x 20) flat-bottom 1 deg
              basin centred on the equator, walls, box forcing; the uneven
              basins of the batched-ensemble workload.
``tiny``, ``tiny_bathy``: small grids for fast parity tests.

Vertical levels: z(k) = (k - 1/2) * 4000 m / nk, i.e. evenly spaced to about
4000 dbar.  The initial profile uses p ~ z (1 dbar per metre).  The vertical
mixing file is treated as all-missing (-> 0.1 cm^2/s, main.f90:326-329).
"""
from __future__ import annotations

import numpy as np

CASES = ("tiny", "tiny_bathy", "box", "global1", "global05", "global025", "basin")


def _grf(nx: int, ny: int, rng: np.random.Generator) -> np.ndarray:
    """Gaussian random field with a k^-2 power spectrum, unit variance."""
    kx = np.fft.fftfreq(nx) * nx
    ky = np.fft.fftfreq(ny) * ny
    kk = np.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2)
    amp = np.zeros_like(kk)
    amp[kk > 0] = 1.0 / kk[kk > 0]  # power ~ k^-2  -> amplitude ~ k^-1
    noise = rng.standard_normal((ny, nx)) + 1j * rng.standard_normal((ny, nx))
    f = np.real(np.fft.ifft2(amp * noise))
    f = (f - f.mean()) / f.std()
    return f


def _levels(nk: int, depth_max: float = 4000.0) -> np.ndarray:
    dz = depth_max / nk
    return (np.arange(1, nk + 1) - 0.5) * dz


def _profile(z: np.ndarray) -> np.ndarray:
    return 2.0 + 23.0 * np.exp(-z / 800.0)


def make_case(name: str = "box", seed: int = 1, noise: float = 0.01,
              glo_ni: int | None = None, glo_nj: int | None = None,
              nk: int | None = None) -> dict:
    """Return the input-file contents for one synthetic case."""
    rng = np.random.default_rng(seed)
    bathy = False
    dtbt, dtbc = 60, 3600
    if name == "box":
        ni_, nj_, nk_ = 128, 64, 20
        lat = 10.0 + np.arange(1, nj_ + 1, dtype=np.float64)          # north edges 11..74
        lon = np.arange(ni_, dtype=np.float64) + 0.5
    elif name == "tiny":
        ni_, nj_, nk_ = 16, 10, 12
        lat = 20.0 + 2.0 * np.arange(1, nj_ + 1, dtype=np.float64)
        lon = 2.0 * np.arange(ni_, dtype=np.float64) + 1.0
    elif name == "basin":
        ni_, nj_, nk_ = glo_ni or 64, glo_nj or 32, nk or 20
        # 1 deg, centred on the equator (256 x 128 spans 63S-64N)
        lat = -float(nj_ // 2) + np.arange(1, nj_ + 1, dtype=np.float64)
        lon = np.arange(ni_, dtype=np.float64) + 0.5
    elif name == "tiny_bathy":
        ni_, nj_, nk_ = 24, 14, 12
        bathy = True
        lat = -30.0 + 4.0 * np.arange(1, nj_ + 1, dtype=np.float64)
        lon = 15.0 * np.arange(ni_, dtype=np.float64) + 7.5             # 360 deg periodic
    elif name == "global1":
        ni_, nj_, nk_ = 360, 160, 30
        bathy = True
        lat = -78.0 + np.arange(nj_, dtype=np.float64) * (158.0 / (nj_ - 1))
        lon = np.arange(ni_, dtype=np.float64) + 0.5
    elif name == "global05":
        ni_, nj_, nk_ = 720, 320, 30
        bathy = True
        lat = -78.0 + np.arange(nj_, dtype=np.float64) * (158.0 / (nj_ - 1))
        lon = 0.5 * np.arange(ni_, dtype=np.float64) + 0.25
        dtbt, dtbc = 30, 1800
    elif name == "global025":
        ni_, nj_, nk_ = 1440, 640, 30
        bathy = True
        lat = -78.0 + np.arange(nj_, dtype=np.float64) * (158.0 / (nj_ - 1))
        lon = 0.25 * np.arange(ni_, dtype=np.float64) + 0.125
        dtbt, dtbc = 20, 1200
    else:
        raise ValueError(f"unknown case {name!r}; known: {CASES}")
    if glo_ni is not None:
        ni_ = glo_ni
    if glo_nj is not None:
        nj_ = glo_nj
    if nk is not None:
        nk_ = nk

    z = _levels(nk_)
    tmn = _profile(z)
    smn = np.full(nk_, 35.0)

    # number of wet levels per column
    if bathy:
        f = _grf(ni_, nj_, rng) + 0.5
        depth = np.where(f > 0.0, 5500.0 * f / f.max(), 0.0)
        dzl = 4000.0 / nk_
        itn = np.where(depth > 0.0, np.clip(np.rint(depth / dzl), 1, nk_), 0).astype(np.int32)
    else:
        itn = np.full((nj_, ni_), nk_, dtype=np.int32)
        itn[0, :] = 0
        itn[-1, :] = 0
        itn[:, 0] = 0
        itn[:, -1] = 0

    # initial state
    pt = np.broadcast_to(tmn[:, None, None], (nk_, nj_, ni_)).copy()
    if noise:
        pt += rng.normal(0.0, noise, size=pt.shape)
    sa = np.full((nk_, nj_, ni_), 35.0)

    # forcing (12 identical months); latitude of T rows (grid 1) and U rows (grid 3/4)
    lat_u = lat
    lat_t = np.empty_like(lat)
    lat_t[1:] = 0.5 * (lat[1:] + lat[:-1])
    lat_t[0] = lat[0] - 0.5 * (lat[1] - lat[0])
    if name in ("box", "tiny", "basin"):
        tx = 0.1 * np.cos(2.0 * np.pi * (lat_u - lat[0] + 1.0) / nj_)
        sst = 28.0 + (2.0 - 28.0) * (lat_t - lat_t[0]) / (lat_t[-1] - lat_t[0])
    else:
        tx = 0.1 * np.sin(3.0 * np.deg2rad(lat_u))
        sst = 2.0 + 26.0 * np.cos(np.deg2rad(lat_t)) ** 2
    taux = np.broadcast_to(tx[None, :, None], (12, nj_, ni_)).copy()
    tauy = np.zeros((12, nj_, ni_))
    bct = np.broadcast_to(sst[None, :, None], (12, nj_, ni_)).copy()
    bcs = np.full((12, nj_, ni_), 35.0)
    pa = np.zeros((12, nj_, ni_))
    fw = np.zeros((12, nj_, ni_))

    return dict(name=name, glo_ni=ni_, glo_nj=nj_, nk=nk_, dtbt=dtbt, dtbc=dtbc,
                r8=0, rst=0, bdate=(1, 1, 1, 0),
                lon=lon, lat=lat, z=z, tmn=tmn, smn=smn, itn=itn,
                pt=pt, sa=sa, taux=taux, tauy=tauy, bct=bct, bcs=bcs, pa=pa, fw=fw,
                vmix=None)


def perturb(case: dict, member: int, sigma: float = 0.05) -> dict:
    """Ensemble member: the same case with an extra seeded N(0, sigma) on T."""
    c = dict(case)
    rng = np.random.default_rng(1000 + member)
    c["pt"] = case["pt"] + rng.normal(0.0, sigma, size=case["pt"].shape)
    return c
