"""The netCDF writers of pcom_b200.output on CPU, driven by a stand-in
model (the device model's own test is tests/test_gpu_output.py)."""
import numpy as np
from scipy.io import netcdf_file

from pcom_b200.output import MEANS, MISSING, read_restart, write_means, write_restart


class FakeModel:
    def __init__(self, ni=6, nj=4, nk=3, seed=0):
        rng = np.random.default_rng(seed)
        self.glo_ni, self.glo_nj, self.nk = ni, nj, nk
        self.ni, self.nj = ni + 2, nj + 2
        self.case = dict(lon=np.arange(ni) + 0.5, lat=np.arange(nj) * 2.0, z=np.arange(nk) * 10.0 + 5)
        self.date = (1, 1, 2, 0)
        lev = rng.integers(0, nk + 1, size=(self.nj, self.ni)).astype(np.int32)
        self._static = dict(lev_t=lev, lev_u=np.minimum(lev, np.roll(lev, -1, axis=1)),
                            rh1=np.cos(np.deg2rad(np.linspace(-30, 30, self.nj)))[:, None] * np.ones((1, self.ni)))
        sh3, sh2 = (nk, self.nj, self.ni), (self.nj, self.ni)
        self._acc = {a: rng.standard_normal(sh2 if a in ("acch", "acssh") else sh3) for a, *_ in MEANS.values()}
        self._acc.update(n_ts=3, n_uv=3, n_w=3, n_ch=3, n_ssh=3)
        self._fields = {f: rng.standard_normal(sh3) for f in
                        ("tc", "sc", "tp", "sp", "uc", "vc", "up", "vp", "auc", "avc", "aup", "avp", "aupp", "avpp", "am")}
        self._fields["prho"] = rng.standard_normal(sh3 + (2,))
        for f in ("chc", "chp", "ubc", "vbc", "ubp", "vbp", "bnd_taux", "bnd_tauy", "bnd_t", "bnd_s", "bnd_pa"):
            self._fields[f] = rng.standard_normal(sh2)
        self.loaded = None
        self.was_reset = False

    def accum(self):
        return self._acc

    def static(self):
        return self._static

    def field(self, n):
        return self._fields[n].copy()

    def reset_accum(self):
        self.was_reset = True

    def set_state(self, **kw):
        self.loaded = kw


def test_means_files(tmp_path):
    m = FakeModel()
    files = write_means(m, str(tmp_path))
    assert len(files) == 8 and m.was_reset
    with netcdf_file(files[0], "r", mmap=False) as f:
        assert f.variables["pt"].dimensions == ("time", "z", "lat", "lon")
        np.testing.assert_allclose(f.variables["pt"][0], (m._acc["act"] / 3)[:, 1:-1, 1:-1], rtol=1e-6)
    with netcdf_file(str(tmp_path / "ssh_0001-01-02_00:00.nc"), "r", mmap=False) as f:
        ssh = f.variables["ssh"][0].astype(np.float64)
    wet = m._static["lev_t"][1:-1, 1:-1] >= 1
    assert np.all(ssh[~wet] == MISSING)
    w = m._static["rh1"][1:-1, 1:-1] * wet
    assert abs((np.where(wet, ssh, 0) * w).sum() / w.sum()) < 1e-6


def test_restart_round_trip_files(tmp_path):
    a = FakeModel(seed=1)
    p = str(tmp_path / "restart.nc")
    write_restart(a, p)
    b = FakeModel(seed=2)
    read_restart(b, p)
    for f in ("tc", "uc", "aupp", "am", "chc", "ubc"):
        np.testing.assert_array_equal(b.loaded[f][..., 1:-1, 1:-1], a._fields[f][..., 1:-1, 1:-1])
        np.testing.assert_array_equal(b.loaded[f][..., :, 0], b.loaded[f][..., :, -2])
    np.testing.assert_array_equal(b.loaded["prho"][:, 1:-1, 1:-1], a._fields["prho"][:, 1:-1, 1:-1])
    with netcdf_file(p, "r", mmap=False) as f:
        assert f.cdate == b"0001-01-02 00:00:00"
