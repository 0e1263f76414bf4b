"""Host-side output (time means of output(), main.f90:726-760) and the
restart file round trip (mod_mympi.f90:133-176, 460-547) on the GPU model."""
import numpy as np
import pytest
from scipy.io import netcdf_file

from pcom_b200.model import Model
from pcom_b200.output import MISSING, read_restart, write_means, write_restart
from pcom_b200.synth import make_case

pytestmark = pytest.mark.gpu


def test_time_means(tmp_path):
    c = make_case("tiny_bathy")
    m = Model(c)
    m.run(24)
    acc = m.accum()
    files = write_means(m, str(tmp_path))
    assert len(files) == 8 and all(f.endswith("_0001-01-02_00:00.nc") for f in files)
    st = m.static()
    with netcdf_file(str(tmp_path / "pt_0001-01-02_00:00.nc"), "r", mmap=False) as f:
        pt = f.variables["pt"][0].astype(np.float64)
        assert pt.shape == (c["nk"], c["glo_nj"], c["glo_ni"])
    ref = (acc["act"] / acc["n_ts"])[:, 1:-1, 1:-1]
    assert np.abs(pt - ref).max() <= 1e-5 * np.abs(ref).max()
    with netcdf_file(str(tmp_path / "ssh_0001-01-02_00:00.nc"), "r", mmap=False) as f:
        ssh = f.variables["ssh"][0].astype(np.float64)
    wet = st["lev_t"][1:-1, 1:-1] >= 1
    assert np.all(ssh[~wet] == MISSING)
    w = st["rh1"][1:-1, 1:-1] * wet
    assert abs((ssh * w)[wet].sum() / w.sum()) < 1e-6 * np.abs(ssh[wet]).max()
    assert m.accum()["n_ts"] == 0  # reset after output
    m.close()


def test_restart_round_trip(tmp_path):
    """N steps, restart file, M steps == N + M steps without the file."""
    c = make_case("tiny_bathy")
    a = Model(c)
    a.run(24)
    path = str(tmp_path / "restart.nc")
    write_restart(a, path)
    date = a.date
    a.run(6)
    cb = dict(c, rst=1, bdate=tuple(date))
    b = Model(cb)
    read_restart(b, path)
    b.run(6)
    for f in ("tc", "sc", "uc", "vc", "chc", "ubc", "vbc"):
        x, y = a.field(f)[..., 1:-1, 1:-1], b.field(f)[..., 1:-1, 1:-1]
        assert np.array_equal(x, y), f
    a.close()
    b.close()
