"""Row-slab decomposition (pcom_b200.decomp) on the CPU.

The split follows the reference's rank map and remainder rule
(mod_param.f90:279-369).  With the oracle as each rank's compute engine and
every row outside a rank's window set to NaN after each subroutine, the
ranks' own rows must come out bit-equal to the single-domain oracle: that
holds only if the halo refresh after each subroutine and the all-gather
before the barotropic subcycle supply every row the rank depends on.  The
same plan drives the CUDA handles (tests/test_gpu_decomp.py).
"""
import os

import numpy as np
import pytest

from pcom_b200 import decomp as D
from pcom_b200.synth import make_case
from decomp_util import OracleSlab, assemble
from parity_util import STATE_FIELDS

HALO = 2


def test_split_extent_remainder_rule():
    # n // parts rows each, the remainder one each to the first parts
    assert D.split_extent(64, 3) == [(1, 22), (23, 43), (44, 64)]
    assert D.split_extent(10, 4) == [(1, 3), (4, 6), (7, 8), (9, 10)]
    assert D.split_extent(160, 8) == [(20 * p + 1, 20 * p + 20) for p in range(8)]
    for n, p in ((37, 5), (640, 7), (14, 2)):
        e = D.split_extent(n, p)
        assert e[0][0] == 1 and e[-1][1] == n
        assert all(b[0] == a[1] + 1 for a, b in zip(e, e[1:]))
        sizes = [b - a + 1 for a, b in e]
        assert max(sizes) - min(sizes) <= 1 and sizes == sorted(sizes, reverse=True)


def test_rank_map_and_neighbours():
    # px = 4, py = 2 (the example of set_ids): ids = [[0, 4], [1, 5], [2, 6], [3, 7]]
    assert [D.rank_position(r, 4, 2) for r in range(8)] == [(1, 1), (2, 1), (3, 1), (4, 1),
                                                           (1, 2), (2, 2), (3, 2), (4, 2)]
    nb = D.neighbours(0, 4, 2)
    assert nb == {"s": None, "n": 4, "w": 3, "e": 1}  # x wraps, y faces MPI_PROC_NULL
    nb = D.neighbours(7, 4, 2)
    assert nb == {"s": 3, "n": None, "w": 6, "e": 4}
    with pytest.raises(ValueError):
        D.rank_position(8, 4, 2)


def test_slabs_partition_the_rows():
    for glo_nj, ranks in ((64, 3), (160, 8), (14, 2), (640, 7)):
        nj = glo_nj + 2
        sl = D.slabs(glo_nj, ranks, HALO)
        rows = [j for s in sl for j in range(s.lo, s.hi + 1)]
        assert rows == list(range(1, nj + 1))
        for s in sl:
            assert s.win_lo == max(1, s.lo - HALO) and s.win_hi == min(nj, s.hi + HALO)
            assert (s.south is None) == (s.rank == 0) and (s.north is None) == (s.rank == ranks - 1)
    with pytest.raises(ValueError, match="halo"):
        D.slabs(6, 4, 2)  # a slab of one row cannot feed a 2-row halo


def _run_local(oracle_lib, name, ranks, steps):
    c = make_case(name)
    ref = oracle_lib.Oracle(c, threads=1)
    ref.step(steps)
    eng = {s.rank: OracleSlab(oracle_lib, c, s) for s in D.slabs(c["glo_nj"], ranks, HALO)}
    drv = D.SlabDriver(D.LocalLinks(eng), HALO, after_phase=lambda ph: [e.poison(ph) for e in eng.values()])
    drv.run(steps)
    for f in STATE_FIELDS + ["acr", "prho1", "prho2", "acssh"]:
        g, r = assemble(eng, f), ref.view(f)
        bad = np.count_nonzero((g != r) & ~(np.isnan(g) & np.isnan(r)))
        assert bad == 0, f"{name} over {ranks} ranks: {f} differs at {bad} points after {steps} steps"


@pytest.mark.parametrize("name,ranks,steps", [("tiny_bathy", 2, 26), ("box", 3, 3), ("tiny", 3, 5)])
def test_slabs_bit_equal_to_single_domain(oracle_lib, name, ranks, steps):
    _run_local(oracle_lib, name, ranks, steps)


def test_halo_of_one_row_is_not_enough(oracle_lib):
    """The check has teeth: with a 1-row halo the poisoned rows reach the
    ranks' own rows and the result differs."""
    c = make_case("tiny_bathy")
    ref = oracle_lib.Oracle(c, threads=1)
    ref.step(2)
    eng = {s.rank: OracleSlab(oracle_lib, c, s) for s in D.slabs(c["glo_nj"], 2, 1)}
    D.SlabDriver(D.LocalLinks(eng), 1, after_phase=lambda ph: [e.poison(ph) for e in eng.values()]).run(2)
    g, r = assemble(eng, "tc"), ref.view("tc")
    assert np.count_nonzero(g != r) > 0


# ------------------------------------------------ two processes over gloo
def _gloo_rank(rank, world, port, steps, out_dir):
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from oracle import pyoracle

        c = make_case("tiny_bathy")
        slab = D.slabs(c["glo_nj"], world, HALO)[rank]
        e = OracleSlab(pyoracle, c, slab)
        D.SlabDriver(D.DistLinks(e, world), HALO, after_phase=e.poison).run(steps)
        ref = pyoracle.Oracle(c, threads=1)
        ref.step(steps)
        bad = {}
        for f in STATE_FIELDS + ["acr", "prho1", "prho2"]:
            g, r = e.views(f)[0].numpy(), ref.view(f)
            g, r = g[:, slab.lo - 1:slab.hi, :], r[:, slab.lo - 1:slab.hi, :]
            n = int(np.count_nonzero((g != r) & ~(np.isnan(g) & np.isnan(r))))
            if n:
                bad[f] = n
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as fh:
            fh.write(repr(bad))
    finally:
        dist.destroy_process_group()


def test_gloo_two_ranks_bit_equal(tmp_path):
    """World size 2 over gloo (127.0.0.1): each rank's own rows after 26
    steps (a day boundary, so den_prho's refresh runs) equal the
    single-domain oracle's."""
    import socket

    import torch.multiprocessing as mp

    from oracle import pyoracle

    pyoracle.build()
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_gloo_rank, args=(2, port, 26, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for r in range(2):
        assert (tmp_path / f"rank{r}.txt").read_text() == "{}", f"rank {r}"
