"""Test helpers for the row-slab decomposition: the oracle as a stand-in
compute engine of one rank (test infrastructure only).

The oracle computes every row of every subroutine; after each subroutine the
rows of the fields it wrote that lie outside the rank's window are set to
NaN, so the rank's own rows can only come out right if the halo refresh and
the all-gather of pcom_b200.decomp supply every row they depend on."""
from __future__ import annotations

import numpy as np

from pcom_b200 import decomp as D


class OracleSlab:
    def __init__(self, oracle_mod, case: dict, slab: D.Slab):
        self.o = oracle_mod.Oracle(case, threads=1)
        self.slab = slab
        self.ni, self.nj, self.nk = case["glo_ni"] + 2, case["glo_nj"] + 2, case["nk"]
        self.dtbc = case["dtbc"]

    def views(self, name: str):
        import torch

        names = ("prho1", "prho2") if name == "prho" else (name,)
        return [torch.from_numpy(self.o.view(n)) for n in names]

    def begin_step(self):
        it = self.o.iter + 1
        self.o.iter = it
        day_of = lambda i: (i - 1) * self.dtbc // 86400
        day = it == 1 or day_of(it) != day_of(it - 1)
        if day:
            self.o.phase("int_bnd")
            self.o.phase("den_prho")
        return it, day

    def phase(self, name: str, it: int):
        self.o.phase(name)

    def end_step(self):
        self.o.phase("advance")

    def sync(self):
        pass

    def poison(self, phase: str):
        poison(self, phase)


def written(phase: str) -> list[str]:
    """Row-split fields a subroutine writes (None: every one of them)."""
    phases = [phase] if phase else list(D.HALO_3D) + list(D.ACCUM_3D) + list(D.GATHER_2D)
    names = []
    for ph in phases:
        names += list(D.HALO_3D.get(ph, [])) + list(D.ACCUM_3D.get(ph, []))
        names += [n for n, _ in D.GATHER_2D.get(ph, [])]
        if ph == "int_ssh":
            names.append("acssh")
    return list(dict.fromkeys(names))


def poison(engine, phase: str | None):
    """NaN outside the engine's window in every field `phase` wrote."""
    s = engine.slab
    for name in written(phase):
        for v in engine.views(name):
            v[:, : s.win_lo - 1, :] = float("nan")
            v[:, s.win_hi:, :] = float("nan")


def assemble(engines: dict, name: str) -> np.ndarray:
    """The whole field from each rank's own rows."""
    first = engines[min(engines)]
    out = np.array(first.views(name)[0].cpu().numpy(), copy=True)
    for e in engines.values():
        s = e.slab
        out[:, s.lo - 1:s.hi, :] = e.views(name)[0].cpu().numpy()[:, s.lo - 1:s.hi, :]
    return out
