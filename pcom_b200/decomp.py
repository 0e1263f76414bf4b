"""Horizontal domain decomposition of the PCOM step: row slabs, one rank each.

The reference splits its domain into npx x npy blocks, one MPI rank each
(mod_param.f90:279-369): ranks are laid out column-major over the px x py
grid (set_ids), each dimension is divided evenly with the remainder going one
row (column) each to the first ranks (get_neighbor), x wraps around and the
north/south edges face MPI_PROC_NULL.  After every operator each rank swaps a
1-wide halo with its four neighbours (mympi_swpbnd, mod_mympi.f90:669-861).

Here the domain is split into row slabs (npx = 1, npy = ranks), with that
remainder rule, and each rank drives one handle on its own GPU:

* Every handle holds the whole domain's arrays (0.9 GB at 1 degree, ~10 GB
  at 0.25 degree: HBM is not the limit) and keeps global row indexing, so
  every kernel evaluates a row exactly as the whole-domain run does.  The
  step's 3-D kernels compute only a window of rows: the rank's own rows plus
  `halo` rows on each side (pcom_gpu_set_rows).
* After every subroutine of the step (and after den_prho) the 3-D fields it
  wrote are refreshed in the halo rows from the ranks that own them, so each
  window starts the next subroutine with current data.  The fused kernels
  recompute their intermediates from their inputs instead of exchanging
  after every operator, so one exchange per subroutine replaces the
  reference's exchange per operator; `halo` rows cover the reach of the
  longest operator chain of any subroutine.
* The barotropic subcycle (2-D, 120 substeps, latency-bound) is not split:
  every rank runs it over the whole domain from the same inputs, after an
  all-gather of the 2-D fields it reads that the 3-D subroutines produce
  (bphi, bgraphi, ut, vt and the first level of am).  Its outputs are then
  identical on every rank, and the per-substep halo exchanges of the
  reference (about 20 per substep) disappear.
* The 2-D preparation kernels read only replicated 2-D fields and cover
  every row on every rank.

Transport: `DistLinks` moves the rows with torch.distributed (NCCL between
GPUs, gloo on the CPU): one batched send/receive per neighbour per
subroutine and one all-gather of the 2-D rows before the subcycle.
`LocalLinks` runs several ranks in one process (copies between their
arrays).  Columns are not split: x is the periodic direction the kernels
close with ring neighbours, and row slabs already divide the 3-D work.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from . import _lib as L

PHASES = ("den_alpha", "int_pgra", "int_readyc", "int_trop", "int_clin", "int_ssh", "int_ts")

# 3-D fields each subroutine writes that other rows read later: their halo
# rows are refreshed after the subroutine
HALO_3D = {
    "den_prho": ["prho"],
    "den_alpha": ["alpha", "adp"],
    "int_pgra": [],
    "int_readyc": ["wm", "auc", "avc", "aup", "avp", "aupp", "avpp", "fx", "fy"],
    "int_trop": [],
    "int_clin": ["uc", "vc", "up", "vp", "am"],
    "int_ssh": ["alpha"],
    "int_ts": ["wm", "tc", "sc", "tp", "sp"],
}
# 2-D fields the barotropic subcycle reads on every row, by the subroutine
# that writes them on its own rows; (name, planes): planes = None for a 2-D
# field, 1 for the first level of a 3-D field
GATHER_2D = {
    "int_pgra": [(f"{b}_{s}", None) for b in ("bphi", "bgraphi") for s in ("xn", "xs", "ye", "yw")],
    "int_readyc": [("ut", None), ("vt", None)],
    "int_clin": [("am", 1)],
}
# accumulators: written on the window, read only at their own point
ACCUM_3D = {"int_clin": ["acu", "acv"], "int_ts": ["act", "acs", "acr", "acw"], "int_ssh": []}


# ------------------------------------------------------------------ the split
def split_extent(n: int, parts: int) -> list[tuple[int, int]]:
    """(first, last) 1-based interior indices of each part: n // parts each,
    one more for the first n % parts parts (mod_param.f90:313-324)."""
    q, m = divmod(n, parts)
    out = []
    for p in range(1, parts + 1):
        if p <= m:
            last = p * (q + 1)
            size = q + 1
        else:
            last = p * q + m
            size = q
        out.append((last - size + 1, last))
    return out


def rank_position(rank: int, px: int, py: int) -> tuple[int, int]:
    """1-based (i, j) of a rank on the px x py grid: ids = reshape(0..npro-1,
    (px, py)), column-major (set_ids, mod_param.f90:344-369)."""
    if not 0 <= rank < px * py:
        raise ValueError(f"rank {rank} outside a {px} x {py} grid")
    return rank % px + 1, rank // px + 1


def neighbours(rank: int, px: int, py: int) -> dict:
    """n/s (None at the edges: MPI_PROC_NULL) and e/w (wrapping) neighbour
    ranks (get_neighbor, mod_param.f90:279-311,326-334)."""
    i, j = rank_position(rank, px, py)
    ids = lambda ii, jj: (ii - 1) + px * (jj - 1)
    return {"s": ids(i, j - 1) if j > 1 else None, "n": ids(i, j + 1) if j < py else None,
            "w": ids(i - 1 if i > 1 else px, j), "e": ids(i + 1 if i < px else 1, j)}


@dataclass(frozen=True)
class Slab:
    rank: int
    lo: int              # first padded row this rank owns (1-based)
    hi: int              # last padded row this rank owns
    south: int | None    # neighbour ranks
    north: int | None
    win_lo: int          # rows its 3-D kernels compute: own rows +- halo
    win_hi: int


def slabs(glo_nj: int, ranks: int, halo: int) -> list[Slab]:
    """Row slabs of a glo_nj-row domain over `ranks` ranks (npx = 1).  The
    padded rows are 1..glo_nj+2; interior row g is padded row g + 1.  The
    south-most rank also owns padded row 1 and the north-most padded row nj
    (the boundary rows the reference leaves to MPI_PROC_NULL)."""
    nj = glo_nj + 2
    ext = split_extent(glo_nj, ranks)
    out = []
    for r, (gs, gn) in enumerate(ext):
        lo = 1 if r == 0 else gs + 1
        hi = nj if r == ranks - 1 else gn + 1
        if gn - gs + 1 < halo:
            raise ValueError(f"{glo_nj} rows over {ranks} ranks leaves rank {r} {gn - gs + 1} rows, "
                             f"fewer than the {halo}-row halo")
        nb = neighbours(r, 1, ranks)
        out.append(Slab(r, lo, hi, nb["s"], nb["n"], max(1, lo - halo), min(nj, hi + halo)))
    return out


# --------------------------------------------------------------- the engine
class _Cai:
    """A device array for torch.as_tensor (CUDA array interface)."""

    def __init__(self, ptr: int, n: int, elem: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8" if elem == 8 else "<f4",
                                         "data": (ptr, False), "version": 3, "strides": None}


class GpuSlab:
    """One rank's handle (pcom_b200.model.Model) computing its window of rows."""

    def __init__(self, model, slab: Slab, stream=None):
        import torch

        if model.host_only:
            raise ValueError("a slab needs a device handle")
        self.m = model
        self.slab = slab
        self.ni, self.nj, self.nk = model.ni, model.nj, model.nk
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        model.set_stream(self.stream.cuda_stream)
        L.check(model.lib.pcom_gpu_set_rows(model.handle, slab.win_lo, slab.win_hi), "set_rows")

    def views(self, name: str):
        """The named device array as [planes, nj, width] torch tensors sharing
        its memory (the current buffer: ask again after every step)."""
        import torch

        ptr, n, eb = C.c_void_p(), C.c_int64(), C.c_int32()
        L.check(self.m.lib.pcom_gpu_field_ptr(self.m.handle, name.encode(), C.byref(ptr), C.byref(n), C.byref(eb)),
                f"field_ptr {name}")
        t = torch.as_tensor(_Cai(ptr.value, n.value, eb.value), device=self.stream.device)
        width = self.ni * (2 if name == "prho" else 1)  # prho: (d/dT, d/dS) pairs per point
        return [t.view(n.value // (width * self.nj), self.nj, width)]

    def begin_step(self):
        it, day = C.c_int64(), C.c_int32()
        L.check(self.m.lib.pcom_model_begin_step(self.m._m, C.byref(it), C.byref(day)), "begin_step")
        return int(it.value), bool(day.value)

    def phase(self, name: str, it: int):
        self.m.phase(name, it)

    def end_step(self):
        L.check(self.m.lib.pcom_model_end_step(self.m._m), "end_step")

    def sync(self):
        self.stream.synchronize()


# ---------------------------------------------------------------- transport
def _rows(t, a: int, b: int):
    """Rows a..b (padded, 1-based) of a [planes, nj, width] tensor."""
    return t[:, a - 1:b, :]


class LocalLinks:
    """Every rank in this process: rows move by copies between the ranks'
    arrays (one device, or several visible to one process)."""

    def __init__(self, engines: dict):
        self.engines = engines

    def local_ranks(self):
        return sorted(self.engines)

    def exchange(self, names: list[str], halo: int):
        if not names:
            return
        for e in self.engines.values():
            e.sync()
        for r, e in self.engines.items():
            s = e.slab
            for nb, a, b in ((s.south, s.lo - halo, s.lo - 1), (s.north, s.hi + 1, s.hi + halo)):
                if nb is None:
                    continue
                src = self.engines[nb]
                for name in names:
                    for d, o in zip(e.views(name), src.views(name)):
                        _rows(d, a, b).copy_(_rows(o, a, b))
        self._settle()

    def gather(self, specs: list[tuple[str, int | None]]):
        if not specs:
            return
        for e in self.engines.values():
            e.sync()
        for r, e in self.engines.items():
            for q, o in self.engines.items():
                if q == r:
                    continue
                for name, planes in specs:
                    for d, sv in zip(e.views(name), o.views(name)):
                        lo, hi = o.slab.lo, o.slab.hi
                        p = d.shape[0] if planes is None else planes
                        d[:p, lo - 1:hi, :].copy_(sv[:p, lo - 1:hi, :])
        self._settle()

    def _settle(self):
        import torch

        if any(getattr(e, "stream", None) is not None for e in self.engines.values()):
            torch.cuda.synchronize()


class DistLinks:
    """One rank per process: rows move with torch.distributed (NCCL for CUDA
    tensors between GPUs, gloo for CPU tensors).  Every rank takes the same
    collective steps in the same order."""

    def __init__(self, engine, world: int, group=None):
        self.engine = engine
        self.world = world
        self.group = group

    def local_ranks(self):
        return [self.engine.slab.rank]

    def exchange(self, names: list[str], halo: int):
        import torch
        import torch.distributed as dist

        if not names or self.world == 1:
            return
        e = self.engine
        e.sync()
        s = e.slab
        sends, recvs, ops = {}, {}, []
        for nb, own, ghost in ((s.south, (s.lo, s.lo + halo - 1), (s.lo - halo, s.lo - 1)),
                               (s.north, (s.hi - halo + 1, s.hi), (s.hi + 1, s.hi + halo))):
            if nb is None:
                continue
            views = [v for name in names for v in e.views(name)]
            sends[nb] = torch.cat([_rows(v, *own).reshape(-1) for v in views])
            recvs[nb] = (torch.empty_like(sends[nb]), views, ghost)
            ops.append(dist.P2POp(dist.isend, sends[nb], nb, group=self.group))
            ops.append(dist.P2POp(dist.irecv, recvs[nb][0], nb, group=self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for nb, (buf, views, (a, b)) in recvs.items():
            o = 0
            for v in views:
                dst = _rows(v, a, b)
                n = dst.numel()
                dst.copy_(buf[o:o + n].view_as(dst))
                o += n
        if buf_device_is_cuda(e):
            torch.cuda.synchronize()

    def gather(self, specs: list[tuple[str, int | None]]):
        import torch
        import torch.distributed as dist

        if not specs or self.world == 1:
            return
        e = self.engine
        e.sync()
        s = e.slab
        allslabs = slabs(e.nj - 2, self.world, 0)
        maxrows = max(x.hi - x.lo + 1 for x in allslabs)
        views = []
        for name, planes in specs:
            for v in e.views(name):
                views.append(v[: (v.shape[0] if planes is None else planes)])
        per_row = sum(v.shape[0] * v.shape[2] for v in views)
        mine = torch.zeros(maxrows * per_row, dtype=views[0].dtype, device=views[0].device)
        o = 0
        for v in views:
            blk = v[:, s.lo - 1:s.hi, :]
            mine[o:o + blk.numel()] = blk.reshape(-1)
            o += v.shape[0] * maxrows * v.shape[2]
        out = torch.empty(self.world * mine.numel(), dtype=mine.dtype, device=mine.device)
        dist.all_gather_into_tensor(out, mine, group=self.group)
        for q, x in enumerate(allslabs):
            if q == s.rank:
                continue
            src = out[q * mine.numel():(q + 1) * mine.numel()]
            o = 0
            for v in views:
                dst = v[:, x.lo - 1:x.hi, :]
                n = dst.numel()
                dst.copy_(src[o:o + n].view_as(dst))
                o += v.shape[0] * maxrows * v.shape[2]
        if buf_device_is_cuda(e):
            torch.cuda.synchronize()


def buf_device_is_cuda(engine) -> bool:
    return getattr(engine, "stream", None) is not None


# ------------------------------------------------------------------- driver
class SlabDriver:
    """The time loop of main.f90:158-238 over row slabs: on every rank, the
    step's subroutines in order, each followed by the refresh of the halo
    rows it invalidated, and the all-gather of the 2-D rows the barotropic
    subcycle reads.  `after_phase(name)` (optional) runs after each refresh,
    before the all-gather."""

    def __init__(self, links, halo: int, after_phase=None):
        self.links = links
        self.halo = halo
        self.after_phase = after_phase

    def _engines(self):
        lk = self.links
        return [lk.engines[r] for r in lk.local_ranks()] if isinstance(lk, LocalLinks) else [lk.engine]

    def _refresh(self, name: str):
        self.links.exchange(HALO_3D.get(name, []), self.halo)
        if self.after_phase:
            self.after_phase(name)
        self.links.gather(GATHER_2D.get(name, []))

    def step(self):
        es = self._engines()
        starts = [e.begin_step() for e in es]
        it, day = starts[0]
        if any(s != starts[0] for s in starts):
            raise RuntimeError("the ranks' calendars differ")
        if day:
            self._refresh("den_prho")
        for ph in PHASES:
            for e in es:
                e.phase(ph, it)
            self._refresh(ph)
        for e in es:
            e.end_step()
        return it

    def run(self, nsteps: int):
        for _ in range(nsteps):
            self.step()
