"""Band-parallel steepest descent of one cell over the ranks of a process
group (one rank per GPU).

Rank r transforms, densifies and steps the contiguous bands [lo_r, hi_r)
(``band_ranges``); per SD step the ranks exchange twice:

* the spin densities, summed over the ranks after the density pass
  (ccpsdv3/cpsd.c:185-194) -- an all-reduce of ispin n^3 doubles;
* the new orbitals and -H psi of every rank's bands after the
  steepest-descent update (cpsd.c:399-400) -- an all-gather of the packed
  coefficient rows.

The overlaps, the Lagrange iteration, the constraint correction and the
energies (cpsd.c:415-646) then run on the full arrays on every rank, so
every rank holds the same state after a step.  The reference's own split is
a grid decomposition with FFT transposes (ccpsdv3-mpi/d3db-mpi.c); bands
shard the dominant cost here (the per-band transforms) with two exchanges
and no transposes.
"""
from __future__ import annotations

from typing import List, Sequence, Tuple


def band_ranges(nbands: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous [lo, hi) per rank, sizes differing by at most one (the
    first nbands % world ranks take one more); ranks beyond nbands get an
    empty range."""
    if world < 1 or nbands < 0:
        raise ValueError("need world >= 1 and nbands >= 0")
    base, extra = divmod(nbands, world)
    out, lo = [], 0
    for r in range(world):
        hi = lo + base + (1 if r < extra else 0)
        out.append((lo, hi))
        lo = hi
    return out


def spin_split(lo: int, hi: int, ne0: int) -> Tuple[int, int]:
    """Bands of spin 0 and of spin 1 inside [lo, hi) (spin 1 starts at ne0)."""
    n0 = max(0, min(hi, ne0) - lo)
    return n0, (hi - lo) - n0


def torch_exchange(dist, ranges: Sequence[Tuple[int, int]]):
    """The two exchanges over a torch.distributed process group, on host
    (numpy) arrays in place: (allreduce_sum(a), allgather_rows(a2d)).  Every
    rank makes the same calls in the same order."""
    import torch

    def allreduce_sum(a):
        t = torch.from_numpy(a)
        dist.all_reduce(t)

    def allgather_rows(a2d):
        t = torch.from_numpy(a2d)
        for r, (lo, hi) in enumerate(ranges):
            if hi > lo:
                dist.broadcast(t[lo:hi], src=r)

    return allreduce_sum, allgather_rows


class _DeviceArray:
    """A device buffer of the library as a __cuda_array_interface__ object
    (float64, C order), so torch can wrap it without a copy."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(int(x) for x in shape), "typestr": "<f8",
                                         "data": (int(ptr), False), "version": 3, "strides": None}


def device_tensor(torch, ptr: int, shape, device: int):
    return torch.as_tensor(_DeviceArray(ptr, shape), device="cuda:%d" % device)


class RankBuffers:
    """torch views of one context's exchanged arrays for the current step."""

    def __init__(self, torch, cell):
        dn_part, dn, c2, cpsi, ld = cell.bp_buffers()
        inp = cell.inp
        n3 = inp.ispin * inp.nfft ** 3
        dev = cell.device
        self.dn_part = device_tensor(torch, dn_part, (n3,), dev)
        self.dn = device_tensor(torch, dn, (n3,), dev)
        self.c2 = device_tensor(torch, c2, (inp.nbands, ld), dev)
        self.cpsi = device_tensor(torch, cpsi, (inp.nbands, ld), dev)


class TorchExchange:
    """The exchanges of one rank per process over a torch.distributed
    process group (NCCL on GPUs): an all-reduce of the densities and one
    broadcast per rank of its orbital rows, on the cell's stream."""

    def __init__(self, torch, dist, cell, ranges):
        self.torch, self.dist, self.cell, self.ranges = torch, dist, cell, list(ranges)
        self.stream = torch.cuda.ExternalStream(cell.stream, device="cuda:%d" % cell.device)

    def sum_densities(self):
        b = RankBuffers(self.torch, self.cell)
        with self.torch.cuda.stream(self.stream):
            b.dn.copy_(b.dn_part)
            self.dist.all_reduce(b.dn)

    def gather_rows(self, which):
        b = RankBuffers(self.torch, self.cell)
        t = getattr(b, which)
        with self.torch.cuda.stream(self.stream):
            for r, (lo, hi) in enumerate(self.ranges):
                if hi > lo:
                    self.dist.broadcast(t[lo:hi], src=r)


class LocalGroup:
    """The same exchanges among contexts of one process (ranks emulated on
    one GPU, stepped phase by phase): the densities summed in rank order,
    every rank's rows copied to the others."""

    def __init__(self, torch, cells, ranges):
        self.torch, self.cells, self.ranges = torch, list(cells), list(ranges)

    def sum_densities(self):
        self.torch.cuda.synchronize()
        bufs = [RankBuffers(self.torch, c) for c in self.cells]
        acc = bufs[0].dn_part.clone()
        for b in bufs[1:]:
            acc += b.dn_part
        for b in bufs:
            b.dn.copy_(acc)
        self.torch.cuda.synchronize()

    def gather_rows(self, which):
        self.torch.cuda.synchronize()
        bufs = [RankBuffers(self.torch, c) for c in self.cells]
        for q, (lo, hi) in enumerate(self.ranges):
            for r, b in enumerate(bufs):
                if r != q and hi > lo:
                    getattr(b, which)[lo:hi].copy_(getattr(bufs[q], which)[lo:hi])
        self.torch.cuda.synchronize()


def run(cells, exchange, inner: int):
    """`inner` band-parallel SD steps and the energies of the call for this
    process's cells (one per rank: one cell with TorchExchange, all of them
    with LocalGroup): the same call order on every rank."""
    for _ in range(inner):
        for c in cells:
            c.step_phase(0)
        exchange.sum_densities()
        for c in cells:
            c.step_phase(1)
        exchange.gather_rows("c2")
        for c in cells:
            c.step_phase(2)
    exchange.gather_rows("cpsi")
    for c in cells:
        c.bp_finish(inner)
    return [c.E.copy() for c in cells]
