"""Slab decomposition of one large box over ranks (one process per GPU).

A single case too large for one GPU splits along its slowest direction (y in 2-D,
z in 3-D) into contiguous slabs, one per rank.  The explicit update of a slab
reads `ghost` cells beyond it along every direction; those along the split
direction belong to the neighbouring ranks, so one step is preceded by one
exchange: each rank sends its first and last `ghost` planes of valid cells to
the rank below and above and receives theirs into its ghost planes.  The domain
ends keep their own ghost planes (the boundary fill, vd_fill_ghosts), or wrap
around in a periodic direction.  The common time step is the minimum over ranks
of each rank's limit (Source/TimeStep.cpp:113-115, ParallelDescriptor::ReduceRealMin).

The exchange uses torch.distributed point-to-point messages: NCCL between GPUs
over NVLink (device tensors), gloo between CPU processes (host tensors).  Every
rank posts the same sends and receives in the same order.  The slab's own update
is the per-box entry point on the slab with the global domain passed in
vd_params (domlo/domhi in the slab's index space), so the domain faces stay where
they are.
"""
from __future__ import annotations

from dataclasses import dataclass

import torch
import torch.distributed as dist


def split_extent(n: int, world: int, rank: int):
    """Cells [lo, hi] (inclusive) of rank's slab when n cells split over world ranks
    as evenly as possible (the first n % world ranks take one more)."""
    if n < world:
        raise ValueError(f"{n} cells cannot give {world} ranks a slab each")
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0) - 1


@dataclass
class Slab:
    """Rank's slab of a box of n_global cells (x, y, z) in `dim` dimensions, with
    `ghost` ghost cells on every side of every active direction."""
    n_global: tuple
    dim: int
    ghost: int
    rank: int
    world: int
    periodic: bool = False

    @property
    def axis(self) -> int:
        """The split direction (0 x, 1 y, 2 z): the slowest active one."""
        return self.dim - 1

    @property
    def extent(self):
        return split_extent(self.n_global[self.axis], self.world, self.rank)

    @property
    def n_local(self) -> tuple:
        lo, hi = self.extent
        n = list(self.n_global)
        n[self.axis] = hi - lo + 1
        return tuple(n)

    def window(self, d: int) -> slice:
        """Index range, along direction d of an array over the global box grown by
        `ghost`, of this slab's cells and ghosts."""
        if d != self.axis:
            return slice(None)
        lo, hi = self.extent
        return slice(lo, hi + 1 + 2 * self.ghost)

    def domain_in_slab(self):
        """(domlo, domhi) of the global domain in the slab's index space (the slab
        starts at 0): the values vd_params takes for the slab's update."""
        lo, _ = self.extent
        domlo = [0, 0, 0]
        domhi = [self.n_global[d] - 1 for d in range(3)]
        domlo[self.axis] -= lo
        domhi[self.axis] -= lo
        return domlo, domhi

    def neighbours(self):
        """(rank below, rank above) along the split direction; None at a domain end
        of a non-periodic direction."""
        below = self.rank - 1 if self.rank > 0 else (self.world - 1 if self.periodic else None)
        above = self.rank + 1 if self.rank < self.world - 1 else (0 if self.periodic else None)
        return below, above

    def exchange(self, state: torch.Tensor, group=None) -> None:
        """Fill the ghost planes of `state` (ncomp, z, y, x over the slab grown by
        `ghost`) along the split direction from the neighbouring ranks, in place."""
        if self.world == 1 and not self.periodic:
            return
        g = self.ghost
        ax = 3 - self.axis                     # tensor axis of the split direction
        n = state.shape[ax] - 2 * g            # valid planes of this slab
        if n < g:
            raise ValueError(f"slab of {n} planes is thinner than the {g} ghost planes")
        if self.world == 1:
            # one rank, periodic: the wrap is local
            lo_src = state.narrow(ax, n, g).clone()
            hi_src = state.narrow(ax, g, g).clone()
            state.narrow(ax, 0, g).copy_(lo_src)
            state.narrow(ax, n + g, g).copy_(hi_src)
            return
        below, above = self.neighbours()
        send_lo = state.narrow(ax, g, g).contiguous()          # first valid planes, to the rank below
        send_hi = state.narrow(ax, n, g).contiguous()          # last valid planes, to the rank above
        recv_lo = torch.empty_like(send_lo)                    # from the rank below: its last planes
        recv_hi = torch.empty_like(send_hi)                    # from the rank above: its first planes
        # Messages between one pair of ranks match in the order they are posted, and
        # with two ranks in a periodic direction the rank below is also the rank
        # above: so every rank posts the upward shift first (its last planes up,
        # the planes of the rank below into its low ghosts), then the downward one.
        ops = []
        if above is not None:
            ops.append(dist.P2POp(dist.isend, send_hi, above, group))
        if below is not None:
            ops.append(dist.P2POp(dist.irecv, recv_lo, below, group))
        if below is not None:
            ops.append(dist.P2POp(dist.isend, send_lo, below, group))
        if above is not None:
            ops.append(dist.P2POp(dist.irecv, recv_hi, above, group))
        if ops:
            for w in dist.batch_isend_irecv(ops):
                w.wait()
        if below is not None:
            state.narrow(ax, 0, g).copy_(recv_lo)
        if above is not None:
            state.narrow(ax, n + g, g).copy_(recv_hi)

    @staticmethod
    def common_dt(local_dt: float, device="cpu", group=None) -> float:
        """The minimum over ranks of the local time-step limits."""
        t = torch.tensor([local_dt], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
        return float(t.item())
