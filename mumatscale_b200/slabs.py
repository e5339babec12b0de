"""One domain split into z-slabs, one process per device (torch.distributed).

The reference runs a domain as NSubblocks MPI ranks that swap halo planes
and new-grain lists inside every step (calculate.c:193-352).  Here each
process owns one z-slab of whole subblock layers (:class:`SlabDomain`) and
a step is three launch phases around two exchange points, whose transfers
the library lists (``mms_slab_exchange_plan``):

* point 0, after nucleation: the cl and fs boundary planes, and an
  all-gather of every slab's {candidates, short of draws};
* point 1, after the stencil: the fs, gr, dc and solid-bitmask boundary
  planes, and an all-gather of every slab's new grains.

Reductions (fraction solid, solid volume, ce sum) are each slab's own sum
followed by an all-reduce over the group.

Transports: ``"nccl"`` runs the plane swaps as batched NCCL send/recv and
the gathers as NCCL all-gathers, straight from device memory on the
slab's stream; ``"host"`` stages every transfer through host memory, for
process groups whose backend only moves host tensors (gloo).
"""
from __future__ import annotations

from . import PREC_F64, XFER_GATHER, XFER_HALO, Params, SlabDomain

__all__ = ["DistributedSlab", "exchange"]


class _DeviceBytes:
    """A device allocation of the library seen as a torch uint8 tensor."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {
            "shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
            "version": 3, "strides": None, "stream": None,
        }


def exchange(entries, group=None) -> None:
    """Runs one exchange point: ``entries`` are (kind, peer, send, recv)
    with torch tensors of bytes.  Halo entries to the same peer are issued
    in list order on both sides, so they pair one to one; a gather entry's
    ``recv`` holds world-size contributions of ``send``'s size in rank
    order."""
    import torch.distributed as dist
    ops = []
    for kind, peer, send, recv in entries:
        if kind == XFER_HALO:
            ops.append(dist.P2POp(dist.isend, send, peer, group))
            ops.append(dist.P2POp(dist.irecv, recv, peer, group))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    world = dist.get_world_size(group)
    for kind, _, send, recv in entries:
        if kind != XFER_GATHER:
            continue
        if dist.get_backend(group) == "nccl":
            dist.all_gather_into_tensor(recv, send, group=group)
        else:
            chunks = list(recv.view(world, -1).unbind(0))
            dist.all_gather(chunks, send, group=group)


class DistributedSlab:
    """This process's slab of a domain split over the ranks of ``group``
    (slab index = rank)."""

    def __init__(self, params: Params, precision: int = PREC_F64, device: int = 0, group=None,
                 transport: str | None = None, chunk: int = 64):
        import torch
        import torch.distributed as dist
        self.group = group
        self.params = params
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        torch.cuda.set_device(device)
        self.device = torch.device("cuda", device)
        self.dom = SlabDomain(params, self.world, self.rank, precision, device)
        self.stream = torch.cuda.Stream(device=self.device)
        self.dom.set_stream(self.stream.cuda_stream)
        if transport is None:
            transport = "nccl" if dist.get_backend(group) == "nccl" else "host"
        if transport not in ("nccl", "host"):
            raise ValueError("transport must be 'nccl' or 'host'")
        self.transport = transport
        self.chunk = chunk

    def _entries(self, point: int, ts: int):
        import torch
        out = []
        for kind, peer, send, recv, nbytes in self.dom.exchange_plan(point, ts):
            s = torch.as_tensor(_DeviceBytes(send, nbytes), device=self.device)
            r_bytes = nbytes * (self.world if kind == XFER_GATHER else 1)
            r = torch.as_tensor(_DeviceBytes(recv, r_bytes), device=self.device)
            out.append((kind, peer, s, r))
        return out

    def _exchange(self, point: int, ts: int) -> None:
        import torch
        entries = self._entries(point, ts)
        if not entries:
            return
        with torch.cuda.stream(self.stream):
            if self.transport == "nccl":
                exchange(entries, self.group)
                return
            host = [(k, p, s.cpu(), r.cpu()) for k, p, s, r in entries]  # ordered after the launches
            exchange(host, self.group)
            for (_, _, _, r), (_, _, _, hr) in zip(entries, host):
                r.copy_(hr)

    def _one(self, ts: int, resume: bool) -> None:
        self.dom.launch(0, resume)
        self._exchange(0, ts)
        self.dom.launch(1)
        self._exchange(1, ts)
        self.dom.launch(2)

    def _agree(self, t: int, stalled: bool) -> None:
        """Every slab must be at the same step with the same stall state."""
        import torch
        import torch.distributed as dist
        dev = self.device if dist.get_backend(self.group) == "nccl" else "cpu"
        v = torch.tensor([t, int(stalled), -t, -int(stalled)], dtype=torch.int64, device=dev)
        dist.all_reduce(v, op=dist.ReduceOp.MAX, group=self.group)
        if int(v[0]) != -int(v[2]) or int(v[1]) != -int(v[3]):
            raise RuntimeError("slabs diverged (timestep or stall state differs between ranks)")

    def step(self, nsteps: int = 1) -> None:
        ts, stalled = self.dom.poll()
        self._agree(ts, stalled)
        if stalled:
            raise RuntimeError("slab is stalled before stepping")
        target = ts + int(nsteps)
        while ts < target:
            for k in range(min(self.chunk, target - ts)):
                self._one(ts + k, False)
            t, stalled = self.dom.poll()
            self._agree(t, stalled)
            if stalled:
                # every slab stalled at step t + 1's activation; the steps
                # launched after it did nothing
                self.dom.refill()
                self._one(t, True)
                ts = t + 1
                continue
            ts = t

    def reduce(self, what: str = "fs_fraction") -> float:
        """The whole domain's value: this slab's sum, then a sum over the
        group's ranks (computeFS's MPI_Allreduce, loop.c:173-183; the
        summation order differs from one domain's).  Every rank calls it."""
        import torch
        import torch.distributed as dist
        local = self.dom.reduce("solid_volume" if what == "fs_fraction" else what)
        dev = self.device if dist.get_backend(self.group) == "nccl" else "cpu"
        t = torch.tensor([local], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        v = float(t.item())
        if what == "fs_fraction":
            nx, ny, nz = self.params.grid
            v /= nx * ny * nz * self.params.cellSize ** 3
        return v

    @property
    def timestep(self) -> int:
        return self.dom.timestep

    def close(self) -> None:
        self.stream.synchronize()
        self.dom.close()
