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

Transports: ``"nccl"`` hands the whole step loop to the library
(``mms_slab_nccl_step``): the phase launches and, at each exchange point,
one NCCL group (send/recv of the planes with the neighbouring slabs, an
all-gather of the lists) on the slab's stream, through a communicator of
the library's own whose id rank 0 sends to the others; Python makes one
call per ``step``.  ``"host"`` stages every transfer through host memory
and drives the step from Python, for process groups whose backend only
moves host tensors (gloo).
"""
from __future__ import annotations

import ctypes as C
import os

from . import PREC_F64, XFER_GATHER, XFER_HALO, Params, SlabDomain, _check, _lib

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


def nccl_library_path() -> str | None:
    """The libnccl torch uses (its nvidia-nccl wheel), so that the library
    binds to the same NCCL the process already has; None: let the dynamic
    loader find libnccl.so.2."""
    try:
        import nvidia.nccl
        for d in nvidia.nccl.__path__:
            f = os.path.join(d, "lib", "libnccl.so.2")
            if os.path.exists(f):
                return f
    except Exception:
        pass
    return None


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
        self._plans = {}
        if transport == "nccl":
            self._nccl_init()

    def _nccl_init(self) -> None:
        """Joins the library's NCCL communicator of the group: rank 0 makes
        the unique id and the group's collective sends it to every rank."""
        import torch.distributed as dist
        path = nccl_library_path()
        self._nccl_path = path.encode() if path else None
        uid = C.create_string_buffer(128)
        if self.rank == 0:
            _check(_lib().mms_slab_nccl_unique_id(self._nccl_path, uid), "mms_slab_nccl_unique_id")
        box = [uid.raw if self.rank == 0 else None]
        dist.broadcast_object_list(box, src=dist.get_global_rank(self.group, 0) if self.group else 0,
                                   group=self.group)
        uid = C.create_string_buffer(box[0], 128)
        _check(_lib().mms_slab_nccl_init(self.dom._ctx, self._nccl_path, uid), "mms_slab_nccl_init", self.dom._ctx)

    def _entries(self, point: int, ts: int):
        """The transfers of an exchange point as tensors over the library's
        buffers.  The plan depends on the step only through its parity
        (which of the two cl / fs buffers is current), so it is built once
        per (point, parity)."""
        import torch
        key = (point, ts & 1)
        if key not in self._plans:
            out = []
            for kind, peer, send, recv, nbytes in self.dom.exchange_plan(point, ts):
                s = torch.as_tensor(_DeviceBytes(send, nbytes), device=self.device)
                r_bytes = nbytes * (self.world if kind == XFER_GATHER else 1)
                r = torch.as_tensor(_DeviceBytes(recv, r_bytes), device=self.device)
                out.append((kind, peer, s, r))
            self._plans[key] = out
        return self._plans[key]

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
        if self.transport == "nccl":
            _check(_lib().mms_slab_nccl_step(self.dom._ctx, int(nsteps)), "mms_slab_nccl_step", self.dom._ctx)
            return
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
        if self.transport == "nccl":
            from . import REDUCE
            v = C.c_double()
            _check(_lib().mms_slab_nccl_reduce(self.dom._ctx, REDUCE[what], C.byref(v)), "mms_slab_nccl_reduce",
                   self.dom._ctx)
            return v.value
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
