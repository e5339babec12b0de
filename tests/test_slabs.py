"""One domain split into z-slabs (the reference's multi-rank run of one
domain, calculate.c:193-352, as slabs of whole subblock layers).

GPU: the slabs stepped together give the single domain's fields and grain
records bit for bit, and the reference's own field dumps for its 2 x 1 x 2
deck; the per-process driver (host transport over gloo, two processes on
one device) gives the same.  CPU: the slab layout and the exchange
function over two gloo ranks."""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import numpy as np
import pytest

import mumatscale_b200 as M
from conftest import ROOT, golden, golden_deck
from digests import mismatches, state_digests

FIELDS = ("ce", "cl", "fs", "gr", "dc")


def _deck(name: str, nsbz: int | None = None, sdimz: int | None = None) -> M.Params:
    p = M.read_deck(golden_deck(name))
    if nsbz:
        p.gnsbz = nsbz
    if sdimz:
        p.gsdimz = sdimz
    return p


def _grain_table(grains) -> np.ndarray:
    return np.array([list(np.array(g.rotmat).reshape(9)) + list(g.rotang) +
                     [g.nuc_x, g.nuc_y, g.nuc_z, g.nuc_threshold, float(g.nuc_timestep)] for g in grains])


# --------------------------------------------------------------------- CPU
def test_slab_layout_partitions_layers(built):
    p = M.default_params()
    p.gnsbx, p.gnsby, p.gnsbz = 2, 3, 7
    p.gsdimx, p.gsdimy, p.gsdimz = 8, 8, 5
    for n in range(1, 8):
        z = r = 0
        for s in range(n):
            lay = M.slab_layout(p, n, s)
            assert (lay.nslabs, lay.slab) == (n, s)
            assert lay.z_begin == z and lay.rank_begin == r
            assert lay.z_cells % p.gsdimz == 0 and lay.z_cells > 0
            assert lay.rank_count == (lay.z_cells // p.gsdimz) * 6
            z += lay.z_cells
            r += lay.rank_count
        assert z == 35 and r == 42
    for bad in ((8, 0), (2, 2), (0, 0), (3, -1)):
        with pytest.raises(M.MmsError):
            M.slab_layout(p, *bad)


def _exchange_rank(rank: int, world: int, port: int, q) -> None:
    import torch
    import torch.distributed as dist
    from mumatscale_b200.slabs import exchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # two fields of 3 planes x 4 bytes; this rank's interior planes hold
        # its rank id + field number, the halo planes are received
        f = [torch.full((3 * 4,), 100 + 10 * rank + i, dtype=torch.uint8) for i in range(2)]
        ents = []
        peer = 1 - rank
        for i in range(2):
            # rank 0 sends its top interior plane up, rank 1 its bottom one down
            recv = f[i][0:4] if rank == 1 else f[i][8:12]
            ents.append((M.XFER_HALO, peer, f[i][4:8], recv))
        g_send = torch.full((5,), rank + 1, dtype=torch.uint8)
        g_recv = torch.zeros(5 * world, dtype=torch.uint8)
        ents.append((M.XFER_GATHER, -1, g_send, g_recv))
        exchange(ents)
        got_halo = [int((f[i][0:4] if rank == 1 else f[i][8:12])[0]) for i in range(2)]
        q.put((rank, got_halo, g_recv.tolist()))
    finally:
        dist.destroy_process_group()


def test_slab_exchange_two_gloo_ranks():
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_exchange_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = {}
    for _ in ps:
        rank, halo, gath = q.get(timeout=120)
        res[rank] = (halo, gath)
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    # each rank's halo planes hold the other rank's boundary planes, field by field
    assert res[0][0] == [110, 111] and res[1][0] == [100, 101]
    assert res[0][1] == res[1][1] == [1] * 5 + [2] * 5


class _StubSlab:
    """A slab whose own sums are given: the group reduction alone."""

    def __init__(self, sums: dict):
        self.sums = sums

    def reduce(self, what: str) -> float:
        return self.sums[what]


def _reduce_rank(rank: int, world: int, port: int, q) -> None:
    import torch.distributed as dist
    from mumatscale_b200.slabs import DistributedSlab
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = object.__new__(DistributedSlab)
        p = M.default_params()
        p.gnsbx, p.gnsby, p.gnsbz = 1, 1, 2
        p.gsdimx, p.gsdimy, p.gsdimz = 4, 4, 4
        p.cellSize = 2.0
        s.group, s.params, s.device, s.transport = None, p, "cpu", "host"
        s.dom = _StubSlab({"solid_volume": 8.0 * (rank + 1), "ce_sum": 10.0 + rank})
        q.put((rank, s.reduce("fs_fraction"), s.reduce("solid_volume"), s.reduce("ce_sum")))
    finally:
        dist.destroy_process_group()


def test_slab_reductions_two_gloo_ranks():
    """Each rank's sum all-reduced; the fraction solid from the total solid
    volume over the whole domain's volume (4 x 4 x 8 cells of 2^3)."""
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_reduce_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(60)
        assert p.exitcode == 0
    for _, fs, vol, ce in res:
        assert vol == 24.0 and ce == 21.0
        assert fs == 24.0 / (4 * 4 * 8 * 8.0)


# --------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_slabs_match_reference_dumps(built, cuda_device):
    """small4 (NSubblocks 2 x 1 x 2, the reference run as 4 MPI ranks) as
    two slabs: every field and grain record equals the reference's dumps."""
    rec = golden("small4")
    p = M.read_deck(golden_deck("small4"))
    with M.SlabGroup(p, 2) as grp:
        assert [d.layout.z_cells for d in grp.slabs] == [p.gsdimz, p.gsdimz]
        last = 0
        for s, want in rec["steps"].items():
            s = int(s)
            grp.step(s - last)
            last = s
            assert grp.timestep == s
            assert grp.num_grains == want["num_grains"]
            bad = mismatches(state_digests(grp), want["digest"])
            assert not bad, f"step {s}: fields differ from the reference: {bad}"
        assert all(d.uses_tma for d in grp.slabs)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [M.PREC_F64, M.PREC_F32])
@pytest.mark.parametrize("nslabs", [2, 3, 4])
def test_slabs_equal_single_domain(built, cuda_device, prec, nslabs):
    """small4 with 4 layers of 4-cell subblocks: 2, 3 and 4 slabs give the
    single domain's fields and grain records bit for bit, in both forms."""
    p = _deck("small4", nsbz=4, sdimz=4)
    with M.Domain(p, precision=prec) as dom, M.SlabGroup(p, nslabs, precision=prec) as grp:
        for n in (1, 60, 140):
            dom.step(n)
            grp.step(n)
            assert grp.timestep == dom.timestep
            assert grp.num_grains == dom.num_grains
            for f in FIELDS:
                a, b = dom.download(f), grp.download(f)
                assert np.array_equal(a, b), f"{f} differs after step {dom.timestep}"
            ga, gb = _grain_table(dom.grains()), _grain_table(grp.grains())
            assert np.array_equal(ga, gb)
            # every slab holds every grain record
            for d in grp.slabs[1:]:
                assert np.array_equal(_grain_table(d.grains()), gb)
        assert dom.num_grains > 20
        v1 = dom.reduce("fs_fraction")
        assert abs(grp.reduce("fs_fraction") - v1) <= 1e-12 * max(v1, 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", [M.PREC_F64, M.PREC_F32])
def test_slabs_am_quadrature(built, cuda_device, prec):
    """AM deck (moving-source quadrature, whole-domain z in the slab's
    temperature; the FP32 form's contraction on the tensor cores) as two
    slabs: bit for bit the single domain's."""
    p = _deck("am1", nsbz=2, sdimz=6)
    with M.Domain(p, precision=prec) as dom, M.SlabGroup(p, 2, precision=prec) as grp:
        for n in (50, 80):
            dom.step(n)
            grp.step(n)
            assert grp.num_grains == dom.num_grains
            for f in FIELDS + ("temperature",):
                assert np.array_equal(dom.download(f), grp.download(f)), f
        assert dom.num_grains > 1


@pytest.mark.gpu
def test_slab_rejects_curvature_and_lone_step(built, cuda_device):
    p = _deck("curv1")
    p.gnsbz, p.gsdimz = 2, 8
    with pytest.raises(M.MmsError):
        M.SlabDomain(p, 2, 0)
    q = _deck("small4")
    with M.SlabDomain(q, 2, 1) as d:
        with pytest.raises(M.MmsError):
            d.step(1)


@pytest.mark.gpu
def test_distributed_slabs_host_transport(built, cuda_device, tmp_path):
    """The per-process driver: two processes, one slab each, exchanging
    through a gloo group; their fields equal the single domain's."""
    steps, nsbz, sdimz = 150, 4, 4
    deck = str(golden_deck("small4"))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    procs = []
    for r in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(r), WORLD_SIZE="2")
        procs.append(subprocess.Popen(
            [sys.executable, str(ROOT / "tests" / "_slab_worker.py"), "--deck", deck, "--nsbz", str(nsbz),
             "--sdimz", str(sdimz), "--steps", str(steps), "--out", str(tmp_path)], env=env))
    for pr in procs:
        assert pr.wait(timeout=600) == 0
    p = _deck("small4", nsbz=nsbz, sdimz=sdimz)
    with M.Domain(p) as dom:
        dom.step(steps)
        parts = [np.load(tmp_path / f"slab{r}.npz") for r in range(2)]
        for f in FIELDS:
            whole = dom.download(f)
            for q in parts:
                z0 = int(q["z_begin"])
                loc = q[f]
                assert np.array_equal(loc[1:-1], whole[z0 + 1:z0 + loc.shape[0] - 1]), f
        ga = _grain_table(dom.grains())
        want = [dom.reduce(w) for w in ("fs_fraction", "solid_volume", "ce_sum")]
        assert want[0] > 0
        for q in parts:
            assert int(q["timestep"]) == steps
            gb = np.concatenate([q["rot"], q["ang"], q["nuc"]], axis=1)
            assert np.array_equal(ga, gb)
            # the group's all-reduced sums: every rank holds the domain's
            for got, w in zip(q["red"], want):
                assert abs(got - w) <= 1e-12 * abs(w), (got, w)


@pytest.mark.gpu
def test_distributed_slab_nccl_one_rank(built, cuda_device, tmp_path):
    """The library's NCCL path (mms_slab_nccl_*) as far as one GPU allows:
    a one-rank NCCL group holding the whole domain as its one slab.  The
    run-time loading of NCCL, the communicator, the agreement all-reduce and
    the all-reduced sums run; a one-slab group steps like a whole domain, so
    the per-step exchanges (halo send/recv and the all-gathers) need two
    GPUs and do not run here.  The state equals the single domain's bit for
    bit."""
    steps = 150
    deck = str(golden_deck("small4"))
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK="0", WORLD_SIZE="1",
               NCCL_NVLS_ENABLE="0")
    pr = subprocess.run([sys.executable, str(ROOT / "tests" / "_slab_worker.py"), "--deck", deck, "--nsbz", "1",
                         "--sdimz", "16", "--steps", str(steps), "--out", str(tmp_path), "--backend", "nccl"],
                        env=env, timeout=600)
    assert pr.returncode == 0
    p = _deck("small4", nsbz=1, sdimz=16)
    q = np.load(tmp_path / "slab0.npz")
    with M.Domain(p) as dom:
        dom.step(steps)
        for f in FIELDS:
            assert np.array_equal(q[f], dom.download(f)), f
        assert int(q["timestep"]) == steps
        assert np.array_equal(_grain_table(dom.grains()), np.concatenate([q["rot"], q["ang"], q["nuc"]], axis=1))
        want = [dom.reduce(w) for w in ("fs_fraction", "solid_volume", "ce_sum")]
        for got, w in zip(q["red"], want):
            assert abs(got - w) <= 1e-12 * abs(w), (got, w)
