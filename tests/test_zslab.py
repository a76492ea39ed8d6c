"""Z-slab decomposition (the reference's MPI scheme along z, mpicomm.F90).

CPU: the partition and the halo schedule, and the halo message pattern of
the one-slab-per-rank form over torch.distributed (gloo, two ranks).  GPU:
the slabs of one process, exchanging their halo planes through device
copies, reproduce the single-domain run bit for bit."""
import os
import socket

import numpy as np

from bits import assert_bits_equal
import pytest

from cases import disp, mdisp, mixed, mur, small
from semba_fdtd_b200 import zslab

CASES = {"small": lambda: small(n=16, steps=40, layers=4), "disp": disp, "mdisp": mdisp, "mur": mur}


def test_partition_tiles_the_swept_planes():
    pb = disp()
    lo, hi = zslab._global_sweep(pb)
    for n in (1, 2, 3, 5):
        b = zslab.partition(pb, n)
        assert len(b) == n and b[0][0] < lo and b[-1][1] > hi
        for q in range(n - 1):
            assert b[q + 1][0] == b[q][1] + 1
        inner = [min(z1, hi) - max(z0, lo) + 1 for z0, z1 in b]
        assert sum(inner) == hi - lo + 1 and min(inner) >= 2 and max(inner) - min(inner) <= 1
    with pytest.raises(ValueError):
        zslab.partition(pb, hi - lo + 1)


def test_halo_schedule():
    b = [(-10, 4), (5, 9), (10, 20)]
    s = zslab.halo_schedule(b)
    assert ("E", 1, 0, (0, 1), 5) in s and ("H", 0, 1, (3, 4), 4) in s
    assert ("E", 2, 1, (0, 1), 10) in s and ("H", 1, 2, (3, 4), 9) in s
    assert len(s) == 4


class _Planes:
    """Host planes standing in for the device planes of each rank."""

    def __init__(self, bounds, n=8):
        import torch
        self.bounds = bounds
        self.store = {}
        self.n = n
        self.torch = torch

    def __call__(self, rank, comp, z):
        key = (rank, comp, z)
        if key not in self.store:
            self.store[key] = self.torch.full((self.n,), float(1000 * rank + 10 * comp + z % 10))
        return self.store[key]


def _gloo_worker(rank, world, port, bounds, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        planes = _Planes(bounds)
        zslab.run_distributed(None, 2, planes=planes)
        out.put((rank, {k: v.tolist() for k, v in planes.store.items()}))
    finally:
        dist.destroy_process_group()


def test_distributed_halo_messages_gloo():
    import torch.multiprocessing as mp
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    bounds = [(-100, 4), (5, 100)]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, bounds, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # after the E exchange rank 0 holds rank 1's Ex, Ey of plane 5; after the
    # H exchange rank 1 holds rank 0's Hx, Hy of plane 4
    for c in (0, 1):
        assert got[0][(0, c, 5)] == [1000.0 + 10 * c + 5] * 8
    for c in (3, 4):
        assert got[1][(1, c, 4)] == [0.0 + 10 * c + 4] * 8


@pytest.mark.gpu
@pytest.mark.parametrize("nslabs", [2, 3])
@pytest.mark.parametrize("name", list(CASES))
def test_zslabs_bit_exact(name, nslabs):
    from semba_fdtd_b200 import Solver
    pb = CASES[name]()
    steps = 37
    with Solver(pb) as s:
        s.step(steps)
        ref_tr = s.probes()
        ref = [s.field(c) for c in range(6)]
    with zslab.ZSlabs(pb, nslabs) as z:
        z.step(steps)
        assert_bits_equal(z.probes(), ref_tr)
        for c in range(6):
            assert_bits_equal(z.field(c), ref[c], err_msg=f"component {c}")


@pytest.mark.gpu
def test_zslabs_reject_periodic_z():
    from semba_fdtd_b200._lib import SembaGpuError
    with pytest.raises(SembaGpuError):
        zslab.ZSlabs(mixed(), 2)


@pytest.mark.gpu
def test_distributed_single_rank_on_the_context_stream():
    """run_distributed with one rank: no halo message, but the whole step
    loop of the distributed form (its messages ordered on the context's own
    stream, from sgpu_get_stream) runs and equals the plain run bit for bit."""
    import torch.distributed as dist
    from semba_fdtd_b200 import Solver
    pb = CASES[next(iter(CASES))]()
    steps = 23
    with Solver(pb) as s:
        s.step(steps)
        ref_tr = s.probes()
        ref = [s.field(c) for c in range(6)]
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
    try:
        d = zslab.run_distributed(pb, steps)
        try:
            d.synchronize()
            assert_bits_equal(d.probes(), ref_tr)
            for c in range(6):
                assert_bits_equal(d.field(c), ref[c])
        finally:
            d.close()
    finally:
        dist.destroy_process_group()
