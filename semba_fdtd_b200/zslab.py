"""Z-slab domain decomposition: the reference's MPI scheme (mpicomm.F90:
122-358, 1507-1677; exchanges at timestepping.F90:1453-1459 and 1661-1669)
over several libsemba_gpu contexts.

Each slab is a context built by ``sgpu_host_create_zslab`` for planes
z0..z1 of the problem; a step is

    every slab: E half step (curl, CPML, ADE, E sources)
    halo E:     Ex, Ey of each slab's first owned plane -> the slab below
    every slab: H half step (curl, CPML, magnetic ADE, H sources, borders)
    halo H:     Hx, Hy of each slab's last owned plane  -> the slab above
    every slab: probes

so every cell computes exactly what the single-domain run computes and the
results are equal bit for bit.  ``ZSlabs`` keeps all slabs in one process
(on one or several devices, copies through ``sgpu_copy_zplane``);
``run_distributed`` is the one-slab-per-rank form over torch.distributed,
sending the halo planes with point-to-point messages.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .solver import Solver

__all__ = ["partition", "ZSlabs", "halo_schedule", "run_distributed"]

_BIG = 1 << 30  # bound of the end slabs: they also own the planes beyond the swept range


def _global_sweep(problem):
    lib = _lib.load()
    desc, keep = problem.to_desc(1)
    h = C.c_void_p()
    rc = lib.sgpu_host_plan(C.byref(desc), 1, C.byref(h))
    if rc:
        raise _lib.SembaGpuError(f"sgpu_host_plan failed ({_lib.ERRORS.get(rc, rc)})")
    try:
        a6, s6, q6 = (_lib.Lim * 6)(), (_lib.Lim * 6)(), (_lib.Lim * 6)()
        lib.sgpu_host_info(h, None, None, a6, s6, q6)
        return min(s.zi for s in s6), max(s.ze for s in s6)
    finally:
        lib.sgpu_destroy(h)


def partition(problem, nslabs: int) -> list[tuple[int, int]]:
    """(z0, z1) of each slab: the problem's swept z planes split into nslabs
    contiguous runs of near-equal length (at least two planes each); the first
    slab starts and the last ends at an unbounded plane."""
    lo, hi = _global_sweep(problem)
    n = hi - lo + 1
    if nslabs < 1 or n < 2 * nslabs:
        raise ValueError(f"{n} swept planes cannot be split into {nslabs} slabs of two or more")
    cuts = [lo + (n * q) // nslabs for q in range(nslabs + 1)]
    out = []
    for q in range(nslabs):
        z0 = -_BIG if q == 0 else cuts[q]
        z1 = _BIG if q == nslabs - 1 else cuts[q + 1] - 1
        out.append((z0, z1))
    return out


def halo_schedule(bounds):
    """The plane copies of one step as (phase, src slab, dst slab, comps, z):
    phase 'E' after the E half step, 'H' after the H half step."""
    sched = []
    for q in range(len(bounds) - 1):
        z_top = bounds[q][1]  # last plane slab q owns
        sched.append(("E", q + 1, q, (0, 1), z_top + 1))
        sched.append(("H", q, q + 1, (3, 4), z_top))
    return sched


class ZSlabs:
    """All slabs of a decomposition in one process.  devices: one CUDA device
    index per slab (default: the current device for all)."""

    def __init__(self, problem, nslabs: int, variant: str = "exact", probe_capacity: int = 1024, devices=None):
        self.problem = problem
        self.bounds = partition(problem, nslabs)
        self.lib = _lib.load(variant)
        self.slabs = []
        for q, b in enumerate(self.bounds):
            if devices is not None:
                _cuda_set_device(devices[q])
            self.slabs.append(Solver(problem, variant=variant, probe_capacity=probe_capacity, zslab=b))
        self.sched = halo_schedule(self.bounds)
        self.n = 0

    def close(self):
        for s in self.slabs:
            s.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _halo(self, phase):
        for ph, src, dst, comps, z in self.sched:
            if ph != phase:
                continue
            for c in comps:
                rc = self.lib.sgpu_copy_zplane(self.slabs[dst].handle, self.slabs[src].handle, c, z)
                if rc:
                    self.slabs[dst]._check(rc, "sgpu_copy_zplane")

    def step(self, count: int = 1) -> None:
        lib = self.lib
        for _ in range(count):
            n = self.n
            for s in self.slabs:
                s._check(lib.sgpu_advance_e(s.handle, n), "sgpu_advance_e")
            self._halo("E")
            for s in self.slabs:
                s._check(lib.sgpu_advance_h(s.handle, n), "sgpu_advance_h")
            self._halo("H")
            for s in self.slabs:
                s._check(lib.sgpu_update_observation(s.handle, n), "sgpu_update_observation")
                s.n = n + 1
                if s.nprobes and s._pending() >= s.probe_capacity:
                    s._drain()
            self.n = n + 1

    def probes(self) -> np.ndarray:
        """Probe rows [step, probe] in the problem's probe order."""
        out = np.zeros((self.n, len(self.problem.probes)), np.float32)
        for s in self.slabs:
            ids = s.probe_ids()
            if ids:
                out[:, ids] = s.probes()
        return out

    def field(self, comp: int) -> np.ndarray:
        """The whole component over the problem's Alloc box, [i, j, k]: each
        slab contributes the planes it owns."""
        parts = []
        for s, (z0, z1) in zip(self.slabs, self.bounds):
            f = s.field(comp)
            zi = s.alloc[comp][4]
            k0 = max(z0, zi) - zi
            k1 = min(z1, s.alloc[comp][5]) - zi
            parts.append(f[:, :, k0:k1 + 1])
        return np.concatenate(parts, axis=2)


def _cuda_set_device(dev: int) -> None:
    import torch
    torch.cuda.set_device(dev)


def run_distributed(problem, steps: int, variant: str = "exact", group=None, planes=None):
    """One slab per rank of torch.distributed (NCCL on GPUs): rank r owns
    slab r of ``partition(problem, world)``; the halo planes travel as
    point-to-point messages, the receiver's copy landing in its own plane.
    ``planes`` replaces the device planes by host buffers for tests of the
    message pattern (gloo on CPU): a function (slab, comp, z) -> array.
    Returns this rank's Solver (None with ``planes``)."""
    import torch
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    bounds = partition(problem, world) if planes is None else planes.bounds
    sched = halo_schedule(bounds)
    s = None
    if planes is None:
        s = Solver(problem, variant=variant, zslab=bounds[rank])

    def plane_tensor(comp, z):
        if planes is not None:
            return planes(rank, comp, z)
        ptr, nbytes = C.c_void_p(), C.c_uint64()
        s._check(s.lib.sgpu_zplane(s.handle, comp, z, C.byref(ptr), C.byref(nbytes)), "sgpu_zplane")
        return torch.as_tensor(_DeviceArray(ptr.value, nbytes.value // 4), device="cuda")

    # The messages are ordered on the context's own stream, with no host
    # wait: made current, it is the stream the process group's sends wait on
    # (the half step that wrote the planes is ahead of them) and the one that
    # waits for the receives (the next half step comes after them).
    ctx_stream = None
    if s is not None:
        ptr = C.c_void_p()
        s._check(s.lib.sgpu_get_stream(s.handle, C.byref(ptr)), "sgpu_get_stream")
        ctx_stream = torch.cuda.ExternalStream(ptr.value) if ptr.value else torch.cuda.default_stream()

    def halo(phase):
        ops = []
        for ph, src, dst, comps, z in sched:
            if ph != phase:
                continue
            for c in comps:
                if rank == src:
                    ops.append(dist.P2POp(dist.isend, plane_tensor(c, z), dst, group))
                elif rank == dst:
                    ops.append(dist.P2POp(dist.irecv, plane_tensor(c, z), src, group))
        if not ops:
            return
        if ctx_stream is None:
            for r in dist.batch_isend_irecv(ops):
                r.wait()
            return
        with torch.cuda.stream(ctx_stream):
            for r in dist.batch_isend_irecv(ops):
                r.wait()  # the context's stream waits for the message, the host does not

    lib = s.lib if s is not None else None
    for n in range(steps):
        if s is not None:
            s._check(lib.sgpu_advance_e(s.handle, n), "sgpu_advance_e")
        halo("E")
        if s is not None:
            s._check(lib.sgpu_advance_h(s.handle, n), "sgpu_advance_h")
        halo("H")
        if s is not None:
            s._check(lib.sgpu_update_observation(s.handle, n), "sgpu_update_observation")
            s.n = n + 1
    return s


class _DeviceArray:
    """A float32 device buffer seen through __cuda_array_interface__."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (ptr, False), "version": 3}
