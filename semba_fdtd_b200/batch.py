"""Batched form: many independent problems advanced together in one device
arena through libsemba_gpu's sgpu_batch_* entry points.

Each instance runs steps 0..nsteps exactly as :class:`Solver` would (same
per-cell arithmetic, bit-identical probe traces and fields); the batch only
decides which instances share a launch.  Instances can be added between
calls that advance the batch and finish at their own last step.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .case import Problem


class Plan:
    """Host-only set-up of one problem (no device memory): its footprint in
    a batch arena, for admission control; consumed by :meth:`Batch.add`."""

    def __init__(self, problem: Problem, nsteps: int | None = None, variant: str = "exact"):
        self.lib = _lib.load(variant)
        self.problem = problem
        self.nsteps = int(problem.nsteps if nsteps is None else nsteps)
        desc, self._keep = problem.to_desc(1)
        h = C.c_void_p()
        rc = self.lib.sgpu_host_plan(C.byref(desc), self.nsteps, C.byref(h))
        self._h = h
        if rc:
            msg = self.lib.sgpu_last_error(h).decode() if h.value else ""
            self.close()
            raise _lib.SembaGpuError(f"sgpu_host_plan failed ({_lib.ERRORS.get(rc, rc)}): {msg}")
        b, big = C.c_uint64(), C.c_uint64()
        rc = self.lib.sgpu_batch_footprint(h, C.byref(b), C.byref(big))
        if rc:
            self.close()
            raise _lib.SembaGpuError(f"sgpu_batch_footprint failed ({_lib.ERRORS.get(rc, rc)})")
        self.footprint = b.value
        self.largest_buffer = big.value

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.sgpu_destroy(self._h)
        self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    def __init__(self, arena_bytes: int, max_instances: int = 256, variant: str = "exact", kernel_family: int = 1):
        self.lib = _lib.load(variant)
        h = C.c_void_p()
        rc = self.lib.sgpu_batch_create(int(arena_bytes), int(max_instances), C.byref(h))
        self._h = h
        if rc:
            msg = self.lib.sgpu_batch_last_error(h).decode() if h.value else ""
            self.close()
            raise _lib.SembaGpuError(f"sgpu_batch_create failed ({_lib.ERRORS.get(rc, rc)}): {msg}")
        self.problems: dict[int, Problem] = {}
        self._check(self.lib.sgpu_batch_set_kernel_family(h, int(kernel_family)), "sgpu_batch_set_kernel_family")

    # -- plumbing ----------------------------------------------------------
    def _check(self, rc: int, what: str) -> None:
        if rc:
            msg = self.lib.sgpu_batch_last_error(self._h).decode()
            raise _lib.SembaGpuError(f"{what} failed ({_lib.ERRORS.get(rc, rc)}): {msg}")

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.sgpu_batch_destroy(self._h)
        self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- instances ---------------------------------------------------------
    def add(self, problem: Problem | Plan, nsteps: int | None = None) -> int:
        """Set up an instance in the arena; returns its slot.  A Plan is
        consumed.  Raises SembaGpuError (OOM) when the arena has no room."""
        slot = C.c_int(-1)
        if isinstance(problem, Plan):
            rc = self.lib.sgpu_batch_add(self._h, None, problem._h, problem.nsteps, C.byref(slot))
            prob = problem.problem
            problem.close()
        else:
            desc, keep = problem.to_desc(1)
            n = int(problem.nsteps if nsteps is None else nsteps)
            rc = self.lib.sgpu_batch_add(self._h, C.byref(desc), None, n, C.byref(slot))
            prob = problem
            del keep
        self._check(rc, "sgpu_batch_add")
        self.problems[slot.value] = prob
        return slot.value

    def remove(self, slot: int) -> None:
        self._check(self.lib.sgpu_batch_remove(self._h, int(slot)), "sgpu_batch_remove")
        self.problems.pop(slot, None)

    def info(self, slot: int) -> tuple[int, int, int]:
        """(steps done, steps in total, probes) of an instance."""
        d, t, p = C.c_int(), C.c_int(), C.c_int()
        self._check(self.lib.sgpu_batch_slot_info(self._h, int(slot), C.byref(d), C.byref(t), C.byref(p)), "slot_info")
        return d.value, t.value, p.value

    def done(self, slot: int) -> bool:
        d, t, _ = self.info(slot)
        return d >= t

    def probes(self, slot: int) -> np.ndarray:
        """Probe traces recorded so far, [step, probe] (FP32)."""
        d, t, p = self.info(slot)
        out = np.zeros((max(d, 1), max(p, 1)), np.float32)
        rows = C.c_int()
        self._check(self.lib.sgpu_batch_read_probes(self._h, int(slot), out.ctypes.data_as(_lib.c_float_p), d,
                                                    C.byref(rows)), "sgpu_batch_read_probes")
        return out[: rows.value, :p]

    def field(self, slot: int, comp: int) -> np.ndarray:
        """Field component over its Alloc range as [i, j, k]."""
        ctx = C.c_void_p()
        self._check(self.lib.sgpu_batch_instance(self._h, int(slot), C.byref(ctx)), "sgpu_batch_instance")
        a6 = (_lib.Lim * 6)()
        self.lib.sgpu_host_info(ctx, None, None, a6, None, None)
        xi, xe, yi, ye, zi, ze = a6[comp].tuple()
        out = np.empty((ze - zi + 1, ye - yi + 1, xe - xi + 1), np.float32)
        rc = self.lib.sgpu_download_field(ctx, comp, out.ctypes.data_as(_lib.c_float_p))
        if rc:
            raise _lib.SembaGpuError(f"sgpu_download_field failed ({_lib.ERRORS.get(rc, rc)})")
        return out.transpose(2, 1, 0)

    # -- stepping ----------------------------------------------------------
    def advance(self, nsteps: int) -> None:
        self._check(self.lib.sgpu_batch_advance(self._h, int(nsteps)), "sgpu_batch_advance")

    def synchronize(self) -> None:
        self._check(self.lib.sgpu_batch_synchronize(self._h), "sgpu_batch_synchronize")

    def elapsed(self, nsteps: int) -> float:
        """Advance nsteps and return their device time in ms."""
        ms = C.c_float()
        self._check(self.lib.sgpu_batch_elapsed(self._h, int(nsteps), C.byref(ms)), "sgpu_batch_elapsed")
        return ms.value

    @property
    def steps(self) -> int:
        n = C.c_int()
        self._check(self.lib.sgpu_batch_steps(self._h, C.byref(n)), "sgpu_batch_steps")
        return n.value

    def run_all(self, chunk: int = 32) -> None:
        """Advance until every instance has finished."""
        while any(not self.done(s) for s in self.problems):
            left = max(self.info(s)[1] - self.info(s)[0] for s in self.problems)
            self.advance(min(chunk, left))
        self.synchronize()

    # -- memory and tuning -------------------------------------------------
    def memory(self) -> tuple[int, int, int]:
        """(arena capacity, bytes in use, largest free block)."""
        a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self._check(self.lib.sgpu_batch_memory(self._h, C.byref(a), C.byref(b), C.byref(c)), "sgpu_batch_memory")
        return a.value, b.value, c.value

    def set_tuning(self, chunks=None, ctas_per_sm: int = 0) -> None:
        arr = (C.c_int * 3)(*chunks) if chunks is not None else None
        self._check(self.lib.sgpu_batch_set_tuning(self._h, arr, int(ctas_per_sm)), "sgpu_batch_set_tuning")

    def tuning(self) -> tuple[list[int], int]:
        arr, ctas = (C.c_int * 3)(), C.c_int()
        self._check(self.lib.sgpu_batch_get_tuning(self._h, arr, C.byref(ctas)), "sgpu_batch_get_tuning")
        return list(arr), ctas.value

    def autotune(self, steps_per_trial: int = 4) -> tuple[list[int], int]:
        """Pick CTAs per SM and per-size-class z chunks by timing real steps."""
        arr, ctas = (C.c_int * 3)(), C.c_int()
        self._check(self.lib.sgpu_batch_autotune(self._h, int(steps_per_trial), arr, C.byref(ctas)), "sgpu_batch_autotune")
        return list(arr), ctas.value

    def profile(self, nsteps: int) -> list[float]:
        """Device ms per phase summed over nsteps real steps (E field, ADE,
        E sources, H field, H sources and borders, probes)."""
        ms = (C.c_float * 6)()
        self._check(self.lib.sgpu_batch_profile_steps(self._h, int(nsteps), ms), "sgpu_batch_profile_steps")
        return list(ms)
