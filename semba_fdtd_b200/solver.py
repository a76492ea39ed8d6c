"""Solver: one FDTD problem on one GPU through libsemba_gpu.

Three ways to advance, all bit-identical:

* ``mode="graph"`` (default) -- ``sgpu_advance_steps``: whole steps replayed
  from a CUDA graph of up to 32 captured steps;
* ``mode="fused"`` -- ``sgpu_advance_e`` / ``sgpu_advance_h`` /
  ``sgpu_update_observation`` per step;
* ``mode="routines"`` -- one call per reference routine, in the order of
  timestepping.F90:1286-1742 (Advance_Ex, Ey, Ez, AdvanceelectricCPML,
  AdvanceEDispersiveE, AdvancePlaneWaveE, AdvanceNodalE, Advance_Hx, Hy, Hz,
  AdvanceMagneticCPML, MinusCloneMagneticPMC, CloneMagneticPeriodic,
  AdvanceMdispersiveH, AdvancePlaneWaveH, AdvanceNodalH, MinusCloneMagneticPMC,
  CloneMagneticPeriodic, AdvanceMagneticMUR, UpdateObservation).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .case import Problem


class Solver:
    def __init__(self, problem: Problem, variant: str = "exact", probe_capacity: int = 1024,
                 max_steps: int | None = None, kernel_family: int | None = None, zslab: tuple[int, int] | None = None):
        """zslab=(z0, z1): only the z-slab sub-domain of planes z0..z1 (see
        semba_fdtd_b200.zslab for the decomposition and its halo copies)."""
        self.problem = problem
        self.lib = _lib.load(variant)
        self.variant = variant
        self.probe_capacity = probe_capacity
        desc, self._keep = problem.to_desc(probe_capacity)
        self.max_steps = int(max_steps if max_steps is not None else problem.nsteps)
        h = C.c_void_p()
        if zslab is None:
            rc = self.lib.sgpu_host_create(C.byref(desc), self.max_steps, C.byref(h))
        else:
            rc = self.lib.sgpu_host_create_zslab(C.byref(desc), self.max_steps, int(zslab[0]), int(zslab[1]),
                                                 C.byref(h))
        self.zslab = zslab
        self._h = h
        if rc:
            msg = self.lib.sgpu_last_error(h).decode() if h.value else ""
            self.close()
            raise _lib.SembaGpuError(f"sgpu_host_create failed ({_lib.ERRORS.get(rc, rc)}): {msg}")
        self.n = 0
        dt = C.c_double()
        nm = C.c_int()
        a6, s6, q6 = (_lib.Lim * 6)(), (_lib.Lim * 6)(), (_lib.Lim * 6)()
        self._check(self.lib.sgpu_host_info(h, C.byref(dt), C.byref(nm), a6, s6, q6))
        self.dt = dt.value
        self.num_media = nm.value
        self.alloc = [a.tuple() for a in a6]
        self.sweep = [s.tuple() for s in s6]
        self.sinpml = [q.tuple() for q in q6]
        self.nprobes = len(problem.probes) if zslab is None else len(self.probe_ids())
        self._probe_rows: list[np.ndarray] = []
        if kernel_family is not None:
            self._check(self.lib.sgpu_set_kernel_family(h, int(kernel_family)), "sgpu_set_kernel_family")

    # -- plumbing ----------------------------------------------------------
    def _check(self, rc: int, what: str = "") -> None:
        if rc:
            msg = self.lib.sgpu_last_error(self._h).decode()
            raise _lib.SembaGpuError(f"{what or 'libsemba_gpu'} failed ({_lib.ERRORS.get(rc, rc)}): {msg}")

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self.lib.sgpu_destroy(self._h)
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

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- stepping ----------------------------------------------------------
    def step(self, count: int = 1, mode: str = "graph") -> None:
        """Advance `count` whole steps from the current step index."""
        if self.n + count > self.max_steps + 1:
            raise _lib.SembaGpuError("beyond the time vector built at creation (max_steps)")
        lib, h = self.lib, self._h
        done = 0
        while done < count:
            room = self.probe_capacity - self._pending() if self.nprobes else count - done
            if room <= 0:
                self._drain()
                continue
            k = min(count - done, room)
            n0 = self.n
            if mode == "graph":
                self._check(lib.sgpu_advance_steps(h, n0, k), "sgpu_advance_steps")
            elif mode == "fused":
                for n in range(n0, n0 + k):
                    self._check(lib.sgpu_advance_e(h, n), "sgpu_advance_e")
                    self._check(lib.sgpu_advance_h(h, n), "sgpu_advance_h")
                    self._check(lib.sgpu_update_observation(h, n), "sgpu_update_observation")
            elif mode == "routines":
                for n in range(n0, n0 + k):
                    for f in (lib.sgpu_advance_ex, lib.sgpu_advance_ey, lib.sgpu_advance_ez,
                              lib.sgpu_advance_electric_cpml, lib.sgpu_advance_edispersive_e):
                        self._check(f(h))
                    self._check(lib.sgpu_advance_planewave_e(h, n))
                    self._check(lib.sgpu_advance_nodal_e(h, n))
                    for f in (lib.sgpu_advance_hx, lib.sgpu_advance_hy, lib.sgpu_advance_hz,
                              lib.sgpu_advance_magnetic_cpml, lib.sgpu_advance_pmc_h, lib.sgpu_advance_periodic_h,
                              lib.sgpu_advance_mdispersive_h):
                        self._check(f(h))
                    self._check(lib.sgpu_advance_planewave_h(h, n))
                    self._check(lib.sgpu_advance_nodal_h(h, n))
                    for f in (lib.sgpu_advance_pmc_h, lib.sgpu_advance_periodic_h, lib.sgpu_advance_magnetic_mur):
                        self._check(f(h))
                    self._check(lib.sgpu_update_observation(h, n))
            else:
                raise ValueError(mode)
            self.n += k
            done += k
            if self.nprobes and self._pending() >= self.probe_capacity:
                self._drain()

    def _pending(self) -> int:
        return self.n - getattr(self, "_probe_base", 0) - sum(len(r) for r in self._probe_rows)

    def _drain(self) -> None:
        if not self.nprobes:
            return
        buf = np.empty((self.probe_capacity, self.nprobes), np.float32)
        ns, first = C.c_int(), C.c_int()
        self._check(self.lib.sgpu_read_probes(self._h, buf.ctypes.data_as(_lib.c_float_p), self.probe_capacity,
                                              C.byref(ns), C.byref(first)), "sgpu_read_probes")
        if ns.value:
            self._probe_rows.append(buf[: ns.value].copy())

    def run(self, nsteps: int | None = None, mode: str = "graph") -> np.ndarray:
        """Run the remaining steps (or `nsteps`) and return the probe traces."""
        nsteps = self.problem.nsteps + 1 - self.n if nsteps is None else nsteps
        self.step(nsteps, mode=mode)
        return self.probes()

    def probes(self) -> np.ndarray:
        """All probe rows recorded so far, [step, probe] (FP32)."""
        self.synchronize()
        self._drain()
        if not self._probe_rows:
            return np.zeros((0, self.nprobes), np.float32)
        return np.concatenate(self._probe_rows, axis=0)

    def synchronize(self) -> None:
        self._check(self.lib.sgpu_synchronize(self._h), "sgpu_synchronize")

    def probe_ids(self) -> list[int]:
        """Indices into problem.probes of the probes this solver records (a
        z-slab records those on the planes it owns)."""
        if self.zslab is None:
            return list(range(len(self.problem.probes)))
        z0, z1 = self.zslab
        return [q for q, p in enumerate(self.problem.probes) if p[3] >= z0 and p[3] <= z1]

    # -- restart files -----------------------------------------------------
    def store_resume(self, path) -> None:
        """Write the restart file of flush_and_save_resume for the state after
        the last step run (n = self.n - 1)."""
        eps0, mu0 = C.c_float(), C.c_float()
        self._check(self.lib.sgpu_host_get_constants(self._h, C.byref(eps0), C.byref(mu0)), "sgpu_host_get_constants")
        self._check(self.lib.sgpu_store_resume(self._h, str(path).encode(), self.n - 1, eps0, mu0), "sgpu_store_resume")

    def load_resume(self, path) -> int:
        """Load a restart file written for the same problem (by this library
        or in the reference's record layout); steps go on at n + 1.  Returns n."""
        n = C.c_int()
        if self.n != 0:
            raise _lib.SembaGpuError("load a restart file into a solver that has not stepped")
        self._check(self.lib.sgpu_load_resume(self._h, str(path).encode(), C.byref(n)), "sgpu_load_resume")
        self.n = n.value + 1
        self._probe_base = self.n  # probe rows start at the first step after the restart
        return n.value

    # -- volume probes -----------------------------------------------------
    def add_freq_probe(self, magnetic: bool, box, stride=(1, 1, 1), freqs=(1e9,)) -> int:
        """Frequency-domain volume probe over box (XI XE YI YE ZI ZE) at the
        nodes whose coordinates are multiples of stride; accumulated after
        every later step.  Returns its id."""
        fr = np.ascontiguousarray(np.asarray(freqs, np.float32))
        d = _lib.FreqProbeDesc(int(bool(magnetic)), (C.c_int * 6)(*map(int, box)), (C.c_int * 3)(*map(int, stride)),
                               len(fr), fr.ctypes.data_as(_lib.c_float_p))
        pid = C.c_int(-1)
        self._check(self.lib.sgpu_add_freq_probe(self._h, C.byref(d), C.byref(pid)), "sgpu_add_freq_probe")
        return pid.value

    def add_movie_probe(self, magnetic: bool, box, stride=(1, 1, 1), n_first: int = 0, n_last: int = 1 << 30,
                        every: int = 1, capacity: int = 16) -> int:
        """Time-domain volume probe: frames of the sampled box after steps
        n_first <= n < n_last, every `every` steps, in a ring of `capacity`."""
        d = _lib.MovieProbeDesc(int(bool(magnetic)), (C.c_int * 6)(*map(int, box)), (C.c_int * 3)(*map(int, stride)),
                                int(n_first), int(n_last), int(every), int(capacity))
        pid = C.c_int(-1)
        self._check(self.lib.sgpu_add_movie_probe(self._h, C.byref(d), C.byref(pid)), "sgpu_add_movie_probe")
        return pid.value

    def volume_probe_shape(self, pid: int):
        """((ni, nj, nk), (i0, j0, k0)) of a volume probe."""
        ni, nj, nk, ijk = C.c_int(), C.c_int(), C.c_int(), (C.c_int * 3)()
        self._check(self.lib.sgpu_volume_probe_shape(self._h, pid, C.byref(ni), C.byref(nj), C.byref(nk), ijk))
        return (ni.value, nj.value, nk.value), tuple(ijk)

    def freq_probe(self, pid: int, nfreq: int) -> np.ndarray:
        """Accumulators of a frequency probe, complex128 [nfreq, 3, nk, nj, ni]."""
        (ni, nj, nk), _ = self.volume_probe_shape(pid)
        out = np.empty(nfreq * 3 * nk * nj * ni * 2, np.float64)
        self._check(self.lib.sgpu_read_freq_probe(self._h, pid, out.ctypes.data_as(C.POINTER(C.c_double))),
                    "sgpu_read_freq_probe")
        return out.view(np.complex128).reshape(nfreq, 3, nk, nj, ni)

    def movie_frames(self, pid: int, max_frames: int = 1 << 20):
        """(first step, frames [F, 3, nk, nj, ni] float32) recorded since the last read."""
        (ni, nj, nk), _ = self.volume_probe_shape(pid)
        cap = max(1, min(max_frames, 4096))
        frames, first = [], None
        while True:
            buf = np.empty((cap, 3, nk, nj, ni), np.float32)
            got, n0 = C.c_int(), C.c_int()
            self._check(self.lib.sgpu_read_movie_probe(self._h, pid, buf.ctypes.data_as(_lib.c_float_p), cap,
                                                       C.byref(got), C.byref(n0)), "sgpu_read_movie_probe")
            if first is None:
                first = n0.value
            if got.value == 0:
                break
            frames.append(buf[: got.value])
            if got.value < cap or sum(len(f) for f in frames) >= max_frames:
                break
        arr = np.concatenate(frames) if frames else np.zeros((0, 3, nk, nj, ni), np.float32)
        return first, arr

    # -- near-to-far field (farfield.F90) -----------------------------------
    def add_farfield(self, box, faces=(1, 1, 1, 1, 1, 1), initial: float = 1e8, final: float = 1e9,
                     step: float = 1e8, logarithmic: bool = False, decimate: bool = False) -> int:
        """InitFarField for the box (esqx1, esqx2, esqy1, esqy2, esqz1, esqz2):
        the faces Tr, Fr, Iz, De, Ab, Ar to sample, the frequency range and
        NF2FFDecim.  The surface DFT then runs on the device every step."""
        spec = _lib.FarFieldSpec()
        spec.box[:] = [int(v) for v in box]
        spec.faces[:] = [int(bool(v)) for v in faces]
        spec.initial_freq, spec.final_freq, spec.freq_step = float(initial), float(final), float(step)
        spec.logarithmic, spec.decimate = int(bool(logarithmic)), int(bool(decimate))
        fid = C.c_int()
        self._check(self.lib.sgpu_host_add_farfield(self._h, C.byref(spec), C.byref(fid)), "sgpu_host_add_farfield")
        return fid.value

    def farfield_array(self, fid: int, face: int, slot: int) -> np.ndarray:
        """One accumulated surface array, complex128 [nfreq, outer, inner]
        (slot 0/1: E t1/t2; 2/3: H partner of t1 on its two planes; 4/5: of t2)."""
        nf, dims = C.c_int(), (C.c_int * 2)()
        self._check(self.lib.sgpu_farfield_shape(self._h, fid, C.byref(nf), None), "sgpu_farfield_shape")
        self._check(self.lib.sgpu_read_farfield(self._h, fid, face, slot, dims, None), "sgpu_read_farfield")
        n = dims[0] * dims[1]
        out = np.zeros(max(1, nf.value * n * 2), np.float64)
        self._check(self.lib.sgpu_read_farfield(self._h, fid, face, slot, dims,
                                                out.ctypes.data_as(C.POINTER(C.c_double))), "sgpu_read_farfield")
        return out[:nf.value * n * 2].view(np.complex128).reshape(nf.value, dims[0], dims[1])

    def farfield_transform(self, fid: int, angles, incident) -> np.ndarray:
        """FlushFarfield on the device: rows [n, 9] of freq, theta, phi,
        |Etheta|, arg Etheta, |Ephi|, arg Ephi, RCS (arithmetic), RCS
        (geometric), one per frequency and direction.  angles = (theta start,
        stop, step, phi start, stop, step) in radians; incident = the (time,
        value) pairs of the normalisation signal."""
        a = _lib.FarFieldAngles(*[float(v) for v in angles])
        inc = np.ascontiguousarray(np.asarray(incident, np.float32).reshape(-1, 2))
        rows = C.c_int()
        self._check(self.lib.sgpu_farfield_transform(self._h, fid, C.byref(a), None, 0, None, 0, C.byref(rows)),
                    "sgpu_farfield_transform")
        out = np.empty((rows.value, 9), np.float64)
        self._check(self.lib.sgpu_farfield_transform(self._h, fid, C.byref(a), inc.ctypes.data_as(_lib.c_float_p),
                                                     len(inc), out.ctypes.data_as(C.POINTER(C.c_double)),
                                                     rows.value, C.byref(rows)), "sgpu_farfield_transform")
        return out

    def set_kernel_family(self, family: int) -> None:
        """1: TMA-pipelined fused field kernels (default); 0: register-marching."""
        self._check(self.lib.sgpu_set_kernel_family(self._h, int(family)), "sgpu_set_kernel_family")

    # -- data --------------------------------------------------------------
    def field_shape(self, comp: int) -> tuple:
        """(nz, ny, nx) of component comp's Alloc box: the C-order shape of
        the buffers ``field(out=...)`` and ``upload_field`` take."""
        xi, xe, yi, ye, zi, ze = self.alloc[comp]
        return (ze - zi + 1, ye - yi + 1, xe - xi + 1)

    def field(self, comp: int, out: np.ndarray | None = None) -> np.ndarray:
        """Field component (0..5) over its Alloc range, Fortran order, as a
        3-D array indexed [i, j, k] relative to the Alloc lower corner.  `out`
        (float32, C-contiguous, shape field_shape(comp)) receives the values;
        a pinned one (``_lib.pinned_empty``) is filled by the copy engine
        directly."""
        shape = self.field_shape(comp)
        if out is None:
            out = np.empty(shape, np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError(f"out must be C-contiguous float32 of shape {shape}")
        self._check(self.lib.sgpu_download_field(self._h, comp, out.ctypes.data_as(_lib.c_float_p)), "download")
        return out.transpose(2, 1, 0)

    def upload_field(self, comp: int, values: np.ndarray) -> None:
        """Set component comp from a C-contiguous float32 array of shape
        field_shape(comp) ([k][j][i]); pinned arrays go straight to the copy
        engine."""
        shape = self.field_shape(comp)
        if values.shape != shape or values.dtype != np.float32 or not values.flags.c_contiguous:
            raise ValueError(f"values must be C-contiguous float32 of shape {shape}")
        self._check(self.lib.sgpu_upload_field(self._h, comp, values.ctypes.data_as(_lib.c_float_p)), "upload")

    def media(self, comp: int) -> np.ndarray:
        xi, xe, yi, ye, zi, ze = self.alloc[comp]
        out = np.empty((ze - zi + 1, ye - yi + 1, xe - xi + 1), np.int16)
        self._check(self.lib.sgpu_host_get_media(self._h, comp, out.ctypes.data_as(C.POINTER(C.c_int16))), "media")
        return out.transpose(2, 1, 0)

    def g_tables(self):
        n = self.num_media + 1
        arrs = [np.empty(n, np.float32) for _ in range(4)]
        self._check(self.lib.sgpu_host_get_g(self._h, *[a.ctypes.data_as(_lib.c_float_p) for a in arrs]))
        return arrs

    def metric(self, which: int):
        lo, hi = C.c_int(), C.c_int()
        self._check(self.lib.sgpu_host_get_metric(self._h, which, None, C.byref(lo), C.byref(hi)))
        out = np.empty(hi.value - lo.value + 1, np.float32)
        self._check(self.lib.sgpu_host_get_metric(self._h, which, out.ctypes.data_as(_lib.c_float_p), None, None))
        return lo.value, out

    def mur_cab1(self, face: int):
        """CAB1 per medium of a Mur face (back, front, left, right, down, up),
        or None when the face has no Mur condition."""
        out = np.empty(self.num_media + 1, np.float32)
        rc = self.lib.sgpu_host_get_mur_cab1(self._h, int(face), out.ctypes.data_as(_lib.c_float_p))
        return None if rc else out

    def time_vector(self, n0: int = 0, count: int | None = None) -> np.ndarray:
        """tiempo(n0 .. n0+count-1), FP64, as the library holds it."""
        count = self.max_steps + 3 - n0 if count is None else count
        out = np.empty(count, np.float64)
        self._check(self.lib.sgpu_get_time(self._h, n0, count, out.ctypes.data_as(C.POINTER(C.c_double))),
                    "sgpu_get_time")
        return out

    def incident(self, comp: int, i: int, j: int, k: int, t) -> np.ndarray:
        """The incident-field column of a point-probe file at node (i, j, k)
        of component comp, at the real(4) times t (sgpu_host_incident)."""
        tt = np.ascontiguousarray(t, np.float32)
        out = np.empty(len(tt), np.float32)
        self._check(self.lib.sgpu_host_incident(self._h, comp, i, j, k, len(tt), tt.ctypes.data_as(_lib.c_float_p),
                                                out.ctypes.data_as(_lib.c_float_p)), "sgpu_host_incident")
        return out

    def check_finite(self) -> bool:
        rc = self.lib.sgpu_check_finite(self._h)
        if rc == 5:
            return False
        self._check(rc, "sgpu_check_finite")
        return True

    def device_bytes(self) -> int:
        b = C.c_uint64()
        self._check(self.lib.sgpu_device_bytes(self._h, C.byref(b)))
        return b.value
