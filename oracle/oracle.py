"""ctypes wrapper of the CPU oracle (oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py, as the checker of the CUDA path.  Parity status:
unpinned -- the reference Fortran cannot be built here and ships no golden
vectors for this path; the oracle is pinned by known-answer tests instead
(tests/test_oracle_kat.py).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"


class OrcLim(C.Structure):
    _fields_ = [("xi", C.c_int), ("xe", C.c_int), ("yi", C.c_int), ("ye", C.c_int), ("zi", C.c_int), ("ze", C.c_int)]


class OrcRegion(C.Structure):
    _fields_ = [("kind", C.c_int), ("eps", C.c_float), ("sigma", C.c_float), ("mu", C.c_float), ("sigmam", C.c_float),
                ("npoles", C.c_int), ("residues", C.POINTER(C.c_float)), ("bpoles", C.POINTER(C.c_float)),
                ("nboxes", C.c_int), ("boxes", C.POINTER(C.c_int)),
                ("mpoles", C.c_int), ("mresidues", C.POINTER(C.c_float)), ("mbpoles", C.POINTER(C.c_float))]


class OrcPW(C.Structure):
    _fields_ = [("x1", C.c_int), ("y1", C.c_int), ("z1", C.c_int), ("x2", C.c_int), ("y2", C.c_int), ("z2", C.c_int),
                ("theta", C.c_float), ("phi", C.c_float), ("alpha", C.c_float), ("beta", C.c_float),
                ("nsamples", C.c_int), ("samples", C.POINTER(C.c_float)), ("dsamples", C.c_float)]


class OrcNodal(C.Structure):
    _fields_ = [("is_elec", C.c_int), ("is_hard", C.c_int), ("npoints", C.c_int), ("boxes", C.POINTER(C.c_int)),
                ("amp", C.POINTER(C.c_float)), ("nsamples", C.c_int), ("samples", C.POINTER(C.c_float)),
                ("dsamples", C.c_float)]


class OrcProblem(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("desx", C.POINTER(C.c_float)), ("desy", C.POINTER(C.c_float)), ("desz", C.POINTER(C.c_float)),
                ("originx", C.c_float), ("originy", C.c_float), ("originz", C.c_float),
                ("dt", C.c_double), ("forcecfl", C.c_int), ("cfl", C.c_float),
                ("pml_layers", C.c_int * 6), ("pml_order", C.c_float * 6), ("pml_refl", C.c_float * 6),
                ("alphamax", C.c_float), ("alphaorder", C.c_float), ("kappamax", C.c_float),
                ("nregions", C.c_int), ("regions", C.POINTER(OrcRegion)),
                ("npw", C.c_int), ("pw", C.POINTER(OrcPW)),
                ("nnodal", C.c_int), ("nodal", C.POINTER(OrcNodal)),
                ("nprobes", C.c_int), ("probes", C.POINTER(C.c_int)),
                ("border", C.c_int * 6), ("mur_after_pml", C.c_int)]


_lib = None


def build() -> Path:
    """Compile the oracle with its Makefile (g++, OpenMP, no FMA contraction)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = C.CDLL(str(LIB))
        vp = C.c_void_p
        lib.orc_create.argtypes = [C.POINTER(OrcProblem), C.c_int, C.c_int, C.POINTER(vp)]
        lib.orc_create.restype = C.c_int
        lib.orc_destroy.argtypes = [vp]
        lib.orc_destroy.restype = None
        lib.orc_run.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_float)]
        lib.orc_run.restype = C.c_int
        lib.orc_get_lims.argtypes = [vp, C.POINTER(OrcLim), C.POINTER(OrcLim), C.POINTER(OrcLim)]
        lib.orc_get_dt.argtypes = [vp]
        lib.orc_get_dt.restype = C.c_double
        lib.orc_get_time.argtypes = [vp, C.c_int]
        lib.orc_get_time.restype = C.c_double
        lib.orc_get_num_media.argtypes = [vp]
        lib.orc_get_field.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        lib.orc_get_field_f64.argtypes = [vp, C.c_int, C.POINTER(C.c_double)]
        lib.orc_get_media.argtypes = [vp, C.c_int, C.POINTER(C.c_short)]
        lib.orc_set_field.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        lib.orc_get_g.argtypes = [vp] + [C.POINTER(C.c_float)] * 4
        lib.orc_get_metric.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        lib.orc_get_metric_range.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        lib.orc_get_edisp.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)] + [C.POINTER(C.c_double)] * 3
        lib.orc_get_mur_cab1.argtypes = [vp, C.c_int, C.POINTER(C.c_float)]
        lib.orc_get_mdisp.argtypes = lib.orc_get_edisp.argtypes
        lib.orc_check_div_dt.argtypes = [C.c_double, C.c_long, C.c_ulonglong]
        lib.orc_check_div_dt.restype = C.c_long
        ip = C.POINTER(C.c_int)
        lib.orc_add_freq_probe.argtypes = [vp, C.c_int, ip, ip, C.c_int, C.POINTER(C.c_float)]
        lib.orc_add_freq_probe.restype = C.c_int
        lib.orc_read_freq_probe.argtypes = [vp, C.c_int, ip, C.POINTER(C.c_double)]
        lib.orc_read_freq_probe.restype = C.c_int
        lib.orc_store_resume.argtypes = [vp, C.c_char_p, C.c_int]
        lib.orc_store_resume.restype = C.c_int
        lib.orc_load_resume.argtypes = [vp, C.c_char_p, ip]
        lib.orc_load_resume.restype = C.c_int
        fp = C.POINTER(C.c_float)
        lib.orc_add_farfield.argtypes = [vp, ip, ip, C.c_float, C.c_float, C.c_float, C.c_int, C.c_int]
        lib.orc_add_farfield.restype = C.c_int
        lib.orc_read_farfield.argtypes = [vp, C.c_int, C.c_int, C.c_int, ip, C.POINTER(C.c_double)]
        lib.orc_read_farfield.restype = C.c_int
        lib.orc_farfield_transform.argtypes = [vp, C.c_int, fp, fp, C.c_int, C.POINTER(C.c_double), C.c_int, ip]
        lib.orc_farfield_transform.restype = C.c_int
        lib.orc_incident.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, fp, fp]
        lib.orc_incident.restype = C.c_int
        lib.orc_set_threads.argtypes = [vp, C.c_int]
        lib.orc_set_threads.restype = None
        _lib = lib
    return _lib


def _problem(pb):
    """orc_problem from a semba_fdtd_b200.case.Problem (input description only)."""
    keep = []

    def f32(a):
        a = np.ascontiguousarray(a, np.float32)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_float))

    def i32(a):
        a = np.ascontiguousarray(a, np.int32)
        keep.append(a)
        return a.ctypes.data_as(C.POINTER(C.c_int))

    p = OrcProblem()
    p.nx, p.ny, p.nz = pb.nx, pb.ny, pb.nz
    p.desx, p.desy, p.desz = f32(pb.desx), f32(pb.desy), f32(pb.desz)
    p.originx, p.originy, p.originz = pb.origin
    p.dt, p.forcecfl, p.cfl = pb.dt, int(pb.forcecfl), pb.cfl
    for f in range(6):
        p.pml_layers[f], p.pml_order[f], p.pml_refl[f] = pb.pml_layers[f], pb.pml_order[f], pb.pml_refl[f]
    p.alphamax, p.alphaorder, p.kappamax = pb.alphamax, pb.alphaorder, pb.kappamax
    regs = (OrcRegion * max(1, len(pb.regions)))()
    for q, r in enumerate(pb.regions):
        g = regs[q]
        g.kind, g.eps, g.sigma, g.mu, g.sigmam = r.kind, r.eps, r.sigma, r.mu, r.sigmam
        g.npoles = len(r.residues)
        g.residues = f32(np.asarray(r.residues, np.complex64).view(np.float32))
        g.bpoles = f32(np.asarray(r.bpoles, np.complex64).view(np.float32))
        g.nboxes = len(r.boxes)
        g.boxes = i32(np.asarray(r.boxes).reshape(-1))
        g.mpoles = len(r.mresidues)
        g.mresidues = f32(np.asarray(r.mresidues, np.complex64).view(np.float32))
        g.mbpoles = f32(np.asarray(r.mbpoles, np.complex64).view(np.float32))
    keep.append(regs)
    p.nregions, p.regions = len(pb.regions), regs
    pws = (OrcPW * max(1, len(pb.planewaves)))()
    for q, w in enumerate(pb.planewaves):
        s = pws[q]
        s.x1, s.y1, s.z1 = w.coor1
        s.x2, s.y2, s.z2 = w.coor2
        s.theta, s.phi, s.alpha, s.beta = w.theta, w.phi, w.alpha, w.beta
        s.nsamples, s.samples, s.dsamples = len(w.wave.samples), f32(w.wave.samples), float(w.wave.dsamples)
    keep.append(pws)
    p.npw, p.pw = len(pb.planewaves), pws
    nds = (OrcNodal * max(1, len(pb.nodals)))()
    for q, n in enumerate(pb.nodals):
        s = nds[q]
        s.is_elec, s.is_hard, s.npoints = int(n.is_elec), int(n.is_hard), len(n.boxes)
        s.boxes, s.amp = i32(np.asarray(n.boxes).reshape(-1)), f32(np.asarray(n.amp).reshape(-1))
        s.nsamples, s.samples, s.dsamples = len(n.wave.samples), f32(n.wave.samples), float(n.wave.dsamples)
    keep.append(nds)
    p.nnodal, p.nodal = len(pb.nodals), nds
    p.nprobes = len(pb.probes)
    p.probes = i32(np.asarray(pb.probes).reshape(-1))
    for f, code in enumerate(pb.border_codes):
        p.border[f] = code
    p.mur_after_pml = int(pb.mur_after_pml)
    return p, keep


class Oracle:
    """The reference algorithm on the CPU (FP32 by default, FP64 with fp64=True)."""

    def __init__(self, problem, fp64: bool = False, threads: int = 0):
        self.lib = load()
        self.problem = problem
        desc, self._keep = _problem(problem)
        h = C.c_void_p()
        rc = self.lib.orc_create(C.byref(desc), int(fp64), int(threads), C.byref(h))
        if rc:
            raise RuntimeError(f"orc_create failed with {rc}")
        self._h = h
        self.n = 0
        a, w, q = (OrcLim * 6)(), (OrcLim * 6)(), (OrcLim * 6)()
        self.lib.orc_get_lims(h, a, w, q)
        tup = lambda l: (l.xi, l.xe, l.yi, l.ye, l.zi, l.ze)
        self.alloc = [tup(x) for x in a]
        self.sweep = [tup(x) for x in w]
        self.sinpml = [tup(x) for x in q]
        self.dt = self.lib.orc_get_dt(h)
        self.num_media = self.lib.orc_get_num_media(h)
        self.nprobes = len(problem.probes)

    def close(self):
        if self._h:
            self.lib.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, count: int) -> np.ndarray:
        out = np.zeros((count, max(1, self.nprobes)), np.float32)
        rc = self.lib.orc_run(self._h, self.n, self.n + count, out.ctypes.data_as(C.POINTER(C.c_float)))
        if rc:
            raise RuntimeError(f"orc_run failed with {rc}")
        self.n += count
        return out[:, : self.nprobes]

    def field(self, comp: int, f64: bool = False) -> np.ndarray:
        xi, xe, yi, ye, zi, ze = self.alloc[comp]
        shape = (ze - zi + 1, ye - yi + 1, xe - xi + 1)
        if f64:
            out = np.empty(shape, np.float64)
            self.lib.orc_get_field_f64(self._h, comp, out.ctypes.data_as(C.POINTER(C.c_double)))
        else:
            out = np.empty(shape, np.float32)
            self.lib.orc_get_field(self._h, comp, out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.transpose(2, 1, 0)

    def set_field(self, comp: int, arr: np.ndarray) -> None:
        """Overwrite a component with an [i, j, k] array over its Alloc range."""
        a = np.ascontiguousarray(np.asarray(arr, np.float32).transpose(2, 1, 0))
        self.lib.orc_set_field(self._h, comp, a.ctypes.data_as(C.POINTER(C.c_float)))

    def media(self, comp: int) -> np.ndarray:
        xi, xe, yi, ye, zi, ze = self.alloc[comp]
        out = np.empty((ze - zi + 1, ye - yi + 1, xe - xi + 1), np.int16)
        self.lib.orc_get_media(self._h, comp, out.ctypes.data_as(C.POINTER(C.c_short)))
        return out.transpose(2, 1, 0)

    def g_tables(self):
        n = self.num_media + 1
        arrs = [np.empty(n, np.float32) for _ in range(4)]
        self.lib.orc_get_g(self._h, *[a.ctypes.data_as(C.POINTER(C.c_float)) for a in arrs])
        return arrs

    def metric(self, which: int):
        lo, hi = C.c_int(), C.c_int()
        self.lib.orc_get_metric_range(self._h, which, C.byref(lo), C.byref(hi))
        out = np.empty(hi.value - lo.value + 1, np.float32)
        self.lib.orc_get_metric(self._h, which, out.ctypes.data_as(C.POINTER(C.c_float)))
        return lo.value, out

    def time(self, n: int) -> float:
        return self.lib.orc_get_time(self._h, n)

    def set_threads(self, n: int) -> None:
        """OpenMP threads of the following steps."""
        self.lib.orc_set_threads(self._h, int(n))

    def incident(self, comp: int, i: int, j: int, k: int, t) -> np.ndarray:
        """Incid as the observation flush calls it, at the real(4) times t."""
        tt = np.ascontiguousarray(t, np.float32)
        out = np.empty(len(tt), np.float32)
        fp = C.POINTER(C.c_float)
        if self.lib.orc_incident(self._h, comp, i, j, k, len(tt), tt.ctypes.data_as(fp), out.ctypes.data_as(fp)):
            raise ValueError("incident field: FP32 oracle and a node inside PhysCoor needed")
        return out

    def store_resume(self, path) -> None:
        """Restart file of the state after the last step run (n = self.n - 1)."""
        if self.lib.orc_store_resume(self._h, str(path).encode(), self.n - 1):
            raise RuntimeError("orc_store_resume failed")

    def load_resume(self, path) -> int:
        """Load a restart file; the next step is n + 1.  Returns n."""
        n = C.c_int()
        if self.lib.orc_load_resume(self._h, str(path).encode(), C.byref(n)):
            raise RuntimeError("orc_load_resume failed (not a restart file of this set-up)")
        self.n = n.value + 1
        return n.value

    def add_freq_probe(self, magnetic: bool, box, stride, freqs) -> int:
        """Frequency-domain volume probe; accumulates after every later step."""
        b = (C.c_int * 6)(*[int(v) for v in box])
        st = (C.c_int * 3)(*[int(v) for v in stride])
        fr = np.ascontiguousarray(np.asarray(freqs, np.float32))
        pid = self.lib.orc_add_freq_probe(self._h, int(bool(magnetic)), b, st, len(fr),
                                          fr.ctypes.data_as(C.POINTER(C.c_float)))
        if pid < 0:
            raise ValueError("frequency probe samples no node")
        return pid

    def freq_probe(self, pid: int) -> np.ndarray:
        """Accumulators as complex128 [nfreq, 3, nk, nj, ni]."""
        sh = (C.c_int * 4)()
        if self.lib.orc_read_freq_probe(self._h, pid, sh, None):
            raise ValueError("no frequency probe with that id")
        nf, nk, nj, ni = list(sh)
        out = np.empty(nf * 3 * nk * nj * ni * 2, np.float64)
        self.lib.orc_read_freq_probe(self._h, pid, None, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out.view(np.complex128).reshape(nf, 3, nk, nj, ni)

    def add_farfield(self, box, faces=(1, 1, 1, 1, 1, 1), initial=1e8, final=1e9, step=1e8,
                     logarithmic=False, decimate=False) -> int:
        """InitFarField (farfield.F90:118-1158) for the box esqx1..esqz2."""
        b = (C.c_int * 6)(*[int(v) for v in box])
        fc = (C.c_int * 6)(*[int(bool(v)) for v in faces])
        fid = self.lib.orc_add_farfield(self._h, b, fc, float(initial), float(final), float(step),
                                        int(bool(logarithmic)), int(bool(decimate)))
        if fid == -2:
            raise ValueError("NF2FF STILL UNSUPPORTED (a face on a PEC/PMC border)")
        if fid < 0:
            raise ValueError("bad far-field request")
        return fid

    def farfield_array(self, fid: int, face: int, slot: int) -> np.ndarray:
        """Accumulated array of a face and slot as complex128 [nfreq, outer, inner]."""
        dims = (C.c_int * 2)()
        if self.lib.orc_read_farfield(self._h, fid, face, slot, dims, None):
            raise ValueError("no far-field array with that id, face and slot")
        n = dims[0] * dims[1]
        nf = self._ff_nfreq(fid)
        out = np.zeros(max(1, nf * n * 2), np.float64)
        self.lib.orc_read_farfield(self._h, fid, face, slot, dims, out.ctypes.data_as(C.POINTER(C.c_double)))
        return out[:nf * n * 2].view(np.complex128).reshape(nf, dims[0], dims[1])

    def _ff_nfreq(self, fid: int) -> int:
        rows = C.c_int()
        ang = (C.c_float * 6)(0, 0, 1, 0, 0, 1)
        self.lib.orc_farfield_transform(self._h, fid, ang, None, 0, None, 0, C.byref(rows))
        return rows.value

    def farfield_transform(self, fid: int, angles, incident) -> np.ndarray:
        """FlushFarfield rows [n, 9]: freq, theta, phi, |Etheta|, arg Etheta,
        |Ephi|, arg Ephi, RCS (arithmetic), RCS (geometric)."""
        ang = (C.c_float * 6)(*[float(v) for v in angles])
        inc = np.ascontiguousarray(np.asarray(incident, np.float32).reshape(-1, 2))
        rows = C.c_int()
        self.lib.orc_farfield_transform(self._h, fid, ang, None, 0, None, 0, C.byref(rows))
        out = np.empty((rows.value, 9), np.float64)
        if self.lib.orc_farfield_transform(self._h, fid, ang, inc.ctypes.data_as(C.POINTER(C.c_float)), len(inc),
                                           out.ctypes.data_as(C.POINTER(C.c_double)), rows.value, C.byref(rows)):
            raise ValueError("far-field transform failed")
        return out

    def mur_cab1(self, face: int):
        """CAB1 per medium of a Mur face (back, front, left, right, down, up),
        or None when the face has no Mur condition."""
        out = np.empty(self.num_media + 1, np.float32)
        rc = self.lib.orc_get_mur_cab1(self._h, face, out.ctypes.data_as(C.POINTER(C.c_float)))
        return None if rc else out
