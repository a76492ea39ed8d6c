"""ctypes bindings of libsemba_gpu.so (include/semba_gpu.h).

The CUDA library is the only compute path: if it cannot be loaded, or no CUDA
device is present, every solver call raises; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
_BUILD = _HERE / "_build"

c_int_p = C.POINTER(C.c_int)
c_float_p = C.POINTER(C.c_float)
c_double_p = C.POINTER(C.c_double)


class Lim(C.Structure):
    _fields_ = [("xi", C.c_int), ("xe", C.c_int), ("yi", C.c_int), ("ye", C.c_int), ("zi", C.c_int), ("ze", C.c_int)]

    def tuple(self):
        return (self.xi, self.xe, self.yi, self.ye, self.zi, self.ze)


class Region(C.Structure):
    _fields_ = [("kind", C.c_int), ("eps", C.c_float), ("sigma", C.c_float), ("mu", C.c_float), ("sigmam", C.c_float),
                ("npoles", C.c_int), ("residues", c_float_p), ("bpoles", c_float_p), ("nboxes", C.c_int),
                ("boxes", c_int_p), ("mpoles", C.c_int), ("mresidues", c_float_p), ("mbpoles", c_float_p)]


class PlaneWaveSrc(C.Structure):
    _fields_ = [("x1", C.c_int), ("y1", C.c_int), ("z1", C.c_int), ("x2", C.c_int), ("y2", C.c_int), ("z2", C.c_int),
                ("theta", C.c_float), ("phi", C.c_float), ("alpha", C.c_float), ("beta", C.c_float),
                ("nsamples", C.c_int), ("samples", c_float_p), ("dsamples", C.c_float)]


class NodalSrc(C.Structure):
    _fields_ = [("is_elec", C.c_int), ("is_hard", C.c_int), ("npoints", C.c_int), ("boxes", c_int_p), ("amp", c_float_p),
                ("nsamples", C.c_int), ("samples", c_float_p), ("dsamples", C.c_float)]


class ProblemDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("desx", c_float_p), ("desy", c_float_p), ("desz", c_float_p),
                ("originx", C.c_float), ("originy", C.c_float), ("originz", C.c_float),
                ("dt", C.c_double), ("forcecfl", C.c_int), ("cfl", C.c_float),
                ("pml_layers", C.c_int * 6), ("pml_order", C.c_float * 6), ("pml_refl", C.c_float * 6),
                ("alphamax", C.c_float), ("alphaorder", C.c_float), ("kappamax", C.c_float),
                ("nregions", C.c_int), ("regions", C.POINTER(Region)),
                ("npw", C.c_int), ("pw", C.POINTER(PlaneWaveSrc)),
                ("nnodal", C.c_int), ("nodal", C.POINTER(NodalSrc)),
                ("nprobes", C.c_int), ("probes", c_int_p), ("probe_capacity", C.c_int),
                ("border", C.c_int * 6), ("mur_after_pml", C.c_int)]


class GridDesc(C.Structure):
    _fields_ = [("alloc", Lim * 6), ("sweep", Lim * 6), ("num_media", C.c_int),
                ("g1", c_float_p), ("g2", c_float_p), ("gm1", c_float_p), ("gm2", c_float_p),
                ("is_pec", C.POINTER(C.c_uint8)),
                ("idxe", c_float_p), ("idye", c_float_p), ("idze", c_float_p),
                ("idxh", c_float_p), ("idyh", c_float_p), ("idzh", c_float_p), ("dt", C.c_double)]


class FreqProbeDesc(C.Structure):
    _fields_ = [("magnetic", C.c_int), ("box", C.c_int * 6), ("stride", C.c_int * 3), ("nfreq", C.c_int),
                ("freq", c_float_p)]


class MovieProbeDesc(C.Structure):
    _fields_ = [("magnetic", C.c_int), ("box", C.c_int * 6), ("stride", C.c_int * 3), ("n_first", C.c_int),
                ("n_last", C.c_int), ("every", C.c_int), ("capacity", C.c_int)]


class FarFieldSpec(C.Structure):
    _fields_ = [("box", C.c_int * 6), ("faces", C.c_int * 6), ("initial_freq", C.c_float),
                ("final_freq", C.c_float), ("freq_step", C.c_float), ("logarithmic", C.c_int),
                ("decimate", C.c_int)]


class FarFieldAngles(C.Structure):
    _fields_ = [("theta_start", C.c_float), ("theta_stop", C.c_float), ("theta_step", C.c_float),
                ("phi_start", C.c_float), ("phi_stop", C.c_float), ("phi_step", C.c_float)]


ERRORS = {0: "ok", 1: "bad argument", 2: "out of memory", 3: "CUDA error", 4: "call out of order",
          5: "non-finite field", 6: "timeout", 7: "unsupported", 8: "size above the stated maximum"}


class SembaGpuError(RuntimeError):
    pass


_libs: dict[str, C.CDLL] = {}


def lib_path(variant: str = "exact") -> Path:
    name = "libsemba_gpu.so" if variant == "exact" else "libsemba_gpu_fast.so"
    return _BUILD / name


def load(variant: str = "exact") -> C.CDLL:
    """Load (once) the exact (-fmad=false) or fast (FMA) library."""
    if variant in _libs:
        return _libs[variant]
    path = lib_path(variant)
    if not path.exists():
        raise SembaGpuError(f"{path} is missing: build it with `python -m semba_fdtd_b200.build` "
                            "(there is no CPU fallback)")
    lib = C.CDLL(str(path))
    _declare(lib)
    _libs[variant] = lib
    return lib


def _declare(lib: C.CDLL) -> None:
    vp = C.c_void_p
    sig = {
        "sgpu_create": ([C.POINTER(GridDesc), C.POINTER(vp)], C.c_int),
        "sgpu_destroy": ([vp], None),
        "sgpu_last_error": ([vp], C.c_char_p),
        "sgpu_synchronize": ([vp], C.c_int),
        "sgpu_get_stream": ([vp, C.POINTER(vp)], C.c_int),
        "sgpu_upload_media": ([vp, C.c_int, C.POINTER(C.c_int16)], C.c_int),
        "sgpu_upload_field": ([vp, C.c_int, c_float_p], C.c_int),
        "sgpu_download_field": ([vp, C.c_int, c_float_p], C.c_int),
        "sgpu_pinned_alloc": ([C.c_uint64, C.POINTER(vp)], C.c_int),
        "sgpu_pinned_free": ([vp], C.c_int),
        "sgpu_set_time": ([vp, C.c_int, C.c_int, c_double_p], C.c_int),
        "sgpu_set_probes": ([vp, C.c_int, c_int_p, C.c_int], C.c_int),
        "sgpu_read_probes": ([vp, c_float_p, C.c_int, c_int_p, c_int_p], C.c_int),
        "sgpu_add_freq_probe": ([vp, C.POINTER(FreqProbeDesc), c_int_p], C.c_int),
        "sgpu_store_resume": ([vp, C.c_char_p, C.c_int, C.c_float, C.c_float], C.c_int),
        "sgpu_host_create_zslab": ([C.POINTER(ProblemDesc), C.c_int, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
        "sgpu_zplane": ([vp, C.c_int, C.c_int, C.POINTER(vp), C.POINTER(C.c_uint64)], C.c_int),
        "sgpu_copy_zplane": ([vp, vp, C.c_int, C.c_int], C.c_int),
        "sgpu_load_resume": ([vp, C.c_char_p, c_int_p], C.c_int),
        "sgpu_host_get_constants": ([vp, c_float_p, c_float_p], C.c_int),
        "sgpu_get_time": ([vp, C.c_int, C.c_int, C.POINTER(C.c_double)], C.c_int),
        "sgpu_host_incident": ([vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, c_float_p, c_float_p], C.c_int),
        "sgpu_add_movie_probe": ([vp, C.POINTER(MovieProbeDesc), c_int_p], C.c_int),
        "sgpu_volume_probe_shape": ([vp, C.c_int, c_int_p, c_int_p, c_int_p, c_int_p], C.c_int),
        "sgpu_read_freq_probe": ([vp, C.c_int, C.POINTER(C.c_double)], C.c_int),
        "sgpu_read_movie_probe": ([vp, C.c_int, c_float_p, C.c_int, c_int_p, c_int_p], C.c_int),
        "sgpu_host_add_farfield": ([vp, C.POINTER(FarFieldSpec), c_int_p], C.c_int),
        "sgpu_farfield_shape": ([vp, C.c_int, c_int_p, c_int_p], C.c_int),
        "sgpu_read_farfield": ([vp, C.c_int, C.c_int, C.c_int, c_int_p, C.POINTER(C.c_double)], C.c_int),
        "sgpu_farfield_transform": ([vp, C.c_int, C.POINTER(FarFieldAngles), c_float_p, C.c_int,
                                     C.POINTER(C.c_double), C.c_int, c_int_p], C.c_int),
        "sgpu_advance_e": ([vp, C.c_int], C.c_int),
        "sgpu_advance_h": ([vp, C.c_int], C.c_int),
        "sgpu_advance_steps": ([vp, C.c_int, C.c_int], C.c_int),
        "sgpu_check_finite": ([vp], C.c_int),
        "sgpu_device_bytes": ([vp, C.POINTER(C.c_uint64)], C.c_int),
        "sgpu_elapsed_steps": ([vp, C.c_int, C.c_int, c_float_p], C.c_int),
        "sgpu_profile_steps": ([vp, C.c_int, C.c_int, c_float_p], C.c_int),
        "sgpu_kernels_per_step": ([vp, c_int_p], C.c_int),
        "sgpu_algorithmic_bytes": ([vp, c_double_p], C.c_int),
        "sgpu_compulsory_bytes": ([vp, c_double_p], C.c_int),
        "sgpu_select_device": ([C.c_int], C.c_int),
        "sgpu_set_kernel_family": ([vp, C.c_int], C.c_int),
        "sgpu_scan_nonfinite_noalloc": ([vp, C.c_uint64, vp, C.POINTER(C.c_uint64), C.POINTER(C.c_int64)], C.c_int),
        "sgpu_host_create": ([C.POINTER(ProblemDesc), C.c_int, C.POINTER(vp)], C.c_int),
        "sgpu_host_plan": ([C.POINTER(ProblemDesc), C.c_int, C.POINTER(vp)], C.c_int),
        "sgpu_host_footprint": ([vp, C.POINTER(C.c_uint64)], C.c_int),
        "sgpu_host_info": ([vp, c_double_p, c_int_p, C.POINTER(Lim), C.POINTER(Lim), C.POINTER(Lim)], C.c_int),
        "sgpu_host_get_g": ([vp, c_float_p, c_float_p, c_float_p, c_float_p], C.c_int),
        "sgpu_host_get_metric": ([vp, C.c_int, c_float_p, c_int_p, c_int_p], C.c_int),
        "sgpu_host_get_media": ([vp, C.c_int, C.POINTER(C.c_int16)], C.c_int),
        "sgpu_host_get_mur_cab1": ([vp, C.c_int, c_float_p], C.c_int),
        "sgpu_batch_create": ([C.c_uint64, C.c_int, C.POINTER(vp)], C.c_int),
        "sgpu_batch_destroy": ([vp], None),
        "sgpu_batch_last_error": ([vp], C.c_char_p),
        "sgpu_batch_add": ([vp, C.POINTER(ProblemDesc), vp, C.c_int, c_int_p], C.c_int),
        "sgpu_batch_remove": ([vp, C.c_int], C.c_int),
        "sgpu_batch_advance": ([vp, C.c_int], C.c_int),
        "sgpu_batch_synchronize": ([vp], C.c_int),
        "sgpu_batch_elapsed": ([vp, C.c_int, c_float_p], C.c_int),
        "sgpu_batch_slot_info": ([vp, C.c_int, c_int_p, c_int_p, c_int_p], C.c_int),
        "sgpu_batch_read_probes": ([vp, C.c_int, c_float_p, C.c_int, c_int_p], C.c_int),
        "sgpu_batch_instance": ([vp, C.c_int, C.POINTER(vp)], C.c_int),
        "sgpu_batch_memory": ([vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
        "sgpu_batch_footprint": ([vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)], C.c_int),
        "sgpu_batch_set_kernel_family": ([vp, C.c_int], C.c_int),
        "sgpu_batch_set_wait_cycles": ([vp, C.c_int64], C.c_int),
        "sgpu_set_wait_cycles": ([vp, C.c_int64], C.c_int),
        "sgpu_trim_device_memory": ([], C.c_int),
        "sgpu_set_wait_drill": ([vp, C.c_int], C.c_int),
        "sgpu_batch_set_wait_drill": ([vp, C.c_int], C.c_int),
        "sgpu_batch_set_tuning": ([vp, c_int_p, C.c_int], C.c_int),
        "sgpu_batch_get_tuning": ([vp, c_int_p, c_int_p], C.c_int),
        "sgpu_batch_autotune": ([vp, C.c_int, c_int_p, c_int_p], C.c_int),
        "sgpu_batch_profile_steps": ([vp, C.c_int, c_float_p], C.c_int),
        "sgpu_batch_steps": ([vp, c_int_p], C.c_int),
    }
    for name, (args, res) in sig.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    for name in ["sgpu_advance_ex", "sgpu_advance_ey", "sgpu_advance_ez", "sgpu_advance_electric_cpml",
                 "sgpu_advance_edispersive_e", "sgpu_advance_hx", "sgpu_advance_hy", "sgpu_advance_hz",
                 "sgpu_advance_magnetic_cpml", "sgpu_advance_pmc_h", "sgpu_advance_periodic_h",
                 "sgpu_advance_magnetic_mur", "sgpu_advance_mdispersive_h"]:
        f = getattr(lib, name)
        f.argtypes = [vp]
        f.restype = C.c_int
    for name in ["sgpu_advance_planewave_e", "sgpu_advance_nodal_e", "sgpu_advance_planewave_h",
                 "sgpu_advance_nodal_h", "sgpu_update_observation"]:
        f = getattr(lib, name)
        f.argtypes = [vp, C.c_int]
        f.restype = C.c_int


def pinned_empty(shape, dtype, variant: str = "exact"):
    """A numpy array in page-locked host memory (sgpu_pinned_alloc): field
    uploads and downloads through it go straight to the copy engine.  The
    memory is freed when the array (and every view of it) is gone."""
    import weakref

    import numpy as np
    lib = load(variant)
    dt = np.dtype(dtype)
    n = int(np.prod(shape)) * dt.itemsize
    p = C.c_void_p()
    rc = lib.sgpu_pinned_alloc(max(n, 1), C.byref(p))
    if rc:
        raise SembaGpuError(f"sgpu_pinned_alloc failed ({ERRORS.get(rc, rc)})")
    buf = (C.c_char * max(n, 1)).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dt, count=int(np.prod(shape))).reshape(shape)
    weakref.finalize(buf, lib.sgpu_pinned_free, C.c_void_p(p.value))
    return arr


def exported_symbols(header: Path | None = None) -> list[str]:
    """Names of the entry points declared in include/semba_gpu.h."""
    import re
    header = header or (_HERE.parent / "include" / "semba_gpu.h")
    txt = header.read_text()
    return sorted(set(re.findall(r"\b(sgpu_[a-z0-9_]+)\s*\(", txt)))
