"""CPU tests of the C ABI library's host side (no GPU needed): the library
loads and exports every entry point of include/semba_gpu.h, and the level-2
set-up (sgpu_host_plan) produces exactly the oracle's dt, coefficient tables,
metric/CPML vectors and media matrices."""
import ctypes as C
from pathlib import Path

import numpy as np

from bits import assert_bits_equal
import pytest

from cases import ALL
from semba_fdtd_b200 import _lib

import oracle


def test_library_exports_every_declared_symbol():
    for variant in ("exact", "fast"):
        lib = C.CDLL(str(_lib.lib_path(variant)))
        missing = [s for s in _lib.exported_symbols() if not hasattr(lib, s)]
        assert not missing, f"{variant}: {missing}"


def _plan(pb):
    lib = _lib.load()
    d, keep = pb.to_desc()
    h = C.c_void_p()
    assert lib.sgpu_host_plan(C.byref(d), pb.nsteps, C.byref(h)) == 0
    return lib, h


@pytest.mark.parametrize("name", list(ALL))
def test_host_plan_matches_oracle_setup(name):
    pb = ALL[name]()
    lib, h = _plan(pb)
    try:
        o = oracle.Oracle(pb)
        dt, nm = C.c_double(), C.c_int()
        a6, s6, q6 = (_lib.Lim * 6)(), (_lib.Lim * 6)(), (_lib.Lim * 6)()
        assert lib.sgpu_host_info(h, C.byref(dt), C.byref(nm), a6, s6, q6) == 0
        # NFDE2sgg time step and the media count after CreatePMLmatrix
        assert dt.value == o.dt
        assert nm.value == o.num_media
        assert [a.tuple() for a in a6] == o.alloc
        assert [s.tuple() for s in s6] == o.sweep
        assert [q.tuple() for q in q6] == o.sinpml
        n1 = nm.value + 1
        hg = [np.empty(n1, np.float32) for _ in range(4)]
        lib.sgpu_host_get_g(h, *[x.ctypes.data_as(_lib.c_float_p) for x in hg])
        for a, b in zip(hg, o.g_tables()):
            assert_bits_equal(a, b)
        for w in range(18):
            lo, hi = C.c_int(), C.c_int()
            lib.sgpu_host_get_metric(h, w, None, C.byref(lo), C.byref(hi))
            arr = np.empty(hi.value - lo.value + 1, np.float32)
            lib.sgpu_host_get_metric(h, w, arr.ctypes.data_as(_lib.c_float_p), None, None)
            olo, oarr = o.metric(w)
            assert olo == lo.value
            assert_bits_equal(arr, oarr)
        # calc_murconstants per Mur face
        for f in range(6):
            oc = o.mur_cab1(f)
            hc = np.empty(n1, np.float32)
            rc = lib.sgpu_host_get_mur_cab1(h, f, hc.ctypes.data_as(_lib.c_float_p))
            assert (rc == 0) == (oc is not None)
            if oc is not None:
                assert_bits_equal(hc, oc)
        for c in range(6):
            xi, xe, yi, ye, zi, ze = a6[c].tuple()
            m = np.empty((ze - zi + 1, ye - yi + 1, xe - xi + 1), np.int16)
            lib.sgpu_host_get_media(h, c, m.ctypes.data_as(C.POINTER(C.c_int16)))
            assert_bits_equal(m, o.media(c).transpose(2, 1, 0))
    finally:
        lib.sgpu_destroy(h)


def test_footprint_counts_fields_media_and_ade_state():
    pb = ALL["disp"]()
    lib, h = _plan(pb)
    try:
        b = C.c_uint64()
        assert lib.sgpu_host_footprint(h, C.byref(b)) == 0
        cells = pb.swept_cells
        # at least 6 fields x 4 B and 6 media x 2 B per swept cell
        assert b.value >= cells * 36
    finally:
        lib.sgpu_destroy(h)


def test_plan_rejects_bad_problems():
    pb = ALL["small"]()
    lib = _lib.load()
    d, keep = pb.to_desc()
    d.pml_layers[0] = 0
    h = C.c_void_p()
    assert lib.sgpu_host_plan(C.byref(d), 10, C.byref(h)) == 1
    d, keep = pb.to_desc()
    d.nx = 1
    assert lib.sgpu_host_plan(C.byref(d), 10, C.byref(h)) == 1
    # a border code outside nfde_types.F90:67-71
    d, keep = pb.to_desc()
    d.border[3] = 3
    assert lib.sgpu_host_plan(C.byref(d), 10, C.byref(h)) == 1
    # a non-CPML face needs no layers
    d, keep = pb.to_desc()
    d.border[0], d.pml_layers[0] = 7, 0
    assert lib.sgpu_host_plan(C.byref(d), 10, C.byref(h)) == 0
    lib.sgpu_destroy(h)


# the reference's own case, copied by tests/golden/make_reference_fixtures.py
REF_CASE = Path(__file__).resolve().parent / "golden" / "ref" / "planewave.fdtd.json"


def test_reference_mur_case_plan_matches_oracle():
    """The reference's own Mur case (testData/cases/planewave.fdtd.json): the
    library's set-up equals the oracle's, including CAB1 of every face."""
    from semba_fdtd_b200 import read_case
    pb = read_case(REF_CASE)
    assert pb.borders == ("mur",) * 6
    lib, h = _plan(pb)
    try:
        o = oracle.Oracle(pb)
        n1 = o.num_media + 1
        for f in range(6):
            hc = np.empty(n1, np.float32)
            assert lib.sgpu_host_get_mur_cab1(h, f, hc.ctypes.data_as(_lib.c_float_p)) == 0
            assert_bits_equal(hc, o.mur_cab1(f))
        for c in range(6):
            xi, xe, yi, ye, zi, ze = o.alloc[c]
            m = np.empty((ze - zi + 1, ye - yi + 1, xe - xi + 1), np.int16)
            lib.sgpu_host_get_media(h, c, m.ctypes.data_as(C.POINTER(C.c_int16)))
            assert_bits_equal(m, o.media(c).transpose(2, 1, 0))
    finally:
        lib.sgpu_destroy(h)


def _device_case(name):
    from semba_fdtd_b200 import read_case
    if name == "reference":
        return read_case(REF_CASE)
    return ALL[name]()


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(ALL) + ["reference"])
def test_device_built_media_equal_host_plan(name):
    """sgpu_host_create builds the media matrices on the device (region
    painting, PML extrusion and copies, PEC borders); they, the media count,
    the coefficient tables and CAB1 equal the host plan's bit for bit."""
    from semba_fdtd_b200 import Solver
    pb = _device_case(name)
    lib, h = _plan(pb)
    try:
        with Solver(pb) as s:
            dt, nm = C.c_double(), C.c_int()
            a6, s6, q6 = (_lib.Lim * 6)(), (_lib.Lim * 6)(), (_lib.Lim * 6)()
            assert lib.sgpu_host_info(h, C.byref(dt), C.byref(nm), a6, s6, q6) == 0
            assert s.num_media == nm.value
            n1 = nm.value + 1
            hg = [np.empty(n1, np.float32) for _ in range(4)]
            lib.sgpu_host_get_g(h, *[x.ctypes.data_as(_lib.c_float_p) for x in hg])
            for a, b in zip(s.g_tables(), hg):
                assert_bits_equal(a, b)
            for f in range(6):
                hc = np.empty(n1, np.float32)
                rc = lib.sgpu_host_get_mur_cab1(h, f, hc.ctypes.data_as(_lib.c_float_p))
                dc = s.mur_cab1(f)
                assert (rc == 0) == (dc is not None)
                if dc is not None:
                    assert_bits_equal(dc, hc)
            for c in range(6):
                xi, xe, yi, ye, zi, ze = a6[c].tuple()
                m = np.empty((ze - zi + 1, ye - yi + 1, xe - xi + 1), np.int16)
                lib.sgpu_host_get_media(h, c, m.ctypes.data_as(C.POINTER(C.c_int16)))
                assert_bits_equal(s.media(c), m.transpose(2, 1, 0), err_msg=f"component {c}")
    finally:
        lib.sgpu_destroy(h)
