"""The allocation-free non-finite scan, checked against sgpu_check_finite.

sgpu_scan_nonfinite_noalloc serves callers that cannot allocate device
memory where they need the check (a Fortran or framework host whose device
memory belongs to its own pool allocator, a service loop that forbids
cudaMalloc after start-up, a watchdog scanning a buffer it does not own).
It keeps its scratch in a file-scope device array instead.  This file sorts
last so that a run stopping at the first failure has run every other test;
it also passes on its own in a fresh process (the first call on the device
takes the scratch address)."""
import ctypes as C

import numpy as np
import pytest

from cases import ALL
from semba_fdtd_b200 import Solver, _lib

pytestmark = pytest.mark.gpu

SGPU_ERR_NONFINITE = 5
SGPU_ERR_SIZE = 8


def _scan(lib, dev_tensor):
    cnt, first = C.c_uint64(), C.c_int64()
    rc = lib.sgpu_scan_nonfinite_noalloc(C.c_void_p(dev_tensor.data_ptr()), dev_tensor.numel(), None,
                                         C.byref(cnt), C.byref(first))
    assert rc == 0, _lib.ERRORS.get(rc, rc)
    return cnt.value, first.value


def test_noalloc_scan_matches_check_finite_on_two_calls():
    import torch

    lib = _lib.load()
    pb = ALL["small"]()
    comp = 2
    with Solver(pb) as s:
        s.step(20)
        clean = np.ascontiguousarray(s.field(comp).transpose(2, 1, 0)).reshape(-1)
        assert np.all(np.isfinite(clean))
        bad = clean.copy()
        planted = [17, 4096 + 3, bad.size - 1]
        bad[planted[0]] = np.nan
        bad[planted[1]] = np.inf
        bad[planted[2]] = -np.inf
        # two calls in a row on different data: the second must not see the
        # first call's results left in the shared scratch
        for arr in (bad, clean):
            assert lib.sgpu_upload_field(s.handle, comp, arr.ctypes.data_as(_lib.c_float_p)) == 0
            rc_existing = lib.sgpu_check_finite(s.handle)
            assert rc_existing in (0, SGPU_ERR_NONFINITE)
            dev = torch.from_numpy(arr).cuda()
            torch.cuda.synchronize()
            count, first = _scan(lib, dev)
            assert (count > 0) == (rc_existing == SGPU_ERR_NONFINITE)
            want = np.flatnonzero(~np.isfinite(arr))
            assert count == want.size
            assert first == (int(want[0]) if want.size else -1)


def test_noalloc_scan_many_blocks_and_size_limit():
    import torch

    lib = _lib.load()
    n = 5 * 4096 * 251 + 7  # many blocks, ragged tail
    host = np.linspace(-1.0, 1.0, n, dtype=np.float32)
    host[n - 2] = np.nan
    host[4096 * 300 + 11] = np.inf
    for arr in (host, np.nan_to_num(host, nan=0.0, posinf=0.0)):
        dev = torch.from_numpy(arr).cuda()
        torch.cuda.synchronize()
        count, first = _scan(lib, dev)
        want = np.flatnonzero(~np.isfinite(arr))
        assert count == want.size
        assert first == (int(want[0]) if want.size else -1)
    # above the stated maximum: rejected before the data is touched
    cnt, first = C.c_uint64(), C.c_int64()
    rc = lib.sgpu_scan_nonfinite_noalloc(C.c_void_p(dev.data_ptr()), 4096 * 65536 + 1, None, C.byref(cnt), C.byref(first))
    assert rc == SGPU_ERR_SIZE
