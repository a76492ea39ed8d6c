"""Restart files (resuming.F90:113-496): the records of flush_and_save_resume
and the resume branches of the Init* routines.

CPU: the oracle's own store -> load -> continue equals an uninterrupted run,
and its file has the reference's record layout.  GPU: the library writes the
oracle's file for the same state (record for record; the currents of a
folded conjugate pole may differ only in the sign of a zero), and a run that
resumes from the oracle's file equals the uninterrupted oracle run."""
import struct

import numpy as np

from bits import assert_bits_equal
import pytest

from cases import disp, mdisp, mixed, mur, small
from semba_fdtd_b200.observation import fortran_records

import oracle

CASES = {"small": lambda: small(n=16, steps=40, layers=4), "disp": disp, "mdisp": mdisp, "mur": mur, "mixed": mixed}
N1, N2 = 23, 17


def _straight(pb, steps):
    o = oracle.Oracle(pb)
    tr = o.step(steps)
    return o, tr


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_resume_continues_exactly(name, tmp_path):
    pb = CASES[name]()
    o_full, tr_full = _straight(pb, N1 + N2)
    a = oracle.Oracle(pb)
    tr_a = a.step(N1)
    a.store_resume(tmp_path / "r.bin")
    b = oracle.Oracle(pb)
    assert b.load_resume(tmp_path / "r.bin") == N1 - 1
    tr_b = b.step(N2)
    assert_bits_equal(np.concatenate([tr_a, tr_b]), tr_full)
    for c in range(6):
        assert_bits_equal(b.field(c), o_full.field(c))


def test_oracle_resume_record_layout(tmp_path):
    pb = CASES["disp"]()
    o = oracle.Oracle(pb)
    o.step(5)
    o.store_resume(tmp_path / "r.bin")
    recs = fortran_records((tmp_path / "r.bin").read_bytes())
    n, t, dt, eps0, mu0 = struct.unpack("<iddff", recs[0])
    assert n == 4 and t == o.time(4) and dt == o.dt and eps0 > 0 and mu0 > 0
    # StoreFields: per component, per (j, k) row of its Alloc box, blocks of
    # 1024 values and a remainder record
    q = 1
    for c in range(6):
        xi, xe, yi, ye, zi, ze = o.alloc[c]
        ax = xe - xi + 1
        f = o.field(c)
        for k in range(ze - zi + 1):
            for j in range(ye - yi + 1):
                nb = ax // 1024
                for b in range(nb):
                    assert len(recs[q]) == 4096
                    q += 1
                row = np.frombuffer(recs[q], np.float32)
                assert len(row) == ax - 1024 * nb
                assert_bits_equal(row, f[1024 * nb:, j, k])
                q += 1
    assert q < len(recs)  # CPML psi and ADE records follow


def _records_equal(ga, oa):
    ra, rb = fortran_records(ga), fortran_records(oa)
    assert len(ra) == len(rb)
    for q, (x, y) in enumerate(zip(ra, rb)):
        assert len(x) == len(y), q
        if x != y:
            # only a 16-byte current record may differ, and only in the sign of
            # zeros (a folded pole's current is written as the conjugate of the
            # kept one), so values are compared here, not bits
            assert len(x) == 16, q
            np.testing.assert_array_equal(np.frombuffer(x, np.float64), np.frombuffer(y, np.float64), err_msg=str(q))


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_gpu_resume_matches_oracle(name, tmp_path):
    from semba_fdtd_b200 import Solver
    pb = CASES[name]()
    o = oracle.Oracle(pb)
    o.step(N1)
    o.store_resume(tmp_path / "o.bin")
    with Solver(pb) as s:
        s.step(N1)
        s.store_resume(tmp_path / "g.bin")
    _records_equal((tmp_path / "g.bin").read_bytes(), (tmp_path / "o.bin").read_bytes())
    o_full, tr_full = _straight(pb, N1 + N2)
    for mode in ("graph", "routines"):
        with Solver(pb) as s:
            assert s.load_resume(tmp_path / "o.bin") == N1 - 1
            s.step(N2, mode=mode)
            assert_bits_equal(s.probes(), tr_full[N1:], err_msg=mode)
            for c in range(6):
                assert_bits_equal(s.field(c), o_full.field(c), err_msg=f"{mode} component {c}")


@pytest.mark.gpu
def test_gpu_resume_rejects_other_setup(tmp_path):
    from semba_fdtd_b200 import Solver
    from semba_fdtd_b200._lib import SembaGpuError
    o = oracle.Oracle(CASES["disp"]())
    o.step(3)
    o.store_resume(tmp_path / "o.bin")
    with Solver(CASES["small"]()) as s:
        with pytest.raises(SembaGpuError):
            s.load_resume(tmp_path / "o.bin")


@pytest.mark.gpu
def test_gpu_resume_rejects_truncated_file(tmp_path):
    from semba_fdtd_b200 import Solver
    from semba_fdtd_b200._lib import SembaGpuError
    pb = CASES["disp"]()
    o = oracle.Oracle(pb)
    o.step(3)
    o.store_resume(tmp_path / "o.bin")
    data = (tmp_path / "o.bin").read_bytes()
    (tmp_path / "cut.bin").write_bytes(data[: len(data) // 2])
    with Solver(pb) as s:
        with pytest.raises(SembaGpuError):
            s.load_resume(tmp_path / "cut.bin")
    # a file that parses is still accepted by a fresh solver after the refusal
    with Solver(pb) as s:
        assert s.load_resume(tmp_path / "o.bin") == 2
        s.step(2)
        assert s.check_finite()
