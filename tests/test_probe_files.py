"""Point-probe output files in the reference's format (row a16).

FlushObservationFiles (observation.F90:3763-3874) writes one text file per
point probe: a header line, then per saved step the time (e27.17e3), the
value and, with plane waves, the incident field there (e19.9e3 each,
fdetypes.F90:229).  CPU tests pin the text format against the reference's
own expected output (tests/golden/ref/probe_format_excerpt.dat) and check
names, windows and line counts on oracle runs; the GPU tests write the files
of library runs and require them byte-identical to the oracle's."""
from dataclasses import replace
from pathlib import Path

import numpy as np
import pytest

from semba_fdtd_b200 import read_case
from semba_fdtd_b200.observation import (fortran_e, point_probe_paths, point_probe_rows, probe_header,
                                         write_point_probes)

import oracle

GOLD = Path(__file__).resolve().parent / "golden" / "ref"
REF_CASE = GOLD / "planewave.fdtd.json"


def test_number_format_matches_reference_output():
    """Every number of the reference's expected probe file re-formats to the
    same characters: the time as real(8) e27.17e3, the values as real(4)
    e19.9e3 (negative zeros included)."""
    lines = (GOLD / "probe_format_excerpt.dat").read_text().splitlines()
    assert len(lines) > 40
    negzero = 0
    for ln in lines[1:]:
        tok = ln.split()
        t = float(tok[0])
        vals = [np.float32(float(v)) for v in tok[1:]]
        negzero += sum(1 for v in tok[1:] if v.startswith("-0.000000000"))
        again = fortran_e(t, 27, 17) + "".join(fortran_e(v, 19, 9) for v in vals)
        assert again == ln
    assert negzero > 0


def test_header_matches_reference_output():
    head = (GOLD / "probe_format_excerpt.dat").read_text().splitlines()[0]
    name = "holland1981.fdtd_mid_point_Wz_11_11_12_s2.dat"
    assert probe_header(name, " -E*dl Vplus Vminus Vplus-Vminus") == head
    assert probe_header("a.dat", "incid") == "t              a.dat       incid"
    assert probe_header("a.dat", " ") == "t              a.dat"


def test_fortran_e_edges():
    assert fortran_e(0.0, 19, 9) == "   0.000000000E+000"
    assert fortran_e(-0.0, 19, 9) == "  -0.000000000E+000"
    assert fortran_e(np.float32(9.9999999e-5), 19, 9) == "   0.999999975E-004"
    assert fortran_e(9.9999999999e9, 19, 9) == "   0.100000000E+011"
    assert fortran_e(1.0, 27, 17) == "   0.10000000000000000E+001"
    assert fortran_e(np.float32(-3.4028235e38), 19, 9) == "  -0.340282347E+039"
    assert fortran_e(np.float32(1.4e-45), 19, 9) == "   0.140129846E-044"


def test_paths_of_the_reference_case():
    pb = read_case(REF_CASE)
    assert pb.root == "planewave.fdtd"
    assert point_probe_paths(pb) == [f"planewave.fdtd_electric_field_point_probe_{c}_4_4_4.dat"
                                     for c in ("Ex", "Ey", "Ez")]
    # the same probe twice: later items get _duplicate_<unit>.dat appended
    pb2 = replace(pb, probes=np.concatenate([pb.probes, pb.probes[:1]]),
                  probe_requests=pb.probe_requests + pb.probe_requests[:1])
    assert point_probe_paths(pb2)[3] == "planewave.fdtd_electric_field_point_probe_Ex_4_4_4.dat_duplicate_1004.dat"


def test_time_window_and_sampling():
    pb = read_case(REF_CASE)
    o = oracle.Oracle(pb)
    try:
        dt = o.dt
        tiempo = np.array([o.time(n) for n in range(0, 60)])
    finally:
        o.close()
    # every step without a window
    steps, tcol, tinc = point_probe_rows(pb, 0, tiempo, dt, 0, 50, 50)
    assert steps == list(range(51)) and np.array_equal(tcol, tiempo[:51])
    # samplingPeriod 3 dt (int(3 dt / dt) may truncate to 2: as the reference)
    t0, t1, ts = np.float32(5 * dt), np.float32(30 * dt), np.float32(3 * dt)
    req = [(r[0], float(t0), float(t1), float(ts)) for r in pb.probe_requests]
    pw = replace(pb, probe_requests=req)
    tr = max(1, int(float(ts) / dt))
    steps, tcol, _ = point_probe_rows(pw, 0, tiempo, dt, 0, 50, 50)
    want = [n for n in range(51) if n % tr == 0 and float(t0) <= tiempo[n] <= float(t1) + dt / 2]
    assert steps == want and len(steps) > 5
    # an H probe: the window on tiempo + dt/2, the time column at - dt/2
    ph = replace(pw, probes=np.asarray([[4, 4, 4, 4]], np.int32), probe_requests=req[:1])
    steps, tcol, tinc = point_probe_rows(ph, 0, tiempo, dt, 0, 50, 50)
    at = tiempo[np.asarray(steps)] + dt / 2
    assert np.array_equal(tcol, at - dt / 2) and np.array_equal(tinc, at.astype(np.float32))


def _oracle_files(pb, steps, outdir):
    o = oracle.Oracle(pb)
    try:
        tr = o.step(steps)
        tiempo = np.array([o.time(n) for n in range(steps + 2)])
        paths = write_point_probes(outdir, pb, tr, tiempo, o.dt, incident=o.incident)
    finally:
        o.close()
    return paths


def test_oracle_files_of_the_reference_case(tmp_path):
    """The reference's own case: three files of steps + 2 lines (header and
    steps 0..nsteps, as test/pyWrapper/test_full_system.py counts them), an
    incident column that carries the Gaussian, and pandas can read them as
    the reference's post-processing does (whitespace-separated, header row)."""
    import pandas as pd
    pb = read_case(REF_CASE)
    steps = 301
    paths = _oracle_files(pb, steps, tmp_path)
    assert [p.name for p in paths] == point_probe_paths(pb)
    for p in paths:
        lines = p.read_text().splitlines()
        assert len(lines) == steps + 1
        assert lines[0] == f"t              {p.name}       incid"
        df = pd.read_csv(p, sep=r"\s+")
        assert list(df.columns) == ["t", p.name, "incid"] and len(df) == steps
    inc = pd.read_csv(paths[0], sep=r"\s+")["incid"].to_numpy()
    assert np.max(np.abs(inc)) > 0.5  # the x-polarised unit plane wave passes the Ex probe


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["reference", "small"])
def test_library_files_equal_oracle_files(tmp_path, case):
    """A library run's probe files are byte-identical to the oracle's: same
    values (bit-exact build), same time vector, same incident column."""
    from semba_fdtd_b200 import Solver
    from cases import small
    pb = read_case(REF_CASE) if case == "reference" else small()
    steps = pb.nsteps + 1
    ref = _oracle_files(pb, steps, tmp_path / "oracle")
    with Solver(pb) as s:
        tr = s.run(steps)
        got = write_point_probes(tmp_path / "gpu", pb, tr, s.time_vector(), s.dt, incident=s.incident)
    assert [p.name for p in got] == [p.name for p in ref]
    for a, b in zip(got, ref):
        assert a.read_bytes() == b.read_bytes(), a.name
        assert len(a.read_text().splitlines()) == steps + 1
