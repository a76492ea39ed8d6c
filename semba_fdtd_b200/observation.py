"""Probe output files that mirror observation.F90's host side.

* ``write_point_probes`` -- the text file of every point probe
  (FlushObservationFiles, observation.F90:3763-3874; names and header,
  :600-731 and :941-945): one line per saved step with the time, the value
  and, when the problem has plane waves, the incident field there, in the
  format '(e27.17e3,11(e19.9e3))' (fdetypes.F90:229);
* ``fortran_e`` -- the Ew.dEe edit descriptor as gfortran writes it;
* ``frequency_list`` -- the frequencies of a frequency-domain probe
  (observation.F90:505-536), in real(4) arithmetic as the reference lists
  them;
* ``write_freq_probe`` / ``read_freq_probe`` -- the unformatted file of a
  frequency-domain volume probe (observation.F90:4013-4046): Fortran
  sequential records, each framed by its byte length as a 4-byte integer
  before and after (gfortran's default record markers).

The sampling and accumulation run on the device (``Solver.probes``,
``Solver.add_freq_probe``).
"""
from __future__ import annotations

import math
import struct
from pathlib import Path

import numpy as np

__all__ = ["frequency_list", "write_freq_probe", "read_freq_probe", "fortran_records", "fortran_e",
           "probe_header", "point_probe_paths", "point_probe_rows", "write_point_probes"]

_TINY32 = float(np.finfo(np.float32).tiny)
_PREFIX = ("Ex_", "Ey_", "Ez_", "Hx_", "Hy_", "Hz_")  # prefix() of observation.F90:4225-4245


def fortran_e(x: float, w: int, d: int, e: int = 3) -> str:
    """``x`` under the Fortran edit descriptor Ew.dEe as gfortran writes it:
    right-justified in w characters, an optional minus sign (also for -0.0),
    "0." and d digits of the correctly rounded decimal significand, then "E",
    the exponent's sign and e digits."""
    x = float(x)
    if math.isnan(x):
        body = "NaN"
    elif math.isinf(x):
        body = "Infinity" if x > 0 else "-Infinity"
    else:
        neg = math.copysign(1.0, x) < 0
        a = abs(x)
        if a == 0.0:
            digits, ex = "0" * d, 0
        else:
            mant, ex10 = f"{a:.{d - 1}e}".split("e")
            digits, ex = mant.replace(".", ""), int(ex10) + 1
        body = ("-" if neg else "") + "0." + digits + "E" + ("-" if ex < 0 else "+") + f"{abs(ex):0{e}d}"
    if len(body) > w:
        return "*" * w
    return body.rjust(w)


def probe_header(name: str, suffix: str) -> str:
    """The first line of a probe file (observation.F90:944-945):
    trim(adjustl(' t' // 14 blanks // name // 7 blanks // suffix)); the
    suffix of E and H probes is 'incid' with plane waves, else blank."""
    return (" t" + " " * 14 + name.strip() + " " * 7 + suffix.strip()).strip()


def point_probe_paths(problem) -> list:
    """File name of every point probe row of `problem` (InitObservation,
    observation.F90:600-731): <root>_<request>_<prefix><i>_<j>_<k>.dat with
    the prefix of the component (Ex_ .. Hz_); a name already taken by an
    earlier item gets "_duplicate_<unit>.dat" appended once per earlier
    match (checkduplicatenames, :2090-2106; units count from 1001)."""
    paths = []
    for q, (c, i, j, k) in enumerate(np.asarray(problem.probes).tolist()):
        req = problem.probe_requests[q][0] if problem.probe_requests else "probe"
        p = f"{problem.root}_{req}_{_PREFIX[c]}{i}_{j}_{k}.dat"
        p1 = p
        for prev in paths:
            if prev == p1:
                p = f"{p}_duplicate_{1001 + q}.dat"
        paths.append(p)
    return paths


def point_probe_rows(problem, q: int, tiempo, dt: float, first_n: int, last_n: int, final_step: int):
    """Steps n (first_n <= n <= last_n) that probe row q writes, with the
    time column and the real(4) time of its incident field.

    The window of FlushObservationFiles (observation.F90:3801-3818) after
    InitObservation's clipping (:268-290): a probe whose finalTime or
    samplingPeriod is below real(4) TINY saves every step; otherwise it
    saves the steps with mod(n, max(1, int(samplingPeriod/dt))) = 0 whose
    time at (tiempo(n), or tiempo(n) + dt/2 for H) lies in [initialTime,
    finalTime + dt/2], finalTime clipped to tiempo(final_step + 2).  The
    time column is at for E and at - dt/2 for H."""
    c = int(problem.probes[q][0])
    _, t0, t1, ts = problem.probe_requests[q] if problem.probe_requests else ("", 0.0, 0.0, 0.0)
    f32 = np.float32
    saveall = f32(t1) < _TINY32 or f32(ts) < _TINY32
    if saveall:
        trancos, init, final = 1, f32(0.0), f32(tiempo[final_step + 2])
    else:
        trancos = max(1, int(float(f32(ts)) / dt))
        init = f32(max(0.0, float(f32(t0))))
        final = f32(min(float(tiempo[final_step + 2]), float(f32(t1))))
        if final < init:
            final = init
    half = dt / 2.0
    steps, tcol, tinc = [], [], []
    for n in range(first_n, last_n + 1):
        if n % trancos:
            continue
        at = float(tiempo[n]) + half if c >= 3 else float(tiempo[n])
        if saveall or (at >= float(init) and at <= float(final) + half):
            steps.append(n)
            tcol.append(at - half if c >= 3 else at)
            tinc.append(at)
    return steps, np.asarray(tcol, np.float64), np.asarray(tinc, np.float64).astype(np.float32)


def write_point_probes(outdir, problem, traces, tiempo, dt: float, first_n: int = 0, final_step: int | None = None,
                       incident=None) -> list:
    """Write the point-probe files of a run (FlushObservationFiles,
    observation.F90:3763-3874, for the steps first_n .. first_n + rows - 1).

    traces: [rows, probes] float32 as ``Solver.probes`` returns them (row r
    is step first_n + r); tiempo: the FP64 time vector indexed by step
    (``Solver.time_vector()``), at least to final_step + 2; final_step: the
    run's last step (default the last row's); incident(comp, i, j, k, t32)
    gives the incident-field column (``Solver.incident``) and is required
    when the problem has plane waves.  Each file starts with the header
    line "t              <name>       incid" ("incid" only with plane
    waves) and holds one line per saved step.  Returns the paths."""
    outdir = Path(outdir)
    outdir.mkdir(parents=True, exist_ok=True)
    tr = np.asarray(traces, np.float32)
    last_n = first_n + tr.shape[0] - 1
    final_step = last_n if final_step is None else final_step
    with_incid = len(problem.planewaves) >= 1
    if with_incid and incident is None:
        raise ValueError("the problem has plane waves: pass incident=Solver.incident (or the oracle's)")
    out = []
    for q, name in enumerate(point_probe_paths(problem)):
        c, i, j, k = (int(v) for v in problem.probes[q])
        steps, tcol, tinc = point_probe_rows(problem, q, tiempo, dt, first_n, last_n, final_step)
        vals = tr[np.asarray(steps, np.int64) - first_n, q] if steps else np.zeros(0, np.float32)
        inc = incident(c, i, j, k, tinc) if with_incid and steps else None
        lines = [probe_header(name, "incid" if with_incid else "")]
        for r in range(len(steps)):
            ln = fortran_e(tcol[r], 27, 17) + fortran_e(vals[r], 19, 9)
            if with_incid:
                ln += fortran_e(inc[r], 19, 9)
            lines.append(ln)
        path = outdir / name
        path.write_text("\n".join(lines) + "\n")
        out.append(path)
    return out


def frequency_list(initial: float, final: float, step: float, logarithmic: bool = False) -> np.ndarray:
    """Freq(1:NumFreqs) of observation.F90:505-536 as float32.

    NumFreqs = int(|initial - final| / step) + 1 (1 when step is 0); linear
    spacing adds (i-1)*step to the initial frequency, logarithmic spacing
    divides the decades between log10(initial) and log10(final) into NumFreqs
    steps and raises 10 to each."""
    f32 = np.float32
    fi, ff, fs = f32(initial), f32(final), f32(step)
    if fs != 0:
        n = int(np.abs(fi - ff) / fs) + 1
    else:
        n = 1
    if n < 0 or n > 100000:
        raise ValueError("frequency range gives %d frequencies (1..100000 allowed)" % n)
    idx = np.arange(n, dtype=np.float32)
    if not logarithmic:
        return (fi + idx * fs).astype(np.float32)
    li, lf = np.log10(fi), np.log10(ff)
    ls = np.abs((li - lf) / f32(n))
    return np.power(f32(10.0), li + idx * ls).astype(np.float32)


def _record(payload: bytes) -> bytes:
    n = struct.pack("<i", len(payload))
    return n + payload + n


def write_freq_probe(path, ijk0, shape, at: float, freqs, values: np.ndarray) -> None:
    """Write a frequency-domain volume probe file.

    ijk0 = (XItrancos, YItrancos, ZItrancos), shape = (ni, nj, nk), `at` the
    time of the final instant, values complex128 [nfreq, 3, nk, nj, ni] (the
    order ``Solver.freq_probe`` returns)."""
    ni, nj, nk = shape
    i0, j0, k0 = ijk0
    v = np.asarray(values, np.complex128)
    fr = np.asarray(freqs, np.float32)
    if v.shape != (len(fr), 3, nk, nj, ni):
        raise ValueError(f"values have shape {v.shape}, expected {(len(fr), 3, nk, nj, ni)}")
    out = [_record(struct.pack("<6i", i0, i0 + ni - 1, j0, j0 + nj - 1, k0, k0 + nk - 1)),
           _record(struct.pack("<d", float(at)))]
    for n in range(len(fr)):
        out.append(_record(fr[n:n + 1].tobytes()))
        for c in range(3):
            for k in range(nk):
                for j in range(nj):
                    out.append(_record(np.ascontiguousarray(v[n, c, k, j]).tobytes()))
    Path(path).write_bytes(b"".join(out))


def fortran_records(data: bytes):
    """Split a Fortran sequential unformatted file into its record payloads."""
    recs, pos = [], 0
    while pos < len(data):
        (n,) = struct.unpack_from("<i", data, pos)
        payload = data[pos + 4:pos + 4 + n]
        (m,) = struct.unpack_from("<i", data, pos + 4 + n)
        if m != n:
            raise ValueError(f"record at byte {pos}: markers {n} and {m} differ")
        recs.append(payload)
        pos += 8 + n
    return recs


def read_freq_probe(path):
    """(ijk0, shape, at, freqs, values) of a file written as above."""
    recs = fortran_records(Path(path).read_bytes())
    xi, xe, yi, ye, zi, ze = struct.unpack("<6i", recs[0])
    (at,) = struct.unpack("<d", recs[1])
    ni, nj, nk = xe - xi + 1, ye - yi + 1, ze - zi + 1
    per = 1 + 3 * nk * nj
    nf = (len(recs) - 2) // per
    freqs = np.empty(nf, np.float32)
    vals = np.empty((nf, 3, nk, nj, ni), np.complex128)
    q = 2
    for n in range(nf):
        freqs[n] = np.frombuffer(recs[q], np.float32)[0]
        q += 1
        for c in range(3):
            for k in range(nk):
                for j in range(nj):
                    vals[n, c, k, j] = np.frombuffer(recs[q], np.complex128)
                    q += 1
    return (xi, yi, zi), (ni, nj, nk), at, freqs, vals
