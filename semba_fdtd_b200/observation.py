"""Volume-probe helpers that mirror observation.F90's host side.

* ``frequency_list`` -- the frequencies of a frequency-domain probe
  (observation.F90:505-536), in real(4) arithmetic as the reference lists
  them;
* ``write_freq_probe`` / ``read_freq_probe`` -- the unformatted file of a
  frequency-domain volume probe (observation.F90:4013-4046): Fortran
  sequential records, each framed by its byte length as a 4-byte integer
  before and after (gfortran's default record markers).

The accumulation itself runs on the device (``Solver.add_freq_probe``).
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

__all__ = ["frequency_list", "write_freq_probe", "read_freq_probe", "fortran_records"]


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
