"""Near-to-far-field transform (farfield.F90): the surface DFT of
UpdateFarField and the radiation integrals of FlushFarfield.

The oracle restates both on the CPU; the device path must give the oracle's
surface accumulators bit for bit (-fmad=false build) and its far-field rows
within a stated tolerance (the transform's sums run in a different order)."""
import numpy as np

from bits import assert_bits_equal
import pytest

from cases import disp, small

import oracle

BOX = (6, 25, 6, 25, 6, 25)
ANGLES = (0.0, float(np.pi), float(np.pi / 6), 0.0, float(2 * np.pi), float(np.pi / 4))
# X faces carry (Ez, Ey), y faces (Ez, Ex), z faces (Ey, Ex); slots 2..5 the H partners
T = {0: (2, 1), 1: (2, 0), 2: (1, 0)}


def _incident(dt, n=300):
    t = (np.arange(n) * dt).astype(np.float32)
    v = np.exp(-(((t - 60 * dt) / (15 * dt)) ** 2)).astype(np.float32)
    return np.stack([t, v], axis=1)


def _weights(o, freqs, nd, dtd, steps):
    """auxExp_E / auxExp_H of every step index 0..steps-1 (None where the
    step is not sampled), restated with numpy: the complex(4) exponential of
    expIwdt, the complex(8) half-step factor and the recursive products."""
    f32 = np.float32
    pi2 = -(f32(2.0) * f32(np.pi))
    out = []
    aE = np.full(len(freqs), complex(float(dtd), 0.0))
    ex = np.exp(np.array([complex(-0.0, float((pi2 * f32(f)) * dtd)) for f in freqs], np.complex64)).astype(np.complex128)
    eh = np.array([np.exp(complex(-0.0, float(pi2 * f32(f)) * (o.dt * 0.5))) for f in freqs])
    aH = float(dtd) * eh
    for n in range(steps):
        if (n - 1) % nd != 0 if n >= 1 else (nd != 1):
            out.append(None)
            continue
        out.append((aE.copy(), aH.copy()))
        aE, aH = aE * ex, aH * ex
    return out


@pytest.mark.parametrize("decimate", [False, True], ids=["every-step", "decimated"])
def test_oracle_surface_dft_matches_numpy(decimate):
    pb = small(n=24, steps=60, layers=4)
    o = oracle.Oracle(pb)
    # a top frequency whose decimation (NF2FFDecim) samples every 4th step
    f32 = np.float32
    ff = f32(0.5 / (5.5 * o.dt))
    fi = fs = f32(ff / f32(3))
    fid = o.add_farfield((5, 18, 5, 18, 5, 18), initial=fi, final=ff, step=fs, decimate=decimate)
    n = int(abs(fi - ff) / fs) + 1
    freqs = (fi + np.arange(n, dtype=f32) * fs).astype(f32)
    nd = max(int((float(f32(0.5) / ff)) / o.dt) - 1, 1) if decimate else 1
    assert nd == (4 if decimate else 1)
    dtd = np.float32(nd * o.dt)
    steps = 60
    w = _weights(o, freqs, nd, dtd, steps)
    ref = oracle.Oracle(pb)
    acc = {}
    # Tr face (x-): Ez on plane 5 over k 5..17, j 5..18; Hy on planes 4, 5
    a = ref.alloc[2]
    for n in range(steps):
        ref.step(1)
        if w[n] is None:
            continue
        ez = ref.field(2).astype(np.float64)[5 - a[0], 5 - a[2]:19 - a[2], 5 - a[4]:18 - a[4]].T  # [k][j]
        hy = ref.field(4).astype(np.float64)[4 - a[0], 5 - a[2]:19 - a[2], 5 - a[4]:18 - a[4]].T
        acc.setdefault("ez", np.zeros((len(freqs),) + ez.shape, np.complex128))
        acc.setdefault("hy", np.zeros((len(freqs),) + hy.shape, np.complex128))
        for q in range(len(freqs)):
            acc["ez"][q] += w[n][0][q] * ez
            acc["hy"][q] += w[n][1][q] * hy
    o.step(steps)
    got_e = o.farfield_array(fid, 0, 0)
    got_h = o.farfield_array(fid, 0, 2)
    assert got_e.shape == acc["ez"].shape and got_h.shape == acc["hy"].shape
    for g, r in ((got_e, acc["ez"]), (got_h, acc["hy"])):
        scale = np.abs(r).max()
        assert scale > 0
        np.testing.assert_allclose(g, r, rtol=0, atol=1e-12 * scale)


def test_oracle_transform_rows_shape_and_reciprocity():
    """Rows come in the reference's order (frequency, theta, phi) with the
    theta / phi sequences of farfield.F90:2520-2525, and the RCS is finite
    and non-negative."""
    pb = small(n=24, steps=60, layers=4)
    o = oracle.Oracle(pb)
    fid = o.add_farfield((5, 18, 5, 18, 5, 18), initial=2e8, final=6e8, step=2e8)
    o.step(60)
    rows = o.farfield_transform(fid, ANGLES, _incident(o.dt))
    def seq(a, b, st):  # theta / phi in real(4), the last step clamped to the stop value
        a, b, st = np.float32(a), np.float32(b), np.float32(st)
        out, x = [], np.float32(a - st)
        while x < b:
            x = np.float32(min(np.float32(x + st), b))
            out.append(x)
        return np.array(out, np.float32)
    th, ph = seq(*ANGLES[:3]), seq(*ANGLES[3:])
    assert rows.shape == (3 * len(th) * len(ph), 9)
    np.testing.assert_array_equal(rows[:, 0], np.repeat(np.float32([2e8, 4e8, 6e8]), len(th) * len(ph)))
    np.testing.assert_array_equal(rows[:, 1], np.tile(np.repeat(th, len(ph)), 3))
    np.testing.assert_array_equal(rows[:, 2], np.tile(ph, 3 * len(th)))
    assert np.all(np.isfinite(rows)) and np.all(rows[:, 7:] >= 0) and rows[:, 7].max() > 0
    # RCS(geom) = 4 pi (|Etheta|^2 + |Ephi|^2) / |DFT(incident)|^2 with the
    # geometric-pass fields, the DFT skipping the first sample
    inc = _incident(o.dt).astype(np.float64)
    dtevol = float(np.float32(inc[1, 0]) - np.float32(inc[0, 0]))
    m = np.arange(1, len(inc))
    for q, f in enumerate(np.float32([2e8, 4e8, 6e8])):
        dft = np.sum(inc[1:, 1] * dtevol * np.exp(-2j * np.pi * float(f) * (m - 1) * dtevol))
        sl = rows[rows[:, 0] == float(f)]
        expect = 4 * np.pi * (sl[:, 3] ** 2 + sl[:, 5] ** 2) / abs(dft) ** 2
        np.testing.assert_allclose(sl[:, 8], expect, rtol=1e-5, atol=1e-6 * expect.max())


@pytest.mark.gpu
@pytest.mark.parametrize("decimate", [False, True], ids=["every-step", "decimated"])
def test_surface_dft_bit_exact(decimate):
    from semba_fdtd_b200 import Solver
    pb = disp()
    steps = 60
    o = oracle.Oracle(pb)
    ofid = o.add_farfield(BOX, initial=1e8, final=9e8, step=4e8, decimate=decimate)
    o.step(steps)
    for mode in ("graph", "routines"):
        with Solver(pb) as s:
            fid = s.add_farfield(BOX, initial=1e8, final=9e8, step=4e8, decimate=decimate)
            s.step(steps, mode=mode)
            for face in range(6):
                for slot in range(6):
                    got, ref = s.farfield_array(fid, face, slot), o.farfield_array(ofid, face, slot)
                    assert got.shape == ref.shape, (mode, face, slot)
                    assert_bits_equal(got, ref, err_msg=f"{mode} face {face} slot {slot}")


@pytest.mark.gpu
def test_transform_matches_oracle():
    """Rows of the device transform against the oracle's serial sums.  Both
    sum in complex(8); the device sums per block in another order, and its
    single-precision sine / cosine of the geometric H mean may differ from
    the host's in the last bit, so the bar is 1e-6 relative to the largest
    value of each column (phases where the magnitude is above 1e-3 of it)."""
    from semba_fdtd_b200 import Solver
    pb = disp()
    steps = 80
    o = oracle.Oracle(pb)
    ofid = o.add_farfield(BOX, initial=1e8, final=9e8, step=4e8)
    o.step(steps)
    inc = _incident(o.dt)
    ref = o.farfield_transform(ofid, ANGLES, inc)
    with Solver(pb) as s:
        fid = s.add_farfield(BOX, initial=1e8, final=9e8, step=4e8)
        s.step(steps)
        got = s.farfield_transform(fid, ANGLES, inc)
    assert got.shape == ref.shape
    np.testing.assert_array_equal(got[:, :3], ref[:, :3])
    for col in (3, 5, 7, 8):
        scale = np.abs(ref[:, col]).max()
        assert scale > 0
        np.testing.assert_allclose(got[:, col], ref[:, col], rtol=0, atol=1e-6 * scale)
    for col, mag in ((4, 3), (6, 5)):
        big = ref[:, mag] > 1e-3 * ref[:, mag].max()
        d = np.angle(np.exp(1j * (got[big, col] - ref[big, col])))
        assert np.abs(d).max() < 1e-5


@pytest.mark.gpu
def test_farfield_arguments_are_checked():
    from semba_fdtd_b200 import Solver
    from semba_fdtd_b200._lib import SembaGpuError
    pb = disp()
    with Solver(pb) as s:
        fid = s.add_farfield(BOX, initial=1e8, final=9e8, step=4e8)
        with pytest.raises(SembaGpuError):
            s.farfield_transform(fid, (0.0, 1.0, 0.0, 0.0, 1.0, 0.1), _incident(1e-11))
        with pytest.raises(SembaGpuError):
            s.farfield_array(fid + 1, 0, 0)
