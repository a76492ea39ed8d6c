"""Volume ("movie") probes: frequency-domain accumulators and time-domain
frames (observation.F90:318-331, 1918-1922, 3527-3600, 4013-4046).

CPU tests pin the oracle's accumulation against an independent numpy DFT of
its own field history and check the host helpers (frequency list, file
records); GPU tests compare the library's device accumulators and frames
with the oracle on the same cases."""
import numpy as np

from bits import assert_bits_equal
import pytest

from cases import disp, mdisp, small
from semba_fdtd_b200 import observation

import oracle

FREQS = np.array([0.6e9, 1.1e9, 2.3e9, 4.0e9], np.float32)


def _mcpi2():
    return complex(-0.0, -float(np.float32(2.0) * np.float32(np.pi)))


def _dft_by_hand(o, pb, box, stride, magnetic, steps):
    """sum_n dt * exp(mcPI2 * f * t_n) [* exp(mcPI2 * f * dt / 2) for H] * F(n)
    over the oracle's own field history, with numpy's complex exp."""
    c0 = 3 if magnetic else 0
    lo = [(-(-box[2 * a] // stride[a])) for a in range(3)]
    hi = [box[2 * a + 1] // stride[a] for a in range(3)]
    ii = np.arange(lo[0], hi[0] + 1) * stride[0]
    jj = np.arange(lo[1], hi[1] + 1) * stride[1]
    kk = np.arange(lo[2], hi[2] + 1) * stride[2]
    acc = np.zeros((len(FREQS), 3, len(kk), len(jj), len(ii)), np.complex128)
    a = o.alloc[c0]
    for n in range(steps):
        o.step(1)
        at = o.time(n)
        for c in range(3):
            fld = o.field(c0 + c).astype(np.float64)
            sub = fld[np.ix_(ii - a[0], jj - a[2], kk - a[4])].transpose(2, 1, 0)
            for q, f in enumerate(FREQS.astype(np.float64)):
                w = o.dt * np.exp(_mcpi2() * f * at)
                if magnetic:
                    w = w * np.exp(_mcpi2() * f * o.dt * 0.5)
                acc[q, c] += w * sub
    return acc


@pytest.mark.parametrize("magnetic", [False, True], ids=["E", "H"])
def test_oracle_dft_matches_numpy(magnetic):
    pb = small(n=16, steps=40, layers=4)
    o = oracle.Oracle(pb)
    box, stride = (6, 14, 5, 13, 7, 12), (2, 3, 1)
    pid = o.add_freq_probe(magnetic, box, stride, FREQS)
    ref = _dft_by_hand(oracle.Oracle(pb), pb, box, stride, magnetic, 40)
    o.step(40)
    got = o.freq_probe(pid)
    assert got.shape == ref.shape
    scale = np.abs(ref).max()
    assert scale > 0
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * scale)


def test_frequency_list():
    lin = observation.frequency_list(1e9, 2e9, 2.5e8)
    assert_bits_equal(lin, np.float32(1e9) + np.arange(5, dtype=np.float32) * np.float32(2.5e8))
    assert observation.frequency_list(1e9, 1e9, 0).tolist() == [np.float32(1e9)]
    lg = observation.frequency_list(1e6, 1e9, 1e8, logarithmic=True)
    assert len(lg) == int(np.float32(1e9 - 1e6) / np.float32(1e8)) + 1
    # 10**log10(f) in real(4) need not return f itself
    assert abs(lg[0] / 1e6 - 1) < 1e-5 and np.all(np.diff(np.log10(lg.astype(np.float64))) > 0)


def test_freq_probe_file_records(tmp_path):
    rng = np.random.default_rng(3)
    vals = rng.standard_normal((2, 3, 2, 3, 4)) + 1j * rng.standard_normal((2, 3, 2, 3, 4))
    p = tmp_path / "probe.bin"
    observation.write_freq_probe(p, (3, 1, 5), (4, 3, 2), 1.25e-9, [1e9, 2e9], vals)
    recs = observation.fortran_records(p.read_bytes())
    # header, time, then per frequency: its value and 3 x nk x nj rows of ni complex(8)
    assert len(recs) == 2 + 2 * (1 + 3 * 2 * 3)
    assert len(recs[0]) == 24 and len(recs[1]) == 8 and len(recs[2]) == 4 and len(recs[3]) == 4 * 16
    ijk0, shape, at, fr, v = observation.read_freq_probe(p)
    assert ijk0 == (3, 1, 5) and shape == (4, 3, 2) and at == 1.25e-9
    assert_bits_equal(fr, np.float32([1e9, 2e9]))
    assert_bits_equal(v, vals)


@pytest.mark.gpu
@pytest.mark.parametrize("case,magnetic,box,stride", [
    ("disp", False, (4, 28, 3, 27, 5, 26), (2, 3, 1)),
    ("disp", True, (1, 31, 2, 30, 1, 31), (3, 2, 4)),
    ("mdisp", True, (5, 20, 6, 18, 4, 22), (1, 1, 2)),
], ids=["disp-E", "disp-H", "mdisp-H"])
def test_freq_probe_bit_exact(case, magnetic, box, stride):
    from semba_fdtd_b200 import Solver
    pb = {"disp": disp, "mdisp": mdisp}[case]()
    steps = 60
    o = oracle.Oracle(pb)
    opid = o.add_freq_probe(magnetic, box, stride, FREQS)
    o.step(steps)
    ref = o.freq_probe(opid)
    for mode in ("graph", "routines"):
        with Solver(pb) as s:
            pid = s.add_freq_probe(magnetic, box, stride, FREQS)
            s.step(steps, mode=mode)
            got = s.freq_probe(pid, len(FREQS))
        assert_bits_equal(got, ref, err_msg=mode)
    with Solver(pb, variant="fast") as s:
        pid = s.add_freq_probe(magnetic, box, stride, FREQS)
        s.step(steps)
        fast = s.freq_probe(pid, len(FREQS))
    err = np.linalg.norm(fast - ref) / np.linalg.norm(ref)
    assert err < 1e-5, err


@pytest.mark.gpu
def test_movie_frames_equal_fields():
    from semba_fdtd_b200 import Solver
    pb = disp()
    box, stride, n_first, every = (2, 30, 3, 29, 4, 27), (2, 2, 3), 5, 7
    o = oracle.Oracle(pb)
    ref, steps = {}, 50
    c0 = 3
    a = o.alloc[c0]
    ii = np.arange(-(-box[0] // 2), box[1] // 2 + 1) * 2
    jj = np.arange(-(-box[2] // 2), box[3] // 2 + 1) * 2
    kk = np.arange(-(-box[4] // 3), box[5] // 3 + 1) * 3
    for n in range(steps):
        o.step(1)
        if n >= n_first and (n - n_first) % every == 0:
            ref[n] = np.stack([o.field(c0 + c)[np.ix_(ii - a[0], jj - a[2], kk - a[4])].transpose(2, 1, 0)
                               for c in range(3)])
    with Solver(pb) as s:
        pid = s.add_movie_probe(True, box, stride, n_first=n_first, n_last=steps, every=every, capacity=3)
        s.step(20)
        first, fr = s.movie_frames(pid)
        assert first == n_first and len(fr) == 3
        for q in range(3):
            assert_bits_equal(fr[q], ref[n_first + q * every])
        s.step(steps - 20)
        first, fr = s.movie_frames(pid)  # 4 more frames were written; the ring kept the last 3
        kept = sorted(ref)[-3:]
        assert first == kept[0] and len(fr) == 3
        for q, n in enumerate(kept):
            assert_bits_equal(fr[q], ref[n])


@pytest.mark.gpu
def test_volume_probe_arguments_are_checked():
    from semba_fdtd_b200 import Solver
    from semba_fdtd_b200._lib import SembaGpuError
    pb = small(n=16, steps=40, layers=4)
    with Solver(pb) as s:
        a = s.alloc[0]
        with pytest.raises(SembaGpuError):  # box outside Alloc
            s.add_freq_probe(False, (a[0] - 5, a[1], a[2], a[3], a[4], a[5]), (1, 1, 1), FREQS)
        with pytest.raises(SembaGpuError):  # stride samples no node
            s.add_freq_probe(False, (5, 6, 5, 6, 5, 6), (7, 7, 7), FREQS)
        with pytest.raises(SembaGpuError):  # no frequencies
            s.add_freq_probe(False, (5, 6, 5, 6, 5, 6), (1, 1, 1), [])
        with pytest.raises(SembaGpuError):  # bad sampling period
            s.add_movie_probe(True, (5, 6, 5, 6, 5, 6), every=0)
        pid = s.add_movie_probe(False, (5, 6, 5, 6, 5, 6), n_first=3, n_last=4, every=1, capacity=2)
        s.step(6)
        first, fr = s.movie_frames(pid)
        assert first == 3 and len(fr) == 1  # one frame in [3, 4)
