"""Known-answer tests that pin the CPU oracle (no GPU).

The reference Fortran cannot be built here and its tests hold no golden
vectors for this path, so the oracle is pinned by physics and by the
reference's own parser fixture:

* one step from a linear Hz ramp gives the analytic discrete curl
  (staggering, G2 of vacuum, metric arrays; timestepping.F90:2165-2285);
* a vacuum plane wave through an empty TF/SF box: unit incident amplitude
  inside, scattered field below -40 dB outside (planewaves.F90:878-1475);
* CPML reflection against a domain large enough to have none in the window
  (borderscpml.F90:584-1176, 1465-1733);
* Debye relaxation of a uniform field in a single-real-pole medium converges
  to the analytic solution (electricdispersive.F90:77-362), and its magnetic
  dual (magneticdispersive.F90:79-360);
* FP32 against FP64 oracle per probe;
* borders (healer.F90:1442-1617, bordersother.F90:65-190,
  bordersmur.F90:1129-1650): a PEC box keeps tangential E and normal H at
  zero on its faces; PMC faces hold the odd image of the first swept H
  (edges the product of two images); a plane wave in a box periodic across
  its wavefront stays uniform over every periodic plane, bit for bit; Mur
  faces absorb a normally incident pulse that PEC faces reflect whole, and
  the first step after a field is planted outside a Mur face follows the
  update formula exactly;
* the reference's parser fixture test/smbjson/test_read_planewave.F90 on
  testData/cases/planewave.fdtd.json (skipped where that tree is absent).
"""
from pathlib import Path

import numpy as np
import pytest

import oracle
from semba_fdtd_b200.case import EPS0, NodalSource, PlaneWave, Problem, Region, Waveform, read_case

ETA0 = 376.730313668


def _box(n, steps, layers, dx=0.01):
    d = np.full(n, dx, np.float32)
    return Problem(nx=n, ny=n, nz=n, desx=d, desy=d.copy(), desz=d.copy(), nsteps=steps, forcecfl=True, cfl=0.8,
                   pml_layers=(layers,) * 6, pml_order=(3.0,) * 6, pml_refl=(1e-6,) * 6)


def _dt():
    return oracle.Oracle(_box(8, 1, 4), fp64=True).dt


def _fill(o, comp, fn):
    xi, xe, yi, ye, zi, ze = o.alloc[comp]
    i, j, k = np.meshgrid(np.arange(xi, xe + 1), np.arange(yi, ye + 1), np.arange(zi, ze + 1), indexing="ij")
    o.set_field(comp, fn(i, j, k).astype(np.float32))


def test_one_step_curl_of_a_ramp_is_exact():
    """Hz = j (absolute cell index), everything else zero.  After one step,
    in the interior: Ex = G2(vacuum) * Idyh(j) exactly, Ey = Ez = 0, Hz
    unchanged, Hx = Hy = 0 (curl E vanishes where Ex is uniform)."""
    n, L = 12, 4
    o = oracle.Oracle(_box(n, 1, L))
    _fill(o, 5, lambda i, j, k: j.astype(np.float32))
    o.step(1)
    g1, g2, gm1, gm2 = o.g_tables()
    assert g1[1] == np.float32(1.0) and gm1[1] == np.float32(1.0)
    assert g2[1] == np.float32(np.float64(o.dt) / np.float64(EPS0))
    lo, idyh = o.metric(4)

    def interior(comp):
        xi, _, yi, _, zi, _ = o.alloc[comp]
        f = o.field(comp)
        return f[2 - xi:n - 2 - xi, 2 - yi:n - 2 - yi, 2 - zi:n - 2 - zi]

    ex = interior(0)
    want = (g2[1] * idyh[np.arange(2, n - 2) - lo]).astype(np.float32)
    np.testing.assert_array_equal(ex, np.broadcast_to(want[None, :, None], ex.shape))
    assert not np.any(interior(1)) and not np.any(interior(2))
    assert not np.any(interior(3)[1:-1, 1:-1, 1:-1]) and not np.any(interior(4)[1:-1, 1:-1, 1:-1])
    hz = interior(5)
    np.testing.assert_array_equal(hz[:, 1:-1, :], np.broadcast_to(np.arange(3, n - 3, dtype=np.float32)[None, :, None],
                                                                  hz[:, 1:-1, :].shape))


def _gauss(dt, steps, sigma, t0):
    ds = dt / 4
    t = np.arange(int(steps * dt / ds) + 2) * ds
    return Waveform(np.exp(-((t - t0) ** 2) / (2 * sigma * sigma)).astype(np.float32), np.float32(ds))


def test_tfsf_unit_incident_and_quiet_scattered_region():
    n, steps, sig = 30, 260, 200e-12
    pb = _box(n, steps, 8)
    pb.planewaves = [PlaneWave((6, 6, 6), (23, 23, 23), 0.0, 0.0, float(np.float32(np.pi / 2)), 0.0,
                               _gauss(_dt(), steps, sig, 4 * sig))]
    # Ex and Hy at the centre (total field); Ex upstream, downstream, lateral (scattered field)
    pb.probes = np.array([[0, 15, 15, 15], [4, 15, 15, 15], [0, 15, 15, 3], [0, 15, 15, 26], [0, 2, 15, 15]], np.int32)
    tr = oracle.Oracle(pb, fp64=True).step(steps).astype(np.float64)
    peak = np.abs(tr[:, 0]).max()
    assert abs(peak - 1.0) < 0.01
    assert abs(np.abs(tr[:, 1]).max() * ETA0 - 1.0) < 0.01
    for q in (2, 3, 4):
        assert np.abs(tr[:, q]).max() / peak < 1e-2, f"probe {q} leaks"


def _dipole(n, c, probe, steps, dt, sig):
    pb = _box(n, steps, 10)
    ds = dt / 4
    t = np.arange(int(steps * dt / ds) + 2) * ds
    x = (t - 4 * sig) / sig
    w = Waveform((-x * np.exp(-0.5 * x * x)).astype(np.float32), np.float32(ds))
    pb.nodals = [NodalSource(True, False, np.array([[c] * 6], np.int32), np.array([[0, 0, 1]], np.float32), w)]
    pb.probes = np.array([[2, *probe]], np.int32)
    return pb


def test_cpml_reflection_below_60_db():
    """Soft Ez dipole, probe 4 cells from the CPML of a 24^3 box, against the
    same source and probe in a 64^3 box whose boundary echo cannot reach the
    probe within the 110 steps."""
    dt, steps = _dt(), 110
    sig = 8 * dt
    small = oracle.Oracle(_dipole(24, 12, (12, 12, 20), steps, dt, sig), fp64=True).step(steps)[:, 0].astype(np.float64)
    big = oracle.Oracle(_dipole(64, 32, (32, 32, 40), steps, dt, sig), fp64=True).step(steps)[:, 0].astype(np.float64)
    assert np.abs(big).max() > 1.0
    assert np.abs(small - big).max() / np.abs(big).max() < 1e-3


def _debye_error(m, n=40, steps=18):
    pb = _box(n, steps, 4)
    dt = oracle.Oracle(pb, fp64=True).dt
    eps_inf, eps_s = 2.0, 6.0
    tau_e = m * dt
    tau = tau_e * eps_s / eps_inf
    a = -1.0 / tau
    r = (eps_s - eps_inf) * float(EPS0) / tau
    pb.regions = [Region(kind=2, boxes=np.array([[0, n - 1] * 3], np.int32), eps=float(np.float32(eps_inf) * EPS0),
                         residues=np.array([r], np.complex64), bpoles=np.array([-a], np.complex64))]
    pb.probes = np.array([[0, n // 2, n // 2, n // 2]], np.int32)
    o = oracle.Oracle(pb, fp64=True)
    for c in range(3):
        _fill(o, c, lambda i, j, k: np.ones(i.shape))
    tr = o.step(steps)[:, 0].astype(np.float64)
    t = np.arange(steps) * dt
    exact = eps_inf / eps_s + (1 - eps_inf / eps_s) * np.exp(-t / tau_e)
    return np.abs(tr - exact).max()


def _magnetic_debye_error(m, n=40, steps=18):
    """The dual of _debye_error: a uniform H = 1 in a single-real-pole
    magnetic medium (mu_inf 2, mu_s 6) relaxes as
    H(t) = mu_inf/mu_s + (1 - mu_inf/mu_s) exp(-t/tau_H)."""
    from semba_fdtd_b200.case import MU0
    pb = _box(n, steps, 4)
    dt = oracle.Oracle(pb, fp64=True).dt
    mu_inf, mu_s = 2.0, 6.0
    tau_h = m * dt
    tau = tau_h * mu_s / mu_inf
    a = -1.0 / tau
    r = (mu_s - mu_inf) * float(MU0) / tau
    pb.regions = [Region(kind=2, boxes=np.array([[0, n - 1] * 3], np.int32), eps=float(EPS0),
                         mu=float(np.float32(mu_inf) * MU0),
                         mresidues=np.array([r], np.complex64), mbpoles=np.array([-a], np.complex64))]
    pb.probes = np.array([[3, n // 2, n // 2, n // 2]], np.int32)
    o = oracle.Oracle(pb, fp64=True)
    for c in range(3, 6):
        _fill(o, c, lambda i, j, k: np.ones(i.shape))
    tr = o.step(steps)[:, 0].astype(np.float64)
    t = np.arange(steps) * dt
    exact = mu_inf / mu_s + (1 - mu_inf / mu_s) * np.exp(-t / tau_h)
    return np.abs(tr - exact).max(), tr


def test_magnetic_debye_relaxation_converges_to_analytic():
    """AdvanceMdispersiveH (magneticdispersive.F90:298-360) by duality with
    the electric test: second-order convergence of the relaxation."""
    e12, tr = _magnetic_debye_error(12)
    e24, _ = _magnetic_debye_error(24)
    assert tr[0] == 1.0 and np.all(np.diff(tr) < 0)  # the state starts at zero
    assert e24 < 5e-3
    assert e12 / e24 > 2.0


def test_debye_relaxation_converges_to_analytic():
    """A uniform E = 1 switched on at t = 0 in a single-real-pole medium
    (eps_inf 2, eps_s 6) with no curl relaxes as
    E(t) = eps_inf/eps_s + (1 - eps_inf/eps_s) exp(-t/tau_E),
    tau_E = tau eps_inf/eps_s (the ADE state lags the field by one step)."""
    e12, e24 = _debye_error(12), _debye_error(24)
    assert e24 < 5e-3
    assert e12 / e24 > 2.0


def test_fp32_tracks_fp64():
    n, steps, sig = 24, 160, 200e-12
    pb = _box(n, steps, 6)
    pb.planewaves = [PlaneWave((5, 5, 5), (18, 18, 18), 0.0, 0.0, float(np.float32(np.pi / 2)), 0.0,
                               _gauss(_dt(), steps, sig, 4 * sig))]
    pb.probes = np.array([[0, 12, 12, 12], [4, 12, 12, 12], [0, 9, 14, 11]], np.int32)
    a = oracle.Oracle(pb).step(steps).astype(np.float64)
    b = oracle.Oracle(pb, fp64=True).step(steps).astype(np.float64)
    for q in range(3):
        assert np.linalg.norm(a[:, q] - b[:, q]) / np.linalg.norm(b[:, q]) < 1e-5


# the reference's own case, copied by tests/golden/make_reference_fixtures.py
REF_CASE = Path(__file__).resolve().parent / "golden" / "ref" / "planewave.fdtd.json"


def test_reader_matches_reference_parser_fixture():
    """Expected values of test/smbjson/test_read_planewave.F90:24-96."""
    pb = read_case(REF_CASE)
    assert pb.dt == pytest.approx(10e-12) and pb.nsteps == 2000
    assert (pb.nx, pb.ny, pb.nz) == (10, 10, 10)
    for d in (pb.desx, pb.desy, pb.desz):
        assert d.shape == (10,) and np.all(d == np.float32(0.1))
    assert pb.boundary == "mur"
    (w,) = pb.planewaves
    assert tuple(int(v) for v in w.coor1) == (1, 1, 1) and tuple(int(v) for v in w.coor2) == (8, 8, 8)
    assert (w.theta, w.phi, w.beta) == (0.0, 0.0, 0.0) and w.alpha == pytest.approx(1.5708)
    np.testing.assert_array_equal(pb.probes, [[0, 4, 4, 4], [1, 4, 4, 4], [2, 4, 4, 4]])


# ---------------------------------------------------------------------------
# borders


def _bordered(n, steps, borders, layers=4):
    pb = _box(n, steps, layers)
    return _with(pb, borders)


def _with(pb, borders):
    from dataclasses import replace
    return replace(pb, borders=tuple(borders))


def _soft_dipole(pb, c, dt, sig):
    ds = dt / 4
    t = np.arange(int(pb.nsteps * dt / ds) + 2) * ds
    x = (t - 4 * sig) / sig
    w = Waveform((-x * np.exp(-0.5 * x * x)).astype(np.float32), np.float32(ds))
    pb.nodals = [NodalSource(True, False, np.array([list(c[:1]) * 2 + list(c[1:2]) * 2 + list(c[2:]) * 2], np.int32),
                             np.array([[1, 1, 1]], np.float32), w)]
    return pb


def _planes(o, comp, axis, idx):
    """The plane(s) `idx` (absolute) of a component along `axis`."""
    f = o.field(comp)
    lo = o.alloc[comp][2 * axis]
    return np.take(f, [i - lo for i in idx], axis=axis)


def test_pec_faces_keep_tangential_e_and_normal_h_zero():
    n, steps = 12, 60
    dt = _dt()
    pb = _soft_dipole(_bordered(n, steps, ["pec"] * 6), (3, 4, 5), dt, 6 * dt)
    o = oracle.Oracle(pb)
    o.step(steps)
    assert np.abs(o.field(0)).max() > 0
    # E tangential to a face sits on its plane (Ex on y = 0, n and z = 0, n ...)
    for comp in range(3):
        for axis in range(3):
            if axis != comp:
                assert not np.any(_planes(o, comp, axis, [0, n])), (comp, axis)
    # H normal to a face (Hx on x = 0, n ...)
    for comp in range(3):
        assert not np.any(_planes(o, 3 + comp, comp, [0, n]))


def test_pmc_faces_hold_the_odd_image():
    n, steps = 12, 40
    dt = _dt()
    pb = _soft_dipole(_bordered(n, steps, ["pmc"] * 6), (3, 4, 5), dt, 6 * dt)
    o = oracle.Oracle(pb)
    o.step(steps)
    hx = o.field(3)  # Alloc x -1..n+1, y -1..n, z -1..n: index = coordinate + 1
    assert np.abs(hx).max() > 0
    # outside y = 0 and y = n-1 (the swept ends of Hx), all x and z
    np.testing.assert_array_equal(hx[:, 0, 1:-1], -hx[:, 1, 1:-1])
    np.testing.assert_array_equal(hx[:, -1, 1:-1], -hx[:, -2, 1:-1])
    np.testing.assert_array_equal(hx[:, 1:-1, 0], -hx[:, 1:-1, 1])
    # an edge outside two PMC faces carries the product of both images
    np.testing.assert_array_equal(hx[:, 0, 0], hx[:, 1, 1])
    np.testing.assert_array_equal(hx[:, -1, -1], hx[:, -2, -2])


def test_periodic_box_keeps_a_normal_plane_wave_uniform():
    """A +z plane wave in a box periodic along x and y, its TF/SF box spanning
    the whole x-y extent (those faces are inactive): every Ex, Hy plane is
    uniform, bit for bit, and the centre sees the unit incident field."""
    n, steps, sig = 10, 200, 150e-12
    pb = _bordered(n, steps, ["periodic"] * 4 + ["pml"] * 2, layers=8)
    pb.nz = 40
    pb.desz = np.full(40, np.float32(0.01))
    pb.planewaves = [PlaneWave((0, 0, 8), (n, n, 32), 0.0, 0.0, float(np.float32(np.pi / 2)), 0.0,
                               _gauss(_dt(), steps, sig, 4 * sig))]
    pb.probes = np.array([[0, 5, 5, 20]], np.int32)
    o = oracle.Oracle(pb)
    tr = [o.step(steps // 2)[:, 0]]
    for comp in (0, 4):
        f = o.field(comp)
        sw = o.sweep[comp]
        al = o.alloc[comp]
        core = f[sw[0] - al[0]:sw[1] - al[0] + 1, sw[2] - al[2]:sw[3] - al[2] + 1, :]
        assert np.abs(core).max() > 1e-3
        assert np.all(core == core[:1, :1, :]), comp
    assert not np.any(o.field(1)) and not np.any(o.field(2))
    tr.append(o.step(steps - steps // 2)[:, 0])
    assert abs(np.abs(np.concatenate(tr)).max() - 1.0) < 0.02


def _sheet_run(borders, n=6, nz=60, steps=320):
    """A soft Ex current sheet across a box periodic in x and y: two plane
    pulses leave it along -z and +z towards the z faces."""
    dt = _dt()
    pb = _bordered(n, steps, ["periodic"] * 4 + borders)
    pb.nz = nz
    pb.desz = np.full(nz, np.float32(0.01))
    ds = dt / 4
    sig = 10 * dt
    t = np.arange(int(steps * dt / ds) + 2) * ds
    w = Waveform(np.exp(-((t - 4 * sig) ** 2) / (2 * sig * sig)).astype(np.float32), np.float32(ds))
    pb.nodals = [NodalSource(True, False, np.array([[0, n - 1, 0, n, nz // 2, nz // 2]], np.int32),
                             np.array([[1, 0, 0]], np.float32), w)]
    pb.probes = np.array([[0, 2, 2, nz // 2 + 10]], np.int32)
    o = oracle.Oracle(pb, fp64=True)
    tr = o.step(steps)[:, 0]
    return np.abs(tr[: steps // 3]).max(), np.abs(o.field(0)).max()


def test_mur_faces_absorb_a_normal_pulse():
    peak, left_mur = _sheet_run(["mur", "mur"])
    _, left_pec = _sheet_run(["pec", "pec"])
    assert peak > 0
    assert left_pec > 0.5 * peak          # PEC faces send the pulses back
    assert left_mur < 0.02 * peak         # Mur faces let them out


def test_mur_update_formula_on_a_planted_field():
    """Hx planted on the first swept layer above the z- face (Mur): after one
    step without sources the outer layer holds Past(inner) + CAB1 * (H(inner)
    - Past(outer)) with Past = 0 (fresh start), i.e. CAB1 * H(inner)."""
    n = 8
    pb = _bordered(n, 1, ["pec"] * 4 + ["mur", "pec"])
    o = oracle.Oracle(pb)
    xi, xe, yi, ye, zi, ze = o.alloc[3]
    hx = np.zeros((xe - xi + 1, ye - yi + 1, ze - zi + 1), np.float32)
    rng = np.random.default_rng(3)
    hx[:, :, 0 - zi] = rng.uniform(-1, 1, size=hx[:, :, 0].shape).astype(np.float32)
    o.set_field(3, hx)
    o.step(1)
    cab = o.mur_cab1(4)
    after = o.field(3)
    inner, outer = after[:, :, 0 - zi], after[:, :, -1 - zi]
    m = o.media(3)[:, :, 0 - zi]
    sw = o.sweep[3]
    sl = (slice(sw[0] - xi, sw[1] - xi + 1), slice(sw[2] - yi, sw[3] - yi + 1))
    want = (np.float32(0) + cab[m[sl]] * (inner[sl] - np.float32(0))).astype(np.float32)
    np.testing.assert_array_equal(outer[sl], want)


def test_corrected_quotient_by_dt_matches_ieee_division():
    """The ADE kernels divide by dt as RN(q + (a - dt*q)*y), y = RN(1/dt),
    q = RN(a*y) (Markstein's correction); it must equal IEEE a/dt.  Checked
    for the time steps of the parity cases and of random grids on 2e6
    operands each, spanning the exponent range."""
    from cases import ALL
    lib = oracle.load()
    dts = {oracle.Oracle(ALL[name]()).dt for name in ("disp", "mdisp", "small")}
    rng = np.random.default_rng(5)
    dts |= {float(v) for v in rng.uniform(1e-13, 1e-10, size=5)}
    for q, dt in enumerate(sorted(dts)):
        assert lib.orc_check_div_dt(dt, 2_000_000, 1234 + q) == 0, dt
