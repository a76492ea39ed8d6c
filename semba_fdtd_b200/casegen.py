"""Seeded synthetic cases for the benchmark configurations.

No external data: every geometry, material and waveform is drawn from a
fixed-seed numpy generator and written as an extended smbjson case
(``<name>.fdtd.json``) plus its excitation files (``*.exc``), which
:func:`semba_fdtd_b200.case.read_case` reads back.  Sizes default to the
benchmark configurations; ``n`` (and the other keyword arguments) give scaled
variants with the same features for parity tests.

* :func:`plain_small`  -- free-space box, CPML 10 (m=3, R=1e-6), cfl 0.8,
  x-polarised +z plane wave through a TF/SF box inset 15 cells, Gaussian
  sigma 100 ps / delay 400 ps, Ex and Hy probes at seeded cells.
* :func:`plain_mid`    -- 256^3, dx 5 mm, CPML 12, lossy sphere r=60
  (eps_r 4, sigma 0.01) and 20 seeded PEC/dielectric blocks, 64 probes.
* :func:`dispersive_large` -- 512^3 graded 1-3 mm cosine mesh, CPML 12,
  30 % of the volume in seeded 2-pair pole-residue blocks, soft Ez dipole
  with a Gaussian-derivative waveform at the centre.
* :func:`batch_instance` / :func:`served_request` -- members of the batched
  and served streams.
"""
from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

from .case import EPS0, read_case, write_waveform

C0 = 299792458.0


def _f32(x) -> float:
    return float(np.float32(x))


def courant_dt(dmin: float, cfl: float = 0.8) -> float:
    """Approximate time step (for choosing waveform sampling only)."""
    return cfl * dmin / (C0 * math.sqrt(3.0))


def gaussian(ds: float, sigma: float, t0: float, duration: float) -> np.ndarray:
    t = np.arange(int(duration / ds) + 2) * ds
    return np.exp(-((t - t0) ** 2) / (2 * sigma * sigma)).astype(np.float32)


def gaussian_derivative(ds: float, sigma: float, t0: float, duration: float) -> np.ndarray:
    t = np.arange(int(duration / ds) + 2) * ds
    x = (t - t0) / sigma
    return (-x * np.exp(-0.5 * x * x)).astype(np.float32)


class _Builder:
    def __init__(self, n, steps, layers, order=3.0, refl=1e-6, cfl=0.8, boundary="pml"):
        bnd = {"type": "pml", "layers": int(layers), "order": order, "reflection": refl} if boundary == "pml" \
            else {"type": boundary}
        self.js = {"format": "FDTD Input file",
                   "general": {"timeStep": 0.0, "numberOfSteps": int(steps), "cfl": cfl},
                   "boundary": {"all": bnd},
                   "mesh": {"grid": {"numberOfCells": [int(v) for v in n], "steps": {}}, "coordinates": [], "elements": []},
                   "materials": [], "materialAssociations": [], "sources": [], "probes": []}
        self._eid = 0
        self._cid = 0
        self._mid = 0
        self.files = {}

    def steps(self, x, y, z):
        self.js["mesh"]["grid"]["steps"] = {"x": [_f32(v) for v in x], "y": [_f32(v) for v in y], "z": [_f32(v) for v in z]}

    def cell(self, intervals):
        self._eid += 1
        self.js["mesh"]["elements"].append({"id": self._eid, "type": "cell",
                                            "intervals": [[[int(a) for a in lo], [int(b) for b in hi]] for lo, hi in intervals]})
        return self._eid

    def node(self, pos):
        self._cid += 1
        self.js["mesh"]["coordinates"].append({"id": self._cid, "relativePosition": [int(v) for v in pos]})
        self._eid += 1
        self.js["mesh"]["elements"].append({"id": self._eid, "type": "node", "coordinateIds": [self._cid]})
        return self._eid

    def material(self, m):
        self._mid += 1
        m = dict(m, id=self._mid)
        self.js["materials"].append(m)
        return self._mid

    def bulk(self, mid, boxes):
        """Associate material mid with cell boxes (inclusive XI..XE etc.)."""
        eid = self.cell([((b[0], b[2], b[4]), (b[1] + 1, b[3] + 1, b[5] + 1)) for b in boxes])
        self.js["materialAssociations"].append({"type": "bulk", "materialId": mid, "elementIds": [eid]})

    def planewave(self, lo, hi, theta, phi, alpha, beta, fname, ds, values):
        eid = self.cell([(lo, hi)])
        self.js["sources"].append({"type": "planewave", "magnitudeFile": fname, "elementIds": [eid],
                                   "direction": {"theta": _f32(theta), "phi": _f32(phi)},
                                   "polarization": {"theta": _f32(alpha), "phi": _f32(beta)}})
        self.files[fname] = (ds, values)

    def nodal(self, lo, hi, fname, ds, values, hard=False):
        eid = self.cell([(lo, hi)])
        self.js["sources"].append({"type": "nodalSource", "field": "electric", "hard": bool(hard),
                                   "magnitudeFile": fname, "elementIds": [eid]})
        self.files[fname] = (ds, values)

    def probe(self, name, field, pos, dirs):
        eid = self.node(pos)
        self.js["probes"].append({"name": name, "type": "point", "field": field, "elementIds": [eid],
                                  "directions": list(dirs), "domain": {"type": "time"}})

    def write(self, outdir: Path, name: str) -> Path:
        outdir = Path(outdir)
        outdir.mkdir(parents=True, exist_ok=True)
        for fname, (ds, values) in self.files.items():
            write_waveform(outdir / fname, ds, values)
        path = outdir / f"{name}.fdtd.json"
        path.write_text(json.dumps(self.js))
        return path


def _pole_pair_material(rng, eps_inf=1.0):
    """Two conjugate pole pairs, f0 in 1-20 GHz, damping 0.05-0.3, residues
    scaled so the static eps_r lies in 2-12."""
    eps_s = rng.uniform(2.0, 12.0)
    delta = eps_s - eps_inf
    u = rng.uniform(0.2, 0.8)
    cs = [u * delta / 2.0, (1.0 - u) * delta / 2.0]
    poles, res = [], []
    for c in cs:
        f0 = rng.uniform(1e9, 20e9)
        z = rng.uniform(0.05, 0.3)
        w0 = 2 * math.pi * f0
        a = complex(-z * w0, w0 * math.sqrt(1 - z * z))
        r = -c * float(EPS0) * a
        for pa, pr in ((a, r), (a.conjugate(), r.conjugate())):
            poles.append([_f32(pa.real), _f32(pa.imag)])
            res.append([_f32(pr.real), _f32(pr.imag)])
    return {"type": "poleResidue", "epsilonInfinity": eps_inf, "electricConductivity": 0.0,
            "poles": poles, "residues": res}


def _magnetic_pole_pair(rng):
    """One conjugate pole pair in the permeability, f0 in 2-15 GHz, damping
    0.1-0.4, residue scaled so the static mu_r lies in 1.5-4."""
    from .case import MU0
    mu_s = rng.uniform(1.5, 4.0)
    f0 = rng.uniform(2e9, 15e9)
    z = rng.uniform(0.1, 0.4)
    w0 = 2 * math.pi * f0
    a = complex(-z * w0, w0 * math.sqrt(1 - z * z))
    r = -(mu_s - 1.0) / 2.0 * float(MU0) * a
    poles, res = [], []
    for pa, pr in ((a, r), (a.conjugate(), r.conjugate())):
        poles.append([_f32(pa.real), _f32(pa.imag)])
        res.append([_f32(pr.real), _f32(pr.imag)])
    return poles, res


def magnetic_dispersive(outdir, n=(26, 24, 22), steps=140, layers=5, seed=9) -> Path:
    """Pole-residue blocks with magnetic poles only, electric poles only, and
    both, next to a TF/SF plane wave and a soft dipole."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    b = _Builder((nx, ny, nz), steps, layers)
    dx = 0.003
    b.steps([dx], [dx], [dx])
    ds = courant_dt(dx) / 4
    th, ph, al, be = _tem_angles(rng)
    b.planewave((3, 3, 3), (nx - 3, ny - 3, nz - 3), th, ph, al, be, "gauss.exc", ds,
                gaussian(ds, 30e-12, 120e-12, 0.4e-9))
    b.nodal((nx // 2, ny // 2, nz // 2), (nx // 2, ny // 2, nz // 2 + 1), "dipole.exc", ds,
            gaussian_derivative(ds, 12e-12, 72e-12, 0.25e-9), hard=False)
    mp, mr = _magnetic_pole_pair(rng)
    mag = b.material({"type": "poleResidue", "epsilonInfinity": 2.0, "muInfinity": 1.2,
                      "magneticConductivity": _f32(rng.uniform(0, 50.0)), "magneticPoles": mp, "magneticResidues": mr})
    b.bulk(mag, [(5, 10, 5, 9, 5, 9)])
    both = dict(_pole_pair_material(rng))
    mp2, mr2 = _magnetic_pole_pair(rng)
    both.update({"muInfinity": 1.5, "magneticPoles": mp2, "magneticResidues": mr2})
    mid = b.material(both)
    b.bulk(mid, [(nx - 11, nx - 6, ny - 10, ny - 6, nz - 10, nz - 6)])
    ele = b.material(_pole_pair_material(rng))
    b.bulk(ele, [(5, 9, ny - 10, ny - 6, 6, 10)])
    spots = [(7, 7, 7), (nx - 8, ny - 8, nz - 8), (7, ny - 8, 8), (nx // 2, ny // 2 + 3, nz // 2)]
    for q, pos in enumerate(spots):
        b.probe(f"e{q}", "electric", pos, "xyz")
        b.probe(f"h{q}", "magnetic", pos, "xyz")
    return b.write(outdir, f"magnetic_dispersive_{nx}x{ny}x{nz}")


def plain_small(outdir, n=64, steps=1000, inset=15, nprobes=8, seed=1, layers=10, dx=0.01) -> Path:
    rng = np.random.default_rng(seed)
    b = _Builder((n, n, n), steps, layers)
    b.steps([dx], [dx], [dx])
    dt = courant_dt(dx)
    ds = dt / 4
    b.planewave((inset,) * 3, (n - inset,) * 3, 0.0, 0.0, math.pi / 2, 0.0, "gauss.exc", ds,
                gaussian(ds, 100e-12, 400e-12, 1.2e-9))
    for q in range(nprobes):
        pos = rng.integers(1, n - 1, size=3)
        b.probe(f"p{q}", "electric", pos, "x")
        b.probe(f"p{q}", "magnetic", pos, "y")
    return b.write(outdir, f"plain_small_{n}")


def plain_mid(outdir, n=256, steps=4000, inset=15, radius=60, nblocks=20, nprobes=64, layers=12, dx=0.005,
              edge=(4, 40), seed_blocks=2, seed_probes=3) -> Path:
    b = _Builder((n, n, n), steps, layers)
    b.steps([dx], [dx], [dx])
    dt = courant_dt(dx)
    ds = dt / 4
    b.planewave((inset,) * 3, (n - inset,) * 3, 0.0, 0.0, math.pi / 2, 0.0, "gauss.exc", ds,
                gaussian(ds, 100e-12, 400e-12, 1.2e-9))
    # staircased sphere as x-runs
    c = n / 2.0
    runs = []
    for k in range(n):
        for j in range(n):
            r2 = radius * radius - (j + 0.5 - c) ** 2 - (k + 0.5 - c) ** 2
            if r2 < 0:
                continue
            h = math.sqrt(r2)
            i0, i1 = int(math.ceil(c - h - 0.5)), int(math.floor(c + h - 0.5))
            if i0 <= i1:
                runs.append((i0, i1, j, j, k, k))
    sphere = b.material({"type": "simple", "relativePermittivity": 4.0, "electricConductivity": 0.01})
    b.bulk(sphere, runs)
    rng = np.random.default_rng(seed_blocks)
    lo_lim, hi_lim = inset + 2, n - inset - 3
    for q in range(nblocks):
        e = rng.integers(edge[0], edge[1] + 1, size=3)
        e = np.minimum(e, hi_lim - lo_lim)
        o = [int(rng.integers(lo_lim, hi_lim - e[a] + 1)) for a in range(3)]
        box = (o[0], o[0] + e[0] - 1, o[1], o[1] + e[1] - 1, o[2], o[2] + e[2] - 1)
        if rng.random() < 0.5:
            mid = b.material({"type": "pec"})
        else:
            mid = b.material({"type": "simple", "relativePermittivity": _f32(rng.uniform(1, 10)),
                              "electricConductivity": _f32(rng.uniform(0, 0.1))})
        b.bulk(mid, [box])
    rng = np.random.default_rng(seed_probes)
    for q in range(nprobes):
        pos = rng.integers(1, n - 1, size=3)
        comp = int(rng.integers(0, 6))
        b.probe(f"p{q}", "electric" if comp < 3 else "magnetic", pos, "xyz"[comp % 3])
    return b.write(outdir, f"plain_mid_{n}")


def bordered(outdir, n=(20, 23, 18), steps=160, boundary="mur", layers=4, seed=7) -> Path:
    """Border test case: a TF/SF plane wave, a soft Ez dipole two cells from
    a corner (so the borders see strong oblique fields early), a PEC block
    and a dielectric block, and probes on and next to the boundary planes."""
    nx, ny, nz = n
    rng = np.random.default_rng(seed)
    b = _Builder((nx, ny, nz), steps, layers, boundary=boundary)
    dx = 0.004
    b.steps([dx], [dx], [dx])
    ds = courant_dt(dx) / 4
    th, ph, al, be = _tem_angles(rng)
    b.planewave((3, 3, 3), (nx - 3, ny - 3, nz - 3), th, ph, al, be, "gauss.exc", ds,
                gaussian(ds, 40e-12, 160e-12, 0.5e-9))
    b.nodal((2, 2, 2), (2, 2, 3), "dipole.exc", ds, gaussian_derivative(ds, 15e-12, 90e-12, 0.3e-9), hard=False)
    pec = b.material({"type": "pec"})
    b.bulk(pec, [(nx // 2, nx // 2 + 2, ny // 2, ny // 2 + 3, 4, 6)])
    die = b.material({"type": "simple", "relativePermittivity": 3.5, "electricConductivity": 0.02})
    b.bulk(die, [(5, 8, ny - 8, ny - 5, nz // 2, nz // 2 + 3)])
    spots = [(0, 0, 0), (nx, ny // 2, nz // 2), (nx // 2, 0, nz // 2), (nx // 2, ny, nz - 1), (1, 1, nz),
             (nx - 1, ny - 1, 1), (2, 2, 2), (nx // 2, ny // 2, nz // 2)]
    for q, pos in enumerate(spots):
        b.probe(f"e{q}", "electric", pos, "xyz")
        b.probe(f"h{q}", "magnetic", pos, "xyz")
    return b.write(outdir, f"bordered_{boundary}_{nx}x{ny}x{nz}")


def graded_steps(n, rng, dmin=1e-3, dmax=3e-3):
    f = int(rng.integers(1, 4))
    ph = rng.uniform(0, 2 * math.pi)
    i = np.arange(n)
    mid, amp = (dmin + dmax) / 2, (dmax - dmin) / 2
    return (mid + amp * np.cos(2 * math.pi * f * i / n + ph)).astype(np.float32)


def dispersive_large(outdir, n=512, steps=2000, fraction=0.30, layers=12, nprobes=8, edge=(32, 128),
                     seed_mesh=4, seed_blocks=5, seed_probes=6, margin=4) -> Path:
    b = _Builder((n, n, n), steps, layers)
    rng = np.random.default_rng(seed_mesh)
    sx, sy, sz = (graded_steps(n, rng) for _ in range(3))
    b.steps(sx, sy, sz)
    dmin = float(min(sx.min(), sy.min(), sz.min()))
    dt = courant_dt(dmin)
    ds = dt / 2
    rng = np.random.default_rng(seed_blocks)
    target = fraction * n ** 3
    lo_lim, hi_lim = margin, n - margin - 1
    blocks = []
    occ = _Occupancy(n)
    while occ.count < target and len(blocks) < 250:
        e = rng.integers(max(2, edge[0]), edge[1] + 1, size=3)
        e = np.minimum(e, hi_lim - lo_lim)
        o = [int(rng.integers(lo_lim, hi_lim - e[a] + 1)) for a in range(3)]
        box = (o[0], o[0] + e[0] - 1, o[1], o[1] + e[1] - 1, o[2], o[2] + e[2] - 1)
        occ.add(box)
        blocks.append(box)
        mid = b.material(_pole_pair_material(rng))
        b.bulk(mid, [box])
    c = n // 2
    sigma = 20e-12
    b.nodal((c, c, c), (c, c, c + 1), "dipole.exc", ds, gaussian_derivative(ds, sigma, 6 * sigma, 12 * sigma), hard=False)
    rng = np.random.default_rng(seed_probes)
    for q in range(nprobes):
        pos = rng.integers(1, n - 1, size=3)
        b.probe(f"p{q}", "electric", pos, "z")
    path = b.write(outdir, f"dispersive_large_{n}")
    return path


class _Occupancy:
    """Counts cells covered by a union of boxes (coarse bitmap for large n)."""

    def __init__(self, n):
        self.n = n
        self.s = max(1, n // 128)
        m = (n + self.s - 1) // self.s
        self.grid = np.zeros((m, m, m), bool)
        self.count = 0

    def add(self, box):
        s = self.s
        x0, x1, y0, y1, z0, z1 = box
        g = self.grid[x0 // s:x1 // s + 1, y0 // s:y1 // s + 1, z0 // s:z1 // s + 1]
        g[...] = True
        self.count = int(self.grid.sum()) * s ** 3


def _tem_angles(rng):
    theta = math.acos(rng.uniform(-1, 1))
    phi = rng.uniform(0, 2 * math.pi)
    k = np.array([math.sin(theta) * math.cos(phi), math.sin(theta) * math.sin(phi), math.cos(theta)])
    th_hat = np.array([math.cos(theta) * math.cos(phi), math.cos(theta) * math.sin(phi), -math.sin(theta)])
    ph_hat = np.array([-math.sin(phi), math.cos(phi), 0.0])
    psi = rng.uniform(0, 2 * math.pi)
    e = math.cos(psi) * th_hat + math.sin(psi) * ph_hat
    alpha = math.acos(max(-1.0, min(1.0, e[2])))
    beta = math.atan2(e[1], e[0])
    return theta, phi, alpha, beta


def batch_instance(outdir, index, rng, layers=8, steps=None, edges=None, inset=5) -> Path:
    """One member of the batched stream: non-cubic grid, 1-6 dielectric
    blocks, a plane wave of seeded direction and polarisation."""
    if edges is None:
        edges = [int(round(math.exp(rng.uniform(math.log(32), math.log(160))))) for _ in range(3)]
    nx, ny, nz = edges
    steps = int(rng.integers(500, 3001)) if steps is None else steps
    b = _Builder((nx, ny, nz), steps, layers)
    dx = 0.005
    b.steps([dx], [dx], [dx])
    ds = courant_dt(dx) / 4
    th, ph, al, be = _tem_angles(rng)
    b.planewave((inset,) * 3, (nx - inset, ny - inset, nz - inset), th, ph, al, be, "gauss.exc", ds,
                gaussian(ds, 60e-12, 240e-12, 0.8e-9))
    for q in range(int(rng.integers(1, 7))):
        box = []
        for a, n in enumerate((nx, ny, nz)):
            lo, hi = inset + 2, n - inset - 3
            e = int(rng.integers(2, max(3, (hi - lo) // 2)))
            o = int(rng.integers(lo, max(lo + 1, hi - e + 1)))
            box += [o, min(hi, o + e - 1)]
        mid = b.material({"type": "simple", "relativePermittivity": _f32(rng.uniform(1, 10)),
                          "electricConductivity": _f32(rng.uniform(0, 0.05))})
        b.bulk(mid, [tuple(box)])
    for q in range(4):
        pos = [int(rng.integers(1, n - 1)) for n in (nx, ny, nz)]
        b.probe(f"p{q}", "electric", pos, "xyz"[q % 3])
    return b.write(outdir, f"batch_{index:03d}")


def served_request(outdir, index, rng, layers=10, steps=None, edges=None) -> Path:
    """One request of the served stream: grid edges log-uniform 48-256,
    0-2 pole-residue blocks, a soft dipole, 4-32 probes."""
    if edges is None:
        edges = [int(round(math.exp(rng.uniform(math.log(48), math.log(256))))) for _ in range(3)]
    nx, ny, nz = edges
    steps = int(rng.integers(500, 4001)) if steps is None else steps
    b = _Builder((nx, ny, nz), steps, layers)
    dx = 0.002
    b.steps([dx], [dx], [dx])
    ds = courant_dt(dx) / 2
    for q in range(int(rng.integers(0, 3))):
        box = []
        for n in (nx, ny, nz):
            lo, hi = 4, n - 5
            e = int(rng.integers(2, max(3, (hi - lo) // 2)))
            o = int(rng.integers(lo, max(lo + 1, hi - e + 1)))
            box += [o, min(hi, o + e - 1)]
        mid = b.material(_pole_pair_material(rng))
        b.bulk(mid, [tuple(box)])
    cx, cy, cz = nx // 2, ny // 2, nz // 2
    sigma = 20e-12
    b.nodal((cx, cy, cz), (cx, cy, cz + 1), "dipole.exc", ds, gaussian_derivative(ds, sigma, 6 * sigma, 12 * sigma))
    for q in range(int(rng.integers(4, 33))):
        pos = [int(rng.integers(1, n - 1)) for n in (nx, ny, nz)]
        b.probe(f"p{q}", "electric", pos, "z")
    return b.write(outdir, f"req_{index:04d}")


def load(path) -> "Problem":  # noqa: F821
    return read_case(path)
