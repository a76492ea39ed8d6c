"""Problem description and the smbjson-subset reader.

A :class:`Problem` is the NFDE-level description the solver needs: grid,
CPML, material regions, plane waves, nodal sources and point probes.  It is
read from the reference's JSON input format (``*.fdtd.json``, parsed by
``src_json_parser/smbjson.F90:118-176``) with three documented extensions the
reference parser does not read:

* ``general.cfl`` -- the ``-cfl`` switch (``interpreta_switches.F90:892-906``)
  given in the case file;
* material ``"type": "simple"`` with ``relativePermittivity``,
  ``electricConductivity``, ``relativePermeability``, ``magneticConductivity``
  -- an isotropic dielectric volume (the NFDE dielectric regions of
  ``preprocess_geom.F90:686-760``), eps stored as ``eps_r * eps0`` in FP32;
* material ``"type": "poleResidue"`` with ``epsilonInfinity``,
  ``electricConductivity``, ``poles`` and ``residues`` (lists of [re, im]),
  and for magnetic dispersion ``muInfinity``, ``magneticConductivity``,
  ``magneticPoles`` and ``magneticResidues`` -- the NFDE frequency-dependent
  volumes (``preprocess_geom.F90:5055-5248``); the NFDE stores minus the pole,
  ``b11 = -pole`` (``bM11`` for the magnetic ones), in complex64;
* nodal sources may set ``"hard": false`` for a soft (current-like) source;
  the reference's JSON path only builds hard ones (``isField``,
  ``preprocess_geom.F90:2913``).

Material associations of type ``bulk`` assign a material to cell elements.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import _lib

# tipofrontera codes of nfde_types.F90:67-71 and the smbjson labels of
# src_json_parser/labels_mod.F90:108-112
BORDER_CODES = {"pec": 1, "pmc": 2, "periodic": 4, "mur": 7, "pml": 9}
EPS0 = np.float32(8.8541878176203898505365630317107502606083701665994498081024171524053950954599821142852891607182008932e-12)
MU0 = np.float32(1.2566370614359172953850573533118011536788677597500423283899778369231265625144835994512139301368468271e-6)
COMP = {"Ex": 0, "Ey": 1, "Ez": 2, "Hx": 3, "Hy": 4, "Hz": 5}


@dataclass
class Region:
    kind: int  # 0 PEC, 1 dielectric, 2 pole-residue
    boxes: np.ndarray  # (n, 6) int32: XI XE YI YE ZI ZE
    eps: float = float(EPS0)
    sigma: float = 0.0
    mu: float = float(MU0)
    sigmam: float = 0.0
    residues: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex64))
    bpoles: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex64))
    # magnetic poles of a pole-residue region (aM11 residues, bM11 = -pole)
    mresidues: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex64))
    mbpoles: np.ndarray = field(default_factory=lambda: np.zeros(0, np.complex64))


@dataclass
class Waveform:
    samples: np.ndarray  # float32, numus + 1 values
    dsamples: np.float32


@dataclass
class PlaneWave:
    coor1: tuple
    coor2: tuple
    theta: float
    phi: float
    alpha: float
    beta: float
    wave: Waveform


@dataclass
class NodalSource:
    is_elec: bool
    is_hard: bool
    boxes: np.ndarray  # (n, 6)
    amp: np.ndarray  # (n, 3) float32
    wave: Waveform


@dataclass
class Problem:
    nx: int
    ny: int
    nz: int
    desx: np.ndarray
    desy: np.ndarray
    desz: np.ndarray
    nsteps: int
    dt: float = 0.0
    forcecfl: bool = True
    cfl: float = 0.8
    pml_layers: tuple = (10,) * 6
    pml_order: tuple = (2.0,) * 6
    pml_refl: tuple = (0.001,) * 6
    alphamax: float = 0.0
    alphaorder: float = 1.0
    kappamax: float = 1.0
    regions: list = field(default_factory=list)
    planewaves: list = field(default_factory=list)
    nodals: list = field(default_factory=list)
    probes: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    probe_names: list = field(default_factory=list)
    # per probe row: (output request name, initialTime, finalTime,
    # samplingPeriod) of its probe, the times real(4) as smbjson reads them
    probe_requests: list = field(default_factory=list)
    origin: tuple = (0.0, 0.0, 0.0)
    name: str = "case"
    # the case file's name without ".json" (nEntradaRoot): output files are
    # named <root>_<request>_...
    root: str = "case.fdtd"
    boundary: str = "pml"
    # per face (back, front, left, right, down, up): "pml", "pec", "pmc",
    # "periodic" or "mur"; only "pml" faces carry layers
    borders: tuple = ("pml",) * 6
    mur_after_pml: bool = False  # the -mur1 / -mur2 switch

    @property
    def border_codes(self) -> tuple:
        return tuple(BORDER_CODES[b] for b in self.borders)

    @property
    def layers(self) -> tuple:
        """CPML layers per face (0 on faces of other kinds)."""
        return tuple(int(L) if b == "pml" else 0 for L, b in zip(self.pml_layers, self.borders))

    @property
    def swept_cells(self) -> int:
        """Cells per E+H update, PML included (the Mcells of errorreport.F90:530)."""
        L = self.layers
        return (self.nx + L[0] + L[1]) * (self.ny + L[2] + L[3]) * (self.nz + L[4] + L[5])

    # -- C description ---------------------------------------------------
    def to_desc(self, probe_capacity: int = 1024):
        """Build the sgpu_problem struct; returns (desc, keepalive)."""
        keep = []

        def fp(a, dtype=np.float32):
            a = np.ascontiguousarray(a, dtype=dtype)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_float if dtype == np.float32 else C.c_int))

        def ip(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            keep.append(a)
            return a.ctypes.data_as(C.POINTER(C.c_int))

        d = _lib.ProblemDesc()
        d.nx, d.ny, d.nz = self.nx, self.ny, self.nz
        d.desx, d.desy, d.desz = fp(self.desx), fp(self.desy), fp(self.desz)
        d.originx, d.originy, d.originz = self.origin
        d.dt = self.dt
        d.forcecfl = int(self.forcecfl)
        d.cfl = self.cfl
        for f in range(6):
            d.pml_layers[f] = int(self.pml_layers[f])
            d.pml_order[f] = float(self.pml_order[f])
            d.pml_refl[f] = float(self.pml_refl[f])
        d.alphamax, d.alphaorder, d.kappamax = self.alphamax, self.alphaorder, self.kappamax
        regs = (_lib.Region * max(1, len(self.regions)))()
        for q, r in enumerate(self.regions):
            g = regs[q]
            g.kind = r.kind
            g.eps, g.sigma, g.mu, g.sigmam = r.eps, r.sigma, r.mu, r.sigmam
            g.npoles = len(r.residues)
            g.residues = fp(np.asarray(r.residues, np.complex64).view(np.float32))
            g.bpoles = fp(np.asarray(r.bpoles, np.complex64).view(np.float32))
            g.nboxes = len(r.boxes)
            g.boxes = ip(np.asarray(r.boxes, np.int32).reshape(-1))
            g.mpoles = len(r.mresidues)
            g.mresidues = fp(np.asarray(r.mresidues, np.complex64).view(np.float32))
            g.mbpoles = fp(np.asarray(r.mbpoles, np.complex64).view(np.float32))
        keep.append(regs)
        d.nregions, d.regions = len(self.regions), regs
        pws = (_lib.PlaneWaveSrc * max(1, len(self.planewaves)))()
        for q, w in enumerate(self.planewaves):
            s = pws[q]
            s.x1, s.y1, s.z1 = w.coor1
            s.x2, s.y2, s.z2 = w.coor2
            s.theta, s.phi, s.alpha, s.beta = w.theta, w.phi, w.alpha, w.beta
            s.nsamples = len(w.wave.samples)
            s.samples = fp(w.wave.samples)
            s.dsamples = float(w.wave.dsamples)
        keep.append(pws)
        d.npw, d.pw = len(self.planewaves), pws
        nds = (_lib.NodalSrc * max(1, len(self.nodals)))()
        for q, n in enumerate(self.nodals):
            s = nds[q]
            s.is_elec, s.is_hard = int(n.is_elec), int(n.is_hard)
            s.npoints = len(n.boxes)
            s.boxes = ip(np.asarray(n.boxes).reshape(-1))
            s.amp = fp(np.asarray(n.amp).reshape(-1))
            s.nsamples = len(n.wave.samples)
            s.samples = fp(n.wave.samples)
            s.dsamples = float(n.wave.dsamples)
        keep.append(nds)
        d.nnodal, d.nodal = len(self.nodals), nds
        d.nprobes = len(self.probes)
        d.probes = ip(np.asarray(self.probes, np.int32).reshape(-1))
        d.probe_capacity = probe_capacity
        for f, code in enumerate(self.border_codes):
            d.border[f] = code
        d.mur_after_pml = int(self.mur_after_pml)
        return d, keep


# ---------------------------------------------------------------------------
# smbjson subset

def _interval_to_box(iv) -> list[int]:
    """cellIntervalsToCoords (src_json_parser/parser_tools.F90:107-140)."""
    a, b = iv
    out = []
    for d in range(3):
        x, y = int(a[d]), int(b[d])
        if x < y:
            out += [x, y - 1]
        elif x == y:
            out += [x, x]
        else:
            out += [y + 1, x - 1]
    return out


def _orientation(iv) -> int:
    """Signed direction (1..3) of a linel interval (cells.F90:95-120)."""
    a, b = iv
    for d in range(3):
        if b[d] - a[d] > 0:
            return d + 1
    for d in range(3):
        if b[d] - a[d] < 0:
            return -(d + 1)
    return 0


def read_waveform(path: Path) -> Waveform:
    """Excitation file: two columns (time, value); the sample step is the
    difference of the first two times in FP32 (preprocess_geom.F90:4963-4997)."""
    rows = [ln.split() for ln in Path(path).read_text().splitlines() if ln.strip()]
    t = np.array([np.float32(float(r[0])) for r in rows], np.float32)
    v = np.array([np.float32(float(r[1])) for r in rows], np.float32)
    return Waveform(samples=v, dsamples=np.float32(t[1] - t[0]))


def write_waveform(path: Path, dt: float, values: np.ndarray) -> None:
    t = np.arange(len(values), dtype=np.float64) * dt
    with open(path, "w") as fh:
        for a, b in zip(t.astype(np.float32), np.asarray(values, np.float32)):
            fh.write(f"{float(a):.9e} {float(b):.9e}\n")


def read_case(path: str | Path, search: tuple = ()) -> Problem:
    """Read a case file.  Waveform (``magnitudeFile``) names are looked up in
    the case file's directory first, then in each directory of `search`."""
    path = Path(path)
    js = json.loads(path.read_text())

    def wave_path(name: str) -> Path:
        for d in (path.parent, *map(Path, search)):
            if (d / name).exists():
                return d / name
        raise FileNotFoundError(f"waveform {name!r} not found next to {path.name} or in {list(search)}")
    grid = js["mesh"]["grid"]
    nx, ny, nz = (int(v) for v in grid["numberOfCells"])
    steps = grid["steps"]

    def des(key, n):
        v = np.asarray(steps[key], dtype=np.float32)
        return np.full(n, v[0], np.float32) if len(v) == 1 else v.astype(np.float32)

    gen = js.get("general", {})
    # readBoundary (smbjson.F90:329-370) reads "all": one kind for the six
    # faces, CPML properties (defaults 8 layers, order 2, R 0.001) only for
    # "pml".  The format's documentation (doc/smbjson.md:72-100) also names
    # per-face labels and a Mur default when "boundary" is absent; both are
    # read here too.
    faces = ("xLower", "xUpper", "yLower", "yUpper", "zLower", "zUpper")
    bjs = js.get("boundary")
    if bjs is None:
        per = [{"type": "mur"}] * 6
    elif "all" in bjs:
        per = [bjs["all"]] * 6
    else:
        missing = [f for f in faces if f not in bjs]
        if missing:
            raise ValueError(f"boundary: no entry for {missing}")
        per = [bjs[f] for f in faces]
    kinds = tuple(str(b.get("type", "pml")) for b in per)
    for k in kinds:
        if k not in BORDER_CODES:
            raise ValueError(f"boundary type {k!r} is not one of {sorted(BORDER_CODES)}")
    layers = tuple(int(b.get("layers", 8)) if k == "pml" else 0 for b, k in zip(per, kinds))
    orders = tuple(float(b.get("order", 2.0)) for b in per)
    refls = tuple(float(b.get("reflection", 0.001)) for b in per)
    first = per[0]
    pb = Problem(nx=nx, ny=ny, nz=nz, desx=des("x", nx), desy=des("y", ny), desz=des("z", nz),
                 nsteps=int(gen.get("numberOfSteps", 0)), dt=float(gen.get("timeStep", 0.0)),
                 forcecfl="cfl" in gen, cfl=float(gen.get("cfl", 1.0)),
                 pml_layers=layers, pml_order=orders, pml_refl=refls,
                 alphamax=float(first.get("pmlAlpha", 0.0)), alphaorder=float(first.get("pmlAlphaOrder", 1.0)),
                 kappamax=float(first.get("pmlKappa", 1.0)), name=path.name.split(".")[0],
                 boundary=kinds[0] if len(set(kinds)) == 1 else "mixed", borders=kinds)
    coords = {c["id"]: c["relativePosition"] for c in js["mesh"].get("coordinates", [])}
    elems = {e["id"]: e for e in js["mesh"].get("elements", [])}
    mats = {m["id"]: m for m in js.get("materials", [])}

    def boxes_of(ids):
        out = []
        for i in ids:
            for iv in elems[i]["intervals"]:
                out.append(_interval_to_box(iv))
        return np.asarray(out, np.int32).reshape(-1, 6)

    pec, diel, disp = [], [], []
    for a in js.get("materialAssociations", []):
        if a.get("type", "bulk") != "bulk":
            continue
        m = mats[a["materialId"]]
        boxes = boxes_of(a["elementIds"])
        t = m["type"]
        if t == "pec":
            pec.append(Region(kind=0, boxes=boxes))
        elif t == "simple":
            er = np.float32(m.get("relativePermittivity", 1.0))
            mr = np.float32(m.get("relativePermeability", 1.0))
            diel.append(Region(kind=1, boxes=boxes, eps=float(er * EPS0), sigma=float(m.get("electricConductivity", 0.0)),
                               mu=float(mr * MU0), sigmam=float(m.get("magneticConductivity", 0.0))))
        elif t == "poleResidue":
            einf = np.float32(m.get("epsilonInfinity", 1.0))
            muinf = np.float32(m.get("muInfinity", 1.0))
            poles = np.array([complex(p[0], p[1]) for p in m.get("poles", [])], np.complex64)
            res = np.array([complex(p[0], p[1]) for p in m.get("residues", [])], np.complex64)
            mpoles = np.array([complex(p[0], p[1]) for p in m.get("magneticPoles", [])], np.complex64)
            mres = np.array([complex(p[0], p[1]) for p in m.get("magneticResidues", [])], np.complex64)
            disp.append(Region(kind=2, boxes=boxes, eps=float(einf * EPS0), sigma=float(m.get("electricConductivity", 0.0)),
                               mu=float(muinf * MU0), sigmam=float(m.get("magneticConductivity", 0.0)),
                               residues=res, bpoles=(-poles).astype(np.complex64),
                               mresidues=mres, mbpoles=(-mpoles).astype(np.complex64)))
        else:
            raise ValueError(f"material type {t!r} is outside this path")
    pb.regions = pec + diel + disp
    for s in js.get("sources", []):
        if s["type"] == "planewave":
            box = boxes_of(s["elementIds"])[0]
            pb.planewaves.append(PlaneWave(coor1=(box[0], box[2], box[4]), coor2=(box[1], box[3], box[5]),
                                           theta=float(s["direction"]["theta"]), phi=float(s["direction"]["phi"]),
                                           alpha=float(s["polarization"]["theta"]), beta=float(s["polarization"]["phi"]),
                                           wave=read_waveform(wave_path(s["magnitudeFile"]))))
        elif s["type"] == "nodalSource":
            bx, amp = [], []
            for i in s["elementIds"]:
                for iv in elems[i]["intervals"]:
                    o = _orientation(iv)
                    a3 = [0.0, 0.0, 0.0]
                    if o:
                        a3[abs(o) - 1] = 1.0 if o > 0 else -1.0
                    bx.append(_interval_to_box(iv))
                    amp.append(a3)
            pb.nodals.append(NodalSource(is_elec=s.get("field", "electric") == "electric", is_hard=bool(s.get("hard", True)),
                                         boxes=np.asarray(bx, np.int32), amp=np.asarray(amp, np.float32),
                                         wave=read_waveform(wave_path(s["magnitudeFile"]))))
        else:
            raise ValueError(f"source type {s['type']!r} is outside this path")
    probes, names, requests = [], [], []
    for p in js.get("probes", []):
        if p["type"] != "point":
            continue
        base_c = 0 if p.get("field", "electric") == "electric" else 3
        # readProbe / getDomain (smbjson.F90:686-730, :1310-1350): the name is
        # the output request, "_log_" appended for a logarithmic frequency
        # spacing; the time window defaults to 0 (save every step)
        dom = p.get("domain", {})
        req = str(p.get("name", " ")).strip()
        if dom.get("frequencySpacing", "linear") == "logarithmic":
            req += "_log_"
        window = tuple(float(np.float32(dom.get(k, 0.0))) for k in ("initialTime", "finalTime", "samplingPeriod"))
        for eid in p["elementIds"]:
            pos = coords[elems[eid]["coordinateIds"][0]]
            for d in p.get("directions", ["x", "y", "z"]):
                c = base_c + "xyz".index(d)
                probes.append([c, int(pos[0]), int(pos[1]), int(pos[2])])
                names.append(f"{p.get('name', 'probe')}_{'EH'[c // 3]}{d}_{pos[0]}_{pos[1]}_{pos[2]}")
                requests.append((req,) + window)
    pb.probes = np.asarray(probes, np.int32).reshape(-1, 4)
    pb.probe_names = names
    pb.probe_requests = requests
    pb.root = path.name[:-5] if path.name.endswith(".json") else path.name
    return pb
