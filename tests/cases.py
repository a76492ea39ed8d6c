"""Scaled variants of the benchmark configurations for parity tests."""
from dataclasses import replace
from functools import lru_cache
from pathlib import Path
import tempfile

from semba_fdtd_b200 import casegen, read_case

_DIR = Path(tempfile.mkdtemp(prefix="semba_cases_"))


@lru_cache(maxsize=None)
def small(n=24, steps=120, layers=6):
    """Plain small: vacuum, CPML, TF/SF plane wave, Ex/Hy probes."""
    return read_case(casegen.plain_small(_DIR / f"small{n}", n=n, steps=steps, inset=5, nprobes=4, layers=layers))


@lru_cache(maxsize=None)
def mid(n=40, steps=120, layers=5):
    """Plain mid: lossy sphere and PEC/dielectric blocks inside the TF/SF box."""
    return read_case(casegen.plain_mid(_DIR / f"mid{n}", n=n, steps=steps, inset=6, radius=max(3, n // 5), nblocks=6,
                                       nprobes=12, layers=layers, edge=(2, max(3, n // 5))))


@lru_cache(maxsize=None)
def disp(n=32, steps=120, layers=5):
    """Dispersive: graded mesh, pole-residue blocks, soft Ez dipole."""
    return read_case(casegen.dispersive_large(_DIR / f"disp{n}", n=n, steps=steps, layers=layers,
                                              edge=(4, max(5, n // 3)), nprobes=6))


@lru_cache(maxsize=None)
def mur(steps=160):
    """First-order Mur on all six faces (the reference's default border)."""
    return read_case(casegen.bordered(_DIR / "mur", steps=steps, boundary="mur"))


@lru_cache(maxsize=None)
def mixed(steps=160):
    """One border kind per face: CPML with Mur behind it (-mur1) at x-, Mur at
    x+, PEC at y-, PMC at y+, periodic along z."""
    pb = read_case(casegen.bordered(_DIR / "mixed", steps=steps, boundary="pml", layers=4))
    return replace(pb, borders=("pml", "mur", "pec", "pmc", "periodic", "periodic"), mur_after_pml=True)


@lru_cache(maxsize=None)
def closed(steps=160):
    """PMC along x, periodic along y, PEC below and Mur above: PMC and
    periodic clones meet on the Hz edges."""
    pb = read_case(casegen.bordered(_DIR / "closed", steps=steps, boundary="pec"))
    return replace(pb, borders=("pmc", "pmc", "periodic", "periodic", "pec", "mur"))


@lru_cache(maxsize=None)
def mdisp(steps=140):
    """Magnetic pole-residue blocks (alone and with electric poles) and an
    electric one."""
    return read_case(casegen.magnetic_dispersive(_DIR / "mdisp", steps=steps))


ALL = {"small": small, "mid": mid, "disp": disp, "mur": mur, "mixed": mixed, "closed": closed, "mdisp": mdisp}
