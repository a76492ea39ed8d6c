"""GPU parity at the benchmarked sizes, compared bit for bit.

The scaled cases of tests/cases.py exercise every feature on small grids; the
configurations the benchmark quotes differ from them in ways that only show
at size: multi-chunk z marching, tensor maps over large boxes, more than
100 M pole-residue nodes and 64-bit offsets (536^3).  Here the exact library
(-fmad=false) runs the configurations themselves against the FP32 oracle:

* the small plain case at its real size: 64^3 + CPML 10 = 84^3 swept cells,
  all 1001 steps (the plane wave switches off at step 153), 8 Ex and 8 Hy
  probes at seeded cells;
* the mid plain case: 256^3 + CPML 12 = 280^3 swept cells (lossy sphere,
  20 PEC / dielectric blocks, 64 probes), the first 200 steps and all six
  final fields;
* the large dispersive case: 512^3 graded mesh + CPML 12 = 536^3 swept
  cells, 30 % of the volume in 2-pair pole-residue blocks, soft Ez dipole,
  the first 6 steps and all six final fields (the oracle takes about a
  minute to set it up and half a second a step on 8-16 host cores; its host
  memory peak is about 15 GB).

Traces and fields are compared as bit patterns (tests/bits.py), so signed
zeros count.  The FMA build's tolerance table is printed for the small case
at full size next to the gate of tests/test_gpu_parity.py.
"""
import tempfile
from pathlib import Path

import numpy as np
import pytest

from bits import assert_bits_equal
from semba_fdtd_b200 import Solver, casegen, read_case

import oracle

pytestmark = pytest.mark.gpu

_DIR = Path(tempfile.mkdtemp(prefix="semba_full_"))
REL_L2_FMA = 1e-5


def _oracle(pb, steps):
    o = oracle.Oracle(pb)
    try:
        tr = o.step(steps)
        fields = [o.field(c) for c in range(6)]
    finally:
        o.close()
    return tr, fields


def _check(pb, steps, ref, family):
    rtr, rf = ref
    with Solver(pb, kernel_family=family, max_steps=max(steps, 1)) as s:
        tr = s.run(steps)
        assert tr.shape == rtr.shape
        assert_bits_equal(tr, rtr, err_msg="probe traces")
        for c in range(6):
            assert_bits_equal(s.field(c), rf[c], err_msg=f"component {c}")
        assert s.check_finite()


@pytest.fixture(scope="module")
def small_full():
    pb = read_case(casegen.plain_small(_DIR / "small"))
    assert (pb.nx, pb.ny, pb.nz) == (64, 64, 64) and pb.nsteps == 1000
    steps = pb.nsteps + 1
    return pb, steps, _oracle(pb, steps)


@pytest.fixture(scope="module")
def mid_full():
    pb = read_case(casegen.plain_mid(_DIR / "mid"))
    assert (pb.nx, pb.ny, pb.nz) == (256, 256, 256)
    steps = 200
    return pb, steps, _oracle(pb, steps)


@pytest.fixture(scope="module")
def large_full():
    pb = read_case(casegen.dispersive_large(_DIR / "large"))
    assert (pb.nx, pb.ny, pb.nz) == (512, 512, 512)
    steps = 6
    return pb, steps, _oracle(pb, steps)


@pytest.mark.parametrize("family", [1, 0], ids=["tma", "regs"])
def test_small_full_size(small_full, family):
    pb, steps, ref = small_full
    _check(pb, steps, ref, family)


@pytest.mark.parametrize("family", [1, 0], ids=["tma", "regs"])
def test_mid_280cube(mid_full, family):
    pb, steps, ref = mid_full
    _check(pb, steps, ref, family)


@pytest.mark.parametrize("family", [1, 0], ids=["tma", "regs"])
def test_large_536cube(large_full, family):
    pb, steps, ref = large_full
    _check(pb, steps, ref, family)


def test_small_full_size_fma_table(small_full):
    """The FMA build on the small case at full size, per probe trace, with the
    classification of tests/test_gpu_parity.py::test_fma_build_within_tolerance
    (resolved / cancellation / noise); the table is printed (pytest -s)."""
    pb, steps, (exact_ref, _) = small_full
    with Solver(pb) as s:
        exact = s.run(steps)
    assert_bits_equal(exact, exact_ref)
    with Solver(pb, variant="fast") as s:
        fast = s.run(steps)
    o = oracle.Oracle(pb, fp64=True)
    try:
        f64 = o.step(steps)
    finally:
        o.close()
    keys = [(int(c) // 3, int(i), int(j), int(k)) for c, i, j, k in pb.probes]
    t = np.asarray(exact, np.float64)
    scale = [np.linalg.norm(t[:, [p for p, k2 in enumerate(keys) if k2 == key]]) for key in keys]
    rows, bad = [], []
    for q in range(exact.shape[1]):
        e = np.asarray(exact[:, q], np.float64)
        f = np.asarray(fast[:, q], np.float64)
        r = np.asarray(f64[:, q], np.float64)
        norm = np.linalg.norm(e)
        if norm == 0:
            continue
        d_fast = np.linalg.norm(f - e) / norm
        e32 = np.linalg.norm(e - r) / np.linalg.norm(r)
        efma = np.linalg.norm(f - r) / np.linalg.norm(r)
        if norm < 0.1 * scale[q]:
            kind, ok = "cancel", np.linalg.norm(f - e) / scale[q] <= REL_L2_FMA
        elif e32 <= REL_L2_FMA:
            kind, ok = "resolved", d_fast <= REL_L2_FMA
        else:
            kind, ok = "noise", efma <= 2 * e32
        c, i, j, k = (int(v) for v in pb.probes[q])
        rows.append(f"  probe {q:2d} {'ExEyEzHxHyHz'[2 * c:2 * c + 2]} ({i:2d},{j:2d},{k:2d}) {kind:8s} "
                    f"fma-vs-exact {d_fast:.3e}  exact-vs-fp64 {e32:.3e}  fma-vs-fp64 {efma:.3e}  {'ok' if ok else 'OUT'}")
        if not ok:
            bad.append(q)
    print("small case 64^3 + CPML 10, 1001 steps, FMA build per probe trace:\n" + "\n".join(rows))
    assert not bad, f"probes {bad} out of tolerance"
