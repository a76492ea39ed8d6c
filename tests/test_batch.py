"""Batched form: instances of uneven sizes in one arena give the same bits
as solo runs of the oracle, whether they start together, join while others
run, or run under autotuned launch shapes; the arena is reused."""
import tempfile
from pathlib import Path

import numpy as np

from bits import assert_bits_equal
import pytest

import oracle
from semba_fdtd_b200 import casegen, read_case
from semba_fdtd_b200.batch import Batch, Plan

pytestmark = pytest.mark.gpu

_DIR = Path(tempfile.mkdtemp(prefix="semba_batch_"))


def _instances():
    rng = np.random.default_rng(11)
    shapes = [((20, 24, 28), 70), ((32, 20, 22), 45), ((24, 30, 20), 100)]
    pbs = [read_case(casegen.batch_instance(_DIR, q, rng, layers=5, steps=s, edges=e, inset=4))
           for q, (e, s) in enumerate(shapes)]
    # a served-stream request with pole-residue blocks (the first seed that draws some)
    for seed in range(100):
        pb = read_case(casegen.served_request(_DIR, 9, np.random.default_rng(seed), layers=5, steps=80, edges=(24, 26, 28)))
        if any(r.kind == 2 for r in pb.regions):
            break
    pbs.append(pb)
    return pbs


_solo_cache = {}


def _solo(i, pb):
    if i not in _solo_cache:
        o = oracle.Oracle(pb)
        _solo_cache[i] = (o.step(pb.nsteps + 1), [o.field(c) for c in range(6)])
    return _solo_cache[i]


def _check(b, slots, pbs):
    for i, (s, pb) in enumerate(zip(slots, pbs)):
        tr, f = _solo(i, pb)
        assert b.done(s)
        assert_bits_equal(b.probes(s), tr, err_msg=f"instance {i}")
        for c in range(6):
            assert_bits_equal(b.field(s, c), f[c], err_msg=f"instance {i} component {c}")


@pytest.mark.parametrize("family", [1, 0], ids=["tma", "regs"])
def test_batch_equals_solo_runs(family):
    pbs = _instances()
    assert any(r.kind == 2 for pb in pbs for r in pb.regions)  # the ADE path is exercised
    with Batch(1 << 30, 16, kernel_family=family) as b:
        slots = [b.add(pb) for pb in pbs]
        b.run_all()
        _check(b, slots, pbs)


def test_instances_set_up_by_several_threads():
    """Instances added from four host threads at once, while steps of the
    first one are queued, give the same bits as their solo runs."""
    from concurrent.futures import ThreadPoolExecutor
    pbs = _instances()
    with Batch(1 << 30, 16) as b:
        first = b.add(pbs[0])
        b.advance(11)
        with ThreadPoolExecutor(4) as pool:
            futs = [pool.submit(b.add, Plan(pb)) for pb in pbs[1:]]
            b.advance(5)
            rest = [f.result() for f in futs]
        slots = [first] + rest
        assert len(set(slots)) == len(slots)
        b.run_all()
        _check(b, slots, pbs)


def test_join_while_running_and_arena_reuse():
    pbs = _instances()
    with Batch(1 << 30, 16) as b:
        slots = [b.add(pbs[0])]
        b.advance(37)
        slots.append(b.add(Plan(pbs[1])))  # planned on the host first
        b.advance(20)
        slots += [b.add(pbs[2]), b.add(pbs[3])]
        b.run_all()
        _check(b, slots, pbs)
        assert b.memory()[1] > 0
        for s in slots:
            b.remove(s)
        cap, used, largest = b.memory()
        assert used == 0 and largest == cap
        # the freed arena takes the same instances again
        slots = [b.add(pb) for pb in pbs]
        b.run_all()
        _check(b, slots, pbs)


def test_autotuned_shapes_keep_results():
    pbs = _instances()
    with Batch(1 << 30, 16) as b:
        slots = [b.add(pb) for pb in pbs]
        chunks, ctas = b.autotune(2)
        assert all(c in (8, 16, 32, 64, 128) for c in chunks) and ctas in (2, 3, 4, 6)
        b.run_all()
        _check(b, slots, pbs)


def test_arena_too_small_is_refused_cleanly():
    pbs = _instances()
    plan = Plan(pbs[2])
    with Batch(plan.footprint // 4, 4) as b:
        with pytest.raises(Exception):
            b.add(pbs[2])
        assert b.memory()[1] == 0
    plan.close()


@pytest.mark.parametrize("family", [1, 0], ids=["tma", "regs"])
def test_batch_with_every_border_kind_and_magnetic_ade(family):
    """Mur, PEC, PMC, periodic and CPML(+Mur) instances and one with magnetic
    pole-residue media next to a CPML one: the clone, Mur and magnetic ADE
    phases run over the instances that have them."""
    from cases import closed, mdisp, mixed, mur
    pbs = [mur(), mixed(), closed(), mdisp(), _instances()[1]]
    with Batch(1 << 30, 8, kernel_family=family) as b:
        slots = [b.add(pb) for pb in pbs]
        b.run_all()
        for s, pb in zip(slots, pbs):
            o = oracle.Oracle(pb)
            tr = o.step(pb.nsteps + 1)
            assert_bits_equal(b.probes(s), tr, err_msg=pb.name)
            for c in range(6):
                assert_bits_equal(b.field(s, c), o.field(c), err_msg=f"{pb.name} component {c}")
