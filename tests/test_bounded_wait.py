"""Failure detection of the pipelined kernels, tested without a GPU fault.

Every wait inside the TMA-pipelined field kernels (a consumer warp waiting
for a plane, the producer waiting for a free ring stage) is bounded; when a
bound runs out the kernel records where in an error word, stops, waits with
the default bound for the loads it still has in flight, and exits, and the
next synchronize reports SGPU_ERR_TIMEOUT.  The failure drill
(sgpu_set_wait_drill) makes the producer warps issue no loads, so no plane
ever arrives -- a flag nothing sets -- and with a short bound
(sgpu_set_wait_cycles, 2e5 cycles, about 0.1 ms) every consumer wait runs
out: no wait is endless, nothing is in flight, nothing faults, and the error
path runs."""
import tempfile
from pathlib import Path

import numpy as np
import pytest

from bits import assert_bits_equal
from cases import small
from semba_fdtd_b200 import Solver, casegen, read_case
from semba_fdtd_b200.batch import Batch

import oracle

pytestmark = pytest.mark.gpu

SGPU_ERR_TIMEOUT = 6
SHORT = 200_000  # clock cycles, about 0.1 ms


def test_expired_wait_reports_timeout_then_a_fresh_context_runs():
    pb = small()
    with Solver(pb, kernel_family=1) as s:
        lib = s.lib
        assert lib.sgpu_set_wait_cycles(s.handle, SHORT) == 0
        assert lib.sgpu_set_wait_drill(s.handle, 1) == 0
        assert lib.sgpu_advance_e(s.handle, 0) == 0
        rc = lib.sgpu_synchronize(s.handle)
        assert rc == SGPU_ERR_TIMEOUT, rc
        assert "bounded wait" in lib.sgpu_last_error(s.handle).decode()
        # the error word is cleared once reported
        assert lib.sgpu_synchronize(s.handle) == 0
        # the H side too, through the graph-replayed steps
        assert lib.sgpu_advance_steps(s.handle, 1, 2) == 0
        assert lib.sgpu_synchronize(s.handle) == SGPU_ERR_TIMEOUT
        # drill off, default bound: the context launches again without error
        assert lib.sgpu_set_wait_drill(s.handle, 0) == 0
        assert lib.sgpu_set_wait_cycles(s.handle, 4_000_000_000) == 0
        assert lib.sgpu_advance_h(s.handle, 3) == 0
        assert lib.sgpu_synchronize(s.handle) == 0
    # a fresh context is unaffected and still equals the oracle
    o = oracle.Oracle(pb)
    try:
        ref = o.step(40)
    finally:
        o.close()
    with Solver(pb, kernel_family=1) as s:
        assert_bits_equal(s.run(40), ref)


def test_expired_wait_in_the_batch_reports_timeout():
    d = Path(tempfile.mkdtemp(prefix="semba_wait_"))
    rng = np.random.default_rng(5)
    pbs = [read_case(casegen.batch_instance(d, q, rng, layers=5, steps=40, edges=e, inset=4))
           for q, e in enumerate([(20, 24, 28), (28, 20, 22)])]
    with Batch(256 << 20, 4, kernel_family=1) as b:
        for pb in pbs:
            b.add(pb)
        assert b.lib.sgpu_batch_set_wait_cycles(b._h, SHORT) == 0
        assert b.lib.sgpu_batch_set_wait_drill(b._h, 1) == 0
        b.advance(1)
        rc = b.lib.sgpu_batch_synchronize(b._h)
        assert rc == SGPU_ERR_TIMEOUT, rc
        assert "bounded wait" in b.lib.sgpu_batch_last_error(b._h).decode()
