"""Served form: a Poisson stream through the continuous-batching server;
every solve's probe traces equal its solo oracle run (alone and in the mix
give the same bits), and the plain one-at-a-time baseline agrees too."""
import tempfile
from pathlib import Path

import numpy as np

from bits import assert_bits_equal
import pytest

import oracle
from semba_fdtd_b200 import casegen, read_case
from semba_fdtd_b200.serve import Request, Server, poisson_arrivals, run_plain

_DIR = Path(tempfile.mkdtemp(prefix="semba_serve_"))


def _stream(n=8, seed=7):
    rng = np.random.default_rng(seed)
    arr = poisson_arrivals(n, rate=40.0, seed=seed)
    reqs = []
    for q in range(n):
        edges = tuple(int(v) for v in rng.integers(18, 30, size=3))
        steps = int(rng.integers(30, 90))
        pb = read_case(casegen.served_request(_DIR, q, rng, layers=4, steps=steps, edges=edges))
        reqs.append(Request(rid=q, arrival=float(arr[q]), problem=pb, nsteps=steps))
    return reqs


def test_poisson_arrivals_are_seeded_and_increasing():
    a, b = poisson_arrivals(100, 5.0, 3), poisson_arrivals(100, 5.0, 3)
    assert_bits_equal(a, b)
    assert np.all(np.diff(a) > 0)
    assert 10.0 < a[-1] < 40.0


@pytest.mark.gpu
def test_served_results_equal_solo_runs():
    reqs = _stream()
    srv = Server(arena_bytes=1 << 30, max_instances=4, chunk=32, backfill=4)
    try:
        st = srv.run(reqs)
    finally:
        srv.close()
    assert st.completed == len(reqs) and st.peak_resident >= 2
    for r in reqs:
        want = oracle.Oracle(r.problem).step(r.nsteps + 1)
        assert_bits_equal(r.traces, want, err_msg=f"request {r.rid}")
    s = st.summary()
    assert s["p50_s"] <= s["p99_s"]


@pytest.mark.gpu
def test_plain_baseline_equals_solo_runs():
    reqs = _stream(n=3)
    st = run_plain(reqs)
    assert st.completed == 3
    for r in reqs:
        want = oracle.Oracle(r.problem).step(r.nsteps + 1)
        assert_bits_equal(r.traces, want)
