"""Committed golden fixtures (tests/golden/, made by make_golden.py).

CPU: the FP32 oracle reproduces the fixtures bit for bit on this machine.
GPU: the -fmad=false library reproduces them bit for bit, with no oracle in
the process."""
import hashlib
import json
from pathlib import Path

import numpy as np

from bits import assert_bits_equal
import pytest

from cases import ALL

GOLD = Path(__file__).resolve().parent / "golden"


def _load():
    traces = np.load(GOLD / "oracle_traces.npz")
    fields = json.loads((GOLD / "oracle_fields.json").read_text())
    return traces, fields


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, np.float32).tobytes()).hexdigest()


@pytest.mark.parametrize("name", list(ALL))
def test_oracle_reproduces_golden(name):
    import oracle
    traces, fields = _load()
    pb = ALL[name]()
    o = oracle.Oracle(pb)
    assert_bits_equal(o.step(fields[name]["steps"]), traces[name])
    assert [_sha(o.field(c)) for c in range(6)] == fields[name]["fields"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(ALL))
def test_gpu_reproduces_golden(name):
    from semba_fdtd_b200 import Solver
    traces, fields = _load()
    pb = ALL[name]()
    with Solver(pb) as s:
        s.step(fields[name]["steps"])
        assert_bits_equal(s.probes(), traces[name])
        assert [_sha(s.field(c)) for c in range(6)] == fields[name]["fields"]
