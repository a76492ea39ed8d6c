"""Regenerate the golden fixtures of the FP32 oracle.

    python tests/golden/make_golden.py

For each scaled parity case of tests/cases.py (seeded, deterministic): the
probe traces of a full run ([step, probe] float32, in oracle_traces.npz) and
the SHA-256 of each final field component over its Alloc range in [i, j, k]
C order (oracle_fields.json).  The GPU parity tests compare the -fmad=false
library against these files without running the oracle; the CPU tests check
that the oracle still reproduces them.
"""
import hashlib
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
for p in (ROOT, ROOT / "oracle", HERE.parent):
    sys.path.insert(0, str(p))


def field_sha(arr) -> str:
    return hashlib.sha256(np.ascontiguousarray(arr, np.float32).tobytes()).hexdigest()


def main():
    import oracle
    from cases import ALL
    traces, hashes = {}, {}
    for name, make in ALL.items():
        pb = make()
        o = oracle.Oracle(pb)
        traces[name] = o.step(pb.nsteps + 1)
        hashes[name] = {"steps": pb.nsteps + 1, "fields": [field_sha(o.field(c)) for c in range(6)]}
        o.close()
    np.savez_compressed(HERE / "oracle_traces.npz", **traces)
    (HERE / "oracle_fields.json").write_text(json.dumps(hashes, indent=1) + "\n")


if __name__ == "__main__":
    main()
