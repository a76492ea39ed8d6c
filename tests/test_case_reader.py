"""The smbjson-subset reader's border handling (no GPU): readBoundary's "all"
entry (src_json_parser/smbjson.F90:329-370), the per-face labels and the Mur
default of the format's documentation (doc/smbjson.md:72-100)."""
import json
import tempfile
from pathlib import Path

import pytest

from semba_fdtd_b200 import casegen, read_case


def _case(tmp, boundary):
    path = casegen.plain_small(Path(tmp), n=12, steps=4, inset=3, nprobes=1, layers=4)
    js = json.loads(path.read_text())
    if boundary is None:
        js.pop("boundary")
    else:
        js["boundary"] = boundary
    path.write_text(json.dumps(js))
    return read_case(path)


def test_all_entry_and_mur_default():
    with tempfile.TemporaryDirectory() as tmp:
        pb = _case(tmp, {"all": {"type": "pml", "layers": 6, "order": 3.0, "reflection": 1e-4}})
        assert pb.borders == ("pml",) * 6 and pb.layers == (6,) * 6
        assert pb.pml_order == (3.0,) * 6 and pb.pml_refl == (1e-4,) * 6
        pb = _case(tmp, {"all": {"type": "pec"}})
        assert pb.borders == ("pec",) * 6 and pb.layers == (0,) * 6 and pb.border_codes == (1,) * 6
        pb = _case(tmp, None)
        assert pb.borders == ("mur",) * 6 and pb.border_codes == (7,) * 6


def test_per_face_entries():
    with tempfile.TemporaryDirectory() as tmp:
        pb = _case(tmp, {"xLower": {"type": "pml", "layers": 5}, "xUpper": {"type": "mur"},
                         "yLower": {"type": "pec"}, "yUpper": {"type": "pmc"},
                         "zLower": {"type": "periodic"}, "zUpper": {"type": "periodic"}})
        assert pb.borders == ("pml", "mur", "pec", "pmc", "periodic", "periodic")
        assert pb.border_codes == (9, 7, 1, 2, 4, 4)
        assert pb.layers == (5, 0, 0, 0, 0, 0)
        assert pb.swept_cells == (12 + 5) * 12 * 12
        with pytest.raises(ValueError):
            _case(tmp, {"xLower": {"type": "mur"}})
        with pytest.raises(ValueError):
            _case(tmp, {"all": {"type": "absorbing"}})
