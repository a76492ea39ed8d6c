"""Copy the reference's own test fixtures used here into tests/golden/ref/.

    python tests/golden/make_reference_fixtures.py [reference tree]

Run where the reference tree is present (default /root/reference); the
tests read only the copies, so they also run where it is absent.

* planewave.fdtd.json and gauss.exc -- the smbjson case of the reference's
  parser test (test/smbjson/test_read_planewave.F90:24-96) and its
  excitation file (testData/cases/, testData/excitations/);
* probe_format_excerpt.dat -- the header and a sample of the data lines of
  the reference's expected probe output
  (testData/outputs/holland1981.fdtd_mid_point_Wz_11_11_12_s2.dat, written
  by FlushObservationFiles with the format '(e27.17e3,11(e19.9e3))'): every
  line whose numbers include a negative zero among the first 40, then every
  25th line.  It pins the text format of the probe files, not their values.
"""
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "ref"


def main(ref: Path) -> None:
    OUT.mkdir(exist_ok=True)
    shutil.copyfile(ref / "testData/cases/planewave.fdtd.json", OUT / "planewave.fdtd.json")
    shutil.copyfile(ref / "testData/excitations/gauss.exc", OUT / "gauss.exc")
    lines = (ref / "testData/outputs/holland1981.fdtd_mid_point_Wz_11_11_12_s2.dat").read_text().splitlines()
    keep = [lines[0]] + [ln for q, ln in enumerate(lines[1:], 1) if q <= 40 or q % 25 == 0]
    (OUT / "probe_format_excerpt.dat").write_text("\n".join(keep) + "\n")


if __name__ == "__main__":
    main(Path(sys.argv[1]) if len(sys.argv) > 1 else Path("/root/reference"))
