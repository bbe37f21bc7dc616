"""Copy the reference's 3-D Taylor-Green trajectory into a fixture.

The reference ships the output of its own validation/tgv3d.cpp run (D = 64,
Re = 1600, u0 = 0.02, D3Q27 central moments, shifted populations, FP64):
kinetic energy E/E0 and enstrophy Psi/Psi0 at t* = 0, 0.5, ..., 10, in
results/E_tgv3d/tgv3d_re1600_d3q27_cm.dat.  This script copies those rows
(and the header naming the run) to tests/golden/tgv3d_re1600_d3q27_cm.txt so
the GPU test can compare against them without the reference tree.

Run from the repository root:  python tests/golden/make_tgv_golden.py
"""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[2]))
from oracle import REFERENCE_DIR  # noqa: E402

SRC = REFERENCE_DIR / "results" / "E_tgv3d" / "tgv3d_re1600_d3q27_cm.dat"
DST = Path(__file__).resolve().parent / "tgv3d_re1600_d3q27_cm.txt"


def main():
    lines = SRC.read_text().splitlines()
    rows = [ln for ln in lines if ln.strip() and not ln.startswith("#")]
    for ln in rows:
        t, e, p = (float(v) for v in ln.split())  # three numbers per row
    head = [ln for ln in lines if ln.startswith("#")]
    DST.write_text("\n".join(
        ["# copied from the reference's results/E_tgv3d/tgv3d_re1600_d3q27_cm.dat "
         "(output of its validation/tgv3d.cpp)"] + head + rows) + "\n")
    print(f"{len(rows)} rows -> {DST}")


if __name__ == "__main__":
    main()
