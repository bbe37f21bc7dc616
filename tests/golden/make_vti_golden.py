"""Make the VTI golden files with the REFERENCE's own writer.

Compiles tests/cpp/vti_case.cpp against the reference's src/ headers (with
the host Kokkos stand-in of oracle/ref) and runs it; the outputs in
tests/golden/vti/ pin this repository's writers byte for byte.  Needs the
reference sources (run where they are available):

    python tests/golden/make_vti_golden.py
"""
from __future__ import annotations

import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
from oracle import REFERENCE_DIR  # noqa: E402

REF_SRC = REFERENCE_DIR / "src"
OUT = HERE / "vti"


def arrays() -> np.ndarray:
    """The 300 float32 inputs of the case: a smooth field, negatives, a
    zero, tiny and large magnitudes (so that the 9-digit ASCII and the raw
    Float32 paths both see varied values)."""
    i = np.arange(300, dtype=np.float64)
    v = np.sin(0.37 * i) * (1.0 + 0.5 * np.cos(0.11 * i))
    v[7] = 0.0
    v[61] = -3.0e-9
    v[250] = 12345.678
    return v.astype(np.float32)


def main() -> int:
    OUT.mkdir(exist_ok=True)
    arrays().tofile(OUT / "arrays.bin")
    with tempfile.TemporaryDirectory() as td:
        exe = Path(td) / "vti_ref"
        cmd = ["g++", "-std=c++20", "-O1", f"-I{REF_SRC}", f"-I{ROOT / 'oracle' / 'ref' / 'kokkos_shim'}",
               str(ROOT / "tests" / "cpp" / "vti_case.cpp"), "-o", str(exe), "-fopenmp"]
        subprocess.run(cmd, check=True)
        subprocess.run([str(exe), str(OUT), str(OUT / "arrays.bin"), "solver"], check=True)
    (OUT / "never.vti").unlink(missing_ok=True)
    for p in sorted(OUT.iterdir()):
        print(p.name, p.stat().st_size)
    return 0


if __name__ == "__main__":
    sys.exit(main())
