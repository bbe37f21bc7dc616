"""Record what the reference's own validation programs print, as fixtures.

Builds the programs of validation/ listed below against the reference's
src/ headers and the host Kokkos stand-in (`make -C oracle ref-validation`,
which needs the reference sources), runs each on the host cores and saves
its standard output under tests/golden/validation/<name>.txt.  The GPU tests
run the same programs built against the B200 drop-in headers
(`make -C oracle facade-drivers`) and compare the printed figures with
these files.

    python tests/golden/make_validation_golden.py [name ...]
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = HERE / "validation"
PROGRAMS = ["specular", "specular_node", "specwall_unsteady", "regularized", "cavity", "thermal",
            "natural_convection", "scalar_walls", "scalar_specular", "gaussian_plume", "scalar_mass"]


def main(names):
    subprocess.run(["make", "-C", str(ROOT / "oracle"), f"-j{os.cpu_count() or 4}", "ref-validation"],
                   check=True, stdout=subprocess.DEVNULL)
    OUT.mkdir(exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    for name in names or PROGRAMS:
        exe = ROOT / "oracle" / "_ref" / f"{name}_cpu"
        r = subprocess.run([str(exe)], capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise SystemExit(f"{name} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
        (OUT / f"{name}.txt").write_text(r.stdout)
        print(name, "ok")


if __name__ == "__main__":
    main(sys.argv[1:])
