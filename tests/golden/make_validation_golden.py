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
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
OUT = HERE / "validation"
PROGRAMS = ["specular", "specular_node", "specwall_unsteady", "regularized", "cavity", "thermal",
            "natural_convection", "scalar_walls", "scalar_specular", "gaussian_plume", "scalar_mass",
            "poiseuille", "galilean", "decaying_flows", "tgv3d_bench_f32_128"]
# Programs run with arguments: fixture name -> (executable, arguments).  The
# 3-D Taylor-Green benchmark at the 128^3 workload: FP32 populations, u0 0.05,
# Re 1600 on L = N / (2 pi), 1000 time steps (t* = 1000 u0 / L; the half step
# added to tmax only keeps the program's floor(tmax L / u0) at exactly 1000).
TGV128_TMAX = 1000.5 * 0.05 / (128 / (2 * 3.141592653589793))
ARGS = {"tgv3d_bench_f32_128": ("tgv3d_bench_f32", ["-d", "128", "-re", "1600", "-u0", "0.05",
                                                    "-tmax", f"{TGV128_TMAX:.9f}"])}


# Results files (validation/Campaign.hpp:133-139 open_out) of reference runs,
# made in a scratch folder whose results/<dir>/ exists and copied to
# tests/golden/dat/: fixture name -> (executable, arguments, results file).
DAT_RUNS = {"tgvb_re1600_d3q27_cm_d32": (
    "tgv3d_bench", ["-d", "32", "-re", "1600", "-u0", "0.05", "-tmax", "1.0"],
    "results/E_tgv3d_bench/tgvb_re1600_d3q27_cm.dat")}


def make_dat(name):
    prog, args, rel = DAT_RUNS[name]
    exe = ROOT / "oracle" / "_ref" / f"{prog}_cpu"
    with tempfile.TemporaryDirectory() as td:
        (Path(td) / rel).parent.mkdir(parents=True)
        r = subprocess.run([str(exe), *args], capture_output=True, text=True, cwd=td,
                           env=dict(os.environ, OMP_NUM_THREADS="4"))
        if r.returncode != 0:
            raise SystemExit(f"{name} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
        (HERE / "dat").mkdir(exist_ok=True)
        (HERE / "dat" / f"{name}.dat").write_bytes((Path(td) / rel).read_bytes())
    print(name, "ok")


def main(names):
    subprocess.run(["make", "-C", str(ROOT / "oracle"), f"-j{os.cpu_count() or 4}", "ref-validation"],
                   check=True, stdout=subprocess.DEVNULL)
    OUT.mkdir(exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS="4")
    for name in names or (PROGRAMS + list(DAT_RUNS)):
        if name in DAT_RUNS:
            make_dat(name)
            continue
        prog, args = ARGS.get(name, (name, []))
        exe = ROOT / "oracle" / "_ref" / f"{prog}_cpu"
        r = subprocess.run([str(exe), *args], capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise SystemExit(f"{name} failed ({r.returncode}):\n{r.stdout}\n{r.stderr}")
        (OUT / f"{name}.txt").write_text(r.stdout)
        print(name, "ok")


if __name__ == "__main__":
    main(sys.argv[1:])
