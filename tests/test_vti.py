"""VTK output (write_vti / write_vti_bin / write_pvd) against the files the
reference's own writer makes for the same inputs (tests/golden/vti/, made by
tests/golden/make_vti_golden.py from tests/cpp/vti_case.cpp): byte for byte,
from the Python writers and from the C++ drop-in headers."""
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from m3lb_b200 import vti

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden" / "vti"
FACADE = ROOT / "m3lb_b200" / "facade"
LIBDIR = ROOT / "m3lb_b200"


def _arrays():
    v = np.fromfile(GOLD / "arrays.bin", dtype="<f4")
    return [vti.VtiArray("rho", 1, v[:60]), vti.VtiArray("u", 3, v[60:240]),
            vti.VtiArray("chi", 1, v[240:])]


def test_python_binary_writer_matches_reference(tmp_path):
    vti.write_vti_bin(tmp_path / "bin.vti", 5, 4, 3, _arrays(), np.pi / 64)
    assert (tmp_path / "bin.vti").read_bytes() == (GOLD / "bin.vti").read_bytes()


def test_python_series_writer_matches_reference(tmp_path):
    vti.write_pvd(tmp_path / "series.pvd", [(0.0, "vti/f_0000.vti"), (0.1234567890123, "vti/f_0001.vti"),
                                            (2.5e-7, "f 2.vti")])
    assert (tmp_path / "series.pvd").read_bytes() == (GOLD / "series.pvd").read_bytes()


def test_python_binary_writer_rejects_wrong_sizes(tmp_path):
    with pytest.raises(ValueError, match="has 60 values, expected 40"):
        vti.write_vti_bin(tmp_path / "x.vti", 5, 4, 2, _arrays())


@pytest.fixture(scope="module")
def facade_case(tmp_path_factory):
    cxx = shutil.which("g++") or "g++"
    exe = tmp_path_factory.mktemp("vti") / "vti_case"
    cmd = [cxx, "-std=c++20", "-O1", "-Wall", "-Werror", f"-I{FACADE}", f"-I{ROOT / 'include'}",
           str(ROOT / "tests" / "cpp" / "vti_case.cpp"), "-o", str(exe), f"-L{LIBDIR}", "-lm3lb",
           f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return exe


def test_facade_writers_match_reference(facade_case, tmp_path):
    r = subprocess.run([str(facade_case), str(tmp_path), str(GOLD / "arrays.bin")],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "has 60 values, expected 40" in r.stdout
    for name in ("bin.vti", "series.pvd"):
        assert (tmp_path / name).read_bytes() == (GOLD / name).read_bytes(), name


@pytest.mark.gpu
def test_facade_solver_file_matches_reference(cuda_device, facade_case, tmp_path):
    r = subprocess.run([str(facade_case), str(tmp_path), str(GOLD / "arrays.bin"), "solver"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert (tmp_path / "rest.vti").read_bytes() == (GOLD / "rest.vti").read_bytes()


@pytest.mark.gpu
def test_python_solver_file_matches_reference(cuda_device, tmp_path):
    from m3lb_b200 import solver as S
    coll = S.BGK(lattice=S.D3Q27, storage=S.ShiftedPopulations, omega=1.25)
    s = S.FluidSolver(S.Domain(6, 5, 4, True, False, True), coll, storage="f64")
    fl = np.zeros((4, 5, 6), np.uint8)
    fl[:, 0, :] = 1
    s.set_geometry(fl)
    s.initialize(1.0)
    vti.write_vti(tmp_path / "rest.vti", s)
    s.close()
    assert (tmp_path / "rest.vti").read_bytes() == (GOLD / "rest.vti").read_bytes()
