"""The C++ drop-in headers (m3lb_b200/facade).

Reference-style C++ call sites compile against the facade and run on the
device through libm3lb.so:
  * tests/cpp/facade_poiseuille.cpp (this repository's driver, written the way
    the reference's validation/poiseuille.cpp drives its solver) reproduces
    the Poiseuille known answers of README.md:178-276;
  * the reference's own src/app/main.cpp (lbm_app) and
    examples/flow_past_square.cpp, compiled unmodified against the facade by
    `make -C oracle facade-drivers`, run to completion.
"""
import os
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import REFERENCE_DIR

ROOT = Path(__file__).resolve().parent.parent
FACADE = ROOT / "m3lb_b200" / "facade"
LIBDIR = ROOT / "m3lb_b200"
REF_APP = ROOT / "oracle" / "_ref" / "lbm_app_b200"
REF_EXAMPLE = ROOT / "oracle" / "_ref" / "flow_past_square_b200"


def _compile(src: Path, out: Path):
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++20", "-O2", "-Wall", "-Werror", f"-I{FACADE}", f"-I{ROOT / 'include'}",
           str(src), "-o", str(out), f"-L{LIBDIR}", "-lm3lb", f"-Wl,-rpath,{LIBDIR}"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


def test_facade_driver_compiles(tmp_path):
    _compile(ROOT / "tests" / "cpp" / "facade_poiseuille.cpp", tmp_path / "fp")


@pytest.mark.skipif(not (REFERENCE_DIR / "src" / "app" / "main.cpp").exists(),
                    reason="reference sources not present")
@pytest.mark.parametrize("src", ["src/app/main.cpp", "examples/flow_past_square.cpp"])
def test_reference_drivers_compile_unmodified(tmp_path, src):
    cxx = shutil.which("g++") or "g++"
    r = subprocess.run([cxx, "-std=c++20", "-O2", "-fsyntax-only", f"-I{FACADE}",
                        f"-I{ROOT / 'include'}", str(REFERENCE_DIR / src)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


@pytest.fixture(scope="module")
def poiseuille_bin(tmp_path_factory):
    return _compile(ROOT / "tests" / "cpp" / "facade_poiseuille.cpp",
                    tmp_path_factory.mktemp("facade") / "facade_poiseuille")


def _run_poiseuille(binary, *args):
    r = subprocess.run([str(binary), *map(str, args)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    m = re.search(r"l2 (\S+) rho_mean (\S+) mass_drift (\S+) steps (\d+)", r.stdout)
    assert m, r.stdout
    return float(m.group(1)), float(m.group(2)), float(m.group(3)), int(m.group(4))


@pytest.mark.gpu
def test_facade_poiseuille_known_answer(cuda_device, poiseuille_bin):
    """D2Q9 BGK, H = 32, tau = 0.8, FP64 storage: L2 6.95e-4 (README.md:178-186)."""
    l2, rho, drift, steps = _run_poiseuille(poiseuille_bin, "bgk", 0.8, 60000)
    assert steps == 60000
    assert l2 == pytest.approx(6.95e-4, rel=0.01)
    assert abs(drift) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("op,tau", [("bgk", 0.5 + 3 ** 0.5 / 4), ("trt", 0.8), ("cm", 0.875),
                                    ("mrt", 0.875)])
def test_facade_poiseuille_magic_parameter(cuda_device, poiseuille_bin, op, tau):
    """At the magic parameter the wall sits exactly midway (README.md:240-276)."""
    l2, _, _, _ = _run_poiseuille(poiseuille_bin, op, tau, 60000)
    assert l2 < 1e-10


@pytest.mark.gpu
@pytest.mark.skipif(not REF_APP.exists(), reason="facade build of the reference lbm_app absent")
def test_reference_lbm_app_runs_on_device(cuda_device):
    """The reference's benchmark harness, unmodified: every operator and
    streaming/storage combination runs, and mass is conserved to its own
    tolerance (src/app/main.cpp:56-59)."""
    r = subprocess.run([str(REF_APP), "-n", "64", "-steps", "20"], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "MASS NOT CONSERVED" not in r.stdout
    rows = [ln for ln in r.stdout.splitlines() if ln.startswith("D3Q27")]
    assert len(rows) == 7


@pytest.mark.gpu
@pytest.mark.skipif(not REF_EXAMPLE.exists(), reason="facade build of the reference example absent")
def test_reference_example_runs_on_device(cuda_device, tmp_path):
    out = tmp_path / "profile.csv"
    r = subprocess.run([str(REF_EXAMPLE), "-n", "48", "-steps", "2000", "-out", str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "DIVERGED" not in r.stdout
    assert out.exists() and len(out.read_text().splitlines()) == 49


# ------------------------------------------------------ wall validations
# The reference's validation/specular.cpp, specular_node.cpp,
# specwall_unsteady.cpp, regularized.cpp and cavity.cpp, built unmodified
# against the facade (`*_b200`, run on the device): each must pass its own
# checks there and print the figures the reference prints on the host
# (tests/golden/validation/<name>.txt, made by make_validation_golden.py).
REF_DIR = ROOT / "oracle" / "_ref"
VGOLD = ROOT / "tests" / "golden" / "validation"
_NUM = r"[-+]?\d+\.\d+(?:e[-+]\d+)?"


def _validation(name, *args):
    exe = REF_DIR / f"{name}_b200"
    if not exe.exists():
        pytest.skip(f"{name}_b200 not built (make -C oracle facade-drivers)")
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=1200)
    return r.returncode, r.stdout, (VGOLD / f"{name}.txt").read_text()


def _figures(text, key):
    return [[float(v) for v in re.findall(_NUM, ln)] for ln in text.splitlines() if key in ln]


def _same_figures(out, ref, key, rtol, atol=0.0):
    got, want = _figures(out, key), _figures(ref, key)
    assert len(got) == len(want) > 0, key
    for a, b in zip(got, want):
        np.testing.assert_allclose(a, b, rtol=rtol, atol=atol, err_msg=key)


@pytest.mark.gpu
def test_reference_specular_validation_on_device(cuda_device):
    """Half channel closed by the ghost mirror = lower half of the full
    channel to round-off, planes at 0.5 / H + 0.5, mass conserved
    (validation/specular.cpp:103-160), for D2Q9 at tau 0.8 and 1.2 and D3Q27."""
    rc, out, ref = _validation("specular")
    assert rc == 0 and out.rstrip().endswith("PASS"), out
    for key in ("no-slip plane", "symmetry plane"):
        _same_figures(out, ref, key, rtol=1e-9)
    _same_figures(out, ref, "u_max", rtol=1e-9, atol=1e-15)


@pytest.mark.gpu
def test_reference_specular_node_validation_on_device(cuda_device):
    """On-node mirror: half box = periodic box to 1e-12 in 2-D, quarter box
    with two-face edges in 3-D (validation/specular_node.cpp:284-368)."""
    rc, out, ref = _validation("specular_node")
    assert rc == 0 and out.rstrip().endswith("PASS"), out
    assert out.count(" ok") == 6
    # the control (halfway mirror on the same box) differs by the same amount
    _same_figures(out, ref, "CONTROL", rtol=1e-9)


@pytest.mark.gpu
def test_reference_specwall_unsteady_on_device(cuda_device):
    """The ghost mirror's first-order error for unsteady modes: the device
    prints the reference's figures (validation/specwall_unsteady.cpp:79-91)."""
    rc, out, ref = _validation("specwall_unsteady")
    assert rc == 0, out
    _same_figures(out, ref, "SpecWall half box", rtol=5e-3)


@pytest.mark.gpu
def test_reference_regularized_validation_on_device(cuda_device):
    """Regularised walls: Couette exact, the wall ON the node at every tau,
    second-order Poiseuille on D2Q9 and D3Q27 (validation/regularized.cpp),
    with the reference's error table to 1e-6."""
    rc, out, ref = _validation("regularized")
    assert rc == 0, out
    # W, L2 error, order, wall position, steps: identical convergence tables
    got = [ln.split() for ln in out.splitlines() if re.match(r"\s+(8|16|32)\s+\d\.\d+e", ln)]
    want = [ln.split() for ln in ref.splitlines() if re.match(r"\s+(8|16|32)\s+\d\.\d+e", ln)]
    assert len(got) == len(want) == 6
    for a, b in zip(got, want):
        assert a[0] == b[0]
        np.testing.assert_allclose(float(a[1]), float(b[1]), rtol=1e-6)
        # steps to steady state: the stopping test sits at round-off level
        assert abs(int(a[-1]) - int(b[-1])) <= 0.05 * int(b[-1])
    # the fitted wall planes: at 0 and W to round-off on both sides
    got_planes = [ln.split() for ln in out.splitlines() if re.match(r"\s+\d\.\d\d\s+(8|16)\s", ln)]
    assert len(got_planes) == 8
    for row in got_planes:
        assert abs(float(row[2])) < 1e-12 and abs(float(row[3]) - float(row[1])) < 1e-9


@pytest.mark.gpu
def test_reference_cavity_validation_on_device(cuda_device):
    """Lid-driven cavity at Re = 100 with regularised walls and
    finite-difference corners against Ghia et al.: the device's centreline
    profiles equal the reference's (validation/cavity.cpp)."""
    rc, out, ref = _validation("cavity")
    assert rc == 0 and "DIVERGED" not in out, out
    rows = lambda t: [ln.split() for ln in t.splitlines() if re.match(r"\s+0\.\d+\s+-?\d\.\d+\s+-?\d", ln)]
    got, want = rows(out), rows(ref)
    assert len(got) == len(want) > 10
    for a, b in zip(got, want):
        np.testing.assert_allclose([float(v) for v in a], [float(v) for v in b], atol=2e-5)


# Scalar and thermal validations: every number the device run prints equals
# the reference's to 1e-6 relative, or to 1e-11 absolute where the figure is
# a round-off residual.
def _all_figures(text):
    rows = [ln for ln in text.splitlines() if ln.strip() and "backend" not in ln]
    return [[float(v) for v in re.findall(r"[-+]?\d+\.?\d*(?:e[-+]?\d+)?", ln)] for ln in rows]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["thermal", "natural_convection", "scalar_walls", "scalar_specular",
                                  "scalar_mass", "gaussian_plume"])
def test_reference_scalar_validation_on_device(cuda_device, name):
    """validation/{thermal, natural_convection, scalar_walls, scalar_specular,
    scalar_mass, gaussian_plume}.cpp built against the facade: the D2Q5 / D3Q7
    scalar solver, its walls, sources and outflow, and the Boussinesq-coupled
    de Vahl Davis cavity (Nusselt numbers and step counts) as the reference
    prints them."""
    rc, out, ref = _validation(name)
    assert rc == 0, out
    assert "FAIL" not in out
    got, want = _all_figures(out), _all_figures(ref)
    assert len(got) == len(want)
    for a, b in zip(got, want):
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-11)


# Known answers of the north-star checks, as the reference's own programs
# print them: validation/poiseuille.cpp (wall slip vs tau, exactness at each
# operator's magic point, resolution behaviour), validation/galilean.cpp (the
# effective viscosity of the ABC flow under a superimposed uniform velocity)
# and validation/decaying_flows.cpp (Taylor-Green, ABC and shear-wave
# resolution ladders).  Built unmodified against the facade, run on the
# device with FP64 populations, they must pass their own acceptance checks
# and print the figures the reference prints on the host.
def _figure_rows(text, skip=("backend",)):
    rows = []
    for ln in text.splitlines():
        if not ln.strip() or any(s in ln for s in skip):
            continue
        vals = re.findall(r"[-+]?\d+\.\d+(?:e[-+]?\d+)?", ln)
        if vals:
            rows.append((ln, [float(v) for v in vals]))
    return rows


def _same_tables(out, ref, rtol, roundoff):
    """Every printed figure equals the reference's to rtol; figures the
    reference prints below `roundoff` (residuals at round-off level) only have
    to stay below it."""
    got, want = _figure_rows(out), _figure_rows(ref)
    assert len(got) == len(want) > 0
    for (lg, a), (lw, b) in zip(got, want):
        assert len(a) == len(b), (lg, lw)
        for x, y in zip(a, b):
            if abs(y) < roundoff:
                assert abs(x) < roundoff, (lg, lw)
            else:
                assert abs(x - y) <= rtol * abs(y) + 1e-12, (lg, lw)


@pytest.mark.gpu
def test_reference_poiseuille_validation_on_device(cuda_device):
    """D2Q9 Poiseuille with Guo forcing (validation/poiseuille.cpp): BGK at
    tau 0.8 slips by -4.06e-3, every operator is exact (L2 ~1e-13) at its
    magic tau, TRT at every tau, and the off-magic error is second order."""
    rc, out, ref = _validation("poiseuille")
    assert rc == 0 and "FAIL" not in out, out
    _same_tables(out, ref, rtol=2e-3, roundoff=1e-11)
    slip = [ln for ln in out.splitlines() if ln.startswith("0.8000000")]
    assert slip and slip[0].split()[1] == "-4.06e-03", slip


@pytest.mark.gpu
def test_reference_galilean_validation_on_device(cuda_device):
    """Galilean invariance (validation/galilean.cpp): the ABC-flow viscosity
    under U0 = 0 ... 0.15 drifts by 6.77e-2 with BGK, 5.87e-5 with raw MRT and
    4.70e-5 with central moments, the residual scaling as U0^2."""
    rc, out, ref = _validation("galilean")
    assert rc == 0 and out.count("PASS") == 4, out
    _same_tables(out, ref, rtol=1e-6, roundoff=0.0)
    # the viscosity table: operator, nu_eff at four U0 (nine decimals), drift
    drift = {ln.split()[0]: ln.split()[-1] for ln in out.splitlines()
             if re.match(r"\s+(BGK|MRT|CentralMoments|TRT)\S*(\s+\(raw\))?(\s+\d\.\d{9}){4}\s", ln)}
    assert drift["BGK"] == "6.77e-02" and drift["CentralMoments"] == "4.70e-05", drift
    assert drift["MRT"] == "5.87e-05", drift


@pytest.mark.gpu
def test_reference_decaying_flows_on_device(cuda_device):
    """Decaying flows with exact Navier-Stokes solutions
    (validation/decaying_flows.cpp): every fitted order of the viscosity and
    velocity error is 2.00 +- 0.11 for BGK, TRT, MRT and CM on the
    Taylor-Green (D2Q9), ABC (D3Q27) and diagonal shear-wave ladders, mass is
    conserved, and each figure equals the reference's."""
    rc, out, ref = _validation("decaying_flows")
    assert rc == 0 and "FAIL" not in out, out
    _same_tables(out, ref, rtol=1e-5, roundoff=1e-11)
    orders = [float(v) for ln in out.splitlines() if "order:" in ln
              for v in re.findall(r"(?:nu|L2) (\d\.\d\d)", ln)]
    assert len(orders) == 40
    assert all(abs(o - 2.0) <= 0.11 for o in orders), orders
