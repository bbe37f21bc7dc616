"""The benchmark's smaller workloads exactly as stated, with their errors.

* The D2Q9 BGK Poiseuille channel: 64 x 32 interior nodes, periodic in x,
  halfway bounce-back walls in y (the non-periodic y axis carries one halo
  row per side, so the 32 rows are all fluid and the no-slip planes sit half
  a node outside them: H = 32), tau = 0.8, Guo body force g_x = 1e-6,
  rho0 = 1, u = 0 initially, 20 000 steps, FP64 populations.  Checked
  against the analytic parabola and against the FP64 oracle (the reference's
  algorithm restated in C, bit-identical to the reference build).
* The D3Q27 central-moment Taylor-Green vortex at 128^3, FP32 shifted
  populations, u0 = 0.05, Re = 1600 on L = N / (2 pi)
  (tau = 0.5 + 3 u0 128 / (2 pi 1600) = 0.501910), 1000 steps: kinetic
  energy and enstrophy against the reference's own validation program run
  on the host (validation/tgv3d_bench.cpp, FP32, recorded in
  tests/golden/validation/tgv3d_bench_f32_128.txt), and the velocity and
  density errors of FP32 storage against FP64 storage of the same run.

Errors stated (measured on the B200) sit in the docstrings of the tests and
in the design notes; the asserted bounds leave a margin above them.
"""
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent


def _poiseuille_solver(storage):
    from m3lb_b200 import solver as S

    dom = S.Domain(64, 32, 1, True, False, True)
    coll = S.BGK(S.D2Q9, S.SecondOrderEquilibrium, S.Guo(1e-6, 0.0, 0.0),
                 S.ShiftedPopulations, omega=1.0 / 0.8)
    s = S.FluidSolver(dom, coll, storage=storage)
    s.initialize(1.0, 0.0, 0.0, 0.0)
    return s


def test_poiseuille_64x32_known_answer(cuda_device):
    """Config 1: after 20 000 steps the velocity profile is the parabola
    u(y) = g / (2 nu) (y + 1/2) (H - 1/2 - y) up to BGK's viscosity-dependent
    wall slip at tau = 0.8: relative L2 error 6.9e-4 (the reference's README
    gives 6.95e-4 for the same H and tau at a larger force; the relative error
    does not depend on the force to leading order), uniform in x, v = 0, and
    the device equals the FP64 oracle to round-off (velocity relative L2
    ~1e-13, density ~1e-15)."""
    import oracle as O

    s = _poiseuille_solver("f64")
    s.steps(20000)
    rho, ux, uy, _ = s.compute_macroscopic()
    s.close()
    nu = (0.8 - 0.5) / 3.0
    y = np.arange(32, dtype=np.float64)
    ua = 1e-6 / (2 * nu) * (y + 0.5) * (32 - 0.5 - y)
    prof = ux[0, :, :].mean(axis=1)
    assert np.max(np.abs(ux[0] - prof[:, None])) < 1e-15 * np.max(ua) * 1e3  # x-uniform
    assert np.max(np.abs(uy)) < 1e-12 * np.max(ua)
    l2 = float(np.sqrt(np.sum((prof - ua) ** 2) / np.sum(ua ** 2)))
    assert 6.0e-4 < l2 < 8.0e-4, l2

    cpu = O.CpuSolver("oracle", lattice=9, op="bgk", shifted=True, forcing=True, nx=64, ny=32,
                      nz=1, px=True, py=False, pz=True, omega=1.0 / 0.8, fx=1e-6,
                      precision="f64")
    cpu.initialize(1.0, 0.0, 0.0, 0.0)
    cpu.step(20000)
    rr, ru, rv, _ = cpu.macro()
    cpu.close()
    ru = ru.reshape(ux.shape)
    rr = rr.reshape(rho.shape)
    eu = float(np.sqrt(np.sum((ux - ru) ** 2) / np.sum(ru ** 2)))
    er = float(np.max(np.abs(rho - rr)))
    assert eu < 1e-11 and er < 1e-13, (eu, er)


def _tgv128_fields(n=128, u0=0.05):
    k = 2 * math.pi / n
    i = np.arange(n, dtype=np.float64) * k
    z, y, x = np.meshgrid(i, i, i, indexing="ij")
    dr = 3.0 * u0 * u0 / 16.0
    rho = 1 + dr * (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2)
    ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
    uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
    return rho, ux, uy, np.zeros_like(ux)


def test_tgv128_fp32_against_fp64_storage(cuda_device):
    """Config 2's precision statement: FP32-stored populations against FP64
    ones after 1000 steps of the 128^3 Taylor-Green vortex, from the same
    initial field.  Measured: velocity relative L2 ~2e-7, max |du| / u0 ~2e-6,
    (rho - 1) relative L2 ~2e-5, max |drho| ~5e-8."""
    from m3lb_b200 import solver as S

    n, u0 = 128, 0.05
    nu = u0 * (n / (2 * math.pi)) / 1600.0
    omega = 1.0 / (3 * nu + 0.5)
    fields = _tgv128_fields(n, u0)
    out = {}
    for st in ("f64", "f32"):
        dom = S.Domain(n, n, n, True, True, True)
        coll = S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=omega)
        s = S.FluidSolver(dom, coll, storage=st)
        s.initialize_field([np.asarray(a, np.float32).astype(np.float64) for a in fields])
        s.steps(1000)
        out[st] = s.compute_macroscopic()
        s.close()
    r64, *u64 = out["f64"]
    r32, *u32 = out["f32"]
    u64, u32 = np.stack(u64), np.stack(u32)
    eu = float(np.sqrt(np.sum((u32 - u64) ** 2) / np.sum(u64 ** 2)))
    emax = float(np.max(np.abs(u32 - u64)) / u0)
    er = float(np.sqrt(np.sum((r32 - r64) ** 2) / np.sum((r64 - 1) ** 2)))
    ermax = float(np.max(np.abs(r32 - r64)))
    assert eu < 5e-6 and emax < 5e-5, (eu, emax)
    assert er < 5e-4 and ermax < 1e-6, (er, ermax)


def _table(text):
    rows = []
    for ln in text.splitlines():
        m = re.match(r"\s+(\d+\.\d{3})\s+(\d+\.\d+)\s+(\S+)\s+(\d+\.\d+)\s+(\S+)\s*$", ln)
        if m:
            rows.append(tuple(float(v) for v in m.groups()[:4]))
    return rows


def test_tgv128_energy_and_enstrophy_match_reference_build(cuda_device):
    """Config 2: the reference's validation/tgv3d_bench.cpp, compiled
    unmodified against the drop-in headers with FP32 populations, runs the
    128^3 workload on the device (41 probes over 1000 steps) and prints the
    kinetic energy Ek* and the enstrophy dissipation eps_zeta the reference's
    host build prints, to 1e-5 relative (measured: Ek* identical to the six
    printed decimals); the energy dissipation eps_E, a backward difference of
    Ek*, to 1e-3 absolute."""
    import sys

    sys.path.insert(0, str(ROOT / "tests" / "golden"))
    from make_validation_golden import ARGS

    prog, args = ARGS["tgv3d_bench_f32_128"]
    exe = ROOT / "oracle" / "_ref" / f"{prog}_b200"
    if not exe.exists():
        pytest.skip(f"{exe.name} not built (make -C oracle facade-drivers)")
    r = subprocess.run([str(exe), *args], capture_output=True, text=True, timeout=900,
                       cwd=str(ROOT))
    assert r.returncode == 0, r.stdout + r.stderr
    got = _table(r.stdout)
    want = _table((ROOT / "tests" / "golden" / "validation" / "tgv3d_bench_f32_128.txt").read_text())
    assert len(got) == len(want) == 41
    for g, w in zip(got, want):
        assert g[0] == w[0]
        assert abs(g[1] - w[1]) <= 1e-5 * w[1] + 1e-6, (g, w)
        assert abs(g[3] - w[3]) <= 1e-5 * w[3] + 1e-6, (g, w)
        if not math.isnan(w[2]):
            assert abs(g[2] - w[2]) <= 1e-3, (g, w)


def test_tgv256_16bit_storage_accuracy(cuda_device):
    """Config 3 (the headline workload): the 256^3 Taylor-Green vortex after
    500 steps with 16-bit shifted populations, against FP64 populations from
    the same initial field.  FP16C (1 sign, 4 exponent, 11 mantissa bits)
    keeps the velocity error under the 1e-3 bound (measured ~6e-4); IEEE
    binary16 does not (~2.0e-3); FP32 storage is ~4e-7."""
    import torch
    from m3lb_b200 import solver as S

    n, u0, steps = 256, 0.05, 500
    nu = u0 * (n / (2 * math.pi)) / 1600.0
    omega = 1.0 / (3 * nu + 0.5)
    k = 2 * math.pi / n
    i = torch.arange(n, dtype=torch.float64, device=cuda_device) * k
    z, y, x = torch.meshgrid(i, i, i, indexing="ij")
    dr = 3.0 * u0 * u0 / 16.0
    f64 = [1 + dr * (torch.cos(2 * x) + torch.cos(2 * y)) * (torch.cos(2 * z) + 2),
           u0 * torch.sin(x) * torch.cos(y) * torch.cos(z),
           -u0 * torch.cos(x) * torch.sin(y) * torch.cos(z)]
    f64.append(torch.zeros_like(f64[0]))
    del x, y, z

    def run(storage):
        dom = S.Domain(n, n, n, True, True, True)
        coll = S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=omega)
        s = S.FluidSolver(dom, coll, storage=storage)
        dt = torch.float64 if storage == "f64" else torch.float32
        s.initialize_field_device(*[t.to(dt).contiguous() for t in f64])
        s.steps(steps)
        rho, ux, uy, uz = s.compute_macroscopic()
        s.close()
        return rho, np.stack([ux, uy, uz])

    r_ref, u_ref = run("f64")
    du = float(np.sqrt(np.sum(u_ref * u_ref)))
    err = {}
    for st in ("f16c", "f16", "f32"):
        _, u = run(st)
        err[st] = float(np.sqrt(np.sum((u - u_ref) ** 2)) / du)
        del u
    assert err["f32"] < 2e-6, err
    assert err["f16c"] < 1e-3, err
    assert err["f16c"] < 0.5 * err["f16"], err
