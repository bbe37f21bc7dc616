"""The scalar lattice and the thermal coupling on the GPU.

D2Q5 / D3Q7 with ScalarBGK / ScalarTRT / ScalarRegularised, every cell type,
per-node rates, sources and a storage reference T_ref, against the oracle
(bit-identical to the reference's ScalarSolver, tests/test_oracle.py); the
fluid's per-node Boussinesq force against the oracle; the two-way coupled
convection fixtures made by the reference.  Tolerances: 64 eps s for the
populations (s their scale) in the storage type, as in test_gpu_parity.py.
"""
import itertools

import numpy as np
import pytest
import torch

from m3lb_b200 import capi
from m3lb_b200 import solver as S
import oracle as O
from tests.golden import make_golden as G
from tests.helpers import EPS, Case

pytestmark = pytest.mark.gpu

SCOLL = {"bgk": S.ScalarBGK, "trt": S.ScalarTRT, "regularised": S.ScalarRegularised}


def _scalar_pair(lat, op, shape, kind, om, prec, T_ref):
    nx, ny, nz = shape
    per = G.SCALAR_PERIODIC[kind]
    L = {5: S.D2Q5, 7: S.D3Q7, 9: S.D2Q9, 27: S.D3Q27}[lat]
    gpu = S.ScalarSolver(S.Domain(nx, ny, nz, *per), SCOLL[op](L, omega=om, T_ref=T_ref), storage=prec)
    cpu = O.ScalarCpuSolver("oracle", lattice=lat, op=op, nx=nx, ny=ny, nz=nz, px=per[0], py=per[1],
                            pz=per[2], omega=om, T_ref=T_ref, precision=prec)
    return gpu, cpu


def _run_both(case, seed, T_ref=0.0, omega_field=False, source=False):
    """run_scalar (tests/golden/make_golden.py) on the device and the oracle."""
    lat, op, shape, kind, om, steps, prec = case
    nx, ny, nz = shape
    gpu, cpu = _scalar_pair(lat, op, shape, kind, om, prec, T_ref)
    cells, tw, codes, masks = G.scalar_geometry(lat, shape, kind)
    for s in (gpu, cpu):
        s.set_geometry(cells)
        s.set_wall_values(tw)
        if codes.any():
            s.set_specular_walls(codes)
        if masks.any():
            s.set_specular_nodes(masks)
        s.finalize_geometry()
    rng, u = G.scalar_fields(shape, lat, seed)
    gpu.set_velocity(*u)
    cpu.set_velocity(*u)
    if omega_field:
        om_f = np.asarray(om + 0.3 * rng.random((nz, ny, nx)), np.float32).astype(np.float64)
        gpu.set_omega_field(om_f)
        cpu.set_omega_field(om_f)
    T = np.asarray(0.5 + 0.2 * rng.standard_normal(cpu.n_padded), np.float32).astype(np.float64)
    gpu.initialize_field(T)
    cpu.initialize_field(T)
    f0 = (gpu.temperature(), cpu.field())
    dC = np.asarray(1e-3 * rng.standard_normal((nz, ny, nx)), np.float32).astype(np.float64)
    for t in range(steps):
        if source and t % 3 == 0:
            gpu.add_source(dC)
            cpu.add_source(dC)
        gpu.step()
        cpu.step()
    out = {"field0": f0, "pops": (gpu.gather_populations(), cpu.gather()),
           "stored": (gpu.temperature(), cpu.field())}
    gpu.compute_field()
    cpu.compute_field()
    out["field"] = (gpu.temperature(), cpu.field())
    out["total"] = (gpu.total_population(), cpu.total())
    gpu.close()
    cpu.close()
    return out


def _check(out, prec, nodes):
    g, o = out["pops"]
    scale = max(float(np.max(np.abs(o))), 1e-3)
    tol = 64 * EPS[prec] * scale
    assert float(np.max(np.abs(g - o))) <= tol, "populations"
    ftol = 64 * EPS[prec] * max(float(np.max(np.abs(out["field"][1]))), 1.0) * 8
    for k in ("field0", "stored", "field"):
        a, b = out[k]
        assert float(np.max(np.abs(a - b))) <= ftol, k
    a, b = out["total"]
    assert abs(a - b) <= nodes * 8 * (tol + EPS[prec] * abs(b) / nodes)


@pytest.mark.parametrize("kind", list(G.SCALAR_PERIODIC))
@pytest.mark.parametrize("lat,op", [(5, "bgk"), (5, "trt"), (5, "regularised"), (7, "bgk"),
                                    (7, "trt"), (7, "regularised"), (9, "bgk"), (27, "bgk")])
@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("extras", [(0.0, False, False), (0.5, True, True)])
def test_scalar_matches_oracle(cuda_device, kind, lat, op, prec, extras):
    T_ref, omf, src = extras
    shape = (10, 9, 1) if lat in (5, 9) else (8, 7, 5)
    out = _run_both((lat, op, shape, kind, 1.2, 9, prec), 3, T_ref=T_ref, omega_field=omf, source=src)
    _check(out, prec, int(np.prod(shape)) * lat)


def test_scalar_wide_lattice(cuda_device):
    """A lattice wider than one chunk row (x-chunk boundaries, 3-D walls)."""
    out = _run_both((7, "trt", (150, 6, 5), "walls", 1.1, 12, "f32"), 9, T_ref=0.25, source=True)
    _check(out, "f32", 150 * 6 * 5 * 7)


@pytest.mark.parametrize("name", list(G.SCALAR_CASES))
def test_scalar_golden_on_device(cuda_device, name):
    """The reference ScalarSolver's fixtures through the CUDA path."""
    d = np.load(G.HERE / f"{name}.npz")
    k = list(G.SCALAR_CASES).index(name)
    lat, op, shape, kind, om, steps, prec = G.SCALAR_CASES[name]
    out = _run_both(G.SCALAR_CASES[name], int(d["seed"]), T_ref=0.25, omega_field=k % 2 == 1,
                    source=True)
    tol = 64 * EPS[prec] * 8 * max(float(np.max(np.abs(d["field"]))), 1.0)
    for key in ("field0", "stored", "field"):
        assert float(np.max(np.abs(out[key][0] - d[key]))) <= tol, key


def test_scalar_rejects(cuda_device):
    coll = S.ScalarBGK(S.D3Q7, omega=1.0)
    s = S.ScalarSolver(S.Domain(6, 5, 4), coll, storage="f32")
    with pytest.raises(capi.M3lbError, match="not 0..6"):
        s.set_geometry(np.full((4, 5, 6), 7, np.uint8))
    with pytest.raises(capi.M3lbError, match="axis normal"):
        s.set_specular_walls(np.full((4, 5, 6), 7, np.uint8))
    with pytest.raises(capi.M3lbError, match="both faces"):
        s.set_specular_nodes(np.full((4, 5, 6), 3, np.uint8))
    h = torch.zeros(1)
    assert capi.lib().m3lb_scalar_create(5, 6, 5, 2, 1, 1, 1, 1, capi.STORE_F32, None) == capi.ERR_INVALID
    s.close()
    del h


# ------------------------------------------------------------- buoyancy
@pytest.mark.parametrize("lat", [9, 27])
@pytest.mark.parametrize("op,eq,om2", [(1, 0, -1.0), (1, 1, -1.0), (2, 0, 1.1), (3, 0, 1.5),
                                       (4, 0, -1.0)])
@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("kernel", [capi.KERNEL_AUTO, capi.KERNEL_NODES])
def test_buoyancy_matches_oracle(cuda_device, lat, op, eq, om2, storage, kernel):
    shape = (16, 7, 5) if lat == 27 else (18, 9, 1)
    c = Case(lat=lat, op=op, eq=eq, storage=storage, shifted=True, forcing=True, shape=shape,
             periodic=(True, False, True), omega2=om2, F=(1e-5, 0.0, 2e-6))
    c.gpu.set_option(capi.OPT_KERNEL, kernel)
    fl = np.zeros(c.shape, np.uint8)
    fl[:, 0, :] = 1
    fl[:, -1, :] = 1
    c.geometry(fl)
    c.init_random(seed=op)
    rng = np.random.default_rng(6)
    dt = torch.float64 if storage == "f64" else torch.float32
    g3 = (0.0, 1.0, 0.5 if lat == 27 else 0.0)
    o0 = c.cpu.gather()
    for _ in range(5):
        T = np.asarray(0.3 * rng.standard_normal(c.shape), np.float32).astype(np.float64)
        Td = torch.as_tensor(T, dtype=dt, device="cuda")
        torch.cuda.synchronize()
        c.gpu.set_buoyancy(Td, g=g3, rho0=1.0, beta=2e-4, T0=0.1)
        c.cpu.set_buoyancy(T, g=g3, rho0=1.0, beta=2e-4, T0=0.1)
        c.step(1, store=True)
        torch.cuda.synchronize()
    scale = float(np.max(np.abs(o0)))
    tol = (64.0 if storage != "f16" else 4.0) * EPS[storage] * scale
    assert float(np.max(np.abs(c.gpu.gather_populations() - c.cpu.gather()))) <= tol
    ar = EPS["f64"] if storage == "f64" else EPS["f32"]
    for a, b in zip(c.gpu.stored_macroscopic(), c.cpu.stored_macro()):
        sc = max(float(np.max(np.abs(b))), 1e-3)
        assert float(np.max(np.abs(a - b))) <= lat * tol / 0.9 + 64 * ar * sc
    c.gpu.set_buoyancy(None)
    c.close()


@pytest.mark.parametrize("kernel", [capi.KERNEL_NODES, capi.KERNEL_STREAM, capi.KERNEL_ROWS])
def test_buoyancy_same_under_every_bulk_kernel(cuda_device, kernel):
    """64-wide periodic rows with walls: the row and streamed kernels apply the
    per-node force as the paired kernel does, bit for bit; the one-node
    kernel's moment operator agrees to a few ulp (test_gpu_parity.py)."""
    out = []
    for k in (capi.KERNEL_PAIRS, kernel):
        coll = S.CentralMoments(S.D3Q27, S.Guo(1e-5, 0.0, 0.0), S.ShiftedPopulations, omega=1.6)
        s = S.FluidSolver(S.Domain(64, 6, 4, True, False, True), coll, storage="f16")
        s.set_option(capi.OPT_KERNEL, k)
        fl = np.zeros((4, 6, 64), np.uint8)
        fl[:, 0, :] = 1
        s.set_geometry(fl)
        s.initialize(1.0, 0.01, 0.0, 0.0)
        rng = np.random.default_rng(2)
        T = torch.as_tensor(rng.standard_normal((4, 6, 64)), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        s.set_buoyancy(T, g=(0.0, 1.0, 0.3), beta=1e-3)
        s.steps(6, True)
        out.append((s.gather_populations(), s.stored_macroscopic()))
        s.close()
    if kernel == capi.KERNEL_NODES:
        scale = float(np.max(np.abs(out[0][0])))
        assert float(np.max(np.abs(out[0][0] - out[1][0]))) <= 8 * EPS["f16"] * scale
        return
    np.testing.assert_array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        np.testing.assert_array_equal(a, b)


def test_buoyancy_needs_forcing(cuda_device):
    coll = S.BGK(lattice=S.D3Q27, storage=S.ShiftedPopulations, omega=1.2)
    s = S.FluidSolver(S.Domain(8, 6, 4), coll, storage="f32")
    T = torch.zeros((4, 6, 8), device="cuda")
    with pytest.raises(capi.M3lbError, match="without forcing"):
        s.set_buoyancy(T)
    s.close()


# ------------------------------------------------------ two-way coupling
@pytest.mark.parametrize("name", list(G.COUPLED_CASES))
def test_coupled_convection_golden_on_device(cuda_device, name):
    """The reference's two-way coupled loop (fluid.step(true); scalar.step())
    through m3lb_couple_thermal: fluid populations, fields and temperature
    against the fixtures of the reference's FluidSolver<..., BoussinesqGuo>
    and ScalarSolver."""
    d = np.load(G.HERE / f"{name}.npz")
    flat, fop, slat, sop, shape, steps, prec = G.COUPLED_CASES[name]
    nx, ny, nz = shape
    opc = {"bgk": 1, "trt": 2, "mrt": 3, "cm": 4}[fop]
    from tests.helpers import make_collision
    coll = make_collision(flat, opc, 0, True, True, 1.4, (1.1 if fop == "trt" else -1.0), (0.0, 0.0, 0.0))
    fl = S.FluidSolver(S.Domain(nx, ny, nz, True, False, True), coll, storage=prec)
    L = S.D2Q5 if slat == 5 else S.D3Q7
    th = S.ScalarSolver(S.Domain(nx, ny, nz, True, False, True), SCOLL[sop](L, omega=1.2), storage=prec)
    flags = np.zeros((nz, ny, nx), np.uint8)
    flags[:, 0, :] = 1
    flags[:, -1, :] = 1
    fl.set_geometry(flags)
    cells = np.zeros((nz, ny, nx), np.uint8)
    tw = np.zeros((nz, ny, nx))
    cells[:, 0, :] = 2
    tw[:, 0, :] = 1.0
    cells[:, -1, :] = 2
    th.set_geometry(cells)
    th.set_wall_values(tw)
    th.finalize_geometry()
    rng = np.random.default_rng(int(d["seed"]))
    T = np.asarray(0.5 + 0.05 * rng.standard_normal(th.dom.n_padded), np.float32).astype(np.float64)
    th.initialize_field(T)
    fl.initialize(1.0)
    S.couple_thermal(fl, th, g=(0.0, 1.0, 0.0), rho0=1.0, beta=5e-3, T0=0.5)
    for _ in range(steps):
        fl.step(True)
        th.step()
    pops = fl.gather_populations()
    scale = float(np.max(np.abs(d["pops"])))
    tol = 64 * EPS[prec] * scale * 4
    assert float(np.max(np.abs(pops - d["pops"]))) <= tol
    ar = EPS[prec]
    for a, b in zip(fl.stored_macroscopic(), d["stored"]):
        assert float(np.max(np.abs(a - b))) <= flat * tol + 64 * ar * max(float(np.max(np.abs(b))), 1e-3)
    assert float(np.max(np.abs(th.temperature() - d["T_stored"]))) <= 512 * ar
    th.compute_field()
    assert float(np.max(np.abs(th.temperature() - d["T"]))) <= 512 * ar
    # the flow is buoyancy-driven: the fluid moves
    assert float(np.max(np.abs(d["stored"][2]))) > 1e-5
    th.close()
    fl.close()


def test_couple_rejects_mismatch(cuda_device):
    coll = S.BGK(lattice=S.D3Q27, forcing=S.Guo(0.0, 0.0, 0.0), storage=S.ShiftedPopulations, omega=1.2)
    fl = S.FluidSolver(S.Domain(8, 6, 4), coll, storage="f32")
    th = S.ScalarSolver(S.Domain(8, 6, 5), S.ScalarBGK(S.D3Q7), storage="f32")
    with pytest.raises(capi.M3lbError, match="extent"):
        S.couple_thermal(fl, th)
    th2 = S.ScalarSolver(S.Domain(8, 6, 4), S.ScalarBGK(S.D3Q7), storage="f64")
    with pytest.raises(capi.M3lbError, match="FP32"):
        S.couple_thermal(fl, th2)
    th.close()
    th2.close()
    fl.close()


def test_scalar_diffusion_rate_on_device(cuda_device):
    """A sinusoid decays at D k^2, D = cs2 (1/omega - 1/2) (validation/thermal.cpp)."""
    for L, cs2 in ((S.D2Q5, 1 / 3), (S.D3Q7, 1 / 4)):
        N, om, steps = 64, 1.2, 400
        nz = 1 if L is S.D2Q5 else 4
        s = S.ScalarSolver(S.Domain(N, 4, nz), S.ScalarBGK(L, omega=om), storage="f64")
        x = np.arange(N)
        s.initialize_field(np.broadcast_to(0.01 * np.sin(2 * np.pi * x / N), (nz, 4, N)).ravel())
        s.steps(steps)
        s.compute_field()
        amp = s.temperature()[0, 0] @ np.sin(2 * np.pi * x / N) * 2 / N
        k = 2 * np.pi / N
        assert abs(amp / 0.01 / np.exp(-cs2 * (1 / om - 0.5) * k * k * steps) - 1) < 1e-3
        s.close()
