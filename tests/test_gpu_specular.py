"""Free-slip walls on the GPU (SpecWall ghost mirror, SpecNode on-node mirror).

The CUDA path against the oracle (itself bit-identical to the reference
build with these walls, tests/test_oracle.py) on the geometries of
tests/golden/make_golden.py: a half channel closed by a ghost mirror, a box
whose x and z faces are on-node mirrors with two-face edges, and the two
mixed.  Tolerances as in test_gpu_parity.py: 64 eps s for 32/64-bit storage,
4 eps s for 16-bit storage, s the population scale.
"""
import ctypes as C
import itertools

import numpy as np
import pytest

from m3lb_b200 import capi
from m3lb_b200 import solver as S
from tests.golden import make_golden as G
from tests.helpers import EPS, Case, make_collision

pytestmark = pytest.mark.gpu

TOL_K = {"f64": 64.0, "f32": 64.0, "f16": 4.0, "bf16": 4.0, "f16c": 4.0}
OPS = [(0, 0, -1.0), (1, 0, -1.0), (1, 1, -1.0), (2, 0, 1.1), (3, 0, 1.5), (4, 0, -1.0)]


def _case(lat, op, eq, om2, storage, shifted, forcing, kind, shape=None):
    shape = shape or ((10, 9, 1) if lat == 9 else (8, 7, 6))
    c = Case(lat=lat, op=op, eq=eq, storage=storage, shifted=shifted, forcing=forcing,
             shape=shape, periodic=G.SPEC_PERIODIC[kind], omega2=om2)
    fl, codes, masks = G.spec_geometry(lat, shape, kind)
    c.geometry(fl)
    c.specular(codes, masks)
    return c


def _cases():
    out = []
    for (op, eq, om2), storage, shifted, forcing in itertools.product(
            OPS, ["f32", "f16", "bf16", "f64", "f16c"], [True, False], [False, True]):
        if storage in ("f16", "bf16", "f16c") and not shifted:
            continue
        if op == 0 and (forcing or not shifted):
            continue
        out.append((op, eq, om2, storage, shifted, forcing))
    return out


@pytest.mark.parametrize("kind", ["wall", "node", "mixed"])
@pytest.mark.parametrize("lat", [27, 9])
@pytest.mark.parametrize("op,eq,om2,storage,shifted,forcing", _cases())
def test_specular_matches_oracle(cuda_device, kind, lat, op, eq, om2, storage, shifted, forcing):
    c = _case(lat, op, eq, om2, storage, shifted, forcing, kind)
    c.init_random(seed=3 + op)
    o0 = c.cpu.gather()
    scale = float(np.max(np.abs(o0)))
    tol = TOL_K[storage] * EPS[storage] * max(scale, 1e-30)
    assert np.max(np.abs(c.gpu.gather_populations() - o0)) <= tol
    c.step(7, store=True)
    g, o = c.gpu.gather_populations(), c.cpu.gather()
    err = float(np.max(np.abs(g - o)))
    assert err <= tol, f"populations differ by {err:.3e}"
    ar = EPS["f64"] if storage == "f64" else EPS["f32"]
    for a, b in list(zip(c.gpu.stored_macroscopic(), c.cpu.stored_macro())) + \
            list(zip(c.gpu.compute_macroscopic(), c.cpu.macro())):
        sc = max(float(np.max(np.abs(b))), 1e-3)
        assert float(np.max(np.abs(a - b))) <= lat * tol / 0.9 + 64 * ar * sc
    red = c.gpu.reduce()
    m = c.cpu.total_mass()
    assert abs(red[0] - m) <= c.gpu.dom.n_interior() * (lat * tol + 64 * ar) + 1e-12 * abs(m)
    c.close()


@pytest.mark.parametrize("name", list(G.SPEC_CASES))
def test_specular_golden_on_device(cuda_device, name):
    """The reference build's own fixtures, through the CUDA path."""
    d = np.load(G.HERE / f"{name}.npz")
    lat, op, eq, sh, fo, shape, kind, om, om2, steps, prec = G.SPEC_CASES[name]
    opc = {"none": 0, "bgk": 1, "trt": 2, "mrt": 3, "cm": 4}[op]
    nx, ny, nz = shape
    F = (2e-5, -1e-5, 3e-6 if lat == 27 else 0.0)
    coll = make_collision(lat, opc, eq, bool(sh), bool(fo), om, om2, F)
    s = S.FluidSolver(S.Domain(nx, ny, nz, *G.SPEC_PERIODIC[kind]), coll, storage=prec)
    fl, codes, masks = G.spec_geometry(lat, shape, kind)
    s.set_geometry(fl)
    if codes.any():
        s.set_specular_walls(codes)
    if masks.any():
        s.set_specular_nodes(masks)
    s.initialize_field(tuple(G.initial_field(shape, int(d["seed"]))))
    scale = float(np.max(np.abs(d["pops0"])))
    tol = TOL_K[prec] * EPS[prec] * scale
    assert np.max(np.abs(s.gather_populations() - d["pops0"])) <= tol
    s.steps(steps, True)
    assert np.max(np.abs(s.gather_populations() - d["pops"])) <= tol
    # the reference sums the mass in its arithmetic type; the device in FP64
    ar = EPS["f64"] if prec == "f64" else EPS["f32"]
    mass = float(d["mass"])
    assert abs(s.total_mass() - mass) <= nx * ny * nz * (lat * tol + ar * abs(mass))
    s.close()


def test_setters_reject_what_the_reference_rejects(cuda_device):
    coll = S.BGK(lattice=S.D3Q27, storage=S.ShiftedPopulations, omega=1.2)
    s = S.FluidSolver(S.Domain(4, 4, 4, False, False, False), coll, storage="f32")
    s.initialize(1.0, 0.02)
    codes = np.zeros((4, 4, 4), np.uint8)
    codes[1, 2, 3] = 7
    with pytest.raises(capi.M3lbError, match="not an axis normal"):
        s.set_specular_walls(codes)
    for bad, msg in ((0x40, "outside"), (0x03, "both faces"), (0x30, "both faces")):
        m = np.zeros((4, 4, 4), np.uint8)
        m[2, 1, 0] = bad
        with pytest.raises(capi.M3lbError, match=msg):
            s.set_specular_nodes(m)
    assert not np.any(s.flags())
    lib = capi.lib()
    assert lib.m3lb_set_specular_walls(s.handle, None) == capi.ERR_INVALID
    # set_flags resets the specular marks: the run equals an unmarked one
    m = np.zeros((4, 4, 4), np.uint8)
    m[:, :, 0] = S.SpecFace.SpecXm
    s.set_specular_nodes(m)
    s.set_geometry(np.zeros((4, 4, 4), np.uint8))
    s.initialize(1.0, 0.02)
    s.steps(3)
    t = S.FluidSolver(S.Domain(4, 4, 4, False, False, False), coll, storage="f32")
    t.initialize(1.0, 0.02)
    t.steps(3)
    np.testing.assert_array_equal(s.gather_populations(), t.gather_populations())
    s.close()
    t.close()


def test_specular_same_under_every_bulk_kernel(cuda_device):
    """Wall nodes are updated by the boundary pass, whatever bulk kernel runs
    the fluid: the one-node, paired and row kernels give one result."""
    res = []
    for kernel in (capi.KERNEL_NODES, capi.KERNEL_ROWS, capi.KERNEL_PAIRS):
        c = _case(27, 4, 0, -1.0, "f16", True, False, "mixed", shape=(64, 6, 4))
        c.gpu.set_option(capi.OPT_KERNEL, kernel)
        c.init_random(seed=1)
        c.gpu.steps(5)
        res.append(c.gpu.gather_populations())
        c.close()
    np.testing.assert_array_equal(res[0], res[1])
    np.testing.assert_array_equal(res[0], res[2])


def test_ghost_mirror_half_channel_conserves_mass(cuda_device):
    """Half channel (solid floor, SpecWall lid, Guo force) in FP64: the ghost
    mirror permutes populations, so the mass stays at round-off
    (validation/specular.cpp:33-38, 141)."""
    coll = S.BGK(lattice=S.D3Q27, forcing=S.Guo(1e-5, 0.0, 0.0),
                 storage=S.ShiftedPopulations, omega=1.25)
    s = S.FluidSolver(S.Domain(6, 10, 6, True, False, True), coll, storage="f64")
    fl, codes, _ = G.spec_geometry(27, (6, 10, 6), "wall")
    s.set_geometry(fl)
    s.set_specular_walls(codes)
    s.initialize(1.0)
    m0 = s.total_mass()
    s.steps(500)
    assert abs(s.total_mass() - m0) / m0 < 1e-13
    s.close()
