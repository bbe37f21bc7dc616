"""Regularised walls on the GPU (RegWall: velocity walls, corners, outlets).

The CUDA path against the oracle, which is bit-identical to the reference
build run on one thread with these walls (tests/test_oracle.py), on the
geometries of tests/golden/make_golden.py: Couette, a lid-driven box with
corners, inlet + pressure outlet, inlet + equilibrium outlet, free outflow on
both faces, and corners whose finite-difference stencil reads fluid nodes
before and after their own update.  Tolerances as in test_gpu_parity.py.
"""
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
KINDS = list(G.WALL_PERIODIC)


def _case(lat, op, eq, om2, storage, shifted, forcing, kind, shape=None, kernel=None):
    shape = shape or ((10, 9, 1) if lat == 9 else (8, 7, 5))
    c = Case(lat=lat, op=op, eq=eq, storage=storage, shifted=shifted, forcing=forcing,
             shape=shape, periodic=G.WALL_PERIODIC[kind], omega2=om2)
    if kernel is not None:
        c.gpu.set_option(capi.OPT_KERNEL, kernel)
    fl, codes, st = G.wall_geometry(lat, shape, kind)
    c.geometry(fl)
    c.regularized(codes, st)
    return c


# A wall rebuilds its populations unshifted, so its rounding is on the scale
# of the raw populations (up to the largest weight, 4/9), whatever the storage.
RAW = 4.0 / 9.0


def _check(c, lat, storage, steps=7):
    c.init_random(seed=5)
    o0 = c.cpu.gather()
    tol = TOL_K[storage] * EPS[storage] * (float(np.max(np.abs(o0))) + RAW)
    assert np.max(np.abs(c.gpu.gather_populations() - o0)) <= tol
    c.step(steps, store=True)
    g, o = c.gpu.gather_populations(), c.cpu.gather()
    tol = TOL_K[storage] * EPS[storage] * (max(float(np.max(np.abs(o0))), float(np.max(np.abs(o)))) + RAW)
    err = float(np.max(np.abs(g - o)))
    assert err <= tol, f"populations differ by {err:.3e}"
    ar = EPS["f64"] if storage == "f64" else EPS["f32"]
    for a, b in list(zip(c.gpu.stored_macroscopic(), c.cpu.stored_macro())) + \
            list(zip(c.gpu.compute_macroscopic(), c.cpu.macro())):
        sc = max(float(np.max(np.abs(b))), 1e-3)
        assert float(np.max(np.abs(a - b))) <= lat * tol / 0.9 + 64 * ar * sc
    m = c.cpu.total_mass()
    assert abs(c.gpu.reduce()[0] - m) <= c.gpu.dom.n_interior() * (lat * tol + 64 * ar) + 1e-12 * abs(m)


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


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("lat", [27, 9])
@pytest.mark.parametrize("op,eq,om2,storage,shifted,forcing", _cases())
def test_regularized_matches_oracle(cuda_device, kind, lat, op, eq, om2, storage, shifted, forcing):
    if op == 0 and kind in ("inout", "outeq", "outfree"):
        pytest.skip("pure streaming has no density at the outlets (0/0 in the reference too)")
    c = _case(lat, op, eq, om2, storage, shifted, forcing, kind)
    _check(c, lat, storage)
    c.close()


@pytest.mark.parametrize("kernel", [capi.KERNEL_NODES, capi.KERNEL_PAIRS, capi.KERNEL_STREAM,
                                    capi.KERNEL_ROWS])
@pytest.mark.parametrize("kind", ["couette", "fdcorner"])
def test_regularized_under_every_bulk_kernel(cuda_device, kernel, kind):
    """64-wide periodic rows, so every bulk kernel runs the fluid."""
    c = _case(27, 4, 0, -1.0, "f16", True, True, kind, shape=(64, 6, 4), kernel=kernel)
    _check(c, 27, "f16", steps=5)
    c.close()


MODIFIERS = [
    ("scale", [("set_wall_velocity_scale", 0.5)]),
    ("density", [("set_wall_density", 1.02)]),
    ("field", [("set_wall_velocity_field", "field"), ("set_wall_velocity_field_scale", 0.7)]),
    ("no_fd", [("set_fd_corners", False)]),
    ("no_force_bc", [("set_force_correction", False)]),
    ("order2", [("set_outflow_order", 2)]),
    ("outflow_rho", [("set_outflow_density", 0.98)]),
]


@pytest.mark.parametrize("name,mods", MODIFIERS, ids=[m[0] for m in MODIFIERS])
@pytest.mark.parametrize("kind", ["cavity", "inout", "outfree", "fdcorner"])
def test_wall_setters_match_oracle(cuda_device, name, mods, kind):
    c = _case(27, 1, 0, -1.0, "f64", True, True, kind)
    for fn, arg in mods:
        if arg == "field":
            rng = np.random.default_rng(2)
            arg = 0.01 * rng.standard_normal(c.shape + (3,))
        c.both(fn, arg)
    _check(c, 27, "f64", steps=6)
    c.close()


@pytest.mark.parametrize("name", list(G.WALL_CASES))
def test_regularized_golden_on_device(cuda_device, name):
    """The reference build's own fixtures, through the CUDA path."""
    d = np.load(G.HERE / f"{name}.npz")
    lat, op, eq, sh, fo, shape, kind, om, om2, steps, prec = G.WALL_CASES[name]
    opc = {"none": 0, "bgk": 1, "trt": 2, "mrt": 3, "cm": 4}[op]
    nx, ny, nz = shape
    F = (2e-5, -1e-5, 3e-6 if lat == 27 else 0.0)
    coll = make_collision(lat, opc, eq, bool(sh), bool(fo), om, om2, F)
    s = S.FluidSolver(S.Domain(nx, ny, nz, *G.WALL_PERIODIC[kind]), coll, storage=prec)
    fl, codes, st = G.wall_geometry(lat, shape, kind)
    s.set_geometry(fl)
    s.set_regularized_walls(codes, st)
    s.initialize_field(tuple(G.initial_field(shape, int(d["seed"]))))
    scale = max(float(np.max(np.abs(d["pops0"]))), float(np.max(np.abs(d["pops"])))) + RAW
    tol = TOL_K[prec] * EPS[prec] * scale
    assert np.max(np.abs(s.gather_populations() - d["pops0"])) <= tol
    s.steps(steps, True)
    assert np.max(np.abs(s.gather_populations() - d["pops"])) <= tol
    ar = EPS["f64"] if prec == "f64" else EPS["f32"]
    mass = float(d["mass"])
    assert abs(s.total_mass() - mass) <= nx * ny * nz * (lat * tol + ar * abs(mass))
    s.close()


def test_wall_setters_reject_what_cannot_run(cuda_device):
    coll = S.BGK(lattice=S.D2Q9, storage=S.ShiftedPopulations, omega=1.2)
    s = S.FluidSolver(S.Domain(8, 6, 1, False, False, True), coll, storage="f32")
    codes = np.zeros((1, 6, 8), np.uint8)
    codes[0, 2, 3] = 11
    with pytest.raises(capi.M3lbError, match="not one of 0..10"):
        s.set_regularized_walls(codes)
    codes[0, 2, 3] = 0
    codes[0, 2, 0] = S.WallCode.NrmOutXp            # no upstream node at x = 0
    with pytest.raises(capi.M3lbError, match="no upstream node"):
        s.set_regularized_walls(codes)
    codes[0, 2, 0] = 0
    codes[0, 2, 1] = S.WallCode.NrmOutXp
    s.set_regularized_walls(codes)
    with pytest.raises(capi.M3lbError, match="second upstream"):
        s.set_outflow_order(2)
    assert capi.lib().m3lb_set_regularized_walls(s.handle, None, None) == capi.ERR_INVALID
    s.close()


def test_couette_profile_is_linear(cuda_device):
    """Couette flow between a resting and a moving regularised wall is exact
    (Regularized.hpp: linear profiles carry no curvature slip): the steady
    profile is linear between the wall nodes to round-off."""
    ny, U = 12, 0.04
    coll = S.BGK(lattice=S.D2Q9, storage=S.ShiftedPopulations, omega=1.1)
    s = S.FluidSolver(S.Domain(4, ny, 1, True, False, True), coll, storage="f64")
    s.set_regularized_walls(lambda x, y, z: S.WallSpec(4) if y == 0 else
                            (S.WallSpec(3, U) if y == ny - 1 else S.WallSpec(0)))
    s.initialize(1.0)
    s.steps(30000)
    ux = s.compute_macroscopic()[1][0, :, 0]
    np.testing.assert_allclose(ux, U * np.arange(ny) / (ny - 1), rtol=0, atol=1e-10)
    s.close()
