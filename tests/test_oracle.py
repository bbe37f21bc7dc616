"""The CPU oracle, pinned to the reference (no GPU).

1. Golden fixtures made by the reference build (tests/golden/make_golden.py):
   the oracle must reproduce them bit for bit.
2. Where the reference build is present (oracle/_ref), the oracle against it,
   live, over every operator / storage / forcing / wall combination.
3. The reference's own known answers for this path:
   - the streaming permutation (tests/test_streaming.cpp:42-77, 129-137),
   - Esoteric Pull against two-lattice streaming (test_streaming.cpp:80-124),
   - plane Poiseuille, D2Q9 BGK tau = 0.8, H = 32: relative L2 6.95e-4 and the
     magic-parameter exactness of BGK / TRT / CM / MRT (README.md:173-276,
     validation/poiseuille.cpp:72-140).
"""
import itertools
import math
from pathlib import Path

import numpy as np
import pytest

import oracle as O
from tests.golden import make_golden as G

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.mark.parametrize("name", list(G.CASES))
def test_oracle_reproduces_golden(name):
    d = np.load(GOLDEN / f"{name}.npz")
    r = G.run("oracle", G.CASES[name], seed=int(d["seed"]))
    for k in ("pops0", "pops", "stored", "macro"):
        np.testing.assert_array_equal(r[k], d[k], err_msg=k)
    assert r["mass"] == float(d["mass"])
    np.testing.assert_array_equal(r["mom"], d["mom"])
    assert r["slots"] == float(d["slots"])


needs_ref = pytest.mark.skipif(not O.ref_available("f64") or not O.ref_available("f32"),
                               reason="reference build (oracle/_ref) not present")


@needs_ref
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("lat", [9, 27])
def test_oracle_bit_identical_to_reference(prec, lat):
    O.set_ref_threads(1, prec)
    rng = np.random.default_rng(0)
    ops = [("none", 0), ("bgk", 0), ("bgk", 1), ("trt", 0), ("trt", 1), ("mrt", 0), ("cm", 0)]
    for (op, eq), shifted, forcing, walls in itertools.product(ops, [1, 0], [0, 1], [0, 1]):
        nx, ny, nz = (7, 6, 1) if lat == 9 else (5, 6, 4)
        kw = dict(lattice=lat, op=op, eq=eq, shifted=shifted, forcing=forcing, nx=nx, ny=ny,
                  nz=nz, px=True, py=not walls, pz=True, omega=1.3,
                  omega2=(1.1 if op == "trt" else -1.0), fx=2e-5, fy=-1e-5,
                  fz=3e-6 if lat == 27 else 0.0, precision=prec)
        a, b = O.CpuSolver("oracle", **kw), O.CpuSolver("ref", **kw)
        fl = np.zeros((nz, ny, nx), np.uint8)
        if walls:
            fl[:, 0, :] = 1
            fl[:, -1, :] = 1
        a.set_geometry(fl)
        b.set_geometry(fl)
        sh = (nz, ny, nx)
        rho = 1 + 0.01 * rng.standard_normal(sh)
        u = [0.03 * rng.standard_normal(sh) for _ in range(3)]
        if lat == 9:
            u[2] = np.zeros(sh)
        a.initialize_field(rho, *u)
        b.initialize_field(rho, *u)
        for t in range(5):
            a.step(1, store_macro=(t == 4))
            b.step(1, store_macro=(t == 4))
        case = (prec, lat, op, eq, shifted, forcing, walls)
        np.testing.assert_array_equal(a.gather(), b.gather(), err_msg=str(case))
        for x, y in zip(a.macro(), b.macro()):
            np.testing.assert_array_equal(x, y, err_msg=str(case))
        for x, y in zip(a.stored_macro(), b.stored_macro()):
            np.testing.assert_array_equal(x, y, err_msg=str(case))
        assert a.total_mass() == b.total_mass(), case
        assert a.total_momentum(0) == b.total_momentum(0), case
        assert a.slot_sum() == b.slot_sum(), case
        a.close()
        b.close()


# ------------------------------------------------------- streaming known answers
def _permutation(lat, shape, steps, backend="oracle", streaming=0):
    nx, ny, nz = shape
    Q = lat
    s = O.CpuSolver(backend, lattice=lat, op="none", nx=nx, ny=ny, nz=nz, precision="f64",
                    streaming=streaming)
    tags = (np.arange(s.n_padded * Q, dtype=np.float64) + 1).reshape(s.n_padded, Q)
    s.seed(tags)
    s.step(steps)
    got = s.gather()
    from m3lb_b200.solver import D2Q9, D3Q27
    L = D3Q27 if lat == 27 else D2Q9
    bad = 0
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                n = (z * ny + y) * nx + x
                for i in range(Q):
                    src = (((z - steps * L.cz[i]) % nz) * ny + (y - steps * L.cy[i]) % ny) * nx + \
                          (x - steps * L.cx[i]) % nx
                    bad += got[n, i] != tags[src, i]
    s.close()
    return bad


@pytest.mark.parametrize("lat,shape,steps", [
    (9, (8, 6, 1), 1), (9, (8, 6, 1), 2), (9, (8, 6, 1), 7), (9, (8, 6, 1), 24),
    (27, (5, 4, 3), 1), (27, (5, 4, 3), 13)])
def test_oracle_permutation(lat, shape, steps):
    assert _permutation(lat, shape, steps) == 0


@needs_ref
@pytest.mark.parametrize("lat", [9, 27])
@pytest.mark.parametrize("shifted", [0, 1])
def test_esoteric_pull_matches_two_lattice(lat, shifted):
    """Oracle (Esoteric Pull) against the reference's two-lattice streaming,
    every step, walls + Guo (test_streaming.cpp:80-124, tolerance 1e-13)."""
    O.set_ref_threads(1, "f64")
    nx, ny, nz = (12, 10, 8 if lat == 27 else 1)
    kw = dict(lattice=lat, op="bgk", shifted=shifted, forcing=1, nx=nx, ny=ny, nz=nz, px=True,
              py=False, pz=True, omega=1.4, fx=2e-5, fy=-1e-5, fz=0.0, precision="f64")
    a = O.CpuSolver("oracle", **kw)
    b = O.CpuSolver("ref", streaming=1, **kw)
    fl = np.zeros((nz, ny, nx), np.uint8)
    fl[:, 0, :] = 1
    fl[:, -1, :] = 1
    a.set_geometry(fl)
    b.set_geometry(fl)
    a.initialize(1.0, 0.03, 0.01, 0.0)
    b.initialize(1.0, 0.03, 0.01, 0.0)
    padded_fluid = None
    for _ in range(40 if lat == 9 else 20):
        a.step()
        b.step()
        ga, gb = a.gather(), b.gather()
        if padded_fluid is None:
            sx, sy, sz = nx, ny + 2, nz
            f3 = np.full((sz, sy, sx), 2, np.uint8)
            f3[:, 1:-1, :] = fl
            padded_fluid = (f3.reshape(-1) == 0)
        assert np.max(np.abs(ga[padded_fluid] - gb[padded_fluid])) <= 1e-13


# ------------------------------------------------------- Poiseuille known answers
def poiseuille(op, tau, H=32, umax=0.01, nx=8, steps=60000, lam=None, precision="f64",
               backend="oracle"):
    """validation/poiseuille.cpp:72-140: periodic x, solid rows y = 0 and
    y = H + 1 (ny = H + 2), uniform Guo force G = 8 rho nu umax / H^2."""
    nu = (tau - 0.5) / 3.0
    omega = 1.0 / tau
    G = 8.0 * nu * umax / (H * H)
    ny = H + 2
    omega2 = -1.0
    if op == "trt":
        omega2 = 1.0 / (lam / (1.0 / omega - 0.5) + 0.5)
    s = O.CpuSolver(backend, lattice=9, op=op, shifted=True, forcing=True, nx=nx, ny=ny, nz=1,
                    px=True, py=False, pz=True, omega=omega, omega2=omega2, fx=G,
                    precision=precision)
    fl = np.zeros((1, ny, nx), np.uint8)
    fl[:, 0, :] = 1
    fl[:, -1, :] = 1
    s.set_geometry(fl)
    s.initialize(1.0)
    s.step(steps)
    rho, ux, _, _ = s.macro()
    s.close()
    j = np.arange(1, H + 1)
    u = ux[0, 1:H + 1, nx // 2]
    rm = rho[0, 1:H + 1, nx // 2].mean()
    A = G / (2 * rm * nu)
    ana = A * (j - 0.5) * (H + 0.5 - j)
    return math.sqrt(np.sum((u - ana) ** 2) / np.sum(ana ** 2))


def test_poiseuille_bgk_tau08_known_answer():
    """README.md:178-186: D2Q9 BGK, H = 32, tau = 0.8 -> L2 relative 6.95e-4."""
    assert poiseuille("bgk", 0.8) == pytest.approx(6.95e-4, rel=0.01)


@pytest.mark.parametrize("op,tau,lam", [("bgk", 0.5 + math.sqrt(3) / 4, None),
                                        ("trt", 0.8, 3.0 / 16.0),
                                        ("cm", 7.0 / 8.0, None), ("mrt", 7.0 / 8.0, None)])
def test_poiseuille_magic_parameter_is_exact(op, tau, lam):
    """README.md:240-276: at the magic parameter the halfway wall sits exactly
    midway; the discrete solution is the parabola to round-off (~1e-14)."""
    assert poiseuille(op, tau, lam=lam) < 1e-11


# ------------------------------------------------------------ free-slip walls
@pytest.mark.parametrize("name", list(G.SPEC_CASES))
def test_oracle_reproduces_specular_golden(name):
    """SpecWall / SpecNode fixtures made by the reference build."""
    d = np.load(GOLDEN / f"{name}.npz")
    r = G.run_spec("oracle", G.SPEC_CASES[name], seed=int(d["seed"]))
    for k in ("pops0", "pops", "stored", "macro"):
        np.testing.assert_array_equal(r[k], d[k], err_msg=k)
    assert r["mass"] == float(d["mass"])
    np.testing.assert_array_equal(r["mom"], d["mom"])
    assert r["slots"] == float(d["slots"])


@needs_ref
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("kind", ["wall", "node", "mixed"])
def test_oracle_specular_bit_identical_to_reference(prec, kind):
    """Every operator, both storage conventions, with and without force, on
    both lattices: ghost mirror, on-node mirror with edges, and the two mixed."""
    O.set_ref_threads(1, prec)
    ops = [("none", 0, -1.0), ("bgk", 0, -1.0), ("bgk", 1, -1.0), ("trt", 0, 1.1),
           ("mrt", 0, 1.5), ("cm", 0, -1.0)]
    for lat, (op, eq, om2), shifted, forcing in itertools.product(
            [9, 27], ops, [1, 0], [0, 1]):
        shape = (7, 6, 1) if lat == 9 else (6, 5, 5)
        case = (lat, op, eq, shifted, forcing, shape, kind, 1.3, om2, 6, prec)
        a = G.run_spec("oracle", case, seed=7)
        b = G.run_spec("ref", case, seed=7)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{case} {k}")


def test_oracle_specular_setters_reject_what_the_reference_rejects():
    kw = dict(lattice=27, op="bgk", nx=4, ny=4, nz=4, px=False, py=False, pz=False,
              precision="f64")
    s = O.CpuSolver("oracle", **kw)
    s.initialize(1.0, 0.02, 0.0, 0.0)
    base = s.gather()
    codes = np.zeros((4, 4, 4), np.uint8)
    codes[1, 2, 3] = 7                       # corner code: not an axis normal
    with pytest.raises(ValueError):
        s.set_specular_walls(codes)
    for bad in (0x40, 0x03, 0x0C, 0x30):     # stray bit, both faces of x / y / z
        m = np.zeros((4, 4, 4), np.uint8)
        m[0, 0, 0] = 0x01
        m[2, 1, 0] = bad
        with pytest.raises(ValueError):
            s.set_specular_nodes(m)
    # nothing was marked: the run equals a plain one
    s.step(3)
    t = O.CpuSolver("oracle", **kw)
    t.initialize(1.0, 0.02, 0.0, 0.0)
    t.step(3)
    np.testing.assert_array_equal(s.gather(), t.gather())
    assert not np.array_equal(base, t.gather())
    s.close()
    t.close()


def test_oracle_specular_wall_conserves_mass():
    """A ghost mirror permutes populations, so a box closed by SpecWall and
    bounce-back conserves mass to round-off (validation/specular.cpp:33-38)."""
    case = (27, "bgk", 0, 1, 1, (6, 8, 5), "wall", 1.2, -1.0, 0, "f64")
    lat, op, eq, sh, fo, shape, kind, om, om2, _, prec = case
    nx, ny, nz = shape
    s = O.CpuSolver("oracle", lattice=27, op="bgk", shifted=1, forcing=1, nx=nx, ny=ny, nz=nz,
                    px=True, py=False, pz=True, omega=1.2, fx=1e-5, precision="f64")
    fl, codes, _ = G.spec_geometry(lat, shape, kind)
    s.set_geometry(fl)
    s.set_specular_walls(codes)
    s.initialize(1.0)
    m0 = s.total_mass()
    s.step(200)
    assert abs(s.total_mass() - m0) / m0 < 1e-13
    s.close()


# ------------------------------------------------------- regularised walls
@pytest.mark.parametrize("name", list(G.WALL_CASES))
def test_oracle_reproduces_wall_golden(name):
    """RegWall fixtures (velocity walls, corners, outlets) made by the reference build."""
    d = np.load(GOLDEN / f"{name}.npz")
    r = G.run_wall("oracle", G.WALL_CASES[name], seed=int(d["seed"]))
    for k in ("pops0", "pops", "stored", "macro"):
        np.testing.assert_array_equal(r[k], d[k], err_msg=k)
    assert r["mass"] == float(d["mass"])
    np.testing.assert_array_equal(r["mom"], d["mom"])
    assert r["slots"] == float(d["slots"])


@needs_ref
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("kind", list(G.WALL_PERIODIC))
def test_oracle_walls_bit_identical_to_reference(prec, kind):
    """Every operator, storage convention and force on both lattices, against
    the reference run on one thread (its outflow and corner branches read
    neighbour nodes inside the in-place sweep, so its result is defined by
    the sweep order; one thread is index order)."""
    O.set_ref_threads(1, prec)
    ops = [("none", 0, -1.0), ("bgk", 0, -1.0), ("bgk", 1, -1.0), ("trt", 0, 1.1),
           ("mrt", 0, 1.5), ("cm", 0, -1.0)]
    for lat, (op, eq, om2), shifted, forcing in itertools.product([9, 27], ops, [1, 0], [0, 1]):
        shape = (10, 9, 1) if lat == 9 else (8, 7, 5)
        case = (lat, op, eq, shifted, forcing, shape, kind, 1.3, om2, 7, prec)
        a = G.run_wall("oracle", case, seed=7)
        b = G.run_wall("ref", case, seed=7)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{case} {k}")


WALL_MODIFIERS = {
    "scale": [("set_wall_velocity_scale", 0.5)],
    "density": [("set_wall_density", 1.02)],
    "field": [("set_wall_velocity_field", "field"), ("set_wall_velocity_field_scale", 0.7)],
    "no_fd": [("set_fd_corners", False)],
    "no_force_bc": [("set_force_correction", False)],
    "order2": [("set_outflow_order", 2)],
    "outflow_rho": [("set_outflow_density", 0.98)],
}


@needs_ref
@pytest.mark.parametrize("mod", list(WALL_MODIFIERS))
@pytest.mark.parametrize("kind", ["cavity", "inout", "outfree", "fdcorner"])
def test_oracle_wall_setters_match_reference(mod, kind):
    O.set_ref_threads(1, "f64")
    lat, shape = 27, (8, 7, 5)
    nx, ny, nz = shape
    per = G.WALL_PERIODIC[kind]
    out = []
    for backend in ("oracle", "ref"):
        s = O.CpuSolver(backend, lattice=lat, op="bgk", shifted=1, forcing=1, nx=nx, ny=ny, nz=nz,
                        px=per[0], py=per[1], pz=per[2], omega=1.3, fx=2e-5, fy=-1e-5, fz=3e-6,
                        precision="f64")
        fl, codes, st = G.wall_geometry(lat, shape, kind)
        s.set_geometry(fl)
        s.set_regularized_walls(codes, st)
        for fn, arg in WALL_MODIFIERS[mod]:
            if arg == "field":
                arg = 0.01 * np.random.default_rng(2).standard_normal((nz, ny, nx, 3))
            getattr(s, fn)(arg)
        s.initialize_field(*G.initial_field(shape, 9))
        s.step(6, store_macro=True)
        out.append((s.gather(), s.stored_macro(), s.macro(), s.total_mass()))
        s.close()
    (ga, sa, ma, mass_a), (gb, sb, mb, mass_b) = out
    np.testing.assert_array_equal(ga, gb)
    for x, y in zip(sa + ma, sb + mb):
        np.testing.assert_array_equal(x, y)
    assert mass_a == mass_b


def test_oracle_wall_setters_reject():
    s = O.CpuSolver("oracle", lattice=9, op="bgk", nx=8, ny=6, nz=1, px=False, py=False,
                    precision="f64")
    codes = np.zeros((1, 6, 8), np.uint8)
    codes[0, 2, 3] = 11
    with pytest.raises(ValueError):
        s.set_regularized_walls(codes)
    codes[0, 2, 3] = 0
    codes[0, 2, 0] = 8
    with pytest.raises(ValueError):
        s.set_regularized_walls(codes)
    codes[0, 2, 0] = 0
    codes[0, 2, 1] = 8
    s.set_regularized_walls(codes)
    with pytest.raises(ValueError):
        s.set_outflow_order(2)
    s.close()


def test_oracle_couette_between_regularized_walls_is_exact():
    """Linear profiles carry no curvature slip (FluidSolver.hpp:1296-1303:
    Couette exact to round-off at every tau)."""
    ny, U = 10, 0.04
    s = O.CpuSolver("oracle", lattice=9, op="bgk", nx=4, ny=ny, nz=1, px=True, py=False,
                    omega=1.1, precision="f64")
    codes = np.zeros((1, ny, 4), np.uint8)
    st = np.zeros((1, ny, 4, 4))
    st[..., 3] = 1.0
    codes[0, 0, :] = 4
    codes[0, -1, :] = 3
    st[0, -1, :, 0] = U
    s.set_regularized_walls(codes, st)
    s.initialize(1.0)
    s.step(6000)
    ux = s.macro()[1][0, :, 0]
    np.testing.assert_allclose(ux, U * np.arange(ny) / (ny - 1), rtol=0, atol=1e-10)
    s.close()


# ------------------------------------------------ scalar lattice and coupling
@pytest.mark.parametrize("name", list(G.SCALAR_CASES))
def test_oracle_reproduces_scalar_golden(name):
    """D2Q5 / D3Q7 fixtures made by the reference's ScalarSolver."""
    d = np.load(GOLDEN / f"{name}.npz")
    k = list(G.SCALAR_CASES).index(name)
    r = G.run_scalar("oracle", G.SCALAR_CASES[name], int(d["seed"]), T_ref=0.25,
                     omega_field=k % 2 == 1, source=True)
    for key in ("field0", "stored", "field"):
        np.testing.assert_array_equal(r[key], d[key], err_msg=key)
    assert r["total"] == float(d["total"])


@needs_ref
@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("kind", list(G.SCALAR_PERIODIC))
def test_oracle_scalar_bit_identical_to_reference(prec, kind):
    """Every scalar operator on D2Q5 / D3Q7, ScalarBGK on D2Q9 / D3Q27, every
    cell type, with and without a storage reference T_ref, per-node rates and
    sources."""
    O.set_ref_threads(1, prec)
    for lat, op, tref, omf, src in itertools.product([5, 7, 9, 27], ["bgk", "trt", "regularised"],
                                                    [0.0, 0.5], [False, True], [False, True]):
        if lat in (9, 27) and op != "bgk":   # TRT / regularised need the axis-pair lattices
            continue
        shape = (10, 9, 1) if lat in (5, 9) else (8, 7, 5)
        case = (lat, op, shape, kind, 1.2, 9, prec)
        a = G.run_scalar("oracle", case, 3, T_ref=tref, omega_field=omf, source=src)
        b = G.run_scalar("ref", case, 3, T_ref=tref, omega_field=omf, source=src)
        for k in a:
            np.testing.assert_array_equal(a[k], b[k], err_msg=f"{case} {tref} {omf} {src} {k}")


@pytest.mark.parametrize("name", list(G.COUPLED_CASES))
def test_oracle_reproduces_coupled_golden(name):
    """Fluid with Boussinesq buoyancy + scalar advected by the fluid: fixtures
    made by the reference's FluidSolver<..., BoussinesqGuo> and ScalarSolver."""
    d = np.load(GOLDEN / f"{name}.npz")
    r = G.run_coupled("oracle", G.COUPLED_CASES[name], int(d["seed"]))
    for key in ("pops", "stored", "macro", "T_stored", "T"):
        np.testing.assert_array_equal(r[key], d[key], err_msg=key)
    assert r["mass"] == float(d["mass"]) and r["total"] == float(d["total"])


@needs_ref
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_oracle_buoyancy_bit_identical_to_reference(prec):
    """The per-node Boussinesq force on every fluid operator, with and without
    walls, against BoussinesqGuo in the reference build."""
    O.set_ref_threads(1, prec)
    for lat, (op, eq, om2), shifted, walls in itertools.product(
            [9, 27], [("bgk", 0, -1.0), ("bgk", 1, -1.0), ("trt", 0, 1.1), ("mrt", 0, 1.5),
                      ("cm", 0, -1.0)], [1, 0], [0, 1]):
        nx, ny, nz = (10, 9, 1) if lat == 9 else (8, 7, 5)
        kw = dict(lattice=lat, op=op, eq=eq, shifted=shifted, nx=nx, ny=ny, nz=nz, px=True,
                  py=not walls, pz=True, omega=1.3, omega2=om2, fx=1e-5, fy=0.0,
                  fz=2e-6 if lat == 27 else 0.0, precision=prec)
        a = O.CpuSolver("oracle", forcing=1, **kw)
        b = O.CpuSolver("ref", forcing=2, **kw)
        rng = np.random.default_rng(4)
        sh = (nz, ny, nx)
        fl = np.zeros(sh, np.uint8)
        if walls:
            fl[:, 0, :] = 1
            fl[:, -1, :] = 1
        fields = [np.asarray(x, np.float32).astype(np.float64) for x in
                  [1 + 0.01 * rng.standard_normal(sh)] + [0.03 * rng.standard_normal(sh) for _ in range(3)]]
        if lat == 9:
            fields[3][:] = 0
        for s in (a, b):
            s.set_geometry(fl)
            s.initialize_field(*fields)
        for _ in range(6):
            T = np.asarray(0.3 * rng.standard_normal(sh), np.float32).astype(np.float64)
            for s in (a, b):
                s.set_buoyancy(T, g=(0.0, 1.0, 0.5 if lat == 27 else 0.0), rho0=1.0, beta=2e-4, T0=0.1)
                s.step(1, store_macro=True)
        np.testing.assert_array_equal(a.gather(), b.gather())
        for x, y in zip(a.stored_macro() + a.macro(), b.stored_macro() + b.macro()):
            np.testing.assert_array_equal(x, y)
        assert a.total_mass() == b.total_mass()
        a.close()
        b.close()


def test_oracle_scalar_diffusion_rate():
    """A sinusoid decays at D k^2 with D = cs2 (1/omega - 1/2) (ScalarBGK.hpp:20-27,
    validation/thermal.cpp): cs2 = 1/3 on D2Q5, 1/4 on D3Q7."""
    for lat, cs2 in ((5, 1 / 3), (7, 1 / 4)):
        N, om, steps = 64, 1.2, 400
        nz = 1 if lat == 5 else 4
        s = O.ScalarCpuSolver("oracle", lattice=lat, op="bgk", nx=N, ny=4, nz=nz, omega=om)
        x = np.arange(N)
        T = np.broadcast_to(0.01 * np.sin(2 * np.pi * x / N), (nz, 4, N)).ravel()
        s.initialize_field(T)
        s.step(steps)
        s.compute_field()
        amp = s.field()[0, 0] @ np.sin(2 * np.pi * x / N) * 2 / N
        D = cs2 * (1 / om - 0.5)
        k = 2 * np.pi / N
        assert abs(amp / 0.01 / np.exp(-D * k * k * steps) - 1) < 1e-3
        s.close()


def _f16c_reference(v):
    """The FP16C format from its definition (1 sign, 4 exponent bits with bias
    15, 11 mantissa bits, subnormals below 2^-14 with step 2^-25, largest
    magnitude 2 - 2^-11): nearest value, ties away from zero, magnitudes
    beyond the largest (and NaN) saturated."""
    v = np.asarray(v, np.float64)
    top = 2.0 - 2.0 ** -11
    m = np.where(np.isnan(v), top, np.minimum(np.abs(v), top))
    _, k = np.frexp(np.where(m > 0, m, 1.0))
    e = np.maximum(k - 1, -14)               # binade exponent, subnormals share -14
    ulp = np.ldexp(1.0, e - 11)
    q = np.floor(m / ulp + 0.5) * ulp
    return np.where(np.signbit(v), -q, q)


def test_oracle_f16c_storage_rounds_as_the_format_defines():
    """The oracle's FP16C storage emulation (what the device's encoder must
    match bit for bit) against the format's definition: exact values stay,
    halfway values go away from zero, subnormals keep a 2^-25 step, large
    magnitudes saturate, and random shifted-population-sized values land on
    the nearest representable value."""
    c = O.CpuSolver("oracle", lattice=27, op="none", shifted=True, nx=4, ny=3, nz=2,
                    px=True, py=True, pz=True, precision="f32", quant="f16c")
    n = c.n_padded * c.Q
    special = [1.0, -1.0, 1 + 2 ** -11, 1 + 2 ** -12, 1 + 3 * 2 ** -12, -(1 + 2 ** -12),
               2 ** -14, 2 ** -25, 2 ** -26, 3 * 2 ** -26, 2 ** -27, 0.0, -0.0,
               1.99951171875, 1.9998, 3.0, -70000.0, 2 ** -14 - 2 ** -26, 0.1, -0.01]
    rng = np.random.default_rng(0)
    rand = (rng.standard_normal(n - len(special)) * 10.0 ** rng.uniform(-7, 0, n - len(special)))
    vals = np.concatenate([special, rand]).astype(np.float32).astype(np.float64)
    c.seed(vals.reshape(c.n_padded, c.Q))
    got = c.gather().reshape(-1)
    c.close()
    want = _f16c_reference(vals)
    assert np.array_equal(got, want), np.flatnonzero(got != want)[:10]
    assert got[3] == 1 + 2 ** -11 and got[5] == -(1 + 2 ** -11)   # ties away from zero
    assert got[8] == 2 ** -25 and got[10] == 0.0                 # subnormal step 2^-25
    assert got[13] == got[14] == got[15] == 1.99951171875 and got[16] == -1.99951171875
