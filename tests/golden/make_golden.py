"""Generate the golden fixtures in this folder from the REFERENCE build.

Runs M3LB's own FluidSolver (oracle/_ref, the reference's src/ headers built
unmodified against the host Kokkos stand-in) on small seeded cases and saves
the resulting populations and fields.  Needs the reference build, i.e. run it
where the reference sources were available:

    make -C oracle ref && python tests/golden/make_golden.py

The fixtures then pin the C oracle (bit for bit) and the GPU path (within the
parity tolerances) on machines without the reference.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

import oracle as O  # noqa: E402

# name -> (lattice, op, eq, shifted, forcing, shape, periodic, omega, omega2, F, steps, precision)
CASES = {
    "d3q27_cm_guo_walls_f64": (27, "cm", 0, 1, 1, (12, 10, 8), (True, False, True), 1.7, -1.0,
                               (2e-5, -1e-5, 3e-6), 10, "f64"),
    "d3q27_trt_pf_walls_f64": (27, "trt", 1, 1, 1, (10, 8, 6), (True, False, False), 1.4, 1.1,
                               (1e-5, 0.0, 0.0), 10, "f64"),
    "d3q27_mrt_raw_f32": (27, "mrt", 0, 0, 0, (8, 8, 8), (True, True, True), 1.2, 1.6,
                          (0.0, 0.0, 0.0), 7, "f32"),
    "d3q27_bgk_f32": (27, "bgk", 0, 1, 0, (9, 7, 6), (False, False, False), 1.3, -1.0,
                      (0.0, 0.0, 0.0), 6, "f32"),
    "d2q9_bgk_guo_walls_f64": (9, "bgk", 0, 1, 1, (16, 12, 1), (True, False, True), 1.25, -1.0,
                               (1e-5, -2e-6, 0.0), 25, "f64"),
    "d2q9_cm_f32": (9, "cm", 0, 1, 0, (12, 10, 1), (True, True, True), 1.6, -1.0,
                    (0.0, 0.0, 0.0), 9, "f32"),
}


def initial_field(shape, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    sh = (nz, ny, nx)
    rho = 1 + 0.01 * rng.standard_normal(sh)
    u = [0.03 * rng.standard_normal(sh) for _ in range(3)]
    if nz == 1:
        u[2] = np.zeros(sh)
    # representable in FP32, so every precision starts from the same values
    return [np.asarray(a, np.float32).astype(np.float64) for a in [rho] + u]


def solid_mask(shape, walls):
    nx, ny, nz = shape
    fl = np.zeros((nz, ny, nx), np.uint8)
    if walls:
        fl[:, 0, :] = 1
    fl.flat[fl.size // 2] = 1
    return fl


def run(backend, case, seed, quant=None):
    lat, op, eq, sh, fo, shape, per, om, om2, F, steps, prec = case
    nx, ny, nz = shape
    s = O.CpuSolver(backend, lattice=lat, op=op, eq=eq, shifted=sh, forcing=fo, nx=nx, ny=ny,
                    nz=nz, px=per[0], py=per[1], pz=per[2], omega=om, omega2=om2, fx=F[0],
                    fy=F[1], fz=F[2], precision=prec, quant=quant)
    s.set_geometry(solid_mask(shape, not per[1]))
    s.initialize_field(*initial_field(shape, seed))
    p0 = s.gather()
    s.step(steps, store_macro=True)
    out = {"pops0": p0, "pops": s.gather(), "stored": np.stack(s.stored_macro()),
           "macro": np.stack(s.macro()), "mass": s.total_mass(),
           "mom": np.array([s.total_momentum(a) for a in range(3)]), "slots": s.slot_sum()}
    s.close()
    return out


# Free-slip walls (FluidSolver.hpp:193-268).  name -> (lattice, op, eq,
# shifted, forcing, shape, kind, omega, omega2, steps, precision); `kind`
# picks the geometry of spec_geometry() and, with it, the periodic axes.
SPEC_CASES = {
    "d2q9_bgk_guo_specwall_f64": (9, "bgk", 0, 1, 1, (10, 9, 1), "wall", 1.25, -1.0, 20, "f64"),
    "d3q27_cm_specnode_f64": (27, "cm", 0, 1, 0, (8, 7, 6), "node", 1.6, -1.0, 9, "f64"),
    "d3q27_trt_guo_specmixed_f32": (27, "trt", 0, 1, 1, (8, 7, 5), "mixed", 1.4, 1.1, 9, "f32"),
    "d2q9_mrt_raw_specnode_f32": (9, "mrt", 0, 0, 0, (9, 8, 1), "node", 1.3, 1.5, 15, "f32"),
}
SPEC_PERIODIC = {"wall": (True, False, True), "node": (False, False, False),
                 "mixed": (False, False, True)}


def spec_geometry(lat, shape, kind):
    """(flags, normal codes, face masks) over the interior, each (nz, ny, nx).

    wall : solid row y = 0, SpecWall row y = ny-1 with normal +y (the
           half-channel of the reference's validation/specular.cpp);
    node : solid row y = 0, SpecNode on the x faces and (3-D) the z faces,
           so the box edges carry two-face masks;
    mixed: solid row y = 0, SpecWall columns on the x faces, SpecNode on the
           top row between them."""
    nx, ny, nz = shape
    fl = np.zeros((nz, ny, nx), np.uint8)
    codes = np.zeros_like(fl)
    masks = np.zeros_like(fl)
    fl[:, 0, :] = 1
    if kind == "wall":
        codes[:, -1, :] = 3
    elif kind == "node":
        masks[:, 1:, 0] |= 0x02
        masks[:, 1:, -1] |= 0x01
        if lat == 27:
            masks[0, 1:, :] |= 0x20
            masks[-1, 1:, :] |= 0x10
    elif kind == "mixed":
        codes[:, 1:, 0] = 2
        codes[:, 1:, -1] = 1
        masks[:, -1, 1:-1] = 0x04
    else:
        raise ValueError(kind)
    return fl, codes, masks


# Regularised walls (FluidSolver.hpp:372-552, 792-1021).  name -> (lattice,
# op, eq, shifted, forcing, shape, kind, omega, omega2, steps, precision).
WALL_CASES = {
    "d2q9_bgk_cavity_f64": (9, "bgk", 0, 1, 0, (10, 9, 1), "cavity", 1.3, -1.0, 25, "f64"),
    "d3q27_cm_inout_guo_f64": (27, "cm", 0, 1, 1, (9, 7, 5), "inout", 1.5, -1.0, 12, "f64"),
    "d3q27_trt_outfree_f32": (27, "trt", 0, 1, 1, (9, 6, 5), "outfree", 1.4, 1.1, 10, "f32"),
    "d2q9_mrt_fdcorner_f32": (9, "mrt", 0, 0, 1, (10, 9, 1), "fdcorner", 1.2, 1.5, 15, "f32"),
}
WALL_PERIODIC = {"couette": (True, False, True), "cavity": (False, False, True),
                 "inout": (False, False, True), "outeq": (False, False, True),
                 "outfree": (False, False, True), "fdcorner": (True, False, True)}


def wall_geometry(lat, shape, kind):
    """(flags, normal codes, states (nz, ny, nx, 4)) over the interior.

    couette : RegWall floor (u = 0) and lid (u = (0.02, 0.01, 0)), periodic x;
    cavity  : a box of RegWall faces, lid u = (0.05, 0, 0), NrmCorner on the
              corners (edges in 3-D, z periodic): corner densities and the
              finite-difference corner stress;
    inout   : solid floor and ceiling, velocity inlet at x = 0, pressure
              outlet (NrmOutXp, rho 1.01) at x = nx-1;
    outeq   : the same with the equilibrium outlet (NrmOutEq);
    outfree : solid floor and ceiling, arbitrary-face outflow (NrmOutFree) on
              both x faces, so one donor precedes its node in index order and
              one follows it;
    fdcorner: RegWall floor and lid, periodic x, with NrmCorner nodes inside
              both rows, whose finite-difference stencil reads fluid nodes
              above (later in index order) and below (earlier) them."""
    nx, ny, nz = shape
    fl = np.zeros((nz, ny, nx), np.uint8)
    codes = np.zeros_like(fl)
    st = np.zeros((nz, ny, nx, 4))
    st[..., 3] = 1.0
    if kind == "couette":
        codes[:, 0, :] = 4
        codes[:, -1, :] = 3
        st[:, -1, :, 0] = 0.02
        st[:, -1, :, 1] = 0.01
    elif kind == "cavity":
        codes[:, :, 0] = 2
        codes[:, :, -1] = 1
        codes[:, 0, :] = 4
        codes[:, -1, :] = 3
        st[:, -1, :, 0] = 0.05
        for y in (0, ny - 1):
            for x in (0, nx - 1):
                codes[:, y, x] = 7
                st[:, y, x, 0] = 0.0
    elif kind in ("inout", "outeq"):
        fl[:, 0, :] = 1
        fl[:, -1, :] = 1
        codes[:, 1:-1, 0] = 2
        st[:, 1:-1, 0, 0] = 0.03
        codes[:, 1:-1, -1] = 8 if kind == "inout" else 10
        st[:, 1:-1, -1, 3] = 1.01
    elif kind == "outfree":
        fl[:, 0, :] = 1
        fl[:, -1, :] = 1
        codes[:, 1:-1, 0] = 9
        codes[:, 1:-1, -1] = 9
    elif kind == "fdcorner":
        codes[:, 0, :] = 4
        codes[:, -1, :] = 3
        st[:, -1, :, 0] = 0.03
        codes[:, 0, 3] = 7
        codes[:, -1, nx - 3] = 7
        st[:, -1, nx - 3, 0] = 0.03
    else:
        raise ValueError(kind)
    return fl, codes, st


def run_wall(backend, case, seed, quant=None):
    lat, op, eq, sh, fo, shape, kind, om, om2, steps, prec = case
    nx, ny, nz = shape
    per = WALL_PERIODIC[kind]
    F = (2e-5, -1e-5, 3e-6 if lat == 27 else 0.0) if fo else (0.0, 0.0, 0.0)
    s = O.CpuSolver(backend, lattice=lat, op=op, eq=eq, shifted=sh, forcing=fo, nx=nx, ny=ny,
                    nz=nz, px=per[0], py=per[1], pz=per[2], omega=om, omega2=om2, fx=F[0],
                    fy=F[1], fz=F[2], precision=prec, quant=quant)
    fl, codes, st = wall_geometry(lat, shape, kind)
    s.set_geometry(fl)
    s.set_regularized_walls(codes, st)
    s.initialize_field(*initial_field(shape, seed))
    p0 = s.gather()
    s.step(steps, store_macro=True)
    out = {"pops0": p0, "pops": s.gather(), "stored": np.stack(s.stored_macro()),
           "macro": np.stack(s.macro()), "mass": s.total_mass(),
           "mom": np.array([s.total_momentum(a) for a in range(3)]), "slots": s.slot_sum()}
    s.close()
    return out


def run_spec(backend, case, seed, quant=None):
    lat, op, eq, sh, fo, shape, kind, om, om2, steps, prec = case
    nx, ny, nz = shape
    per = SPEC_PERIODIC[kind]
    F = (2e-5, -1e-5, 3e-6 if lat == 27 else 0.0) if fo else (0.0, 0.0, 0.0)
    s = O.CpuSolver(backend, lattice=lat, op=op, eq=eq, shifted=sh, forcing=fo, nx=nx, ny=ny,
                    nz=nz, px=per[0], py=per[1], pz=per[2], omega=om, omega2=om2, fx=F[0],
                    fy=F[1], fz=F[2], precision=prec, quant=quant)
    fl, codes, masks = spec_geometry(lat, shape, kind)
    s.set_geometry(fl)
    if codes.any():
        s.set_specular_walls(codes)
    if masks.any():
        s.set_specular_nodes(masks)
    s.initialize_field(*initial_field(shape, seed))
    p0 = s.gather()
    s.step(steps, store_macro=True)
    out = {"pops0": p0, "pops": s.gather(), "stored": np.stack(s.stored_macro()),
           "macro": np.stack(s.macro()), "mass": s.total_mass(),
           "mom": np.array([s.total_momentum(a) for a in range(3)]), "slots": s.slot_sum()}
    s.close()
    return out


# Scalar lattice (src/solver/ScalarSolver.hpp).  name -> (lattice, op, shape,
# kind, omega, steps, precision).
SCALAR_CASES = {
    "d3q7_bgk_walls_f64": (7, "bgk", (8, 7, 6), "walls", 1.3, 12, "f64"),
    "d3q7_trt_outflow_f32": (7, "trt", (9, 6, 5), "outflow", 1.1, 10, "f32"),
    "d2q5_regularised_moment_f64": (5, "regularised", (10, 9, 1), "moment", 1.5, 15, "f64"),
    "d2q5_bgk_specular_f32": (5, "bgk", (10, 9, 1), "specular", 0.9, 15, "f32"),
}
SCALAR_PERIODIC = {"periodic": (True, True, True), "walls": (True, False, True),
                   "moment": (True, False, True), "outflow": (False, True, True),
                   "specular": (True, False, True)}


def scalar_geometry(lattice, shape, kind):
    """(cells, wall values, specular codes, specular masks) over the interior.

    periodic: bulk everywhere;
    walls   : Dirichlet floor (T = 1, anti-bounce-back) and adiabatic lid;
    moment  : on-node Dirichlet (ScalarMoment) floor at T = 1 and lid at T = 0;
    outflow : Dirichlet inlet column at x = 0, outflow column at x = nx-1;
    specular: on-node mirror floor (set_specular_nodes) and lid
              (set_specular_walls), a Dirichlet node in the middle."""
    nx, ny, nz = shape
    cells = np.zeros((nz, ny, nx), np.uint8)
    tw = np.zeros((nz, ny, nx))
    codes = np.zeros_like(cells)
    masks = np.zeros_like(cells)
    if kind == "walls":
        cells[:, 0, :] = 2
        tw[:, 0, :] = 1.0
        cells[:, -1, :] = 1
    elif kind == "moment":
        cells[:, 0, :] = 4
        tw[:, 0, :] = 1.0
        cells[:, -1, :] = 4
    elif kind == "outflow":
        cells[:, :, 0] = 2
        tw[:, :, 0] = 1.0
        cells[:, :, -1] = 5
    elif kind == "specular":
        cells[:, 0, :] = 6
        masks[:, 0, :] = 0x08
        cells[:, -1, :] = 6
        codes[:, -1, :] = 3
        cells[nz // 2, ny // 2, nx // 2] = 2
        tw[nz // 2, ny // 2, nx // 2] = 2.0
    elif kind != "periodic":
        raise ValueError(kind)
    return cells, tw, codes, masks


def scalar_fields(shape, lattice, seed):
    """Seeded temperature (per padded node) and advecting velocity (interior)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    u = [0.04 * rng.standard_normal((nz, ny, nx)) for _ in range(3)]
    if lattice == 5:
        u[2][:] = 0.0
    return rng, [np.asarray(a, np.float32).astype(np.float64) for a in u]


def run_scalar(backend, case, seed, T_ref=0.0, omega_field=False, source=False):
    lat, op, shape, kind, om, steps, prec = case
    nx, ny, nz = shape
    per = SCALAR_PERIODIC[kind]
    s = O.ScalarCpuSolver(backend, lattice=lat, op=op, nx=nx, ny=ny, nz=nz, px=per[0],
                          py=per[1], pz=per[2], omega=om, T_ref=T_ref, precision=prec)
    cells, tw, codes, masks = scalar_geometry(lat, shape, kind)
    s.set_geometry(cells)
    s.set_wall_values(tw)
    if codes.any():
        s.set_specular_walls(codes)
    if masks.any():
        s.set_specular_nodes(masks)
    s.finalize_geometry()
    rng, u = scalar_fields(shape, lat, seed)
    s.set_velocity(*u)
    if omega_field:
        s.set_omega_field(np.asarray(om + 0.3 * rng.random((nz, ny, nx)), np.float32).astype(np.float64))
    T = np.asarray(0.5 + 0.2 * rng.standard_normal(s.n_padded), np.float32).astype(np.float64)
    s.initialize_field(T)
    f0 = s.field()
    dC = np.asarray(1e-3 * rng.standard_normal((nz, ny, nx)), np.float32).astype(np.float64)
    for t in range(steps):
        if source and t % 3 == 0:
            s.add_source(dC)
        s.step()
    stored = s.field()
    s.compute_field()
    out = {"field0": f0, "stored": stored, "field": s.field(), "total": s.total()}
    s.close()
    return out


# Thermal coupling: fluid (Boussinesq buoyancy, BoussinesqGuo) and scalar
# advected by the fluid, in the reference's loop order (fluid step storing u,
# then scalar step; validation/rayleigh_benard.cpp:178-188).  name ->
# (fluid lattice, fluid op, scalar lattice, scalar op, shape, steps, precision).
COUPLED_CASES = {
    "d2q9_bgk_d2q5_convection_f64": (9, "bgk", 5, "bgk", (12, 9, 1), 30, "f64"),
    "d3q27_cm_d3q7_convection_f32": (27, "cm", 7, "trt", (8, 7, 6), 20, "f32"),
}


def run_coupled(backend, case, seed):
    """Heated floor (T = 1) and cooled lid (T = 0) as scalar Dirichlet rows on
    the fluid's solid rows; periodic x (and z); buoyancy along +y."""
    flat, fop, slat, sop, shape, steps, prec = case
    nx, ny, nz = shape
    fl_kw = dict(lattice=flat, op=fop, shifted=1, nx=nx, ny=ny, nz=nz, px=True, py=False, pz=True,
                 omega=1.4, omega2=(1.1 if fop == "trt" else -1.0), precision=prec)
    fl = O.CpuSolver(backend, forcing=(2 if backend == "ref" else 1), **fl_kw)
    th = O.ScalarCpuSolver(backend, lattice=slat, op=sop, nx=nx, ny=ny, nz=nz, px=True, py=False,
                           pz=True, omega=1.2, precision=prec)
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
    rng = np.random.default_rng(seed)
    T = np.asarray(0.5 + 0.05 * rng.standard_normal(th.n_padded), np.float32).astype(np.float64)
    th.initialize_field(T)
    fl.initialize(1.0)
    g = (0.0, 1.0, 0.0)
    for _ in range(steps):
        fl.set_buoyancy(th.field(), g=g, rho0=1.0, beta=5e-3, T0=0.5)
        fl.step(1, store_macro=True)
        _, ux, uy, uz = fl.stored_macro()
        th.set_velocity(ux, uy, uz)
        th.step()
    stored_T = th.field()
    th.compute_field()
    out = {"pops": fl.gather(), "stored": np.stack(fl.stored_macro()), "macro": np.stack(fl.macro()),
           "T_stored": stored_T, "T": th.field(), "mass": fl.total_mass(), "total": th.total()}
    fl.close()
    th.close()
    return out


def main():
    if not O.ref_available("f64"):
        raise SystemExit("reference build missing: make -C oracle ref")
    O.set_ref_threads(1, "f64")
    O.set_ref_threads(1, "f32")
    for k, (name, case) in enumerate(CASES.items()):
        r = run("ref", case, seed=100 + k)
        np.savez_compressed(HERE / f"{name}.npz", case=np.array(repr(case)), seed=100 + k, **r)
        print(name, "mass", r["mass"])
    for k, (name, case) in enumerate(SPEC_CASES.items()):
        r = run_spec("ref", case, seed=200 + k)
        np.savez_compressed(HERE / f"{name}.npz", case=np.array(repr(case)), seed=200 + k, **r)
        print(name, "mass", r["mass"])
    for k, (name, case) in enumerate(SCALAR_CASES.items()):
        r = run_scalar("ref", case, seed=400 + k, T_ref=0.25, omega_field=k % 2 == 1, source=True)
        np.savez_compressed(HERE / f"{name}.npz", case=np.array(repr(case)), seed=400 + k, **r)
        print(name, "total", r["total"])
    for k, (name, case) in enumerate(COUPLED_CASES.items()):
        r = run_coupled("ref", case, seed=500 + k)
        np.savez_compressed(HERE / f"{name}.npz", case=np.array(repr(case)), seed=500 + k, **r)
        print(name, "mass", r["mass"])
    for k, (name, case) in enumerate(WALL_CASES.items()):
        r = run_wall("ref", case, seed=300 + k)
        np.savez_compressed(HERE / f"{name}.npz", case=np.array(repr(case)), seed=300 + k, **r)
        print(name, "mass", r["mass"])


if __name__ == "__main__":
    main()
