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
    for k, (name, case) in enumerate(WALL_CASES.items()):
        r = run_wall("ref", case, seed=300 + k)
        np.savez_compressed(HERE / f"{name}.npz", case=np.array(repr(case)), seed=300 + k, **r)
        print(name, "mass", r["mass"])


if __name__ == "__main__":
    main()
