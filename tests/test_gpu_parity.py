"""Collision parity on the GPU against the CPU oracle.

Every operator, equilibrium, storage format, storage convention and forcing
combination is run on the CUDA path and on the oracle (the reference's
algorithm restated in C, itself bit-identical to the reference build) from the
same random initial field, with walls and solid cells.  The oracle emulates
16-bit storage by rounding every stored value exactly as the GPU store does.

Tolerances (absolute, on populations after 8 steps), stated per storage unit
roundoff eps and the population scale s = max |population|:
    f64: 64 eps s          (reassociation and fused multiply-add only)
    f32: 64 eps s          (the reference's own cross-check uses 1e-6)
    f16, bf16: 4 eps s     (a rounding decision may flip by one ulp)
Macroscopic fields and the FP64 reductions use the same bound scaled to
their magnitude.  The paired and the one-node kernels must agree bit for bit.
"""
import itertools

import numpy as np
import pytest

from tests.helpers import EPS, Case

pytestmark = pytest.mark.gpu

OPS = [(1, 0), (1, 1), (2, 0), (2, 1), (3, 0), (4, 0)]
TOL_K = {"f64": 64.0, "f32": 64.0, "f16": 4.0, "bf16": 4.0, "f16c": 4.0}


def _tol(storage, scale):
    return TOL_K[storage] * EPS[storage] * max(scale, 1e-30)


def _cases():
    out = []
    for (op, eq), storage, shifted, forcing in itertools.product(
            OPS, ["f32", "f16", "bf16", "f64", "f16c"], [True, False], [False, True]):
        if storage in ("f16", "bf16", "f16c") and not shifted:
            continue
        out.append((op, eq, storage, shifted, forcing))
    return out


def _flags(shape):
    fl = np.zeros(shape, np.uint8)
    fl[..., 0, :] = 1            # a solid wall row
    fl.flat[len(fl.flat) // 2] = 1
    return fl


@pytest.mark.parametrize("lat", [27, 9])
@pytest.mark.parametrize("op,eq,storage,shifted,forcing", _cases())
def test_collision_matches_oracle(cuda_device, lat, op, eq, storage, shifted, forcing):
    shape = (16, 6, 5) if lat == 27 else (18, 10, 1)
    omega2 = 1.1 if op == 2 else (1.6 if op >= 3 else -1.0)
    c = Case(lat=lat, op=op, eq=eq, storage=storage, shifted=shifted, forcing=forcing,
             shape=shape, periodic=(True, False, True), omega2=omega2)
    c.geometry(_flags(c.shape))
    c.init_random(seed=op * 10 + eq)
    g0, o0 = c.gpu.gather_populations(), c.cpu.gather()
    scale = float(np.max(np.abs(o0)))
    # initial state: the seeding arithmetic is the reference's, in the same order
    assert np.max(np.abs(g0 - o0)) <= _tol(storage, scale)
    c.step(8, store=True)
    g, o = c.gpu.gather_populations(), c.cpu.gather()
    err = float(np.max(np.abs(g - o)))
    assert err <= _tol(storage, scale), f"populations differ by {err:.3e}"

    # Derived fields: rho and u are sums of Q populations, so their bound is
    # Q times the population bound plus the arithmetic's own rounding.
    Q = lat
    ar = EPS["f64"] if storage == "f64" else EPS["f32"]
    pop_tol = _tol(storage, scale)
    for a, b in zip(c.gpu.stored_macroscopic(), c.cpu.stored_macro()):
        sc = max(float(np.max(np.abs(b))), 1e-3)
        assert float(np.max(np.abs(a - b))) <= Q * pop_tol / 0.9 + 64 * ar * sc
    for a, b in zip(c.gpu.compute_macroscopic(), c.cpu.macro()):
        sc = max(float(np.max(np.abs(b))), 1e-3)
        assert float(np.max(np.abs(a - b))) <= Q * pop_tol / 0.9 + 64 * ar * sc

    # FP64 device reductions against the oracle's sums (which accumulate in
    # the arithmetic type, hence the sqrt(n) summation term)
    red = c.gpu.reduce()
    nf = float(np.sum(c.gpu.flags() == 0))
    sum_err = 8 * ar * nf * np.sqrt(nf)
    assert abs(red[0] - c.cpu.total_mass()) <= nf * Q * pop_tol + sum_err
    for a in range(3 if lat == 27 else 2):
        assert abs(red[1 + a] - c.cpu.total_momentum(a)) <= nf * Q * pop_tol + 0.1 * sum_err
    assert abs(red[5] - c.cpu.slot_sum()) <= c.dom.n_padded * Q * pop_tol + 1e-12 * nf * Q
    c.close()


@pytest.mark.parametrize("lat", [27, 9])
@pytest.mark.parametrize("op,eq", OPS)
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64", "f16c"])
def test_pair_kernel_equals_node_kernel(cuda_device, lat, op, eq, storage):
    """The paired kernel (f32x2 arithmetic, warp exchange) and the one-node
    kernel run the same sequence of rounded operations: identical stored bits
    and stored macroscopic fields for every operator (the moment operators'
    one product that the compiler could fuse into a sum in the paired kernel
    only is written as an explicit FMA)."""
    shape = (130, 4, 3) if lat == 27 else (130, 6, 1)
    a = Case(lat=lat, op=op, eq=eq, storage=storage, forcing=True, shape=shape,
             periodic=(True, False, True), omega2=1.1 if op == 2 else -1.0)
    b = Case(lat=lat, op=op, eq=eq, storage=storage, forcing=True, shape=shape,
             periodic=(True, False, True), omega2=1.1 if op == 2 else -1.0, node_kernel=True)
    fl = _flags(a.shape)
    a.gpu.set_geometry(fl)
    b.gpu.set_geometry(fl)
    rng = np.random.default_rng(3)
    fields = [1 + 0.01 * rng.standard_normal(a.shape)] + \
             [0.03 * rng.standard_normal(a.shape) for _ in range(3)]
    a.gpu.initialize_field(fields)
    b.gpu.initialize_field(fields)
    a.gpu.steps(5, True)
    b.gpu.steps(5, True)
    np.testing.assert_array_equal(a.gpu.gather_raw(), b.gpu.gather_raw())
    for x, y in zip(a.gpu.stored_macroscopic(), b.gpu.stored_macroscopic()):
        np.testing.assert_array_equal(x, y)
    a.close()
    b.close()


@pytest.mark.parametrize("storage", ["f32", "f64"])
def test_init_eq_matches_oracle(cuda_device, storage):
    """initialize(rho0, u0) with halo walls: the clamped halo writes of the
    reference's sequential scatter are reproduced (highest node wins)."""
    c = Case(lat=27, op=1, storage=storage, shape=(6, 5, 4), periodic=(False, False, True))
    fl = _flags(c.shape)
    c.geometry(fl)
    c.gpu.initialize(1.01, 0.03, -0.02, 0.01)
    c.cpu.initialize(1.01, 0.03, -0.02, 0.01)
    np.testing.assert_array_equal(c.gpu.gather_populations(), c.cpu.gather())
    c.close()


STREAM_SHAPES = [(27, (64, 5, 4)), (27, (192, 3, 3)), (27, (130, 4, 3)), (27, (2, 5, 4)),
                 (9, (70, 6, 1))]


@pytest.mark.parametrize("lat,shape", STREAM_SHAPES)
@pytest.mark.parametrize("op", [0, 1, 2, 4])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64", "f16c"])
def test_streamed_kernel_equals_paired_kernel(cuda_device, storage, lat, shape, op):
    """The persistent copy-pipelined kernel and the paired kernel: identical
    stored bits after several steps, on full, multi-chunk, partial-chunk and
    two-node rows, with walls and solid cells."""
    from m3lb_b200 import capi

    cases = []
    for kern in (capi.KERNEL_PAIRS, capi.KERNEL_STREAM):
        c = Case(lat=lat, op=op, storage=storage, forcing=True, shape=shape,
                 periodic=(True, False, True), omega2=1.1 if op == 2 else -1.0)
        c.gpu.set_option(capi.OPT_KERNEL, kern)
        c.gpu.set_geometry(_flags(c.shape))
        rng = np.random.default_rng(11)
        c.gpu.initialize_field([1 + 0.01 * rng.standard_normal(c.shape)] +
                               [0.03 * rng.standard_normal(c.shape) for _ in range(3)])
        c.gpu.steps(7, True)
        cases.append(c)
    np.testing.assert_array_equal(cases[0].gpu.gather_raw(), cases[1].gpu.gather_raw())
    if op != 0:
        for x, y in zip(cases[0].gpu.stored_macroscopic(), cases[1].gpu.stored_macroscopic()):
            np.testing.assert_array_equal(x, y)
    for c in cases:
        c.close()


# the last four have a partial last chunk (lanes past nx store nothing)
ROWS_SHAPES = [(27, (64, 5, 4)), (27, (128, 4, 3)), (27, (192, 3, 3)), (27, (256, 2, 3)),
               (9, (128, 6, 1)), (27, (160, 3, 3)), (27, (208, 2, 3)), (27, (96, 4, 3)),
               (9, (146, 6, 1))]


@pytest.mark.parametrize("lat,shape", ROWS_SHAPES)
@pytest.mark.parametrize("op", [0, 1, 2, 3, 4])
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64", "f16c"])
def test_row_kernel_equals_paired_kernel(cuda_device, storage, lat, shape, op):
    """The TMA row kernel (whole rows through shared memory) and the paired
    kernel: identical stored bits after several steps, one to four chunks per
    row, with walls (non-periodic y) and solid cells."""
    from m3lb_b200 import capi

    cases = []
    for kern in (capi.KERNEL_PAIRS, capi.KERNEL_ROWS):
        c = Case(lat=lat, op=op, storage=storage, forcing=True, shape=shape,
                 periodic=(True, False, True), omega2=1.1 if op == 2 else -1.0)
        c.gpu.set_option(capi.OPT_KERNEL, kern)
        c.gpu.set_geometry(_flags(c.shape))
        rng = np.random.default_rng(12)
        c.gpu.initialize_field([1 + 0.01 * rng.standard_normal(c.shape)] +
                               [0.03 * rng.standard_normal(c.shape) for _ in range(3)])
        c.gpu.steps(7, True)
        c.gpu.sync()
        cases.append(c)
    np.testing.assert_array_equal(cases[0].gpu.gather_raw(), cases[1].gpu.gather_raw())
    if op != 0:
        for x, y in zip(cases[0].gpu.stored_macroscopic(), cases[1].gpu.stored_macroscopic()):
            np.testing.assert_array_equal(x, y)
    for c in cases:
        c.close()


def _kernels_equal(kernels, lat, shape, op, eq, storage, forcing, periodic, steps=7, seed=13):
    """Run the same lattice under each kernel choice and require identical
    stored bits and identical stored macroscopic fields."""
    from m3lb_b200 import capi

    cases = []
    for kern in kernels:
        c = Case(lat=lat, op=op, eq=eq, storage=storage, forcing=forcing, shape=shape,
                 periodic=periodic, omega2=1.1 if op == 2 else -1.0)
        c.gpu.set_option(capi.OPT_KERNEL, kern)
        if not all(periodic):
            c.gpu.set_geometry(_flags(c.shape))
        rng = np.random.default_rng(seed)
        c.gpu.initialize_field([1 + 0.01 * rng.standard_normal(c.shape)] +
                               [0.03 * rng.standard_normal(c.shape) for _ in range(3)])
        c.gpu.steps(steps, True)
        c.gpu.sync()
        cases.append(c)
    ref = cases[0].gpu.gather_raw()
    for c in cases[1:]:
        np.testing.assert_array_equal(ref, c.gpu.gather_raw())
        if op != 0:
            for x, y in zip(cases[0].gpu.stored_macroscopic(), c.gpu.stored_macroscopic()):
                np.testing.assert_array_equal(x, y)
    for c in cases:
        c.close()


VARIANT_SHAPES = [(27, (128, 4, 3)), (27, (160, 3, 3)), (27, (256, 2, 2)), (9, (128, 6, 1))]


@pytest.mark.parametrize("lat,shape", VARIANT_SHAPES)
@pytest.mark.parametrize("op,eq", OPS)
@pytest.mark.parametrize("forcing", [False, True])
@pytest.mark.parametrize("periodic", [(True, True, True), (True, False, True)],
                         ids=["periodic", "ywalls"])
@pytest.mark.parametrize("storage", ["f16", "bf16", "f16c"])
def test_auto_kernels_equal_paired_kernel(cuda_device, storage, periodic, forcing, op, eq,
                                          lat, shape):
    """Every operator instantiation that the automatic choice sends to the row
    kernel or the streamed kernel (16-bit storage: BGK, TRT, MRT, CM; both
    equilibria; forced and unforced; a fully periodic lattice, whose rows wrap
    in y through the row kernel's neighbour-row copies, and one with walls)
    gives the paired kernel's bits."""
    from m3lb_b200 import capi

    _kernels_equal([capi.KERNEL_PAIRS, capi.KERNEL_ROWS, capi.KERNEL_STREAM, capi.KERNEL_AUTO],
                   lat, shape, op, eq, storage, forcing, periodic)


@pytest.mark.parametrize("lat,shape", [(9, (6, 70000, 1)), (27, (4, 300, 250))])
def test_rows_beyond_one_grid_dimension(cuda_device, lat, shape):
    """More rows (y, z pairs) than one grid dimension holds (65535): the
    per-node kernels (one-node step, seed, gather, macroscopic readout,
    reduction) stride over rows.  A non-periodic x axis selects the one-node
    step kernel."""
    op = 4 if lat == 27 else 1
    c = Case(lat=lat, op=op, storage="f32", shape=shape, periodic=(False, True, True),
             omega2=1.6 if op == 4 else -1.0)
    c.init_random(seed=5)
    o0 = c.cpu.gather()
    scale = float(np.max(np.abs(o0)))
    tol = _tol("f32", scale)
    assert np.max(np.abs(c.gpu.gather_populations() - o0)) <= tol
    c.step(3, store=True)
    assert float(np.max(np.abs(c.gpu.gather_populations() - c.cpu.gather()))) <= tol
    ar = EPS["f32"]
    for a, b in zip(c.gpu.compute_macroscopic(), c.cpu.macro()):
        sc = max(float(np.max(np.abs(b))), 1e-3)
        assert float(np.max(np.abs(a - b))) <= lat * tol / 0.9 + 64 * ar * sc
    red = c.gpu.reduce()
    nf = float(np.prod(shape))
    assert abs(red[0] - c.cpu.total_mass()) <= nf * lat * tol + 8 * ar * nf * np.sqrt(nf)
    assert abs(red[5] - c.cpu.slot_sum()) <= c.dom.n_padded * lat * tol + 1e-12 * nf * lat
    c.close()


@pytest.mark.parametrize("nx", [256, 128])
def test_row_kernel_wait_that_runs_out_is_reported(cuda_device, nx):
    """The row kernel's waits for a row's copies are bounded.  With the
    consume wait cut to one clock cycle (a test-only option; the drain of the
    copies still in flight keeps its full limit), CTAs give up on rows whose
    copies have not landed yet: the kernel records a status instead of
    hanging, and the next m3lb_sync returns it as an error, once.  The handle
    stays usable: with the default limit restored and the lattice seeded
    again, a step is clean.  nx = 256: rows of 4 chunks moved by a copy
    warp; nx = 128: rows of 2 chunks moved by the update warps themselves."""
    from m3lb_b200 import capi

    c = Case(lat=27, op=4, storage="f16", shape=(nx, 16, 16), periodic=(True, True, True))
    c.gpu.set_option(capi.OPT_KERNEL, capi.KERNEL_ROWS)
    c.gpu.initialize(1.0, 0.01, 0.0, 0.0)
    c.gpu.sync()
    c.gpu.set_option(capi.OPT_WAIT_CYCLES, 1)
    c.gpu.steps(2)
    with pytest.raises(capi.M3lbError, match="gave up waiting"):
        c.gpu.sync()
    c.gpu.sync()  # reported once
    c.gpu.set_option(capi.OPT_WAIT_CYCLES, 0)
    c.gpu.initialize(1.0, 0.01, 0.0, 0.0)
    c.gpu.steps(2)
    c.gpu.sync()
    assert np.isfinite(c.gpu.reduce()).all()
    c.close()
