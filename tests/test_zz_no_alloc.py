"""m3lb_reduce_static against m3lb_reduce, through the C ABI.

m3lb_reduce_static serves callers that cannot allocate device memory: it
takes the population array and flags they hold and keeps its partial sums in
a fixed array inside the library.  Here the arrays come from an ordinary
handle, and the sums of two consecutive calls (at time steps 3 and 6, so both
Esoteric-Pull parities, the second over partials the first call left behind)
must equal m3lb_reduce's bit for bit: both run the same kernels with the same
block count and summation order.  This file sorts last so that a run stopping
at its first failure has run every other test already.
"""
import ctypes as C

import numpy as np
import pytest

from m3lb_b200 import capi
from m3lb_b200 import solver as S

pytestmark = pytest.mark.gpu


def _padded_flags(dom, interior):
    fl = np.full((dom.sz, dom.sy, dom.sx), 2, np.uint8)
    fl[dom.hz:dom.hz + dom.nz, dom.hy:dom.hy + dom.ny, dom.hx:dom.hx + dom.nx] = interior
    return fl


@pytest.mark.parametrize("storage,lat,op,shape,periodic", [
    ("f16", 27, capi.OP_CM, (40, 24, 20), (True, False, True)),
    ("f32", 27, capi.OP_TRT, (33, 16, 12), (False, False, True)),
    ("f64", 9, capi.OP_BGK, (96, 40, 1), (True, False, True)),
])
def test_reduce_static_matches_reduce(cuda_device, storage, lat, op, shape, periodic):
    import torch

    L = S.D3Q27 if lat == 27 else S.D2Q9
    F = (2e-5, -1e-5, 3e-6 if lat == 27 else 0.0)
    if op == capi.OP_CM:
        coll = S.MomentCollision(L, S.Guo(*F), S.ShiftedPopulations, central=True, omega=1.7)
    elif op == capi.OP_TRT:
        coll = S.TRT(L, S.SecondOrderEquilibrium, S.Guo(*F), S.ShiftedPopulations,
                     omega_p=1.5, omega_m=1.2)
    else:
        coll = S.BGK(L, S.SecondOrderEquilibrium, S.Guo(*F), S.RawPopulations, omega=1.25)
    dom = S.Domain(*shape, *periodic)
    s = S.FluidSolver(dom, coll, storage=storage)
    flags = np.zeros((dom.nz, dom.ny, dom.nx), np.uint8)
    flags[:, 0, :] = 1
    flags.flat[flags.size // 2] = 1
    s.set_geometry(flags)
    rng = np.random.default_rng(7)
    sh = (dom.nz, dom.ny, dom.nx)
    s.initialize_field([1 + 0.01 * rng.standard_normal(sh)] +
                       [0.03 * rng.standard_normal(sh) for _ in range(3)])
    dev_flags = torch.from_numpy(_padded_flags(dom, flags)).to(cuda_device)
    out = torch.full((6,), float("nan"), dtype=torch.float64, device=cuda_device)
    pops, _ = s.populations()
    lib = capi.lib()

    for steps in (3, 3):  # two calls in a row, at t = 3 (odd) and t = 6 (even)
        s.steps(steps)
        s.sync()
        want = s.reduce()
        rc = lib.m3lb_reduce_static(lat, dom.nx, dom.ny, dom.nz, *[int(p) for p in periodic],
                                    coll.op, s.storage, int(coll.storage.shifted), 1,
                                    F[0], F[1], F[2], C.c_void_p(pops),
                                    C.c_void_p(dev_flags.data_ptr()), s.timestep(), None,
                                    C.c_void_p(out.data_ptr()))
        assert rc == capi.OK, capi.last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.array_equal(got, want), (s.timestep(), got, want)
    s.close()


def test_reduce_static_rejects_large_lattice(cuda_device):
    """Beyond the fixed scratch (4,194,304 interior nodes) the call fails with
    a message instead of touching memory."""
    import torch

    lib = capi.lib()
    pops = torch.zeros(64, dtype=torch.float16, device=cuda_device)
    out = torch.zeros(6, dtype=torch.float64, device=cuda_device)
    rc = lib.m3lb_reduce_static(27, 256, 256, 256, 1, 1, 1, capi.OP_CM, capi.STORE_F16, 1, 0,
                                0.0, 0.0, 0.0, C.c_void_p(pops.data_ptr()), None, 0, None,
                                C.c_void_p(out.data_ptr()))
    assert rc == capi.ERR_INVALID
    assert "fixed scratch" in capi.last_error()
