"""Channel flow past a square block: D3Q27 TRT, the workload's fourth case.

384 x 128 x 128 nodes, periodic in x; the y and z axes are not periodic, so
their halo nodes (Excluded) close the channel with halfway bounce-back
walls; a solid 24 x 24 block spans z at x in [96, 120), y in [52, 76)
(centred); Guo body force g_x = 2e-6; TRT with the magic parameter 3/16.
The case states no relaxation time: tau+ = 0.8 (nu = 0.1), the Poiseuille
case's value.

  * At 1/8 scale (48 x 16 x 16, block 3 x 3 x 16 at x = 12, y = 6..8), the
    device matches the oracle populations, fields and sums (FP32 storage).
  * At full size, 5000 steps: FP32 and FP16 storage (FP32 arithmetic)
    against FP64 storage, relative L2 and max of the velocity and of
    rho - 1; FP64 mass drift; and the z mirror symmetry of the geometry
    holding in the FP64 field.
"""
import numpy as np
import pytest

from m3lb_b200 import solver as S
from tests.helpers import EPS, Case

pytestmark = pytest.mark.gpu

TAU = 0.8
OMEGA = 1.0 / TAU
OMEGA_M = S.TRT.omega_minus_for(OMEGA, S.TRT.magic_3_16)
G = 2e-6


def _block(nx, ny, nz, x0, x1, y0, y1):
    flags = np.zeros((nz, ny, nx), np.uint8)
    flags[:, y0:y1, x0:x1] = 1
    return flags


def test_block_channel_matches_oracle_at_small_scale(cuda_device):
    c = Case(lat=27, op=2, storage="f32", forcing=True, shape=(48, 16, 16),
             periodic=(True, False, False), omega=OMEGA, omega2=OMEGA_M, F=(G, 0.0, 0.0))
    c.geometry(_block(48, 16, 16, 12, 15, 6, 9))
    c.both("initialize", 1.0, 0.0, 0.0, 0.0)
    c.step(300, store=True)
    g, o = c.gpu.gather_populations(), c.cpu.gather()
    scale = float(np.max(np.abs(o)))
    tol = 16 * EPS["f32"] * scale * 300 ** 0.5
    assert float(np.max(np.abs(g - o))) <= tol
    for a, b in zip(c.gpu.compute_macroscopic(), c.cpu.macro()):
        assert float(np.max(np.abs(a - b))) <= 27 * tol + 64 * EPS["f32"]
    red = c.gpu.reduce()
    nf = float(np.sum(c.gpu.flags() == 0))
    assert abs(red[0] - c.cpu.total_mass()) <= nf * 27 * tol + 8 * EPS["f32"] * nf ** 1.5
    assert red[1] > 0  # the force drives +x momentum
    c.close()


def _run_full(storage, steps=5000):
    nx, ny, nz = 384, 128, 128
    coll = S.TRT(S.D3Q27, S.SecondOrderEquilibrium, S.Guo(G, 0.0, 0.0), S.ShiftedPopulations,
                 omega_p=OMEGA, omega_m=OMEGA_M)
    s = S.FluidSolver(S.Domain(nx, ny, nz, True, False, False), coll, storage=storage)
    s.set_geometry(_block(nx, ny, nz, 96, 120, 52, 76))
    s.initialize(1.0)
    r0 = s.reduce()
    s.steps(steps)
    r1 = s.reduce()
    rho, ux, uy, uz = s.compute_macroscopic()
    solid = s.flags() != 0
    s.close()
    return rho, ux, uy, uz, solid, r0, r1


def test_block_channel_full_size_precisions(cuda_device):
    rho, ux, uy, uz, solid, r0, r1 = _run_full("f64")
    fluid = ~solid
    # the sum over every stored slot is conserved (bounce-back and Guo add no
    # mass); the fluid nodes' rho alone is not, since populations on their way
    # back from a wall sit in wall slots between steps
    n_slots = 384 * 130 * 130 * 27
    print(f"f64: slot-sum drift {r1[5] - r0[5]:.3e}, fluid-mass change {(r1[0] - r0[0]) / r0[0]:.3e}")
    assert abs(r1[5] - r0[5]) <= 1e-16 * n_slots
    assert abs(r1[0] - r0[0]) <= 1e-6 * r0[0]
    assert float(ux[fluid].mean()) > 0
    # the geometry is symmetric under z -> nz - 1 - z
    amp = float(np.max(np.abs(ux)))
    assert float(np.max(np.abs(ux - ux[::-1]))) <= 1e-9 * amp
    assert float(np.max(np.abs(uz + uz[::-1]))) <= 1e-9 * amp
    u64 = np.stack([ux[fluid], uy[fluid], uz[fluid]])
    r64 = rho[fluid] - 1.0
    for storage, bound in (("f32", 1e-4), ("f16", 2e-2)):
        r, x, y, z, _, _, _ = _run_full(storage)
        u = np.stack([x[fluid], y[fluid], z[fluid]])
        l2 = float(np.linalg.norm(u - u64) / np.linalg.norm(u64))
        mx = float(np.max(np.abs(u - u64)) / np.max(np.abs(u64)))
        l2r = float(np.linalg.norm((r[fluid] - 1.0) - r64) / np.linalg.norm(r64))
        print(f"{storage}: velocity rel L2 {l2:.3e} max {mx:.3e}; rho-1 rel L2 {l2r:.3e}")
        assert l2 <= bound and mx <= 10 * bound
