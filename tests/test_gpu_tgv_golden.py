"""The reference's own 3-D Taylor-Green trajectory, reproduced on the GPU.

The reference ships the output of validation/tgv3d.cpp (copied to
tests/golden/tgv3d_re1600_d3q27_cm.txt by make_tgv_golden.py): D3Q27 central
moments on shifted populations in FP64, a periodic 64^3 box with
ux = u0 cos x sin y sin z, uy = -u0/2 sin x cos y sin z,
uz = -u0/2 sin x sin y cos z, u0 = 0.02, Re = 1600 (nu = u0 D / Re,
tau = 0.5024), 32000 steps, kinetic energy and enstrophy (central-difference
vorticity, validation/Campaign.hpp:96-131) every 1600 steps, normalised by
their initial values.  The same run through FluidSolver:
  * FP64 storage matches every printed value (nine digits) to 2e-8;
  * FP32 storage with FP32 arithmetic stays within 2e-4, FP16 storage
    within 1e-2, FP16C storage (one more mantissa bit) within 5e-3:
    precision changes the storage, not the scheme.
(BF16 storage leaves the trajectory at this amplitude: its 8-bit mantissa is
coarser than the shifted populations' variation, and the decay stalls.)
"""
from pathlib import Path

import numpy as np
import pytest

from m3lb_b200 import solver as S

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "tgv3d_re1600_d3q27_cm.txt"
D, RE, U0, TMAX = 64, 1600.0, 0.02, 10.0


def _diagnostics(s):
    """Energy and enstrophy as validation/Campaign.hpp:96-131 sums them."""
    ux, uy, uz = s.compute_macroscopic()[1:]  # (z, y, x)
    e = 0.5 * float(np.sum(ux * ux + uy * uy + uz * uz))

    def d(a, axis):  # central difference with periodic wrap
        return 0.5 * (np.roll(a, -1, axis) - np.roll(a, 1, axis))

    wz = d(uy, 2) - d(ux, 1)
    wx = d(uz, 1) - d(uy, 0)
    wy = d(ux, 0) - d(uz, 2)
    return e, 0.5 * float(np.sum(wx * wx + wy * wy + wz * wz))


def _trajectory(storage):
    nu = U0 * D / RE
    omega = 1.0 / (nu * 3.0 + 0.5)  # omega_from_viscosity, MomentCollision.hpp:93-95
    T = int(TMAX * D / U0)
    probe = T // 20
    s = S.FluidSolver(S.Domain(D, D, D, True, True, True),
                      S.CentralMoments(S.D3Q27, S.NoForcing(), S.ShiftedPopulations, omega=omega),
                      storage=storage)
    k = 2.0 * np.pi / D

    def field(x, y, z):
        X, Y, Z = k * x, k * y, k * z
        return (1.0, U0 * np.cos(X) * np.sin(Y) * np.sin(Z),
                -0.5 * U0 * np.sin(X) * np.cos(Y) * np.sin(Z),
                -0.5 * U0 * np.sin(X) * np.sin(Y) * np.cos(Z))

    s.initialize_field(field)
    e0, w0 = _diagnostics(s)
    rows = [(0.0, 1.0, 1.0)]
    for j in range(1, 21):
        s.steps(probe)
        e, w = _diagnostics(s)
        rows.append((TMAX * j * probe / T, e / e0, w / w0))
    s.close()
    return np.array(rows)


@pytest.mark.parametrize("storage,rtol", [("f64", 2e-8), ("f32", 2e-4), ("f16", 1e-2),
                                          ("f16c", 5e-3)])
def test_taylor_green_matches_reference_trajectory(cuda_device, storage, rtol):
    gold = np.loadtxt(GOLD)
    got = _trajectory(storage)
    assert got.shape == gold.shape
    np.testing.assert_allclose(got[:, 0], gold[:, 0], rtol=0, atol=1e-6)
    np.testing.assert_allclose(got[:, 1], gold[:, 1], rtol=rtol)   # E / E0
    np.testing.assert_allclose(got[:, 2], gold[:, 2], rtol=rtol)   # Psi / Psi0
