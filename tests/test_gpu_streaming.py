"""Streaming on the GPU: the Esoteric-Pull permutation, bit for bit.

Restates the reference's permutation test (tests/test_streaming.cpp:42-77):
tag every population with a unique value, disable collision, run T steps on a
periodic domain, and require every value to have moved exactly T * c_i.  Then
the same with walls and solid cells against the CPU oracle, slot for slot.
16-bit storage moves raw bit patterns, so those runs are bit-exact too.
"""
import numpy as np
import pytest

from m3lb_b200 import capi
from m3lb_b200 import solver as S
from tests.helpers import Case

pytestmark = pytest.mark.gpu


def _tags(dom, Q, storage):
    n = dom.n_padded * Q
    if storage in ("f16", "bf16", "f16c"):
        # unique finite 16-bit patterns (exponent field not all ones)
        pats = np.arange(1, 0x7000, dtype=np.uint16)
        assert n <= len(pats)
        return pats[:n].reshape(dom.n_padded, Q)
    return (np.arange(n, dtype=np.float64) + 1.0).reshape(dom.n_padded, Q)


def _permutation(lat, shape, steps, storage, node_kernel):
    L = S.D3Q27 if lat == 27 else S.D2Q9
    nx, ny, nz = shape
    dom = S.Domain(nx, ny, nz, True, True, True)
    s = S.FluidSolver(dom, S.NullCollision(L), storage=storage)
    if node_kernel:
        s.set_option(capi.OPT_NODE_KERNEL, 1)
    tags = _tags(dom, L.Q, storage)
    raw = storage in ("f16", "bf16", "f16c")
    if raw:
        s.seed_raw(tags)
    else:
        s.seed_populations(tags)
    s.steps(steps)
    got = s.gather_raw() if raw else s.gather_populations()
    bad = 0
    for z in range(nz):
        for y in range(ny):
            for x in range(nx):
                n = dom.id(x, y, z)
                for i in range(L.Q):
                    sx = (x - steps * L.cx[i]) % nx
                    sy = (y - steps * L.cy[i]) % ny
                    sz = (z - steps * L.cz[i]) % nz
                    if got[n, i] != tags[dom.id(sx, sy, sz), i]:
                        bad += 1
    s.close()
    return bad


# the reference's cases, plus shapes that exercise multi-chunk rows, partial
# chunks and the chunk-edge exchange of the paired kernel
CASES = [
    (9, (8, 6, 1), 1), (9, (8, 6, 1), 2), (9, (8, 6, 1), 7), (9, (8, 6, 1), 24),
    (27, (5, 4, 3), 1), (27, (5, 4, 3), 13),
    (27, (6, 4, 3), 1), (27, (6, 4, 3), 13),
    (27, (64, 3, 2), 3), (27, (130, 3, 2), 5), (27, (2, 3, 3), 4), (9, (128, 5, 1), 9),
    (9, (66, 3, 1), 4),
]


@pytest.mark.parametrize("lat,shape,steps", CASES)
@pytest.mark.parametrize("storage", ["f32", "f16", "bf16", "f64", "f16c"])
def test_permutation(cuda_device, lat, shape, steps, storage):
    assert _permutation(lat, shape, steps, storage, node_kernel=False) == 0


@pytest.mark.parametrize("lat,shape,steps", [(9, (8, 6, 1), 7), (27, (6, 4, 3), 13),
                                             (27, (130, 3, 2), 5)])
def test_permutation_node_kernel(cuda_device, lat, shape, steps):
    assert _permutation(lat, shape, steps, "f32", node_kernel=True) == 0


@pytest.mark.parametrize("storage", ["f32", "f16", "f64"])
@pytest.mark.parametrize("lat,shape,periodic", [
    (27, (10, 7, 5), (True, False, True)),    # walls in y through the halo
    (27, (9, 6, 5), (False, False, False)),   # closed box, odd nx: one-node kernel
    (9, (12, 9, 1), (True, False, True)),
])
def test_streaming_walls_match_oracle(cuda_device, storage, lat, shape, periodic):
    """Pure streaming with solid cells and halo walls: every logical
    population equal to the oracle's, bit for bit, after odd and even T."""
    c = Case(lat=lat, op=0, storage=storage, shape=shape, periodic=periodic)
    fl = np.zeros(c.shape, np.uint8)
    fl[..., 0, :] = 1
    fl.flat[len(fl.flat) // 2] = 1
    fl.flat[len(fl.flat) // 3] = 2
    c.geometry(fl)
    dom = c.dom
    rng = np.random.default_rng(1)
    vals = rng.integers(1, 2000, size=(dom.n_padded, c.coll.lattice.Q)).astype(np.float64) / 64.0
    c.gpu.seed_populations(vals)
    c.cpu.seed(vals)
    for t in (1, 2, 5):
        c.step(t)
        np.testing.assert_array_equal(c.gpu.gather_populations(), c.cpu.gather())
    c.close()
