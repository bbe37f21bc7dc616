"""One test case on both sides: the CUDA path (m3lb_b200) and the CPU oracle."""
from __future__ import annotations

import numpy as np

import oracle as O
from m3lb_b200 import capi
from m3lb_b200 import solver as S

LATS = {9: S.D2Q9, 27: S.D3Q27}
OPNAMES = {0: "none", 1: "bgk", 2: "trt", 3: "mrt", 4: "cm"}
# storage -> (oracle precision, oracle storage rounding)
ORACLE_PREC = {"f32": ("f32", None), "f16": ("f32", "f16"), "bf16": ("f32", "bf16"),
               "f64": ("f64", None), "f16c": ("f32", "f16c")}


def make_collision(lat, op, eq=0, shifted=True, forcing=False, omega=1.3, omega2=-1.0,
                   F=(2e-5, -1e-5, 3e-6)):
    L = LATS[lat]
    fo = S.Guo(*F) if forcing else S.NoForcing()
    st = S.ShiftedPopulations if shifted else S.RawPopulations
    eqc = S.ProductFormEquilibrium if eq else S.SecondOrderEquilibrium
    if op == 0:
        return S.NullCollision(L, fo, st)
    if op == 1:
        return S.BGK(L, eqc, fo, st, omega=omega)
    if op == 2:
        return S.TRT(L, eqc, fo, st, omega_p=omega, omega_m=omega2)
    return S.MomentCollision(L, fo, st, central=(op == 4), omega=omega, omega_bulk=omega2)


class Case:
    def __init__(self, lat=27, op=4, eq=0, storage="f32", shifted=True, forcing=False,
                 shape=(16, 6, 5), periodic=(True, True, True), omega=1.3, omega2=-1.0,
                 F=(2e-5, -1e-5, 3e-6), node_kernel=False):
        nx, ny, nz = shape
        if lat == 9:
            nz = 1
            F = (F[0], F[1], 0.0)
        self.lat, self.op, self.storage = lat, op, storage
        self.shape = (nz, ny, nx)
        self.coll = make_collision(lat, op, eq, shifted, forcing, omega, omega2, F)
        self.dom = S.Domain(nx, ny, nz, *periodic)
        self.gpu = S.FluidSolver(self.dom, self.coll, storage=storage)
        if node_kernel:
            self.gpu.set_option(capi.OPT_NODE_KERNEL, 1)
        prec, quant = ORACLE_PREC[storage]
        self.cpu = O.CpuSolver("oracle", lattice=lat, op=OPNAMES[op], eq=eq, shifted=shifted,
                               forcing=forcing, nx=nx, ny=ny, nz=nz, px=periodic[0],
                               py=periodic[1], pz=periodic[2], omega=omega, omega2=omega2,
                               fx=F[0] if forcing else 0.0, fy=F[1] if forcing else 0.0,
                               fz=F[2] if forcing else 0.0, precision=prec, quant=quant)

    def geometry(self, flags):
        self.gpu.set_geometry(flags)
        self.cpu.set_geometry(flags)

    def specular(self, codes=None, masks=None):
        """Free-slip walls on both sides: normal codes (SpecWall) and face
        masks (SpecNode) per interior node, (nz, ny, nx)."""
        if codes is not None and np.any(codes):
            self.gpu.set_specular_walls(codes)
            self.cpu.set_specular_walls(codes)
        if masks is not None and np.any(masks):
            self.gpu.set_specular_nodes(masks)
            self.cpu.set_specular_nodes(masks)

    def regularized(self, codes, states=None):
        """Regularised walls on both sides (codes per interior node, states
        (nz, ny, nx, 4) or None)."""
        self.gpu.set_regularized_walls(codes, states)
        self.cpu.set_regularized_walls(codes, states)

    def both(self, name, *args):
        """Call the same setter on the device solver and the oracle."""
        getattr(self.gpu, name)(*args)
        getattr(self.cpu, name)(*args)

    def init_random(self, seed=0, amp=0.03):
        rng = np.random.default_rng(seed)
        rho = 1 + 0.01 * rng.standard_normal(self.shape)
        u = [amp * rng.standard_normal(self.shape) for _ in range(3)]
        if self.lat == 9:
            u[2] = np.zeros(self.shape)
        # values representable in the arithmetic type so both sides start alike
        real = np.float64 if self.storage == "f64" else np.float32
        rho, *u = [np.asarray(a, real).astype(np.float64) for a in [rho] + u]
        self.gpu.initialize_field((rho, *u))
        self.cpu.initialize_field(rho, *u)

    def step(self, n=1, store=False):
        self.gpu.steps(n, store)
        self.cpu.step(n, store)

    def close(self):
        self.gpu.close()
        self.cpu.close()


# Storage unit roundoff, for tolerances.
EPS = {"f64": 2.0 ** -53, "f32": 2.0 ** -24, "f16": 2.0 ** -11, "bf16": 2.0 ** -8,
       "f16c": 2.0 ** -12}
