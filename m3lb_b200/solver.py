"""Python mirror of the reference's solver / collision-policy API, on libm3lb.

The names, defaults and argument meanings follow M3LB's C++ headers
(src/lattice/Lattices.hpp, src/grid/Domain.hpp, src/memory/*,
src/collision/{BGK,TRT,MomentCollision}.hpp, src/forcing/Forcing.hpp,
src/boundary/Flags.hpp, src/solver/FluidSolver.hpp), so a reference test or
driver reads the same here.  Compile-time policies there become constructor
arguments here; every time step runs in one fused CUDA kernel on the device.

Added over the reference: the storage precision of the populations
(``storage="f32" | "f16" | "f16c" | "bf16" | "f64"``; arithmetic is FP32, or
FP64 for "f64"; "f16c" is a 16-bit float with one more mantissa bit than
IEEE binary16, include/m3lb.h M3LB_STORE_F16C), and a CUDA stream to queue
the work on.
"""
from __future__ import annotations

import ctypes as C
import enum
from dataclasses import dataclass, field

import numpy as np

from . import capi

# ---------------------------------------------------------------- lattices
# Lattices.hpp:75-159: rest first, opposite directions at adjacent indices.


class D2Q9:
    name = "D2Q9"
    D, Q = 2, 9
    cs2 = 1.0 / 3.0
    cx = (0, 1, -1, 0, 0, 1, -1, 1, -1)
    cy = (0, 0, 0, 1, -1, 1, -1, -1, 1)
    cz = (0,) * 9
    w = tuple(v / 36.0 for v in (16, 4, 4, 4, 4, 1, 1, 1, 1))


class D3Q27:
    name = "D3Q27"
    D, Q = 3, 27
    cs2 = 1.0 / 3.0
    cx = (0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, -1, 1)
    cy = (0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, 1, -1)
    cz = (0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, 1, -1)
    w = tuple(v / 216.0 for v in (64, 16, 16, 16, 16, 16, 16, 4, 4, 4, 4, 4, 4, 4,
                                  4, 4, 4, 4, 4, 1, 1, 1, 1, 1, 1, 1, 1))


class D2Q5:
    """Scalar lattice (Lattices.hpp:51-70): advection-diffusion only."""
    name = "D2Q5"
    D, Q = 2, 5
    cs2 = 1.0 / 3.0
    cx = (0, 1, -1, 0, 0)
    cy = (0, 0, 0, 1, -1)
    cz = (0,) * 5
    w = tuple(v / 6.0 for v in (2, 1, 1, 1, 1))


class D3Q7:
    """Scalar lattice (Lattices.hpp:100-121): cs2 = 1/4, not 1/3."""
    name = "D3Q7"
    D, Q = 3, 7
    cs2 = 1.0 / 4.0
    cx = (0, 1, -1, 0, 0, 0, 0)
    cy = (0, 0, 0, 1, -1, 0, 0)
    cz = (0, 0, 0, 0, 0, 1, -1)
    w = tuple(v / 8.0 for v in (2, 1, 1, 1, 1, 1, 1))


def opp(i: int) -> int:
    """Esoteric-Pull pairing rule (Lattices.hpp:43-45)."""
    return 0 if i == 0 else (i + 1 if i & 1 else i - 1)


# ---------------------------------------------------------------- domain
class Domain:
    """Cartesian block (Domain.hpp:37-123): halo only along non-periodic axes,
    padded index idp = (pz*sy + py)*sx + px."""

    def __init__(self, nx, ny, nz=1, px=True, py=True, pz=True, mpi_halo=0):
        if mpi_halo:
            raise NotImplementedError("mpi_halo: distributed slabs are not offered")
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.periodic = [bool(px), bool(py), bool(pz)]

        def halo(n, per):
            return 0 if n <= 1 else (0 if per else 1)

        self.hx, self.hy, self.hz = halo(nx, px), halo(ny, py), halo(nz, pz)
        self.sx, self.sy, self.sz = nx + 2 * self.hx, ny + 2 * self.hy, nz + 2 * self.hz
        self.n_padded = self.sx * self.sy * self.sz

    def n_interior(self):
        return self.nx * self.ny * self.nz

    def idp(self, px, py, pz=0):
        return (pz * self.sy + py) * self.sx + px

    def id(self, x, y, z=0):
        return self.idp(x + self.hx, y + self.hy, z + self.hz)

    def coords(self, n):
        return n % self.sx, (n // self.sx) % self.sy, n // (self.sx * self.sy)

    def is_interior(self, px, py, pz):
        return (self.hx <= px < self.hx + self.nx and self.hy <= py < self.hy + self.ny
                and self.hz <= pz < self.hz + self.nz)


class CellType(enum.IntEnum):
    """Flags.hpp:20-33."""
    Fluid = 0
    Solid = 1
    Excluded = 2
    RegWall = 3
    SpecWall = 4
    SpecNode = 5


class NormalCode(enum.IntEnum):
    """Outward wall normals (Regularized.hpp:97-102), as set_specular_walls takes them."""
    NrmNone = 0
    NrmXp = 1
    NrmXm = 2
    NrmYp = 3
    NrmYm = 4
    NrmZp = 5
    NrmZm = 6


class WallCode(enum.IntEnum):
    """Regularised-wall codes beyond the axis normals (Regularized.hpp:97-105)."""
    NrmCorner = 7
    NrmOutXp = 8
    NrmOutFree = 9
    NrmOutEq = 10


@dataclass
class WallSpec:
    """One regularised wall node (FluidSolver.hpp:97-103): outward normal code,
    imposed velocity, and the density the outlet codes impose."""
    normal: int = 0
    ux: float = 0.0
    uy: float = 0.0
    uz: float = 0.0
    rho: float = 1.0


class SpecFace(enum.IntFlag):
    """Face bits of an on-node specular mask (Specular.hpp:226-234)."""
    SpecNone = 0
    SpecXp = 0x01
    SpecXm = 0x02
    SpecYp = 0x04
    SpecYm = 0x08
    SpecZp = 0x10
    SpecZm = 0x20


# ---------------------------------------------------------------- policies
class RawPopulations:
    name, shifted = "raw", False


class ShiftedPopulations:
    name, shifted = "shifted", True


class EsotericPull:
    """In-place single-array streaming (EsotericPull.hpp); the only scheme the
    device path runs."""
    name = "EsotericPull"
    implicit_bounce_back = True


class SecondOrderEquilibrium:
    name, code = "SecondOrder", capi.EQ_SECOND_ORDER


class ProductFormEquilibrium:
    name, code = "ProductForm", capi.EQ_PRODUCT_FORM


HighOrderEquilibrium = ProductFormEquilibrium


@dataclass
class NoForcing:
    name = "None"
    active = False


@dataclass
class Guo:
    """Uniform Guo body force (Forcing.hpp:58-82)."""
    fx: float = 0.0
    fy: float = 0.0
    fz: float = 0.0
    name = "Guo"
    active = True


def _store(s):
    return s.shifted if hasattr(s, "shifted") else bool(s)


@dataclass
class BGK:
    """BGK.hpp:33-102.  Defaults as the reference template arguments."""
    lattice: type = D3Q27
    equilibrium: type = SecondOrderEquilibrium
    forcing: object = field(default_factory=NoForcing)
    storage: type = RawPopulations
    omega: float = 1.0
    name = "BGK"
    op = capi.OP_BGK

    @staticmethod
    def omega_from_viscosity(nu, lattice=D3Q27):
        return 1.0 / (nu / lattice.cs2 + 0.5)

    @staticmethod
    def viscosity_from_omega(w, lattice=D3Q27):
        return (1.0 / w - 0.5) * lattice.cs2

    def rates(self):
        return self.omega, -1.0


@dataclass
class TRT:
    """TRT.hpp:35-136."""
    lattice: type = D3Q27
    equilibrium: type = SecondOrderEquilibrium
    forcing: object = field(default_factory=NoForcing)
    storage: type = RawPopulations
    omega_p: float = 1.0
    omega_m: float = 1.0
    name = "TRT"
    op = capi.OP_TRT
    magic_3_16 = 3.0 / 16.0

    omega_from_viscosity = BGK.omega_from_viscosity
    viscosity_from_omega = BGK.viscosity_from_omega

    @staticmethod
    def omega_minus_for(omega_plus, lam):
        return 1.0 / (lam / (1.0 / omega_plus - 0.5) + 0.5)

    @staticmethod
    def magic_parameter(omega_plus, omega_minus):
        return (1.0 / omega_plus - 0.5) * (1.0 / omega_minus - 0.5)

    def rates(self):
        return self.omega_p, self.omega_m


@dataclass
class MomentCollision:
    """MomentCollision.hpp:66-376: central moments (central=True) or raw MRT."""
    lattice: type = D3Q27
    forcing: object = field(default_factory=NoForcing)
    storage: type = RawPopulations
    central: bool = True
    omega: float = 1.0
    omega_bulk: float = -1.0
    equilibrium = SecondOrderEquilibrium  # unused: closed form in moment space

    omega_from_viscosity = BGK.omega_from_viscosity
    viscosity_from_omega = BGK.viscosity_from_omega

    @property
    def name(self):
        return "CentralMoments" if self.central else "MRT"

    @property
    def op(self):
        return capi.OP_CM if self.central else capi.OP_MRT

    def bulk(self):
        return self.omega if self.omega_bulk < 0 else self.omega_bulk

    def rates(self):
        return self.omega, self.omega_bulk


def CentralMoments(lattice=D3Q27, forcing=None, storage=RawPopulations, **kw):
    return MomentCollision(lattice, forcing or NoForcing(), storage, True, **kw)


def MRT(lattice=D3Q27, forcing=None, storage=RawPopulations, **kw):
    return MomentCollision(lattice, forcing or NoForcing(), storage, False, **kw)


@dataclass
class NullCollision:
    """Collision that does nothing (tests/test_streaming.cpp:28-38): pure streaming."""
    lattice: type = D3Q27
    forcing: object = field(default_factory=NoForcing)
    storage: type = RawPopulations
    equilibrium = SecondOrderEquilibrium
    name = "None"
    op = capi.OP_NONE

    def rates(self):
        return 1.0, -1.0


# ---------------------------------------------------------------- solver
def _ptr(a):
    return C.c_void_p(a.ctypes.data)


class FluidSolver:
    """FluidSolver<L, EsotericPull<L>, Collision> (FluidSolver.hpp:34-637),
    resident on the current CUDA device."""

    def __init__(self, domain: Domain, collision, streaming=EsotericPull, storage="f32",
                 stream=None):
        if streaming is not EsotericPull:
            raise NotImplementedError("only Esoteric Pull streaming runs on the device")
        self.dom = domain
        self.coll = collision
        L = collision.lattice
        self.L = L
        self.Q = L.Q
        self.storage = capi.STORAGE_NAMES[storage] if isinstance(storage, str) else int(storage)
        self.real = np.float64 if self.storage == capi.STORE_F64 else np.float32
        lib = capi.lib()
        h = C.c_void_p()
        d = domain
        capi.check(lib.m3lb_create(L.Q, d.nx, d.ny, d.nz, int(d.periodic[0]), int(d.periodic[1]),
                                   int(d.periodic[2]), collision.op,
                                   collision.equilibrium.code, self.storage,
                                   int(_store(collision.storage)),
                                   int(collision.forcing.active), C.byref(h)))
        self._h = h
        self._flags = np.zeros((d.nz, d.ny, d.nx), np.uint8)
        self._push_params()
        if stream is not None:
            self.set_stream(stream)

    # -- plumbing
    @property
    def handle(self):
        return self._h

    def _push_params(self):
        w1, w2 = self.coll.rates()
        f = self.coll.forcing
        fx, fy, fz = (f.fx, f.fy, f.fz) if f.active else (0.0, 0.0, 0.0)
        capi.check(capi.lib().m3lb_set_params(self._h, w1, w2, fx, fy, fz))

    def set_stream(self, stream):
        """Queue work on a CUDA stream (a torch.cuda.Stream or a raw handle)."""
        raw = getattr(stream, "cuda_stream", stream)
        capi.check(capi.lib().m3lb_set_stream(self._h, C.c_void_p(raw)))

    def set_option(self, option, value):
        capi.check(capi.lib().m3lb_set_option(self._h, option, int(value)))

    def sync(self):
        capi.check(capi.lib().m3lb_sync(self._h))

    def close(self):
        if getattr(self, "_h", None):
            capi.lib().m3lb_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- reference API
    def set_geometry(self, fn_or_flags):
        """fn(x, y, z) -> CellType over interior coordinates (:74-82), or an
        array of flags shaped (nz, ny, nx)."""
        d = self.dom
        if callable(fn_or_flags):
            z, y, x = np.meshgrid(np.arange(d.nz), np.arange(d.ny), np.arange(d.nx), indexing="ij")
            fl = np.vectorize(lambda a, b, c: int(fn_or_flags(a, b, c)), otypes=[np.uint8])(x, y, z)
        else:
            fl = np.asarray(fn_or_flags)
        fl = np.ascontiguousarray(fl, dtype=np.uint8).reshape(d.nz, d.ny, d.nx)
        capi.check(capi.lib().m3lb_set_flags(self._h, _ptr(fl)))
        self._flags = fl.copy()

    def _per_node(self, fn_or_array):
        d = self.dom
        if callable(fn_or_array):
            z, y, x = np.meshgrid(np.arange(d.nz), np.arange(d.ny), np.arange(d.nx), indexing="ij")
            a = np.vectorize(lambda p, q, r: int(fn_or_array(p, q, r)), otypes=[np.uint8])(x, y, z)
        else:
            a = np.asarray(fn_or_array)
        return np.ascontiguousarray(a, dtype=np.uint8).reshape(d.nz, d.ny, d.nx)

    def set_specular_walls(self, fn_or_codes):
        """Free-slip ghost walls (FluidSolver.hpp:193-218): fn(x, y, z) ->
        NormalCode over interior coordinates, or the codes as an (nz, ny, nx)
        array; NrmNone leaves a node as it is.  Call after set_geometry."""
        codes = self._per_node(fn_or_codes)
        capi.check(capi.lib().m3lb_set_specular_walls(self._h, _ptr(codes)))
        self._flags = np.where(codes != 0, np.uint8(CellType.SpecWall), self._flags).astype(np.uint8)

    def set_specular_nodes(self, fn_or_masks):
        """On-node free-slip walls (FluidSolver.hpp:236-268): fn(x, y, z) ->
        SpecFace mask, or the masks as an (nz, ny, nx) array; SpecNone leaves
        a node as it is.  Call after set_geometry."""
        masks = self._per_node(fn_or_masks)
        capi.check(capi.lib().m3lb_set_specular_nodes(self._h, _ptr(masks)))
        self._flags = np.where(masks != 0, np.uint8(CellType.SpecNode), self._flags).astype(np.uint8)

    def set_regularized_walls(self, fn_or_codes, states=None):
        """Regularised on-node walls (FluidSolver.hpp:372-552): fn(x, y, z) ->
        WallSpec over interior coordinates, or the normal codes as an
        (nz, ny, nx) array with `states` (nz, ny, nx, 4) = (ux, uy, uz, rho)
        or None for (0, 0, 0, 1).  Call after set_geometry."""
        d = self.dom
        if callable(fn_or_codes):
            codes = np.zeros((d.nz, d.ny, d.nx), np.uint8)
            st = np.zeros((d.nz, d.ny, d.nx, 4))
            st[..., 3] = 1.0
            for z in range(d.nz):
                for y in range(d.ny):
                    for x in range(d.nx):
                        w = fn_or_codes(x, y, z)
                        if int(w.normal) == 0:
                            continue
                        codes[z, y, x] = int(w.normal)
                        st[z, y, x] = (w.ux, w.uy, w.uz, w.rho)
        else:
            codes = self._per_node(fn_or_codes)
            st = None if states is None else np.broadcast_to(states, (d.nz, d.ny, d.nx, 4))
        st_arr = None if st is None else np.ascontiguousarray(st, dtype=np.float64)
        capi.check(capi.lib().m3lb_set_regularized_walls(
            self._h, _ptr(codes), _ptr(st_arr) if st_arr is not None else None))
        self._flags = np.where(codes != 0, np.uint8(CellType.RegWall), self._flags).astype(np.uint8)

    def set_wall_velocity_scale(self, sc):
        capi.check(capi.lib().m3lb_set_wall_velocity_scale(self._h, float(sc)))

    def set_wall_density(self, r):
        capi.check(capi.lib().m3lb_set_wall_density(self._h, float(r)))

    def set_wall_velocity_field(self, fn_or_array):
        """fn(x, y, z) -> (ux, uy, uz), or an (nz, ny, nx, 3) array."""
        d = self.dom
        if callable(fn_or_array):
            u = np.array([[[fn_or_array(x, y, z) for x in range(d.nx)] for y in range(d.ny)]
                          for z in range(d.nz)], dtype=np.float64)
        else:
            u = np.asarray(fn_or_array, dtype=np.float64)
        u = np.ascontiguousarray(np.broadcast_to(u, (d.nz, d.ny, d.nx, 3)))
        capi.check(capi.lib().m3lb_set_wall_velocity_field(self._h, _ptr(u)))

    def set_wall_velocity_field_scale(self, sc):
        capi.check(capi.lib().m3lb_set_wall_velocity_field_scale(self._h, float(sc)))

    def set_fd_corners(self, on):
        capi.check(capi.lib().m3lb_set_fd_corners(self._h, int(bool(on))))

    def set_force_correction(self, on):
        capi.check(capi.lib().m3lb_set_force_correction(self._h, int(bool(on))))

    def set_outflow_order(self, k):
        capi.check(capi.lib().m3lb_set_outflow_order(self._h, int(k)))

    def set_outflow_density(self, r):
        capi.check(capi.lib().m3lb_set_outflow_density(self._h, float(r)))

    def set_buoyancy(self, T, g=(0.0, 1.0, 0.0), rho0=1.0, beta=1.0, T0=0.0):
        """Boussinesq force (BoussinesqGuo): F = (fx, fy, fz) + g rho0 beta (T - T0)
        with T a device array / tensor per interior node in the arithmetic
        type, or None to return to the uniform force."""
        ptr = None
        if T is not None:
            ptr = C.c_void_p(T.data_ptr() if hasattr(T, "data_ptr") else int(T))
            self._buoy_keep = T
        capi.check(capi.lib().m3lb_set_buoyancy(self._h, ptr, *map(float, g), float(rho0),
                                               float(beta), float(T0)))

    def initialize(self, rho0=1.0, ux0=0.0, uy0=0.0, uz0=0.0):
        self._push_params()
        capi.check(capi.lib().m3lb_init_eq(self._h, rho0, ux0, uy0, uz0))

    def initialize_field(self, fn_or_arrays):
        """fn(x, y, z) -> (rho, ux, uy, uz) vectorised over interior coordinate
        arrays, or the four arrays themselves (:568-579)."""
        d = self.dom
        if callable(fn_or_arrays):
            z, y, x = np.meshgrid(np.arange(d.nz), np.arange(d.ny), np.arange(d.nx), indexing="ij")
            fields = fn_or_arrays(x, y, z)
        else:
            fields = fn_or_arrays
        arrs = [np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64), (d.nz, d.ny, d.nx)))
                for a in fields]
        self._push_params()
        capi.check(capi.lib().m3lb_init_field_f64(self._h, *[_ptr(a) for a in arrs]))

    @staticmethod
    def _addr(a):
        if hasattr(a, "data_ptr"):
            return C.c_void_p(a.data_ptr())
        if isinstance(a, np.ndarray):
            return C.c_void_p(a.ctypes.data)
        return C.c_void_p(int(a))

    def initialize_field_f32(self, rho, ux, uy, uz):
        """Four host float32 arrays (numpy, or pinned torch tensors) over the
        interior, copied as they are (m3lb_init_field_f32)."""
        self._push_params()
        capi.check(capi.lib().m3lb_init_field_f32(self._h, *[self._addr(a) for a in
                                                             (rho, ux, uy, uz)]))

    def compute_macroscopic_f32(self, rho, ux, uy, uz):
        """compute_macroscopic() into four host float32 buffers."""
        capi.check(capi.lib().m3lb_macro_f32(self._h, *[self._addr(a) for a in
                                                        (rho, ux, uy, uz)]))

    def initialize_field_device(self, rho, ux, uy, uz):
        """Four device arrays of the arithmetic type: torch tensors, or raw
        device pointers.  The handle queues its work on its own stream, so
        for tensors the seed first waits for the work torch has queued on its
        current stream (which may still be writing them), and the call
        returns once the seed has read them (torch may reuse their memory as
        soon as they are freed)."""
        arrs = (rho, ux, uy, uz)
        ptrs = [C.c_void_p(getattr(a, "data_ptr", lambda: a)()) for a in arrs]
        self._push_params()
        lib = capi.lib()
        dev = getattr(rho, "device", None)
        if dev is not None and getattr(dev, "type", "") == "cuda":
            import torch
            mine = C.c_void_p()
            capi.check(lib.m3lb_get_stream(self._h, C.byref(mine)))
            theirs = torch.cuda.current_stream(dev).cuda_stream
            if theirs != (mine.value or 0):
                capi.check(lib.m3lb_stream_order(C.c_void_p(theirs), mine))
        capi.check(lib.m3lb_init_field_device(self._h, *ptrs))
        if dev is not None:
            self.sync()

    def step(self, store_macroscopic=False):
        capi.check(capi.lib().m3lb_step(self._h, 1, int(store_macroscopic)))

    def steps(self, n, store_macroscopic=False):
        capi.check(capi.lib().m3lb_step(self._h, int(n), int(store_macroscopic)))

    def compute_macroscopic(self):
        d = self.dom
        out = [np.empty((d.nz, d.ny, d.nx), np.float64) for _ in range(4)]
        capi.check(capi.lib().m3lb_macro_f64(self._h, *[_ptr(a) for a in out]))
        self._macro = out
        return tuple(out)

    def stored_macroscopic(self):
        d = self.dom
        out = [np.empty((d.nz, d.ny, d.nx), np.float64) for _ in range(4)]
        capi.check(capi.lib().m3lb_stored_macro_f64(self._h, *[_ptr(a) for a in out]))
        self._macro = out
        return tuple(out)

    def _field(self, k):
        if not hasattr(self, "_macro"):
            self.stored_macroscopic()
        return self._macro[k]

    def rho(self):
        return self._field(0)

    def ux(self):
        return self._field(1)

    def uy(self):
        return self._field(2)

    def uz(self):
        return self._field(3)

    def reduce(self):
        out = np.zeros(6, np.float64)
        capi.check(capi.lib().m3lb_reduce(self._h, _ptr(out)))
        return out

    def diagnostics(self):
        """The validation campaign's flow diagnostics on the device
        (validation/Campaign.hpp:99-130): (kinetic energy sum 0.5 |u|^2,
        enstrophy sum 0.5 |w|^2 over the interior, finite) -- the reference's
        Diag {energy, enstrophy, finite}."""
        out = np.zeros(3, np.float64)
        capi.check(capi.lib().m3lb_diagnostics(self._h, _ptr(out)))
        return float(out[0]), float(out[1]), bool(out[2] == 0)

    def total_mass(self):
        return float(self.reduce()[0])

    def total_momentum(self, a):
        return float(self.reduce()[1 + a])

    def flags(self):
        return self._flags

    def timestep(self):
        t = C.c_longlong()
        capi.check(capi.lib().m3lb_timestep(self._h, C.byref(t)))
        return int(t.value)

    def domain(self):
        return self.dom

    def collision(self):
        return self.coll

    def gather_populations(self):
        out = np.empty((self.dom.n_padded, self.Q), np.float64)
        capi.check(capi.lib().m3lb_gather(self._h, _ptr(out)))
        return out

    def gather_raw(self):
        dt = {capi.STORE_F32: np.float32, capi.STORE_F64: np.float64,
              capi.STORE_F16: np.uint16, capi.STORE_BF16: np.uint16,
              capi.STORE_F16C: np.uint16}[self.storage]
        out = np.empty((self.dom.n_padded, self.Q), dt)
        capi.check(capi.lib().m3lb_gather_raw(self._h, _ptr(out)))
        return out

    def seed_populations(self, fn_or_array):
        """fn(n, i) -> value over padded node indices, or an (n_padded, Q) array."""
        if callable(fn_or_array):
            n = np.arange(self.dom.n_padded)
            arr = np.stack([np.broadcast_to(fn_or_array(n, i), n.shape) for i in range(self.Q)], 1)
        else:
            arr = fn_or_array
        arr = np.ascontiguousarray(arr, dtype=np.float64).reshape(self.dom.n_padded, self.Q)
        capi.check(capi.lib().m3lb_scatter(self._h, _ptr(arr)))

    def seed_raw(self, arr):
        arr = np.ascontiguousarray(arr)
        assert arr.size == self.dom.n_padded * self.Q
        capi.check(capi.lib().m3lb_scatter_raw(self._h, _ptr(arr)))

    def dims(self):
        d = (C.c_int * 12)()
        capi.check(capi.lib().m3lb_dims(self._h, d))
        return list(d)

    def populations(self):
        p, b = C.c_void_p(), C.c_size_t()
        capi.check(capi.lib().m3lb_populations(self._h, C.byref(p), C.byref(b)))
        return p.value, b.value

    def launch_count(self):
        n = C.c_longlong()
        capi.check(capi.lib().m3lb_launch_count(self._h, C.byref(n)))
        return int(n.value)


# ---------------------------------------------------------- scalar lattice
class ScalarCell(enum.IntEnum):
    """ScalarBGK.hpp ScalarCell."""
    ScalarBulk = 0
    ScalarAdiabatic = 1
    ScalarDirichlet = 2
    ScalarExcluded = 3
    ScalarMoment = 4
    ScalarOutflow = 5
    ScalarSpecular = 6


class ScalarBGK:
    """ScalarBGK<L> (src/collision/ScalarBGK.hpp): raw storage with an
    optional reference T_ref; D = cs2 (1/omega - 1/2)."""
    code = 1

    def __init__(self, lattice=D3Q7, omega=1.0, T_ref=0.0):
        self.lattice, self.omega, self.T_ref = lattice, float(omega), float(T_ref)
        self.Lambda = 0.25
        self.omega_of = None

    @staticmethod
    def omega_from_diffusivity(d, lattice=D3Q7):
        return 1.0 / (d / lattice.cs2 + 0.5)

    @staticmethod
    def diffusivity_from_omega(w, lattice=D3Q7):
        return (1.0 / w - 0.5) * lattice.cs2


class ScalarTRT(ScalarBGK):
    """ScalarTRT<L> (src/collision/ScalarTRT.hpp): the odd moments at omega,
    the even ones at omega_plus from the magic parameter Lambda."""
    code = 2

    def __init__(self, lattice=D3Q7, omega=1.0, T_ref=0.0, Lambda=0.25):
        super().__init__(lattice, omega, T_ref)
        self.Lambda = float(Lambda)


class ScalarRegularised(ScalarBGK):
    """ScalarRegularised<L> (src/collision/ScalarRegularised.hpp)."""
    code = 3


class ScalarSolver:
    """ScalarSolver<L, EsotericPull<L>, Collision> (src/solver/ScalarSolver.hpp)
    on the device.  Interior arrays are (nz, ny, nx); ``storage`` is "f32" or
    "f64"."""

    def __init__(self, domain: Domain, collision, storage="f32"):
        self.dom, self.coll = domain, collision
        self.storage = storage
        L = collision.lattice
        self.Q = L.Q
        d = domain
        h = C.c_void_p()
        capi.check(capi.lib().m3lb_scalar_create(L.Q, d.nx, d.ny, d.nz, int(d.periodic[0]),
                                                 int(d.periodic[1]), int(d.periodic[2]),
                                                 collision.code, capi.STORAGE_NAMES[storage],
                                                 C.byref(h)))
        self._h = h
        self._keep = []
        self._cells = np.zeros((d.nz, d.ny, d.nx), np.uint8)
        self._push()
        if collision.omega_of is not None:
            self.set_omega_field(collision.omega_of)

    def _push(self):
        c = self.coll
        capi.check(capi.lib().m3lb_scalar_set_params(self._h, c.omega, c.T_ref, c.Lambda))

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            capi.lib().m3lb_scalar_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _u8(self, fn_or_array):
        d = self.dom
        if callable(fn_or_array):
            z, y, x = np.meshgrid(np.arange(d.nz), np.arange(d.ny), np.arange(d.nx), indexing="ij")
            a = np.vectorize(lambda p, q, r: int(fn_or_array(p, q, r)), otypes=[np.uint8])(x, y, z)
        else:
            a = np.asarray(fn_or_array)
        return np.ascontiguousarray(np.broadcast_to(a, (d.nz, d.ny, d.nx)), dtype=np.uint8)

    def _f64(self, fn_or_array, shape):
        d = self.dom
        if callable(fn_or_array):
            z, y, x = np.meshgrid(np.arange(d.nz), np.arange(d.ny), np.arange(d.nx), indexing="ij")
            a = fn_or_array(x, y, z)
        else:
            a = fn_or_array
        return np.ascontiguousarray(np.broadcast_to(a, shape), dtype=np.float64)

    def set_geometry(self, fn_or_cells):
        """fn(x, y, z) -> ScalarCell, or the cells as an (nz, ny, nx) array (:92-99)."""
        c = self._u8(fn_or_cells)
        capi.check(capi.lib().m3lb_scalar_set_cells(self._h, _ptr(c)))
        self._cells = c.copy()

    def set_wall_values(self, fn_or_values):
        d = self.dom
        v = self._f64(fn_or_values, (d.nz, d.ny, d.nx))
        capi.check(capi.lib().m3lb_scalar_set_wall_values(self._h, _ptr(v)))

    def set_specular_walls(self, fn_or_codes):
        capi.check(capi.lib().m3lb_scalar_set_specular_walls(self._h, _ptr(self._u8(fn_or_codes))))

    def set_specular_nodes(self, fn_or_masks):
        capi.check(capi.lib().m3lb_scalar_set_specular_nodes(self._h, _ptr(self._u8(fn_or_masks))))

    def set_omega_field(self, fn_or_values):
        d = self.dom
        v = None if fn_or_values is None else self._f64(fn_or_values, (d.nz, d.ny, d.nx))
        capi.check(capi.lib().m3lb_scalar_set_omega_field(self._h, None if v is None else _ptr(v)))

    def set_velocity(self, ux, uy=None, uz=None):
        """The advecting velocity: device tensors / pointers of the arithmetic
        type, or host arrays (uploaded once), or None (at rest)."""
        if ux is None:
            capi.check(capi.lib().m3lb_scalar_set_velocity_device(self._h, None, None, None))
            self._keep = []
            return
        import torch
        dt = torch.float64 if self.storage == "f64" else torch.float32
        d = self.dom
        ts = []
        for a in (ux, uy, uz):
            if isinstance(a, torch.Tensor):
                t = a.to(device="cuda", dtype=dt).contiguous()
            else:
                t = torch.as_tensor(np.array(np.broadcast_to(a, (d.nz, d.ny, d.nx))),
                                    dtype=dt, device="cuda")
            ts.append(t)
        torch.cuda.synchronize()
        self._keep = ts
        capi.check(capi.lib().m3lb_scalar_set_velocity_device(
            self._h, *[C.c_void_p(t.data_ptr()) for t in ts]))

    def finalize_geometry(self):
        capi.check(capi.lib().m3lb_scalar_finalize_geometry(self._h))

    def initialize(self, T0):
        self._push()
        capi.check(capi.lib().m3lb_scalar_init(self._h, float(T0)))

    def initialize_field(self, T_padded):
        """T per padded node (n_padded values), as the reference's fn(n)."""
        self._push()
        v = np.ascontiguousarray(np.ravel(T_padded), dtype=np.float64)
        if v.size != self.dom.n_padded:
            raise ValueError(f"initialize_field: {v.size} values, the lattice has {self.dom.n_padded} padded nodes")
        capi.check(capi.lib().m3lb_scalar_init_field(self._h, _ptr(v)))

    def step(self):
        self._push()
        capi.check(capi.lib().m3lb_scalar_step(self._h, 1))

    def steps(self, n):
        self._push()
        capi.check(capi.lib().m3lb_scalar_step(self._h, int(n)))

    def add_source(self, fn_or_values):
        d = self.dom
        v = self._f64(fn_or_values, (d.nz, d.ny, d.nx))
        capi.check(capi.lib().m3lb_scalar_add_source(self._h, _ptr(v)))

    def compute_field(self):
        capi.check(capi.lib().m3lb_scalar_compute_field(self._h))

    def temperature(self):
        """The field per interior node as it stands (ScalarSolver::temperature)."""
        d = self.dom
        out = np.empty((d.nz, d.ny, d.nx), np.float64)
        capi.check(capi.lib().m3lb_scalar_field(self._h, _ptr(out)))
        return out

    def field_device(self):
        p = C.c_void_p()
        capi.check(capi.lib().m3lb_scalar_field_device(self._h, C.byref(p)))
        return p.value

    def total_population(self):
        out = C.c_double()
        capi.check(capi.lib().m3lb_scalar_total(self._h, C.byref(out)))
        return out.value

    def gather_populations(self):
        out = np.empty((self.dom.n_padded, self.Q), np.float64)
        capi.check(capi.lib().m3lb_scalar_gather(self._h, _ptr(out)))
        return out

    def flags(self):
        return self._cells

    def timestep(self):
        t = C.c_longlong()
        capi.check(capi.lib().m3lb_scalar_info(self._h, None, C.byref(t), None))
        return int(t.value)

    def domain(self):
        return self.dom

    def sync(self):
        capi.check(capi.lib().m3lb_scalar_sync(self._h))


def couple_thermal(fluid: "FluidSolver", scalar: ScalarSolver, g=(0.0, 1.0, 0.0), rho0=1.0,
                   beta=1.0, T0=0.0):
    """Two-way coupling (BoussinesqGuo + set_velocity, as in the reference's
    validation/rayleigh_benard.cpp): the fluid's force reads the scalar's
    field, the scalar is advected by the fluid's stored velocity, both on the
    fluid's stream.  Step as fluid.step(True); scalar.step()."""
    capi.check(capi.lib().m3lb_couple_thermal(fluid.handle, scalar.handle, *map(float, g),
                                             float(rho0), float(beta), float(T0)))
    scalar._keep = [fluid]
