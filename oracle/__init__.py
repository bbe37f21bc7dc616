"""CPU checkers for the lattice-Boltzmann hot path -- TEST INFRASTRUCTURE.

Two implementations behind one Python interface (:class:`CpuSolver`):

* ``backend="oracle"``: ``liboracle.so``, the plain-C restatement of the
  reference algorithm in ``lbm_oracle_body.h`` (double or float arithmetic,
  optional binary16 / bfloat16 storage rounding).
* ``backend="ref"``: ``_ref/libm3lb_ref_{f64,f32}.so``, the reference's own
  ``FluidSolver`` headers compiled unmodified against a host stand-in for the
  Kokkos API (``ref/``).  Present only where the reference sources were
  available at build time, or where the built libraries were carried along.

Only the tests, the smoke check and the CPU-baseline leg of ``bench.py`` use
this package, as the checker.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
# Where the reference tree (M3LB's sources) is mounted: the one place that
# names it.  Recipes that read the reference (the reference build, the
# fixture scripts, the facade-driver tests) take it from here.
REFERENCE_DIR = Path(os.environ.get("M3LB_REFERENCE", "/root/reference"))


def reference_present() -> bool:
    """The reference sources are available to build from."""
    return (REFERENCE_DIR / "src" / "solver" / "FluidSolver.hpp").exists()
REF_LIBS = {"f64": HERE / "_ref" / "libm3lb_ref_f64.so", "f32": HERE / "_ref" / "libm3lb_ref_f32.so"}

OPS = {"none": 0, "bgk": 1, "trt": 2, "mrt": 3, "cm": 4}
QUANT = {None: 0, "none": 0, "f16": 1, "bf16": 2, "f16c": 3}

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)
_vp = C.c_void_p


_SCALAR_SIG = {
    "screate": (_vp, [C.c_int] * 8 + [C.c_double] * 3),
    "sdestroy": (None, [_vp]),
    "sset_geometry": (None, [_vp, _u8p]),
    "sset_wall_values": (None, [_vp, _dp]),
    "sset_specular_walls": (C.c_int, [_vp, _u8p]),
    "sset_specular_nodes": (C.c_int, [_vp, _u8p]),
    "sset_omega_field": (None, [_vp, _dp]),
    "sset_velocity": (None, [_vp, _dp, _dp, _dp]),
    "sfinalize_geometry": (None, [_vp]),
    "sinitialize": (None, [_vp, C.c_double]),
    "sinitialize_field": (None, [_vp, _dp]),
    "sstep": (None, [_vp, C.c_int]),
    "sadd_source": (None, [_vp, _dp]),
    "scompute_field": (None, [_vp]),
    "sfield": (None, [_vp, _dp]),
    "stotal": (C.c_double, [_vp]),
    "sn_padded": (C.c_longlong, [_vp]),
    "stimestep": (C.c_longlong, [_vp]),
}


def _bind(lib, prefix):
    sig = {
        "create": (_vp, [C.c_int] * 6 + [C.c_int] * 6 + [C.c_double] * 5),
        "destroy": (None, [_vp]),
        "set_geometry": (None, [_vp, _u8p]),
        "set_specular_walls": (C.c_int, [_vp, _u8p]),
        "set_specular_nodes": (C.c_int, [_vp, _u8p]),
        "set_regularized_walls": (C.c_int, [_vp, _u8p, _dp]),
        "set_wall_velocity_scale": (None, [_vp, C.c_double]),
        "set_wall_density": (None, [_vp, C.c_double]),
        "set_wall_velocity_field": (None, [_vp, _dp]),
        "set_wall_velocity_field_scale": (None, [_vp, C.c_double]),
        "set_fd_corners": (None, [_vp, C.c_int]),
        "set_force_correction": (None, [_vp, C.c_int]),
        "set_outflow_order": (C.c_int, [_vp, C.c_int]),
        "set_outflow_density": (None, [_vp, C.c_double]),
        "initialize": (None, [_vp] + [C.c_double] * 4),
        "initialize_field": (None, [_vp] + [_dp] * 4),
        "step": (None, [_vp, C.c_int, C.c_int]),
        "macro": (None, [_vp] + [_dp] * 4),
        "stored_macro": (None, [_vp] + [_dp] * 4),
        "total_mass": (C.c_double, [_vp]),
        "total_momentum": (C.c_double, [_vp, C.c_int]),
        "gather": (None, [_vp, _dp]),
        "seed": (None, [_vp, _dp]),
        "slot_sum": (C.c_double, [_vp]),
        "n_padded": (C.c_longlong, [_vp]),
        "timestep": (C.c_longlong, [_vp]),
    }
    sig["set_buoyancy"] = ((C.c_int if prefix == "ref_" else None),
                           [_vp, _dp] + [C.c_double] * 6)
    sig.update(_SCALAR_SIG)
    if prefix != "ref_":  # the reference solver has no population readout
        sig["sgather"] = (None, [_vp, _dp])
    fns = {}
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name)
        fn.restype = res
        fn.argtypes = args
        fns[name] = fn
    return fns


_cache: dict = {}


def _lib(backend: str, precision: str):
    key = (backend, precision)
    if key in _cache:
        return _cache[key]
    if backend == "oracle":
        if not ORACLE_LIB.exists():
            raise FileNotFoundError(f"{ORACLE_LIB} not built (make -C oracle oracle)")
        lib = C.CDLL(str(ORACLE_LIB))
        fns = _bind(lib, "lbmo_f64_" if precision == "f64" else "lbmo_f32_")
    elif backend == "ref":
        path = REF_LIBS[precision]
        if not path.exists():
            raise FileNotFoundError(f"{path} not built (make -C oracle ref)")
        lib = C.CDLL(str(path))
        fns = _bind(lib, "ref_")
        lib.ref_set_threads.argtypes = [C.c_int]
        lib.ref_get_threads.restype = C.c_int
        fns["_lib"] = lib
    else:
        raise ValueError(backend)
    _cache[key] = fns
    return fns


def ref_available(precision: str = "f64") -> bool:
    return REF_LIBS[precision].exists()


def set_ref_threads(n: int, precision: str = "f64") -> None:
    """OpenMP threads the reference build uses (1 gives a deterministic order)."""
    _lib("ref", precision)["_lib"].ref_set_threads(int(n))


def _ptr(a):
    return a.ctypes.data_as(_dp)


class CpuSolver:
    """One lattice on the CPU, reference-shaped API (FluidSolver.hpp:34-637).

    Arrays exchanged with the caller are interior-only, shaped (nz, ny, nx),
    x fastest; populations (``gather``/``seed``) are (n_padded, Q), node-major.
    """

    def __init__(self, backend="oracle", lattice=27, op="bgk", eq=0, shifted=True,
                 forcing=False, nx=8, ny=8, nz=8, px=True, py=True, pz=True,
                 omega=1.0, omega2=-1.0, fx=0.0, fy=0.0, fz=0.0, precision="f64",
                 quant=None, streaming=0):
        self.backend, self.precision = backend, precision
        self.lattice, self.Q = lattice, lattice
        self.nx, self.ny, self.nz = nx, ny, nz
        self.shape = (nz, ny, nx)
        self._f = _lib(backend, precision)
        opc = OPS[op] if isinstance(op, str) else int(op)
        if backend == "oracle":
            if streaming:
                raise ValueError("the C oracle implements Esoteric Pull only")
            h = self._f["create"](lattice, opc, int(eq), int(shifted), int(forcing),
                                  QUANT[quant], nx, ny, nz, int(px), int(py), int(pz),
                                  omega, omega2, fx, fy, fz)
        else:
            if quant not in (None, "none"):
                raise ValueError("the reference build has no narrow storage")
            h = self._f["create"](lattice, int(streaming), opc, int(eq), int(shifted),
                                  int(forcing), nx, ny, nz, int(px), int(py), int(pz),
                                  omega, omega2, fx, fy, fz)
        if not h:
            raise ValueError("unsupported configuration")
        self._h = h
        self.n_padded = int(self._f["n_padded"](h))

    def close(self):
        if getattr(self, "_h", None):
            self._f["destroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- reference API ----
    def set_geometry(self, flags):
        fl = np.ascontiguousarray(flags, dtype=np.uint8).reshape(self.shape)
        self._f["set_geometry"](self._h, fl.ctypes.data_as(_u8p))

    def set_specular_walls(self, codes):
        """Normal code per interior node (0 none, 1..6 = +x -x +y -y +z -z);
        FluidSolver.hpp:193-218.  Raises ValueError on a rejected code."""
        a = np.ascontiguousarray(codes, dtype=np.uint8).reshape(self.shape)
        if self._f["set_specular_walls"](self._h, a.ctypes.data_as(_u8p)) != 0:
            raise ValueError("set_specular_walls: normal code outside 0..6")

    def set_specular_nodes(self, masks):
        """Face mask per interior node (bit 2a outward +a, bit 2a+1 outward
        -a); FluidSolver.hpp:236-268.  Raises ValueError on a rejected mask."""
        a = np.ascontiguousarray(masks, dtype=np.uint8).reshape(self.shape)
        if self._f["set_specular_nodes"](self._h, a.ctypes.data_as(_u8p)) != 0:
            raise ValueError("set_specular_nodes: mask outside 0x3F or with both faces of an axis")

    def set_regularized_walls(self, codes, spec=None):
        """Normal code per interior node (0 none, 1..6 axis walls, 7 corner,
        8 pressure outlet, 9 free outflow, 10 equilibrium outlet) and the
        state (ux, uy, uz, rho) per node, shaped (nz, ny, nx, 4), or None for
        (0, 0, 0, 1); FluidSolver.hpp:372-552."""
        a = np.ascontiguousarray(codes, dtype=np.uint8).reshape(self.shape)
        sp = None
        if spec is not None:
            sp = np.ascontiguousarray(np.broadcast_to(spec, self.shape + (4,)), dtype=np.float64)
        if self._f["set_regularized_walls"](self._h, a.ctypes.data_as(_u8p),
                                             _ptr(sp) if sp is not None else None) != 0:
            raise ValueError("set_regularized_walls: rejected normal code or outlet position")

    def set_wall_velocity_scale(self, sc):
        self._f["set_wall_velocity_scale"](self._h, float(sc))

    def set_wall_density(self, r):
        self._f["set_wall_density"](self._h, float(r))

    def set_wall_velocity_field(self, u3):
        a = np.ascontiguousarray(np.broadcast_to(u3, self.shape + (3,)), dtype=np.float64)
        self._f["set_wall_velocity_field"](self._h, _ptr(a))

    def set_wall_velocity_field_scale(self, sc):
        self._f["set_wall_velocity_field_scale"](self._h, float(sc))

    def set_fd_corners(self, on):
        self._f["set_fd_corners"](self._h, int(bool(on)))

    def set_force_correction(self, on):
        self._f["set_force_correction"](self._h, int(bool(on)))

    def set_outflow_order(self, k):
        if self._f["set_outflow_order"](self._h, int(k)) != 0:
            raise ValueError("set_outflow_order: a pressure outlet lacks the upstream nodes")

    def set_outflow_density(self, r):
        self._f["set_outflow_density"](self._h, float(r))

    def set_buoyancy(self, T, g=(0.0, 1.0, 0.0), rho0=1.0, beta=1.0, T0=0.0):
        """Boussinesq force F = f + g rho0 beta (T - T0) per node (BoussinesqGuo,
        Forcing.hpp:93-127); T per interior node.  The reference build needs a
        solver made with forcing=2 for this."""
        a = np.ascontiguousarray(np.broadcast_to(T, self.shape), dtype=np.float64)
        rc = self._f["set_buoyancy"](self._h, _ptr(a), *map(float, g), float(rho0), float(beta),
                                     float(T0))
        if rc is not None and rc != 0:
            raise ValueError("set_buoyancy: this solver has no Boussinesq forcing")

    def initialize(self, rho0=1.0, ux=0.0, uy=0.0, uz=0.0):
        self._f["initialize"](self._h, rho0, ux, uy, uz)

    def initialize_field(self, rho, ux, uy, uz):
        arrs = [np.ascontiguousarray(np.broadcast_to(a, self.shape), dtype=np.float64)
                for a in (rho, ux, uy, uz)]
        self._f["initialize_field"](self._h, *[_ptr(a) for a in arrs])

    def step(self, n=1, store_macro=False):
        self._f["step"](self._h, int(n), int(store_macro))

    def _four(self, fn):
        out = [np.empty(self.shape, np.float64) for _ in range(4)]
        fn(self._h, *[_ptr(a) for a in out])
        return tuple(out)

    def macro(self):
        return self._four(self._f["macro"])

    def stored_macro(self):
        return self._four(self._f["stored_macro"])

    def total_mass(self):
        return float(self._f["total_mass"](self._h))

    def total_momentum(self, a):
        return float(self._f["total_momentum"](self._h, int(a)))

    def gather(self):
        out = np.empty((self.n_padded, self.Q), np.float64)
        self._f["gather"](self._h, _ptr(out))
        return out

    def seed(self, pops):
        arr = np.ascontiguousarray(pops, dtype=np.float64).reshape(self.n_padded, self.Q)
        self._f["seed"](self._h, _ptr(arr))

    def slot_sum(self):
        return float(self._f["slot_sum"](self._h))

    @property
    def timestep(self):
        return int(self._f["timestep"](self._h))


SOPS = {"bgk": 1, "trt": 2, "regularised": 3}


class ScalarCpuSolver:
    """One scalar (advection-diffusion) lattice on the CPU, the API of the
    reference's ScalarSolver (src/solver/ScalarSolver.hpp): D2Q5 (lattice 5)
    or D3Q7 (7), ScalarBGK / ScalarTRT / ScalarRegularised.  Interior arrays
    are (nz, ny, nx); initialize_field takes one value per padded node."""

    def __init__(self, backend="oracle", lattice=7, op="bgk", nx=8, ny=8, nz=8, px=True, py=True,
                 pz=True, omega=1.0, T_ref=0.0, Lambda=0.25, precision="f64"):
        self.backend, self.precision = backend, precision
        self.Q = lattice
        self.nx, self.ny, self.nz = nx, ny, nz
        self.shape = (nz, ny, nx)
        self.per = (bool(px), bool(py), bool(pz))
        self._f = _lib(backend, precision)
        opc = SOPS[op] if isinstance(op, str) else int(op)
        h = self._f["screate"](lattice, opc, nx, ny, nz, int(px), int(py), int(pz), omega, T_ref,
                               Lambda)
        if not h:
            raise ValueError("unsupported scalar configuration")
        self._h = h
        self.n_padded = int(self._f["sn_padded"](h))

    def close(self):
        if getattr(self, "_h", None):
            self._f["sdestroy"](self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _u8(self, a):
        return np.ascontiguousarray(np.broadcast_to(a, self.shape), dtype=np.uint8)

    def _f64(self, a, shape=None):
        return np.ascontiguousarray(np.broadcast_to(a, shape or self.shape), dtype=np.float64)

    def set_geometry(self, cells):
        a = self._u8(cells)
        self._f["sset_geometry"](self._h, a.ctypes.data_as(_u8p))

    def set_wall_values(self, tw):
        a = self._f64(tw)
        self._f["sset_wall_values"](self._h, _ptr(a))

    def set_specular_walls(self, codes):
        a = self._u8(codes)
        if self._f["sset_specular_walls"](self._h, a.ctypes.data_as(_u8p)) != 0:
            raise ValueError("set_specular_walls: normal code outside 0..6")

    def set_specular_nodes(self, masks):
        a = self._u8(masks)
        if self._f["sset_specular_nodes"](self._h, a.ctypes.data_as(_u8p)) != 0:
            raise ValueError("set_specular_nodes: rejected mask")

    def set_omega_field(self, om):
        a = self._f64(om)
        self._f["sset_omega_field"](self._h, _ptr(a))

    def set_velocity(self, ux, uy=None, uz=None):
        if ux is None:
            self._f["sset_velocity"](self._h, None, None, None)
            return
        arrs = [self._f64(v) for v in (ux, uy, uz)]
        self._f["sset_velocity"](self._h, *[_ptr(v) for v in arrs])

    def finalize_geometry(self):
        self._f["sfinalize_geometry"](self._h)

    def initialize(self, T0):
        self._f["sinitialize"](self._h, float(T0))

    def initialize_field(self, T_padded):
        a = self._f64(T_padded, (self.n_padded,))
        self._f["sinitialize_field"](self._h, _ptr(a))

    def step(self, n=1):
        self._f["sstep"](self._h, int(n))

    def add_source(self, dC):
        a = self._f64(dC)
        self._f["sadd_source"](self._h, _ptr(a))

    def compute_field(self):
        self._f["scompute_field"](self._h)

    def field(self):
        out = np.empty(self.shape, np.float64)
        self._f["sfield"](self._h, _ptr(out))
        return out

    def total(self):
        return float(self._f["stotal"](self._h))

    def gather(self):
        out = np.empty((self.n_padded, self.Q), np.float64)
        self._f["sgather"](self._h, _ptr(out))
        return out

    @property
    def timestep(self):
        return int(self._f["stimestep"](self._h))


def build(ref: bool = True, jobs: int | None = None) -> None:
    """Build the C oracle and, when the reference sources exist, the reference."""
    import subprocess
    jobs = jobs or os.cpu_count() or 4
    target = "all" if ref else "oracle"
    subprocess.run(["make", "-C", str(HERE), f"-j{jobs}", target, f"REF={REFERENCE_DIR}"], check=True,
                   stdout=subprocess.DEVNULL)
