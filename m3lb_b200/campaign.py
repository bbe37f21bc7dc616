"""Results files of the validation campaign, and the 3-D Taylor-Green
benchmark that writes one, on the B200.

The reference's validation programs share one harness
(validation/Campaign.hpp): ``diagnostics()`` (:99-130) integrates the kinetic
energy and the enstrophy of the velocity field, and ``open_out()`` (:133-139)
opens ``results/<dir>/<test>_<lat>_<op>.dat`` for the program's rows, which
the plotting scripts read.  Here the diagnostics run on the device
(``FluidSolver.diagnostics``, C ABI ``m3lb_diagnostics``), :func:`open_out`
opens the same path with the same failure behaviour, and :func:`c_format`
prints numbers exactly as C's ``printf`` does, so a run through this library
writes the same file, byte for byte, as the reference's program run on the
host.  :func:`tgv3d_bench` is the benchmark configuration of
validation/tgv3d_bench.cpp (Re on L = D / (2 pi), the initial field of the
Taylor-Green vortex with its analytic pressure) writing
``results/E_tgv3d_bench/tgvb_re<Re>_<lat>_<op>.dat``.
"""
from __future__ import annotations

import math
import os
import re
import sys

from . import solver as S

_SPEC = re.compile(r"%([-+ #0]*)(\d*)(?:\.(\d+))?([fed])")


def c_format(fmt: str, *values) -> str:
    """``printf``-style formatting as glibc prints it: Python's own ``%``
    formatting agrees for finite numbers and infinities, and here NaN keeps
    its sign ("-nan" when the sign bit is set, as glibc writes the default NaN
    that 0.0 / 0.0 gives on x86-64)."""
    vals = iter(values)

    def one(m):
        flags, width, prec, conv = m.group(1), m.group(2), m.group(3), m.group(4)
        if conv == "d":
            return ("%" + flags + width + "d") % int(next(vals))
        v = float(next(vals))
        if math.isnan(v):
            txt = ("-" if math.copysign(1.0, v) < 0 else "") + "nan"
            w = int(width) if width else 0
            return txt.ljust(w) if "-" in flags else txt.rjust(w)
        spec = "%" + flags + width + ("." + prec if prec is not None else "") + conv
        return spec % v

    return _SPEC.sub(one, fmt)


def results_path(dir: str, test: str, lat: str, op: str) -> str:
    """The results file of a test: results/<dir>/<test>_<lat>_<op>.dat."""
    return "results/" + dir + "/" + test + "_" + lat + "_" + op + ".dat"


def open_out(dir: str, test: str, lat: str, op: str, root: str = ".", out=None):
    """open_out (Campaign.hpp:133-139): the results file opened for writing
    under `root`, or None when it cannot be opened (its folder does not exist),
    in which case the run only prints; prints "  -> <path>" when opened."""
    path = results_path(dir, test, lat, op)
    try:
        f = open(os.path.join(root, path), "w", newline="\n")
    except OSError:
        return None
    print(f"  -> {path}", file=out or sys.stdout)
    return f


def _collision(lat: str, op: str):
    """The campaign's operators (Campaign.hpp:37-39, dispatch :70-90): BGK
    with the highest-order (product-form) equilibrium, raw MRT and central
    moments, shifted populations, no force."""
    L = {"d2q9": S.D2Q9, "d3q27": S.D3Q27}.get(lat)
    if L is None or op not in ("bgk", "mrt", "cm"):
        raise ValueError(f"unknown configuration -lat {lat} -op {op} (lattices d2q9 d3q27, "
                         "operators bgk mrt cm)")
    if op == "bgk":
        return L, S.BGK(L, S.ProductFormEquilibrium, S.NoForcing(), S.ShiftedPopulations)
    return L, S.MomentCollision(L, S.NoForcing(), S.ShiftedPopulations, central=(op == "cm"))


def tgv3d_bench(D: int = 64, Re: float = 1600.0, tmax: float = 20.0, u0: float = 0.02,
                lat: str = "d3q27", op: str = "cm", storage: str = "f64", root: str = ".",
                out=None):
    """The 3-D Taylor-Green vortex in the benchmark configuration
    (validation/tgv3d_bench.cpp): a periodic D^3 box, Re = u0 L / nu on
    L = D / (2 pi), T = floor(tmax L / u0) steps, 41 probes (every T / 40
    steps) of the non-dimensional kinetic energy Ek*, its dissipation eps_E
    (backward difference; undefined at the first probe) and the enstrophy
    dissipation eps_zeta = 2 zeta / Re.  Prints the reference's table and
    writes the rows to results/E_tgv3d_bench/tgvb_re<Re>_<lat>_<op>.dat under
    `root` when that folder exists.  Returns the rows (t*, Ek*, eps_E,
    eps_zeta)."""
    out = out or sys.stdout
    L = D / (2.0 * math.pi)
    nu = u0 * L / Re
    T = int(tmax * L / u0)
    Lat, coll = _collision(lat, op)
    coll.omega = 1.0 / (3.0 * nu + 0.5)  # omega_from_viscosity (BGK.hpp, MomentCollision.hpp)
    dom = S.Domain(D, D, D, True, True, True)
    s = S.FluidSolver(dom, coll, storage=storage)
    try:
        # initial field (tgv3d_bench.cpp:24-36), per interior node
        import numpy as np
        k = 2.0 * math.pi / D
        i = np.arange(D, dtype=np.float64) * k
        z, y, x = np.meshgrid(i, i, i, indexing="ij")
        dr = 3.0 * u0 * u0 / 16.0
        rho = 1.0 + dr * (np.cos(2.0 * x) + np.cos(2.0 * y)) * (np.cos(2.0 * z) + 2.0)
        ux = u0 * np.sin(x) * np.cos(y) * np.cos(z)
        uy = -u0 * np.cos(x) * np.sin(y) * np.cos(z)
        s.initialize_field((rho, ux, uy, np.zeros_like(ux)))

        N = float(D) ** 3
        sE = 1.0 / (u0 * u0)
        sZ = (L / u0) * (L / u0)
        nus = 1.0 / Re
        f = open_out("E_tgv3d_bench", "tgvb_re" + str(int(Re)), lat, op, root=root, out=out)
        if f:
            f.write(c_format("# t*  Ek*  eps_E  eps_zeta   D=%d Re=%.0f u0=%.4f tau=%.6f\n",
                             D, Re, u0, 3.0 * nu + 0.5))
        print("  %8s %13s %13s %13s %11s" % ("t*", "Ek*", "eps_E", "eps_zeta", "gap %"), file=out)
        print("  " + "-" * 64, file=out)
        probe = T // 40 if T // 40 else 1
        rows = []
        prev_E = prev_t = 0.0
        first = True
        for t in range(T + 1):
            if t % probe == 0:
                energy, enstrophy, finite = s.diagnostics()
                ts = tmax * float(t) / float(T)
                if not finite:
                    print(c_format("  DIVERGED at t* = %.3f", ts), file=out)
                    if f:
                        f.write("# DIVERGED\n")
                    break
                Ek = energy / N * sE
                zeta = enstrophy / N * sZ
                eps_z = 2.0 * nus * zeta
                eps_E = float("-nan") if first else -(Ek - prev_E) / (ts - prev_t)
                gap = (100.0 * (eps_E - eps_z) / eps_z
                       if (eps_z > 0 and not first) else float("-nan"))
                print(c_format("  %8.3f %13.6f %13.6f %13.6f %11.1f", ts, Ek, eps_E, eps_z, gap),
                      file=out)
                if f:
                    f.write(c_format("%.6f %.8e %.8e %.8e\n", ts, Ek, eps_E, eps_z))
                    f.flush()
                rows.append((ts, Ek, eps_E, eps_z))
                prev_E, prev_t, first = Ek, ts, False
            if t < T:
                s.step()
        if f:
            f.close()
        return rows
    finally:
        s.close()
