"""VTK ImageData output (the reference's src/io/VtiWriter.hpp interface).

``write_vti(path, solver)`` writes one solver's rho, u and cell flags as an
ASCII file; ``write_vti_bin(path, nx, ny, nz, arrays, spacing)`` writes any
named Float32 point arrays as a raw-appended binary file; ``write_pvd(path,
frames)`` writes the time series that ties frames to their times.  The bytes
are those the reference writes for the same values (checked against files
from the reference's own writer in tests/golden/vti/): the same XML text,
x-fastest point order, numbers at 9 significant digits (the spacing at 6),
appended blocks each led by a UInt32 byte count.
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np


def _g(v: float, digits: int = 9) -> str:
    return "%.*g" % (digits, v)


def _extent(nx: int, ny: int, nz: int) -> str:
    return f"0 {nx - 1} 0 {ny - 1} 0 {nz - 1}"


def write_vti(path, solver) -> None:
    """ASCII file of rho, u and the cell flags (FluidSolver)."""
    rho, ux, uy, uz = solver.compute_macroscopic()
    fl = solver.flags()
    nz, ny, nx = rho.shape
    ext = _extent(nx, ny, nz)
    parts = ['<?xml version="1.0"?>\n',
             '<VTKFile type="ImageData" version="0.1" byte_order="LittleEndian">\n',
             f'  <ImageData WholeExtent="{ext}" Origin="0 0 0" Spacing="1 1 1">\n',
             f'    <Piece Extent="{ext}">\n',
             '      <PointData Scalars="rho" Vectors="u">\n',
             '        <DataArray type="Float64" Name="rho" format="ascii">\n']
    parts.append("".join(_g(v) + " " for v in np.ravel(rho)))
    parts.append('\n        </DataArray>\n'
                 '        <DataArray type="Float64" Name="u" NumberOfComponents="3" format="ascii">\n')
    u = np.stack([np.ravel(ux), np.ravel(uy), np.ravel(uz)], axis=1)
    parts.append("".join(_g(v) + " " for v in np.ravel(u)))
    parts.append('\n        </DataArray>\n'
                 '        <DataArray type="UInt8" Name="flag" format="ascii">\n')
    parts.append("".join(f"{int(v)} " for v in np.ravel(fl)))
    parts.append('\n        </DataArray>\n'
                 '      </PointData>\n    </Piece>\n  </ImageData>\n</VTKFile>\n')
    with open(path, "w", newline="") as f:
        f.write("".join(parts))


@dataclass
class VtiArray:
    """One named point array: npoints * ncomp values, x fastest."""
    name: str
    ncomp: int = 1
    data: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))


def write_vti_bin(path, nx: int, ny: int, nz: int, arrays, spacing: float = 1.0) -> None:
    """Binary (raw appended, Float32) file of named arrays; raises
    ValueError when an array does not have nx * ny * nz * ncomp values."""
    npts = nx * ny * nz
    blocks = []
    for a in arrays:
        d = np.ascontiguousarray(np.ravel(a.data), dtype="<f4")
        if d.size != npts * a.ncomp:
            raise ValueError(f"write_vti_bin: array '{a.name}' has {d.size} values, "
                             f"expected {npts * a.ncomp}")
        blocks.append((a, d))
    scalar = next((a.name for a, _ in blocks if a.ncomp == 1), None)
    vector = next((a.name for a, _ in blocks if a.ncomp == 3), None)
    ext = _extent(nx, ny, nz)
    sp = _g(spacing, 6)
    head = ['<?xml version="1.0"?>\n',
            '<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian"'
            ' header_type="UInt32">\n',
            f'  <ImageData WholeExtent="{ext}" Origin="0 0 0" Spacing="{sp} {sp} {sp}">\n',
            f'    <Piece Extent="{ext}">\n      <PointData']
    if scalar is not None:
        head.append(f' Scalars="{scalar}"')
    if vector is not None:
        head.append(f' Vectors="{vector}"')
    head.append(">\n")
    offset = 0
    for a, d in blocks:
        head.append(f'        <DataArray type="Float32" Name="{a.name}" NumberOfComponents='
                    f'"{a.ncomp}" format="appended" offset="{offset}"/>\n')
        offset += 4 + d.size * 4
    head.append('      </PointData>\n    </Piece>\n  </ImageData>\n'
                '  <AppendedData encoding="raw">\n_')
    with open(path, "wb") as f:
        f.write("".join(head).encode())
        for _, d in blocks:
            f.write(struct.pack("<I", d.size * 4))
            f.write(d.tobytes())
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")


def write_pvd(path, frames) -> None:
    """Time series: frames = [(time, file path), ...], paths as given."""
    parts = ['<?xml version="1.0"?>\n',
             '<VTKFile type="Collection" version="0.1" byte_order="LittleEndian">\n',
             '  <Collection>\n']
    for t, name in frames:
        parts.append(f'    <DataSet timestep="{_g(t)}" group="" part="0" file="{name}"/>\n')
    parts.append('  </Collection>\n</VTKFile>\n')
    with open(path, "w", newline="") as f:
        f.write("".join(parts))
