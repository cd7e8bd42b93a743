"""Legacy-VTK output of frames and slices, in the format of the reference's
writers (OutputUVW and the scalar outputs, src/outputs.f90:2260-2300): a
binary RECTILINEAR_GRID with float32 big-endian coordinates and point data,
one SCALARS block per field.  Host-side; the arrays come from
Domain.download() / frame_wait() / scalar_slices().
"""
from __future__ import annotations

import numpy as np

from .config import Grid
from .workloads import interior


def _be32(a) -> bytes:
    return np.ascontiguousarray(a, dtype=">f4").tobytes()


def write_rectilinear(path: str, x, y, z, fields: dict, title: str = "CLMM output file"):
    """fields: name -> array of shape (len(z), len(y), len(x)), x fastest."""
    x, y, z = (np.asarray(a, dtype=np.float64) for a in (x, y, z))
    n = (len(x), len(y), len(z))
    with open(path, "wb") as f:
        w = f.write
        w(b"# vtk DataFile Version 2.0\n")
        w(title.encode() + b"\n")
        w(b"BINARY\n")
        w(b"DATASET RECTILINEAR_GRID\n")
        w(b"DIMENSIONS %d %d %d\n" % n)
        for name, c in (("X", x), ("Y", y), ("Z", z)):
            w(b"%s_COORDINATES %d float\n" % (name.encode(), len(c)))
            w(_be32(c) + b"\n")
        w(b"POINT_DATA %d\n" % (n[0] * n[1] * n[2]))
        for name, a in fields.items():
            a = np.asarray(a)
            assert a.shape == (n[2], n[1], n[0]), (name, a.shape, n)
            w(b"SCALARS %s float\n" % name.encode())
            w(b"LOOKUP_TABLE default\n")
            w(_be32(a) + b"\n")


def read_rectilinear(path: str):
    """The coordinates and fields of a file written by write_rectilinear."""
    data = open(path, "rb").read()
    pos = 0

    def line():
        nonlocal pos
        e = data.index(b"\n", pos)
        s = data[pos:e].decode()
        pos = e + 1
        return s

    for _ in range(4):
        line()
    dims = tuple(int(v) for v in line().split()[1:4])
    coords = []
    for n in dims:
        line()
        coords.append(np.frombuffer(data[pos:pos + 4 * n], dtype=">f4").astype(np.float64))
        pos += 4 * n + 1
    npts = int(line().split()[1])
    fields = {}
    while pos < len(data):
        name = line().split()[1]
        line()
        fields[name] = np.frombuffer(data[pos:pos + 4 * npts], dtype=">f4").reshape(dims[2], dims[1], dims[0])
        pos += 4 * npts + 1
    return coords, fields


def staggered_coords(grid: Grid, *, dx=1.0, dy=1.0, dz=1.0, origin=(0.0, 0.0, 0.0)):
    """xU, yV, zW (faces) and xPr, yPr, zPr (centres) of a uniform grid,
    index 1..n (src/initial.f90:4395-4480)."""
    x0, y0, z0 = origin
    g = grid
    xU = x0 + dx * np.arange(1, g.Prnx + 1)
    yV = y0 + dy * np.arange(1, g.Prny + 1)
    zW = z0 + dz * np.arange(1, g.Prnz + 1)
    return xU, yV, zW, xU - dx / 2, yV - dy / 2, zW - dz / 2


def write_uvw(grid: Grid, U, V, W, prefix: str, **grid_kw):
    """OutputUVW: one file per velocity component on its own staggered
    points, U on (xU, yPr, zPr), V on (xPr, yV, zPr), W on (xPr, yPr, zW)."""
    g = grid
    xU, yV, zW, xP, yP, zP = staggered_coords(g, **grid_kw)
    write_rectilinear(prefix + "U.vtk", xU[:g.Unx], yP[:g.Uny], zP[:g.Unz],
                      {"U": interior(U, -2, (g.Unx, g.Uny, g.Unz))})
    write_rectilinear(prefix + "V.vtk", xP[:g.Vnx], yV[:g.Vny], zP[:g.Vnz],
                      {"V": interior(V, -2, (g.Vnx, g.Vny, g.Vnz))})
    write_rectilinear(prefix + "W.vtk", xP[:g.Wnx], yP[:g.Wny], zW[:g.Wnz],
                      {"W": interior(W, -2, (g.Wnx, g.Wny, g.Wnz))})


def write_scalar_slices(grid: Grid, xy, xz, k: int, j: int, path: str, name: str = "scalar01_avg", **grid_kw):
    """The time-averaged slices of a scalar as two planar rectilinear grids:
    the horizontal plane through level k and the vertical plane through row
    j (files path + "_xy.vtk" and path + "_xz.vtk")."""
    g = grid
    _, _, _, xP, yP, zP = staggered_coords(g, **grid_kw)
    if xy is not None:
        write_rectilinear(path + "_xy.vtk", xP, yP, zP[k - 1:k], {name: np.asarray(xy)[None, :, :]})
    if xz is not None:
        write_rectilinear(path + "_xz.vtk", xP, yP[j - 1:j], zP, {name: np.asarray(xz)[:, None, :]})
