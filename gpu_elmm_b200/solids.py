"""Solid bodies on the staggered grid: the start-up geometry pass of the
reference for bodies that are axis-aligned boxes or spheres, producing the
point lists that `elmm_set_solids` (include/elmm_gpu.h) takes.

This is the host side of the immersed-boundary method, run once per domain;
the library applies the lists every RK3 stage.  It restates, for a body
given by its inside test, closest point and closest point outwards
(methods of Box and Sphere):

  * FindInsideCells (src/solidbodies.f90:75-206): Prtype/Utype/Vtype/Wtype
    = body number where the point lies inside the body grown by
    delta = (dx dy dz)^(1/3) / 20, over the index range -2..n+3;
  * FindNeighbouringCells / AuxNeighbours (src/immersedboundary.f90:1475-1506):
    free points with a solid point in their 3x3x3 neighbourhood get type -1;
  * InitImBoundaries (:1650-1747) with TVelIBPoint_Create (:690-904),
    InterpolationPoints (:907-1020, first-order least-squares coefficients
    :1047-1062, weights of Peller et al.) and TScalFlIBPoint_Create
    (:1065-1410);
  * GetSolidBodiesWM_UVW (:139-306): wall-model points of free velocity
    points next to a solid one;
  * SetNullifiedPoints (src/initial.f90:4861-4962);
  * the bottom-wall points that GetOutsideBoundariesWM_UVW leaves out
    (src/wallmodels.f90:700-820: only Xtype(i,j,1) == 0 and Xtype(i,j,0) <= 0).

Geometry of a sphere (GeometricShapes Sphere, src/geometricshapes.f90:1128-
1149): inside within r + eps of the centre, Closest along the ray from the
centre, ClosestOut = Closest (GeometricShape_ClosestOut, :343-349).

Geometry of a box (GeometricShapes ConvexPolyhedron, src/geometricshapes.f90):
its planes are, in this order, x >= x0, x <= x1, y >= y0, y <= y1, z >= z0,
z <= z1 (unit normals; Plane_Inside :632-642).  Inside tests every plane;
ClosestOut projects onto the nearest plane (the first one on ties,
:940-966); Closest of a point outside is the nearest point of the box, which
is what ConvexPolyhedron_Closest (:721-938) finds for a box in exact
arithmetic (face, edge line, or corner); ClosestOnLineOut is the bisection of
Body (:2976-3013).  Periodic x and y wrap the coordinates as CInside does
(:2920-2950).
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from .config import (BC_NOSLIP, BC_PERIODIC, IB_MAX_INTERP, ElmmConfig, ElmmIBPoint, ElmmSolids, ElmmWMPoint,
                     grid_of)

MINUSX, PLUSX, MINUSY, PLUSY, MINUSZ, PLUSZ = 1, 2, 3, 4, 5, 6
_DIRS = {MINUSX: (-1, 0, 0), PLUSX: (1, 0, 0), MINUSY: (0, -1, 0), PLUSY: (0, 1, 0),
         MINUSZ: (0, 0, -1), PLUSZ: (0, 0, 1)}
N_LS = 2  # least-squares interpolation points per direction (immersedboundary.f90:584)


@dataclass
class Box:
    """An axis-aligned solid body [x0,x1] x [y0,y1] x [z0,z1] with roughness z0r
    (SolidBody: rough when z0r > 0)."""
    x0: float
    x1: float
    y0: float
    y1: float
    z0: float
    z1: float
    z0r: float = 0.1
    heat_flux: float = 0.0

    def planes(self):
        # (axis, offset, gl): gl -> coordinate - offset >= -eps, else <= eps
        return ((0, self.x0, True), (0, self.x1, False), (1, self.y0, True), (1, self.y1, False),
                (2, self.z0, True), (2, self.z1, False))

    def inside(self, x, y, z, eps):
        """ConvexPolyhedron_Inside: every plane (Plane_Inside, :632-642)."""
        p = (x, y, z)
        for axis, off, gl in self.planes():
            v = p[axis] - off
            if gl:
                if not v >= -eps:
                    return False
            elif not v <= eps:
                return False
        return True

    def mask(self, x, y, z, eps):
        """inside() on the grid lines x, y, z (1-D arrays): a [k, j, i] mask."""
        mx = (x - self.x0 >= -eps) & (x - self.x1 <= eps)
        my = (y - self.y0 >= -eps) & (y - self.y1 <= eps)
        mz = (z - self.z0 >= -eps) & (z - self.z1 <= eps)
        return mz[:, None, None] & my[None, :, None] & mx[None, None, :]

    def closest(self, x, y, z):
        """The nearest point of the box (ConvexPolyhedron_Closest, :721-938)."""
        return (min(max(x, self.x0), self.x1), min(max(y, self.y0), self.y1), min(max(z, self.z0), self.z1))

    def closest_out(self, x, y, z):
        """The projection onto the nearest face plane, the first on ties
        (ConvexPolyhedron_ClosestOut, :940-966)."""
        p = [x, y, z]
        best, arg = math.inf, None
        for axis, off, _ in self.planes():
            d = abs(p[axis] - off)
            if d >= 0 and d < best:
                best, arg = d, (axis, off)
        q = list(p)
        q[arg[0]] = arg[1]
        return tuple(q)


@dataclass
class Sphere:
    """A solid sphere of radius r centred at (xc, yc, zc) with roughness z0r
    (GeometricShapes Sphere, src/geometricshapes.f90:142-147)."""
    xc: float
    yc: float
    zc: float
    r: float
    z0r: float = 0.1
    heat_flux: float = 0.0

    def inside(self, x, y, z, eps):
        """Sphere_Inside (:1128-1134)."""
        return (self.xc - x) ** 2 + (self.yc - y) ** 2 + (self.zc - z) ** 2 <= (self.r + eps) ** 2

    def mask(self, x, y, z, eps):
        return ((self.xc - x[None, None, :]) ** 2 + (self.yc - y[None, :, None]) ** 2 +
                (self.zc - z[:, None, None]) ** 2) <= (self.r + eps) ** 2

    def closest(self, x, y, z):
        """Sphere_Closest (:1136-1149): the point of the sphere on the ray
        from the centre through (x, y, z)."""
        a, b, c = x - self.xc, y - self.yc, z - self.zc
        t = self.r / math.sqrt(a ** 2 + b ** 2 + c ** 2)
        return (a * t + self.xc, b * t + self.yc, c * t + self.zc)

    def closest_out(self, x, y, z):
        """GeometricShape_ClosestOut (:343-349): Closest."""
        return self.closest(x, y, z)


_EPS10 = 10 * 2.220446049250313e-16  # the default eps of GeometricShape_Inside, 10 * epsilon(1._knd)
_TINY = 2.2250738585072014e-308      # tiny(1._knd)


@dataclass
class Cylinder:
    """A solid cylinder between the centres p1 and p2 of its end caps, radius
    r, roughness z0r (Cylinder, src/geometricshapes.f90:171-177, 1278-1440:
    a CylJacket through p1 along p2 - p1 and, unless infinite, the cap planes
    through p1 and p2 with the outward normals p1 - p2 and p2 - p1).  The
    reference's Plane_Closest moves a point by the plane's signed distance
    times the normal, which the cap planes leave unnormalised, so a cap's
    closest point lies |p2 - p1| times the distance away; restated as
    written, the wall-model distance vectors to a cap carry that factor (it
    is 1 for a cylinder of unit length)."""
    p1: tuple
    p2: tuple
    r: float
    z0r: float = 0.1
    infinite: bool = False
    heat_flux: float = 0.0

    def __post_init__(self):
        x1, y1, z1 = (float(v) for v in self.p1)
        x2, y2, z2 = (float(v) for v in self.p2)
        self.jac = (x1, y1, z1, x2 - x1, y2 - y1, z2 - z1)  # CylJacket_Init(point1, point2 - point1, radius)
        # Plane_Init_3r(point, normal): d = -(a xc + b yc + c zc)
        def plane(xc, yc, zc, a, b, c):
            return (a, b, c, -(a * xc + b * yc + c * zc))
        self.planes = () if self.infinite else (plane(x1, y1, z1, x1 - x2, y1 - y2, z1 - z2),
                                                 plane(x2, y2, z2, x2 - x1, y2 - y1, z2 - z1))

    # ------------------------------------------------------------ parts
    def _jacket_inside(self, x, y, z, eps):
        """CylJacket_Inside with LineDist (:380-391, :1300-1306)."""
        xl, yl, zl, a, b, c = self.jac
        t = (a * (x - xl) + b * (y - yl) + c * (z - zl)) / (a ** 2 + b ** 2 + c ** 2) \
            if (a != 0 or b != 0 or c != 0) else 0 * x
        return np.sqrt((xl + a * t - x) ** 2 + (yl + b * t - y) ** 2 + (zl + c * t - z) ** 2) <= self.r + eps

    @staticmethod
    def _plane_inside(pl, x, y, z, eps):
        """Plane_Inside (:632-642) of a plane built with GL false."""
        a, b, c, d = pl
        return a * x + b * y + c * z + d <= eps * math.sqrt(a ** 2 + b ** 2 + c ** 2)

    @staticmethod
    def _plane_closest(pl, x, y, z):
        """Plane_Closest (:644-660), the unnormalised step as written."""
        a, b, c, d = pl
        if abs(a) > _TINY or abs(b) > _TINY or abs(c) > _TINY:
            t = -(a * x + b * y + c * z + d) / math.sqrt(a ** 2 + b ** 2 + c ** 2)
        else:
            t = 0.0
        return (x + a * t, y + b * t, z + c * t)

    def _jacket_closest(self, x, y, z):
        """CylJacket_Closest (:1308-1325) through Line_Closest (:441-456)."""
        xc, yc, zc, a, b, c = self.jac
        t = (a * (x - xc) + b * (y - yc) + c * (z - zc)) / (a ** 2 + b ** 2 + c ** 2) \
            if (a != 0 or b != 0 or c != 0) else 0.0
        xl, yl, zl = xc + a * t, yc + b * t, zc + c * t
        p, q, w = x - xl, y - yl, z - zl
        with np.errstate(all="ignore"):  # a point on the axis: IEEE inf and nan, unused by the callers then
            t = np.float64(self.r) / np.sqrt(np.float64(p ** 2 + q ** 2 + w ** 2))
            return (float(p * t + xl), float(q * t + yl), float(w * t + zl))

    @staticmethod
    def _dist(x1, y1, z1, x2, y2, z2):
        """PointDist (:374-378)."""
        return math.sqrt((x1 - x2) ** 2 + (y1 - y2) ** 2 + (z1 - z2) ** 2)

    # -------------------------------------------------------- interface
    def inside(self, x, y, z, eps):
        """Cylinder_Inside (:1330-1345)."""
        if not self._jacket_inside(x, y, z, eps):
            return False
        return all(self._plane_inside(pl, x, y, z, eps) for pl in self.planes)

    def mask(self, x, y, z, eps):
        X, Y, Z = x[None, None, :], y[None, :, None], z[:, None, None]
        m = self._jacket_inside(X, Y, Z, eps)
        for pl in self.planes:
            m = m & self._plane_inside(pl, X, Y, Z, eps)
        return np.broadcast_to(m, (len(z), len(y), len(x)))

    def closest(self, x, y, z):
        """Cylinder_Closest (:1347-1400), for caps perpendicular to the axis."""
        if not self.planes:
            return self._jacket_closest(x, y, z)
        pl1, pl2 = self.planes
        j = self._jacket_closest(x, y, z)
        p1 = self._plane_closest(pl1, x, y, z)
        p2 = self._plane_closest(pl2, x, y, z)
        if self._jacket_inside(x, y, z, _EPS10):
            return p1 if self._dist(x, y, z, *p1) <= self._dist(x, y, z, *p2) else p2
        if self._plane_inside(pl1, x, y, z, _EPS10) and self._plane_inside(pl2, x, y, z, _EPS10):
            return j
        if self._dist(x, y, z, *p1) <= self._dist(x, y, z, *p2):
            return self._jacket_closest(*p1)
        return self._jacket_closest(*p2)

    def closest_out(self, x, y, z):
        """Cylinder_ClosestOut (:1402-1440)."""
        far = math.sqrt(1.7976931348623157e308) / 10
        p1 = self._plane_closest(self.planes[0], x, y, z) if self.planes else (far, far, far)
        p2 = self._plane_closest(self.planes[1], x, y, z) if self.planes else (far, far, far)
        j = self._jacket_closest(x, y, z)
        d1, d2, dj = self._dist(x, y, z, *p1), self._dist(x, y, z, *p2), self._dist(x, y, z, *j)
        if d1 <= d2 and d1 <= dj:
            return p1
        if d2 <= d1 and d2 <= dj:
            return p2
        return j  # dj <= d1, d2; also when a NaN fails all three tests (a point on the axis)


def cube_array(n_per_side: int, edge: float, pitch: float, height: float, *, offset: float, depth: float,
               z0r: float = 0.1):
    """n x n cubes of the given edge (x, y) and height at `pitch` spacing,
    the first at `offset`; they reach `depth` below the ground so that the
    ghost layer under them is solid too."""
    return [Box(offset + a * pitch, offset + a * pitch + edge, offset + b * pitch, offset + b * pitch + edge,
                -depth, height, z0r) for b in range(n_per_side) for a in range(n_per_side)]


class _Coords:
    """xU, yV, zW and the cell centres over index -3..n+3 with the formulas of
    src/initial.f90:4395-4480 (z ghosts as the library builds them)."""

    def __init__(self, cfg: ElmmConfig):
        nx, ny, nz = cfg.Prnx, cfg.Prny, cfg.Prnz
        self.nx, self.ny, self.nz = nx, ny, nz
        self.o = 3  # array position of index 0
        i = np.arange(-3, nx + 4)
        j = np.arange(-3, ny + 4)
        self.xU = i * cfg.dxmin + cfg.xmin
        self.yV = j * cfg.dymin + cfg.ymin
        Z = np.zeros(nz + 7)
        if cfg.zW:
            zw = np.ctypeslib.as_array(cfg.zW, shape=(nz + 1,))
            Z[3:nz + 4] = zw
            if cfg.Btype[4] == BC_PERIODIC:
                for k in range(-1, -4, -1):
                    Z[k + 3] = Z[3] - (Z[nz - 1 + 3] - Z[nz - 1 + k + 3])
            else:
                for k in range(-1, -4, -1):
                    Z[k + 3] = Z[3] - (Z[-k + 3] - Z[3])
            if cfg.Btype[5] == BC_PERIODIC:
                for k in range(nz + 1, nz + 4):
                    Z[k + 3] = Z[nz - 1 + 3] + (Z[k - nz + 1 + 3] - Z[3])
            else:
                for k in range(nz + 1, nz + 4):
                    Z[k + 3] = Z[nz - 1 + 3] + (Z[nz - 1 + 3] - Z[nz - 1 - (k - nz + 1) + 3])
            dz = np.diff(Z[1:])  # dzPr(k) = zW(k) - zW(k-1), k = -2..nz+3
            self.dzmin = float(dz.min())
        else:
            Z = np.arange(-3, nz + 4) * cfg.dzmin + cfg.zmin
            self.dzmin = cfg.dzmin
        self.zW = Z
        self.xPr = np.concatenate([[np.nan], (self.xU[:-1] + self.xU[1:]) / 2])
        self.yPr = np.concatenate([[np.nan], (self.yV[:-1] + self.yV[1:]) / 2])
        self.zPr = np.concatenate([[np.nan], (self.zW[:-1] + self.zW[1:]) / 2])
        self.dx, self.dy = cfg.dxmin, cfg.dymin
        self.px = cfg.Btype[0] == BC_PERIODIC
        self.py = cfg.Btype[2] == BC_PERIODIC
        self.lx = self.xU[nx + 3] - self.xU[3]
        self.ly = self.yV[ny + 3] - self.yV[3]

    def x(self, a, i):
        return float(a[i + self.o])


class Geometry:
    def __init__(self, cfg: ElmmConfig, boxes):
        self.cfg = cfg
        self.c = _Coords(cfg)
        self.boxes = list(boxes)
        g = grid_of(cfg)
        self.g = g
        c = self.c
        # the four grids: (sizes, x coordinates, y coordinates, z coordinates)
        self.grids = {
            0: ((g.Prnx, g.Prny, g.Prnz), c.xPr, c.yPr, c.zPr),
            1: ((g.Unx, g.Uny, g.Unz), c.xU, c.yPr, c.zPr),
            2: ((g.Vnx, g.Vny, g.Vnz), c.xPr, c.yV, c.zPr),
            3: ((g.Wnx, g.Wny, g.Wnz), c.xPr, c.yPr, c.zW),
        }
        self.delta = (cfg.dxmin * cfg.dymin * c.dzmin) ** (1.0 / 3) / 20
        self.types = {q: self._find_inside(q) for q in range(4)}
        for q in range(4):
            self._aux_neighbours(q)

    # --------------------------------------------------------- geometry
    def _wrap(self, x, y, z):
        c = self.c
        if c.px and x > c.xU[c.nx + 1 + 3]:
            x = x - c.lx
        if c.py and y > c.yV[c.ny + 1 + 3]:
            y = y - c.ly
        if c.px and x < c.xU[3]:
            x = x + c.lx
        if c.py and y < c.yV[3]:
            y = y + c.ly
        return x, y, z

    def inside(self, b, x, y, z, eps):
        """CInside: the body's inside test of the periodically wrapped point."""
        x, y, z = self._wrap(x, y, z)
        return b.inside(x, y, z, eps)

    @staticmethod
    def closest(b, x, y, z):
        return b.closest(x, y, z)

    @staticmethod
    def closest_out(b, x, y, z):
        return b.closest_out(x, y, z)

    def closest_on_line_out(self, b, x, y, z, x2, y2, z2):
        t1, t2 = 0.0, 1.0
        if self.inside(b, x2, y2, z2, 0.0):
            t1 = 1.0
            while True:
                t2 = t2 * 1.1
                if not self.inside(b, x + (x2 - x) * t2, y + (y2 - y) * t2, z + (z2 - z) * t2, 0.0):
                    break
                if t2 >= 2:
                    return 10.0
        t = (t1 + t2) / 2.0
        lim = min(self.cfg.dxmin / 1000.0, self.cfg.dymin / 1000.0, self.c.dzmin / 1000.0)
        for _ in range(20):
            if self.inside(b, x + (x2 - x) * t, y + (y2 - y) * t, z + (z2 - z) * t, 0.0):
                t1 = t
            else:
                t2 = t
            t = (t1 + t2) / 2.0
            if abs(t1 - t2) < lim:
                break
        return t

    # ------------------------------------------------------------ types
    def _find_inside(self, q):
        (nx, ny, nz), X, Y, Z = self.grids[q]
        o = self.c.o
        xs, ys, zs = X[o - 2:o + nx + 4], Y[o - 2:o + ny + 4], Z[o - 2:o + nz + 4]
        t = np.zeros((nz + 6, ny + 6, nx + 6), dtype=np.int32)  # [k+2, j+2, i+2]
        e = self.delta
        xw, yw = np.array([self._wrap(x, 0, 0)[0] for x in xs]), np.array([self._wrap(0, y, 0)[1] for y in ys])
        for nb, b in enumerate(self.boxes, start=1):
            t[b.mask(xw, yw, zs, e)] = nb
        return t

    def _aux_neighbours(self, q):
        t = self.types[q]
        solid = t > 0
        near = np.zeros_like(solid)
        K, J, I = t.shape
        # points -1..n+2 (array 1..n+4) look at their 3x3x3 neighbourhood
        for dk in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for di in (-1, 0, 1):
                    near[1:K - 1, 1:J - 1, 1:I - 1] |= solid[1 + dk:K - 1 + dk, 1 + dj:J - 1 + dj, 1 + di:I - 1 + di]
        m = (t == 0) & near
        m[0, :, :] = m[-1, :, :] = False
        m[:, 0, :] = m[:, -1, :] = False
        m[:, :, 0] = m[:, :, -1] = False
        t[m] = -1

    def typ(self, q, i, j, k):
        return int(self.types[q][k + 2, j + 2, i + 2])

    # ------------------------------------------------------ IB velocity
    def vel_ib_point(self, comp, xi, yj, zk):
        """TVelIBPoint_Create + InterpolationPoints: (interp points, coefs)."""
        (nx, ny, nz), X, Y, Z = self.grids[comp]
        c = self.c
        T = lambda i, j, k: self.typ(comp, i, j, k)
        x, y, z = c.x(X, xi), c.x(Y, yj), c.x(Z, zk)
        b = self.boxes[T(xi, yj, zk) - 1]
        null = ([], [])
        if not self.inside(b, x, y, z, 0.0):
            return null
        xn, yn, zn = self.closest_out(b, x, y, z)
        if math.sqrt((x - xn) ** 2 + (y - yn) ** 2 + (z - zn) ** 2) <= 0.1 * (
                self.cfg.dxmin * self.cfg.dymin * c.dzmin) ** (1.0 / 3):
            return null
        free = lambda i, j, k: T(i, j, k) <= 0
        fxm = all(free(xi - i, yj, zk) for i in range(1, N_LS + 1))
        fym = all(free(xi, yj - i, zk) for i in range(1, N_LS + 1))
        fzm = all(free(xi, yj, zk - i) for i in range(1, N_LS + 1))
        fxp = all(free(xi + i, yj, zk) for i in range(1, N_LS + 1))
        fyp = all(free(xi, yj + i, zk) for i in range(1, N_LS + 1))
        fzp = all(free(xi, yj, zk + i) for i in range(1, N_LS + 1))
        f1xm, f1ym, f1zm = free(xi - 1, yj, zk), free(xi, yj - 1, zk), free(xi, yj, zk - 1)
        f1xp, f1yp, f1zp = free(xi + 1, yj, zk), free(xi, yj + 1, zk), free(xi, yj, zk + 1)
        if ((f1xm and not fxm) or (f1ym and not fym) or (f1zm and not fzm) or (f1xp and not fxp) or
                (f1yp and not fyp) or (f1zp and not fzp)):
            return null
        blk = self.types[comp][zk + 1:zk + 4, yj + 1:yj + 4, xi + 1:xi + 4]
        if int((blk > 0).sum()) > 21:
            return null
        if (f1xm and f1xp) or (f1ym and f1yp) or (f1zm and f1zp):
            return null
        dirs = []
        for fm, fp in ((fxm, fxp), (fym, fyp), (fzm, fzp)):
            dirs.append(0 if (not fm and not fp) else (-1 if fm else 1))
        dist = [0.0, 0.0, 0.0]
        coords = (X, Y, Z)
        idx = [xi, yj, zk]
        pt = [x, y, z]
        for a in range(3):
            if dirs[a] != 0:
                p2 = list(pt)
                p2[a] = c.x(coords[a], idx[a] + dirs[a])
                t = self.closest_on_line_out(b, x, y, z, *p2)
                if t > 1 or t < 0.05:
                    dirs[a] = 0
                    t = 0.0
                dist[a] = t * (c.x(coords[a], idx[a] + dirs[a]) - c.x(coords[a], idx[a]))
        if dirs == [0, 0, 0]:
            return null
        # InterpolationPoints (first order): per direction N_LS points, then the
        # weights beta of Peller et al. (eq. 17-19)
        d = [1.0, 1.0, 1.0]
        parts = []
        for a in range(3):
            if dirs[a] == 0:
                continue
            xr = c.x(coords[a], idx[a]) + dist[a]
            xs = [c.x(coords[a], idx[a] + i * dirs[a]) for i in range(0, N_LS + 1)]
            A = sum((xs[i] - xr) ** 2 for i in range(1, N_LS + 1))
            cf = [(xs[i] - xr) * (xs[0] - xr) / A for i in range(1, N_LS + 1)]
            d[a] = abs(xs[0] - xr)
            pts = []
            for i in range(1, N_LS + 1):
                q = list(idx)
                q[a] += i * dirs[a]
                pts.append(tuple(q))
            parts.append((a, pts, cf))
        prod = d[0] * d[1] * d[2]
        beta = [prod / d[a] ** 2 if dirs[a] != 0 else 0.0 for a in range(3)]
        csum = beta[0] + beta[1] + beta[2]
        out_p, out_c = [], []
        for a, pts, cf in parts:
            out_p += pts
            out_c += [v * beta[a] / csum for v in cf]
        return out_p, out_c

    # ----------------------------------------------------- IB viscosity
    def scalfl_point(self, xi, yj, zk):
        """TScalFlIBPoint_Create: (interp points, coefs) of a solid Pr cell."""
        c = self.c
        X, Y, Z = c.xPr, c.yPr, c.zPr
        T = lambda i, j, k: self.typ(0, i, j, k)
        x, y, z = c.x(X, xi), c.x(Y, yj), c.x(Z, zk)
        b = self.boxes[T(xi, yj, zk) - 1]
        xn, yn, zn = self.closest_out(b, x, y, z)
        distx, disty, distz = xn - x, yn - y, zn - z
        sgn = lambda v: 1 if math.copysign(1.0, v) > 0 else -1
        dirx, diry, dirz = sgn(distx), sgn(disty), sgn(distz)
        if abs(distx) < (c.x(X, xi + 1) - c.x(X, xi - 1)) / 100.0:
            distx, dirx = 0.0, 0
        if abs(disty) < (c.x(Y, yj + 1) - c.x(Y, yj - 1)) / 100.0:
            disty, diry = 0.0, 0
        if abs(distz) < (c.x(c.zW, zk + 1) - c.x(c.zW, zk - 1)) / 100.0:
            distz, dirz = 0.0, 0
        fp00, fm00 = T(xi + 1, yj, zk) <= 0, T(xi - 1, yj, zk) <= 0
        f0p0, f0m0 = T(xi, yj + 1, zk) <= 0, T(xi, yj - 1, zk) <= 0
        f00p, f00m = T(xi, yj, zk + 1) <= 0, T(xi, yj, zk - 1) <= 0
        if not (fp00 or fm00):
            dirx, distx = 0, 0.0
        if not (f0p0 or f0m0):
            diry, disty = 0, 0.0
        if not (f00p or f00m):
            dirz, distz = 0, 0.0
        nfree = sum((fp00, f0p0, f00p, fm00, f0m0, f00m))
        ndirs = (dirx != 0) + (diry != 0) + (dirz != 0)
        if nfree > ndirs or (fp00 and fm00) or (f0p0 and f0m0) or (f00p and f00m):
            distx = disty = distz = 0.0
            dirx = diry = dirz = 0
        if dirx == 0 and diry == 0 and dirz == 0:
            dx2 = (1 if fp00 else 0) - (1 if fm00 else 0)
            dy2 = (1 if f0p0 else 0) - (1 if f0m0 else 0)
            dz2 = (1 if f00p else 0) - (1 if f00m else 0)
            if dx2 == 0 and dy2 == 0 and dz2 == 0:
                pts = []
                for f, q in ((fp00, (xi + 1, yj, zk)), (fm00, (xi - 1, yj, zk)), (f0p0, (xi, yj + 1, zk)),
                             (f0m0, (xi, yj - 1, zk)), (f00p, (xi, yj, zk + 1)), (f00m, (xi, yj, zk - 1))):
                    if f:
                        pts.append(q)
                return pts, [1.0 / nfree] * nfree
            return [(xi + dx2, yj + dy2, zk + dz2)], [1.0]
        if nfree == 1 or ndirs == 1:
            return [(xi + dirx, yj + diry, zk + dirz)], [1.0]
        if nfree == 2 or ndirs == 2:
            if dirx == 0:  # plane yz
                if abs(disty / distz) < abs(c.x(Y, yj + diry) - y) / abs(c.x(Z, zk + dirz) - z):
                    t = (c.x(Z, zk + dirz) - z) / distz
                    c1 = abs(disty * t) / abs(c.x(Y, yj + diry) - c.x(Y, yj))
                    return [(xi, yj + diry, zk + dirz), (xi, yj, zk + dirz)], [c1, 1 - c1]
                t = (c.x(Y, yj + diry) - y) / disty
                c1 = abs(distz * t) / abs(c.x(Z, zk + dirz) - c.x(Z, zk))
                return [(xi, yj + diry, zk + dirz), (xi, yj + diry, zk)], [c1, 1 - c1]
            if diry == 0:  # plane xz
                if abs(distx / distz) < abs(c.x(X, xi + dirx) - x) / abs(c.x(Z, zk + dirz) - z):
                    t = (c.x(Z, zk + dirz) - z) / distz
                    c1 = abs(distx * t) / abs(c.x(X, xi + dirx) - c.x(X, xi))
                    return [(xi + dirx, yj, zk + dirz), (xi, yj, zk + dirz)], [c1, 1 - c1]
                t = (c.x(X, xi + dirx) - x) / distx
                c1 = abs(distz * t) / abs(c.x(Z, zk + dirz) - c.x(Z, zk))
                return [(xi + dirx, yj, zk + dirz), (xi + dirx, yj, zk)], [c1, 1 - c1]
            # plane xy
            if abs(distx / disty) < abs(c.x(X, xi + dirx) - x) / abs(c.x(Y, yj + diry) - y):
                t = (c.x(Y, yj + diry) - y) / disty
                c1 = abs(distx * t) / abs(c.x(X, xi + dirx) - c.x(X, xi))
                return [(xi + dirx, yj + diry, zk), (xi, yj + diry, zk)], [c1, 1 - c1]
            t = (c.x(X, xi + dirx) - x) / distx
            c1 = abs(disty * t) / abs(c.x(Y, yj + diry) - c.x(Y, yj))
            return [(xi + dirx, yj + diry, zk), (xi + dirx, yj, zk)], [c1, 1 - c1]
        # three directions: the gridline plane crossed first
        tx = (c.x(X, xi + dirx) - x) / distx
        ty = (c.x(Y, yj + diry) - y) / disty
        tz = (c.x(Z, zk + dirz) - z) / distz
        ax = lambda t: abs(distx * t) / abs(c.x(X, xi + dirx) - x)
        ay = lambda t: abs(disty * t) / abs(c.x(Y, yj + diry) - y)
        az = lambda t: abs(distz * t) / abs(c.x(Z, zk + dirz) - z)
        if tx <= ty and tx <= tz:
            a, bb = ay(tx), az(tx)
            return ([(xi + dirx, yj + diry, zk + dirz), (xi + dirx, yj, zk + dirz), (xi + dirx, yj + diry, zk),
                     (xi + dirx, yj, zk)], [a * bb, (1 - a) * bb, a * (1 - bb), (1 - a) * (1 - bb)])
        if ty <= tx and ty <= tz:
            a, bb = ax(ty), az(ty)
            return ([(xi + dirx, yj + diry, zk + dirz), (xi, yj + diry, zk + dirz), (xi + dirx, yj + diry, zk),
                     (xi, yj + diry, zk)], [a * bb, (1 - a) * bb, a * (1 - bb), (1 - a) * (1 - bb)])
        a, bb = ax(tz), ay(tz)
        return ([(xi + dirx, yj + diry, zk + dirz), (xi, yj + diry, zk + dirz), (xi + dirx, yj, zk + dirz),
                 (xi, yj, zk + dirz)], [a * bb, (1 - a) * bb, a * (1 - bb), (1 - a) * (1 - bb)])

    # --------------------------------------------------- lists
    def _boundary_points(self, q):
        """Solid points of grid q with a free 6-neighbour, k, j, i order."""
        (nx, ny, nz), _, _, _ = self.grids[q]
        t = self.types[q]
        s = t[3:nz + 3, 3:ny + 3, 3:nx + 3] > 0  # points 1..n sit at array position index + 2
        f = np.zeros_like(s)
        for dk, dj, di in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)):
            f |= t[3 + dk:nz + 3 + dk, 3 + dj:ny + 3 + dj, 3 + di:nx + 3 + di] <= 0
        k, j, i = np.nonzero(s & f)
        return [(int(a) + 1, int(b) + 1, int(cc) + 1) for cc, b, a in zip(k, j, i)]

    def null_points(self, q):
        (nx, ny, nz), _, _, _ = self.grids[q]
        t = self.types[q]
        s = t[3:nz + 3, 3:ny + 3, 3:nx + 3] > 0
        for dk, dj, di in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)):
            s &= t[3 + dk:nz + 3 + dk, 3 + dj:ny + 3 + dj, 3 + di:nx + 3 + di] > 0
        k, j, i = np.nonzero(s)
        return np.stack([i + 1, j + 1, k + 1], axis=1).astype(np.int32) if len(i) else np.zeros((0, 3), np.int32)

    def wm_points(self):
        """GetSolidBodiesWM_UVW: (component, direction, i, j, k, dist, z0)."""
        out = []
        c = self.c
        mwd = (self.cfg.dxmin * self.cfg.dymin * c.dzmin) ** (1.0 / 3) / 20
        for comp in (1, 2, 3):
            (nx, ny, nz), X, Y, Z = self.grids[comp]
            t = self.types[comp]
            ks, js, is_ = np.nonzero(t[3:nz + 3, 3:ny + 3, 3:nx + 3] < 0)
            for kk, jj, ii in zip(ks, js, is_):
                i, j, k = int(ii) + 1, int(jj) + 1, int(kk) + 1
                for dr in range(1, 7):
                    m, n, o = _DIRS[dr]
                    nb = self.typ(comp, i + m, j + n, k + o)
                    if nb <= 0:
                        continue
                    b = self.boxes[nb - 1]
                    x, y, z = c.x(X, i), c.x(Y, j), c.x(Z, k)
                    near = self.closest(b, x, y, z)
                    dv = [near[0] - x, near[1] - y, near[2] - z]
                    dist = math.sqrt(dv[0] ** 2 + dv[1] ** 2 + dv[2] ** 2)
                    dot = dv[0] * m + dv[1] * n + dv[2] * o
                    if not (dot / (dist * 1.0) > 0.4 if dist > 0 else False):
                        xm, ym, zm = c.x(X, i + m), c.x(Y, j + n), c.x(Z, k + o)
                        tt = self.closest_on_line_out(b, xm, ym, zm, x, y, z)
                        near = (xm + tt * (x - xm), ym + tt * (y - ym), zm + tt * (z - zm))
                        dv2 = [near[0] - x, near[1] - y, near[2] - z]
                        d2 = math.sqrt(dv2[0] ** 2 + dv2[1] ** 2 + dv2[2] ** 2)
                        if d2 < dist and d2 < mwd:
                            pass  # keeps the closest-point vector (immersedboundary.f90:211-224)
                        else:
                            dv = dv2
                    if math.sqrt(dv[0] ** 2 + dv[1] ** 2 + dv[2] ** 2) < mwd:
                        raise ValueError(f"wall-model point too close to the wall: {comp} {(i, j, k)}")
                    rough = b.z0r > 0  # a rough body's points carry its z0 and heat flux
                    out.append((comp, dr, i, j, k, tuple(dv), b.z0r if rough else 0.0,
                                b.heat_flux if rough else 0.0))
        return out

    def solid_pr(self):
        """Pr cells with Prtype > 0: i, j in 1..n (the x and y ghosts are
        periodic images) and k in -1..nz+2 (the z ghost layers the
        temperature's fill of the solid cells reaches)."""
        g = self.g
        t = self.types[0][1:g.Prnz + 5, 3:g.Prny + 3, 3:g.Prnx + 3]
        k, j, i = np.nonzero(t > 0)
        return np.stack([i + 1, j + 1, k - 1], axis=1).astype(np.int32) if len(i) else np.zeros((0, 3), np.int32)

    def wm_pr(self):
        """The Pr wall-model points of the scalar equations, each cell once:
        GetSolidBodiesWM's free cells (Prtype <= 0) with a solid 6-neighbour
        and GetOutsideBoundariesWM_Pr's cells of a no-slip z wall with
        Prtype == 0 (the domain's x and y are periodic)."""
        g, cfg = self.g, self.cfg
        t = self.types[0]
        nx, ny, nz = g.Prnx, g.Prny, g.Prnz
        inner = t[3:nz + 3, 3:ny + 3, 3:nx + 3]
        near = np.zeros(inner.shape, dtype=bool)
        for dk, dj, di in ((0, 0, 1), (0, 0, -1), (0, 1, 0), (0, -1, 0), (1, 0, 0), (-1, 0, 0)):
            near |= t[3 + dk:nz + 3 + dk, 3 + dj:ny + 3 + dj, 3 + di:nx + 3 + di] > 0
        pts = (inner <= 0) & near
        if cfg.Btype[4] == BC_NOSLIP:
            pts[0] |= inner[0] == 0
        if cfg.Btype[5] == BC_NOSLIP:
            pts[nz - 1] |= inner[nz - 1] == 0
        k, j, i = np.nonzero(pts)
        return np.stack([i + 1, j + 1, k + 1], axis=1).astype(np.int32) if len(i) else np.zeros((0, 3), np.int32)

    def _face_point(self, i, j, k):
        """GetSolidBodiesWM's choice for a free cell: the nearest body among
        its solid 6-neighbours' (Closest, in the order +x, -x, +y, -y, +z,
        -z) and the distance vector, or (0, inf, None)."""
        c = self.c
        nb, dist, dv = 0, math.inf, None
        x, y, z = c.x(c.xPr, i), c.x(c.yPr, j), c.x(c.zPr, k)
        for m, n, o in ((1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)):
            t = self.typ(0, i + m, j + n, k + o)
            if t > 0 and t != nb:
                near = self.closest(self.boxes[t - 1], x, y, z)
                dd = math.sqrt((near[0] - x) ** 2 + (near[1] - y) ** 2 + (near[2] - z) ** 2)
                if dd < dist:
                    dist, nb, dv = dd, t, (near[0] - x, near[1] - y, near[2] - z)
        return nb, dist, dv

    def _wall_wins(self, i, j, k, dv):
        """RemoveDuplicateWMPoints (src/wallmodels.f90:373-410) for a cell that
        is a point of a no-slip z wall (Prtype == 0) and of a solid face: the
        wall point is kept if it is strictly closer to its wall (on a tie the
        solid-face point, the first added, which a stable sort keeps)."""
        g, cfg, c = self.g, self.cfg, self.c
        if self.typ(0, i, j, k) != 0:
            return False
        if k == 1 and cfg.Btype[4] == BC_NOSLIP:
            dz = c.x(c.zW, 0) - c.x(c.zPr, 1)
        elif k == g.Prnz and cfg.Btype[5] == BC_NOSLIP:
            dz = c.x(c.zW, g.Prnz) - c.x(c.zPr, g.Prnz)
        else:
            return False
        return dv is None or dz * dz < dv[0] ** 2 + dv[1] ** 2 + dv[2] ** 2

    def wall_pr(self):
        """The Pr wall-model points of the no-slip z walls that the
        deduplication keeps (each carries its wall's temperature flux)."""
        g, cfg = self.g, self.cfg
        out = []
        for k, side in ((1, 4), (g.Prnz, 5)):
            if cfg.Btype[side] != BC_NOSLIP:
                continue
            for j in range(1, g.Prny + 1):
                for i in range(1, g.Prnx + 1):
                    if self.typ(0, i, j, k) != 0:
                        continue
                    nb, _, dv = self._face_point(i, j, k)
                    if nb == 0 or self._wall_wins(i, j, k, dv):
                        out.append((i, j, k))
        return np.array(out, dtype=np.int32).reshape(-1, 3)

    def heat_pr(self):
        """The Pr wall-model points at solid faces that carry a heat flux:
        (i, j, k, temperature_flux x area_factor).  GetSolidBodiesWM
        (src/immersedboundary.f90:14-138) gives a free cell with solid
        6-neighbours the nearest of their bodies (_face_point) and that
        body's flux if it is rough;
        ComputeAreaFactor (src/wallmodels.f90:173-203) the boundary area over
        the cell volume along the distance's dominant axis.  A cell that is
        also a point of a no-slip bottom keeps one of the two
        (RemoveDuplicateWMPoints, src/wallmodels.f90:373-410: the one closer
        to its wall; on a tie the solid-face point, the first added, which
        a stable sort keeps first)."""
        g, cfg, c = self.g, self.cfg, self.c
        nx, ny, nz = g.Prnx, g.Prny, g.Prnz
        dzmin = c.dzmin
        out = []
        for k in range(1, nz + 1):
            for j in range(1, ny + 1):
                for i in range(1, nx + 1):
                    if self.typ(0, i, j, k) > 0:
                        continue
                    nb, dist, dv = self._face_point(i, j, k)
                    if nb == 0 or self._wall_wins(i, j, k, dv):
                        continue
                    b = self.boxes[nb - 1]
                    flux = b.heat_flux if b.z0r > 0 else 0.0
                    if flux == 0:
                        continue
                    on = [abs(-v) / dist for v in dv]
                    if on[0] > on[1] and on[0] > on[2]:
                        o, d = on[0], math.sqrt(cfg.dymin * dzmin)
                    elif on[1] > on[0] and on[1] > on[2]:
                        o, d = on[1], math.sqrt(cfg.dxmin * dzmin)
                    else:
                        o, d = on[2], math.sqrt(cfg.dxmin * cfg.dymin)
                    af = d * (d / o) / (cfg.dxmin * cfg.dymin * dzmin)
                    out.append((i, j, k, flux * af))
        return out

    def bottom_skip(self, q):
        (nx, ny, nz), _, _, _ = self.grids[q]
        t = self.types[q]
        keep = (t[1 + 2, 3:ny + 3, 3:nx + 3] == 0) & (t[0 + 2, 3:ny + 3, 3:nx + 3] <= 0)
        j, i = np.nonzero(~keep)
        return np.stack([i + 1, j + 1], axis=1).astype(np.int32) if len(i) else np.zeros((0, 2), np.int32)


def _ib_array(points):
    arr = (ElmmIBPoint * max(1, len(points)))()
    for n, ((xi, yj, zk), pts, cf) in enumerate(points):
        p = arr[n]
        p.xi, p.yj, p.zk, p.interp = xi, yj, zk, len(pts)
        for m, ((a, b, c), w) in enumerate(zip(pts, cf)):
            p.ii[m], p.jj[m], p.kk[m] = a, b, c
            p.coef[m] = w
    return arr


@dataclass
class Solids:
    """The point lists of one domain's solid bodies (see the module doc)."""
    ib: list = field(default_factory=lambda: [[], [], []])      # per component: ((i,j,k), pts, coefs)
    null: list = field(default_factory=lambda: [np.zeros((0, 3), np.int32)] * 3)
    scalfl: list = field(default_factory=list)
    wm: list = field(default_factory=list)
    bottom_skip: list = field(default_factory=lambda: [np.zeros((0, 2), np.int32)] * 3)
    solid_pr: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    wm_pr: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    heat_pr: list = field(default_factory=list)
    wall_pr: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))

    def struct(self) -> ElmmSolids:
        """The elmm_solids view; the arrays stay referenced by this object."""
        s = ElmmSolids()
        self._keep = []
        for q in range(3):
            a = _ib_array(self.ib[q])
            self._keep.append(a)
            s.n_ib[q] = len(self.ib[q])
            s.ib[q] = C.cast(a, C.POINTER(ElmmIBPoint))
            nl = np.ascontiguousarray(self.null[q], dtype=np.int32).reshape(-1)
            self._keep.append(nl)
            s.n_null[q] = len(nl) // 3
            s.null_ijk[q] = nl.ctypes.data_as(C.POINTER(C.c_int32))
            bs = np.ascontiguousarray(self.bottom_skip[q], dtype=np.int32).reshape(-1)
            self._keep.append(bs)
            s.n_bottom_skip[q] = len(bs) // 2
            s.bottom_skip_ij[q] = bs.ctypes.data_as(C.POINTER(C.c_int32))
        a = _ib_array(self.scalfl)
        self._keep.append(a)
        s.n_scalfl = len(self.scalfl)
        s.scalfl = C.cast(a, C.POINTER(ElmmIBPoint))
        w = (ElmmWMPoint * max(1, len(self.wm)))()
        for n, (comp, dr, i, j, k, dv, z0, tf) in enumerate(self.wm):
            w[n].component, w[n].direction, w[n].xi, w[n].yj, w[n].zk = comp, dr, i, j, k
            w[n].dist[0], w[n].dist[1], w[n].dist[2] = dv
            w[n].z0 = z0
            w[n].temperature_flux = tf
        self._keep.append(w)
        s.n_wm = len(self.wm)
        s.wm = C.cast(w, C.POINTER(ElmmWMPoint))
        for name, arr in (("solid_pr", self.solid_pr), ("wm_pr", self.wm_pr), ("wall_pr", self.wall_pr)):
            a = np.ascontiguousarray(arr, dtype=np.int32).reshape(-1)
            self._keep.append(a)
            setattr(s, "n_" + name, len(a) // 3)
            setattr(s, name + "_ijk", a.ctypes.data_as(C.POINTER(C.c_int32)))
        hi = np.ascontiguousarray([p[:3] for p in self.heat_pr], dtype=np.int32).reshape(-1)
        hq = np.ascontiguousarray([p[3] for p in self.heat_pr], dtype=np.float64)
        self._keep += [hi, hq]
        s.n_heat_pr = len(self.heat_pr)
        s.heat_pr_ijk = hi.ctypes.data_as(C.POINTER(C.c_int32))
        s.heat_pr_q = hq.ctypes.data_as(C.POINTER(C.c_double))
        return s

    def counts(self) -> dict:
        return {"ib": [len(x) for x in self.ib], "null": [len(x) for x in self.null],
                "scalfl": len(self.scalfl), "wm": len(self.wm), "bottom_skip": [len(x) for x in self.bottom_skip],
                "solid_pr": len(self.solid_pr), "wm_pr": len(self.wm_pr)}


def build_solids(cfg: ElmmConfig, boxes) -> Solids:
    """GetSolidBodiesBC + SetNullifiedPoints for the given bodies (Box and
    Sphere objects, numbered in list order)."""
    g = Geometry(cfg, boxes)
    s = Solids()
    for comp in (1, 2, 3):
        pts = []
        for (i, j, k) in g._boundary_points(comp):
            ip, cf = g.vel_ib_point(comp, i, j, k)
            assert len(ip) <= IB_MAX_INTERP
            pts.append(((i, j, k), ip, cf))
        s.ib[comp - 1] = pts
    s.null = [g.null_points(q) for q in (1, 2, 3)]
    s.scalfl = [((i, j, k),) + g.scalfl_point(i, j, k) for (i, j, k) in g._boundary_points(0)]
    s.wm = g.wm_points()
    s.bottom_skip = [g.bottom_skip(q) for q in (1, 2, 3)]
    s.solid_pr = g.solid_pr()
    s.wm_pr = g.wm_pr()
    s.heat_pr = g.heat_pr() if any(b.heat_flux != 0 for b in boxes) else []
    s.wall_pr = g.wall_pr()
    s.geometry = g
    return s
