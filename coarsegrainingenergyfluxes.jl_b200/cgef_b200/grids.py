"""Uniform structured grids (FlowGeometries.Grids.StructuredGrid over two ranges).

Arrays follow the reference's column-major (Nx, Ny) layout, which numpy holds as shape
(ny, nx) with the x (longitude) index fastest.  Spherical coordinates are radians.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Optional, Sequence, Tuple, Union

import numpy as np

from . import _lib


class CartesianGeometry:
    """Planar geometry (FlowGeometries.Geometry.CartesianGeometry)."""

    code = _lib.CARTESIAN

    def __repr__(self) -> str:
        return "CartesianGeometry()"


@dataclass(frozen=True)
class SphericalGeometry:
    """Sphere of radius R metres (FlowGeometries.Geometry.SphericalGeometry)."""

    R: float = 6.371e6
    code = _lib.SPHERICAL


@dataclass(frozen=True)
class Axis:
    """A uniform axis start + i*step, i = 0..length-1 (a Julia range)."""

    start: float
    step: float
    length: int

    def values(self) -> np.ndarray:
        # fma(i, step, start), the library's own evaluation
        i = np.arange(self.length, dtype=np.longdouble)
        return (np.longdouble(self.start) + i * np.longdouble(self.step)).astype(np.float64)

    def __len__(self) -> int:
        return self.length


def axis(start: float, step: float, length: int) -> Axis:
    return Axis(float(start), float(step), int(length))


def _as_axis(a: Union[Axis, Sequence[float], np.ndarray]) -> Axis:
    if isinstance(a, Axis):
        return a
    v = np.asarray(a, dtype=np.float64)
    if v.ndim != 1 or v.size < 1:
        raise ValueError("an axis is a 1-D sequence of coordinates")
    if v.size == 1:
        return Axis(float(v[0]), 1.0, 1)
    step = (v[-1] - v[0]) / (v.size - 1)
    if not np.allclose(np.diff(v), step, rtol=1e-9, atol=0.0) or step <= 0:
        raise ValueError("only uniform ascending axes are supported (the reference's Range-axis path)")
    return Axis(float(v[0]), float(step), int(v.size))


class StructuredGrid:
    """2-D grid: geometry, uniform x and y axes, optional active-cell mask of shape (ny, nx).

    `periodic` defaults as the reference's constructor does: a spherical longitude axis that
    spans the whole circle wraps; every other axis is bounded.
    """

    def __init__(self, geometry, x, y, mask: Optional[np.ndarray] = None,
                 periodic: Optional[Tuple[bool, bool]] = None):
        self.geometry = geometry
        self.x = _as_axis(x)
        self.y = _as_axis(y)
        if periodic is None:
            full = isinstance(geometry, SphericalGeometry) and abs(self.x.length * self.x.step - 2 * math.pi) < 1e-9
            periodic = (bool(full), False)
        self.periodic = (bool(periodic[0]), bool(periodic[1]))
        if mask is not None:
            mask = np.ascontiguousarray(np.asarray(mask).astype(bool))
            if mask.shape != (self.y.length, self.x.length):
                raise ValueError(f"mask shape {mask.shape} != (ny, nx) = {(self.y.length, self.x.length)}")
            if mask.all():
                mask = None
        self.mask = mask

    @property
    def nx(self) -> int:
        return self.x.length

    @property
    def ny(self) -> int:
        return self.y.length

    @property
    def shape(self) -> Tuple[int, int]:
        """numpy shape (ny, nx) of a field on this grid."""
        return (self.y.length, self.x.length)

    def size_tuple(self) -> Tuple[int, int]:
        """The reference's (Nx, Ny)."""
        return (self.x.length, self.y.length)

    @property
    def is_spherical(self) -> bool:
        return isinstance(self.geometry, SphericalGeometry)

    def isactive(self, i: int, j: int) -> bool:
        return True if self.mask is None else bool(self.mask[j, i])

    def with_mask(self, mask) -> "StructuredGrid":
        return StructuredGrid(self.geometry, self.x, self.y, mask, self.periodic)

    def coords(self) -> Tuple[np.ndarray, np.ndarray]:
        return self.x.values(), self.y.values()

    def area(self) -> np.ndarray:
        """Cell measure per row (ny,): R^2 cos(phi) dlambda dphi on the sphere, dx dy on the plane."""
        if self.is_spherical:
            R = self.geometry.R
            return R * R * np.cos(self.y.values()) * self.x.step * self.y.step
        return np.full(self.ny, self.x.step * self.y.step)

    def _desc(self, keep):
        m = None if self.mask is None else np.ascontiguousarray(self.mask, dtype=np.uint8)
        keep.append(m)
        d = _lib.GridDesc()
        d.geometry = self.geometry.code
        d.periodic_x, d.periodic_y = int(self.periodic[0]), int(self.periodic[1])
        d.nx, d.ny = self.nx, self.ny
        d.x0, d.dx, d.y0, d.dy = self.x.start, self.x.step, self.y.start, self.y.step
        d.radius = self.geometry.R if self.is_spherical else 0.0
        d.mask = None if m is None else m.ctypes.data
        return d

    def same_geometry(self, other: "StructuredGrid") -> bool:
        return (type(self.geometry) is type(other.geometry) and self.x == other.x and self.y == other.y
                and self.periodic == other.periodic
                and (not self.is_spherical or self.geometry.R == other.geometry.R))

    def __repr__(self) -> str:
        return (f"StructuredGrid({self.geometry!r}, nx={self.nx}, ny={self.ny}, periodic={self.periodic}, "
                f"masked={self.mask is not None})")
