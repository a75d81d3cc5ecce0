"""Physical and spectral grids: the inputs of SpectralWaveModel.

RectilinearGrid covers the Oceananigans grid accessors the reference uses on this
path (src/Grids.jl:53-76: nodes, faces, spacings); PolarWaveVectorGrid restates
src/CoordinateGrids/polar_wavevector_grid.jl:18-68 with the face rules of
src/CoordinateGrids/spectral_grids.jl:4-27 and the validation of :176-214.
"""
import math

import numpy as np

from ._lib import ArgumentError

Periodic, Bounded, Flat = "Periodic", "Bounded", "Flat"


class InfiniteDepth:
    """Deep-water dispersion marker (src/Grids.jl:8-15)."""

    def __repr__(self):
        return "InfiniteDepth()"


def _faces(spec, n, name):
    if isinstance(spec, (tuple, list)) and len(spec) == 2 and n != 1 and not isinstance(spec[0], (list, tuple)):
        a, b = float(spec[0]), float(spec[1])
        if not b > a:
            raise ArgumentError(f"{name} interval must be increasing")
        d = (b - a) / n
        return np.array([a + k * d for k in range(n + 1)], dtype=np.float64)
    f = np.asarray(spec, dtype=np.float64)
    if f.shape == (2,) and n == 1:
        return f.copy()
    if f.shape != (n + 1,):
        raise ArgumentError(f"{name} faces must have length {n + 1}")
    if not np.all(np.diff(f) > 0):
        raise ArgumentError(f"{name} faces must be strictly increasing")
    return f


class RectilinearGrid:
    """Rectilinear physical grid with cell-centre nodes and faces.

    RectilinearGrid(size=(Nx, Ny, Nz), x=(x0, x1), y=(y0, y1), z=(z0, z1) or faces,
    halo=(3, 3, 3), topology=("Periodic", "Periodic", "Bounded")). A 2-tuple size
    means a Flat vertical direction.
    """

    def __init__(self, arch=None, FT=np.float64, *, size, x, y, z=None, halo=(3, 3, 3),
                 topology=(Periodic, Periodic, Bounded), first_spacings=None):
        size = tuple(int(s) for s in size)
        if len(size) == 2:
            size = size + (0,)
            topology = tuple(topology[:2]) + (Flat,)
        self.Nx, self.Ny, self.Nz = size
        if self.Nx < 1 or self.Ny < 1:
            raise ArgumentError("grid size must be positive")
        self.topology = tuple(topology)
        self.halo = tuple(halo)
        self.FT = FT
        self._xf = _faces(x, self.Nx, "x")
        self._yf = _faces(y, self.Ny, "y")
        if self.Nz > 0:
            if z is None:
                raise ArgumentError("a grid with vertical cells needs z")
            self._zf = _faces(z, self.Nz, "z")
        else:
            self._zf = np.zeros(0)
        # (dx, dy) the stencils use, first(xspacings), first(yspacings) unless given (a slab of a larger
        # uniform grid keeps the parent's values)
        self._first = None if first_spacings is None else (float(first_spacings[0]), float(first_spacings[1]))

    # Oceananigans-style accessors (src/Grids.jl:53-76)
    def xfaces(self):
        return self._xf.copy()

    def yfaces(self):
        return self._yf.copy()

    def zfaces(self):
        return self._zf.copy()

    def xnodes(self):
        return 0.5 * (self._xf[:-1] + self._xf[1:])

    def ynodes(self):
        return 0.5 * (self._yf[:-1] + self._yf[1:])

    def znodes(self):
        return 0.5 * (self._zf[:-1] + self._zf[1:]) if self.Nz else np.zeros(0)

    def first_spacings(self):
        """(first(xspacings), first(yspacings)): the spacings the stencils use."""
        if self._first is not None:
            return self._first
        return float(self.xspacings()[0]), float(self.yspacings()[0])

    def xspacings(self):
        return np.diff(self._xf)

    def yspacings(self):
        return np.diff(self._yf)

    def zspacings(self):
        return np.diff(self._zf)

    @property
    def Lx(self):
        return float(self._xf[-1] - self._xf[0])

    @property
    def Ly(self):
        return float(self._yf[-1] - self._yf[0])

    @property
    def Lz(self):
        return float(self._zf[-1] - self._zf[0]) if self.Nz else 0.0

    def horizontal_size(self):
        return (self.Nx, self.Ny)

    def has_flat_vertical(self):
        return self.topology[2] == Flat or self.Nz == 0

    def periodic_xy(self):
        return self.topology[0] == Periodic and self.topology[1] == Periodic

    def __repr__(self):
        return f"RectilinearGrid(size=({self.Nx}, {self.Ny}, {self.Nz}), topology={self.topology})"


def centers_to_faces(centers):
    """Midpoint faces with linear end extrapolation (spectral_grids.jl:4-19)."""
    c = np.asarray(centers, dtype=np.float64)
    n = len(c)
    if n == 0:
        raise ArgumentError("coordinate vectors must be non-empty")
    f = np.empty(n + 1)
    if n == 1:
        f[0], f[1] = c[0] - 0.5, c[0] + 0.5
    else:
        f[1:n] = (c[:-1] + c[1:]) / 2.0
        f[0] = c[0] - (f[1] - c[0])
        f[n] = c[-1] + (c[-1] - f[n - 1])
    return f


def lower_bounded_centers_to_faces(centers, lower):
    f = centers_to_faces(centers)
    f[0] = max(f[0], lower)
    return f


def _validate_centers(name, c):
    if len(c) == 0:
        raise ArgumentError(f"{name} centers must be non-empty")
    if not np.all(np.diff(c) > 0):
        raise ArgumentError(f"{name} centers must be strictly increasing")


def _validate_faces(name, c, f):
    if len(f) != len(c) + 1:
        raise ArgumentError(f"{name} faces must have length length(centers) + 1")
    if not np.all(np.diff(f) > 0):
        raise ArgumentError(f"{name} faces must be strictly increasing")
    for i in range(len(c)):
        if not (f[i] <= c[i] <= f[i + 1]):
            raise ArgumentError(f"{name} center {i + 1} must lie inside its cell faces")


class PolarWaveVectorGrid:
    """Polar (kappa, phi) spectral grid (polar_wavevector_grid.jl:18-56).

    kappa faces default to midpoints floored at 0; phi faces default to uniform
    2pi/Nphi bins centred on phi[0]. weights[m, n] = (k2^2 - k1^2)/2 * dphi_n.
    """

    def __init__(self, arch=None, FT=np.float64, *, κ=None, φ=None, κ_faces=None, φ_faces=None,
                 kappa=None, phi=None, kappa_faces=None, phi_faces=None):
        k = κ if κ is not None else kappa
        p = φ if φ is not None else phi
        kf = κ_faces if κ_faces is not None else kappa_faces
        pf = φ_faces if φ_faces is not None else phi_faces
        if k is None:
            raise ArgumentError("PolarWaveVectorGrid requires `κ`")
        if p is None:
            raise ArgumentError("PolarWaveVectorGrid requires `φ`")
        kc = np.array(list(k), dtype=np.float64)
        pc = np.array(list(p), dtype=np.float64)
        _validate_centers("φ", pc)
        kf = lower_bounded_centers_to_faces(kc, 0.0) if kf is None else np.array(list(kf), dtype=np.float64)
        if pf is None:
            dphi = 2.0 * math.pi if len(pc) == 1 else 2.0 * math.pi / len(pc)
            pf = np.array([pc[0] - dphi / 2.0 + i * dphi for i in range(len(pc) + 1)])
        else:
            pf = np.array(list(pf), dtype=np.float64)
        _validate_centers("κ", kc)
        if not np.all(kc > 0):
            raise ArgumentError("κ centers must be positive")
        _validate_faces("κ", kc, kf)
        if not np.all(kf >= 0):
            raise ArgumentError("κ faces must be >= 0.0")
        _validate_faces("φ", pc, pf)
        self.κ, self.φ, self.κ_faces, self.φ_faces = kc, pc, kf, pf
        radial = (kf[1:] ** 2 - kf[:-1] ** 2) / 2.0
        angular = np.diff(pf)
        self.weights = np.array([[radial[m] * angular[n] for n in range(len(pc))] for m in range(len(kc))])

    kappa = property(lambda self: self.κ)
    phi = property(lambda self: self.φ)
    kappa_faces = property(lambda self: self.κ_faces)
    phi_faces = property(lambda self: self.φ_faces)

    def coordinate_size(self):
        return (len(self.κ), len(self.φ))

    def k_components(self, m, n):
        return (self.κ[m] * math.cos(self.φ[n]), self.κ[m] * math.sin(self.φ[n]))

    def spectral_weight(self, m, n):
        return float(self.weights[m, n])

    def __repr__(self):
        return f"{len(self.κ)}×{len(self.φ)} PolarWaveVectorGrid"
