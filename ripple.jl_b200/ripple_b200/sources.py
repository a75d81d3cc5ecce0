"""Source terms on this path and the wind forcing that drives them.

Parameter defaults and validation follow the reference:
PressureCorrelationInput (src/Physics/WindInput/pressure_correlation.jl:24-52),
LocalSaturationDissipation (src/Physics/Dissipation/local_saturation.jl:18-28),
BulkWindDrag (src/Physics/shared/drag.jl:73-86),
PrecomputedSources (src/Physics/Packages/precomputed_sources.jl:179-191),
HollandHurricaneWind / LinearStormTrack (src/Forcing/winds.jl:115-229).
The rates themselves are evaluated by librpl.so on the device.
"""
import math

import numpy as np

from ._lib import ArgumentError


class Counterclockwise:
    sign = 1


class Clockwise:
    sign = -1


class BulkWindDrag:
    """u* = U10 sqrt(Cd(U10)); form "linear" (Wu 1982) or "capped" (Hwang 2001)."""

    def __init__(self, form="linear"):
        form = str(form).lstrip(":")
        if form not in ("linear", "capped"):
            raise ArgumentError(f"unsupported BulkWindDrag form {form}")
        self.form = form

    def drag_coefficient(self, U10):
        if self.form == "linear":
            return (0.8 + 0.065 * U10) * 1e-3
        return max((8.058 + 0.967 * U10 - 0.016 * U10 ** 2) * 1e-4, 4e-4)

    def friction_velocity(self, U10):
        return U10 * math.sqrt(max(self.drag_coefficient(U10), 0.0))


class LinearStormTrack:
    """Piecewise-linear storm centre in time (winds.jl:115-152)."""

    def __init__(self, times, centers):
        t = [float(v) for v in times]
        c = list(centers)
        if len(t) != len(c):
            raise ArgumentError("storm-track times and centers must have the same length")
        if len(t) == 0:
            raise ArgumentError("storm-track times and centers must be non-empty")
        for k in range(1, len(t)):
            if not t[k] > t[k - 1]:
                raise ArgumentError("storm-track times must be strictly increasing")
        for cc in c:
            if len(cc) != 2:
                raise ArgumentError("storm-track centers must be two-component coordinates")
        self.times = t
        self.centers = [(float(a), float(b)) for a, b in c]

    def __call__(self, t):
        times, centers = self.times, self.centers
        if t <= times[0]:
            return centers[0]
        if t >= times[-1]:
            return centers[-1]
        up = next(k for k, v in enumerate(times) if v >= t)
        lo = up - 1
        w = (t - times[lo]) / (times[up] - times[lo])
        return ((1 - w) * centers[lo][0] + w * centers[up][0], (1 - w) * centers[lo][1] + w * centers[up][1])


class HollandHurricaneWind:
    """Holland (1980) vortex with exponential decay beyond `radius` (winds.jl:200-229)."""

    def __init__(self, *, center=(0.0, 0.0), vmax=1.0, rmax=1.0, radius=4.0, shape_parameter=1.5,
                 inflow_angle=0.0, background=(0.0, 0.0), rotation=Counterclockwise):
        if not vmax >= 0:
            raise ArgumentError("Holland hurricane vmax must be nonnegative")
        if not rmax > 0:
            raise ArgumentError("Holland hurricane rmax must be positive")
        if not radius > rmax:
            raise ArgumentError("Holland hurricane radius must exceed rmax")
        if not shape_parameter > 0:
            raise ArgumentError("Holland hurricane shape_parameter must be positive")
        if not (isinstance(center, LinearStormTrack) or (len(center) == 2)):
            raise ArgumentError("Holland hurricane center must be a point or a LinearStormTrack")
        self.center = center
        self.vmax, self.rmax, self.radius = float(vmax), float(rmax), float(radius)
        self.shape_parameter, self.inflow_angle = float(shape_parameter), float(inflow_angle)
        self.background = (float(background[0]), float(background[1]))
        self.rotation = rotation


class PressureCorrelationInput:
    """Janssen wind input, ST3-lite (pressure_correlation.jl:24-52). `wind` is a speed or a wind struct."""

    def __init__(self, *, drag, wind, direction=0.0, β_max=1.2, z_α=0.011, p_in=2.0, α0=0.0095,
                 ρ_air=1.225, ρ_water=1025.0, von_karman=0.4, gravity=9.81, **ascii_names):
        self.drag = drag
        self.wind = wind
        self.direction = float(direction)
        self.β_max = float(ascii_names.pop("beta_max", β_max))
        self.z_α = float(ascii_names.pop("z_alpha", z_α))
        self.p_in = float(p_in)
        self.α0 = float(ascii_names.pop("alpha0", α0))
        self.ρ_air = float(ascii_names.pop("rho_air", ρ_air))
        self.ρ_water = float(ascii_names.pop("rho_water", ρ_water))
        self.von_karman = float(von_karman)
        self.gravity = float(gravity)
        if ascii_names:
            raise ArgumentError(f"unknown PressureCorrelationInput keywords {sorted(ascii_names)}")
        if not isinstance(drag, BulkWindDrag):
            raise ArgumentError("PressureCorrelationInput drag must be a BulkWindDrag on this path")


class LocalSaturationDissipation:
    """Local-saturation whitecapping (local_saturation.jl:18-28)."""

    def __init__(self, *, C_ds=-2.2e-5, B_r=9.0e-4, p=2.0, σ_power=1.0, gravity=9.81, sigma_power=None):
        self.C_ds, self.B_r, self.p = float(C_ds), float(B_r), float(p)
        self.σ_power = float(sigma_power if sigma_power is not None else σ_power)
        self.gravity = float(gravity)


class PrecomputedSources:
    """Bundle whose wind input gets the wave-supported stress cap (precomputed_sources.jl:179-191)."""

    def __init__(self, *, wind_input=None, dissipation=None, nonlinear=None, extras=()):
        if nonlinear is not None or len(tuple(extras)) > 0:
            raise ArgumentError("nonlinear transfer and extra source terms are outside this path")
        self.wind_input = wind_input
        self.dissipation = dissipation


def evaluate_wind(wind, x, y, t):
    """Host evaluation of a generic callable wind: returns (U10, direction) arrays over the grid."""
    X, Y = np.meshgrid(x, y, indexing="ij")
    vel = wind(X, Y, t)
    vx, vy = (np.asarray(v, dtype=np.float64) for v in vel)
    return np.hypot(vx, vy), np.arctan2(vy, vx)
