"""Source terms on this path and the wind forcing that drives them.

Parameter defaults and validation follow the reference:
PressureCorrelationInput (src/Physics/WindInput/pressure_correlation.jl:24-52),
LocalSaturationDissipation (src/Physics/Dissipation/local_saturation.jl:18-28),
BulkWindDrag (src/Physics/shared/drag.jl:73-86),
PrecomputedSources (src/Physics/Packages/precomputed_sources.jl:179-191),
HollandHurricaneWind / LinearStormTrack (src/Forcing/winds.jl:115-229), and the SourceTermSet terms
whose tendency is linear in the action: ExponentialWindInput, WaveAgeWindInput, WhitecappingDissipation
(src/Sources/Sources.jl:5-11,32-39,67-122) and MeanSpectrumWhitecapping
(src/Physics/Dissipation/mean_spectrum.jl:20-40).
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


def source_parameter(value, name):
    """A rate or speed parameter (Sources.jl:480-482): a number, an (Nx, Ny) array, or a callable of
    (x, y) evaluated once at the cell centres. Time-dependent callables are outside this path."""
    if value is None:
        return None
    if np.isscalar(value):
        return float(value)
    if callable(value):
        return value
    a = np.asarray(value, dtype=np.float64)
    if a.ndim != 2:
        raise ArgumentError(f"{name} must be a number, an (Nx, Ny) array or a callable of (x, y)")
    return a


def _integer_spreading_power(p):
    """Sources.jl:1387-1392"""
    if not p >= 0:
        raise ArgumentError("directional spreading power must be nonnegative")
    if float(p) != int(p):
        raise ArgumentError("finite-volume directional spreading currently supports nonnegative integer powers; "
                            f"got {float(p)}")
    return int(p)


class ExponentialWindInput:
    """rate * cell average of max(cos(phi - direction), 0)^spreading_power (Sources.jl:32-39,492-496)."""

    def __init__(self, *, rate=0.0, direction=0.0, spreading_power=2.0):
        self.rate = source_parameter(rate, "rate")
        if not np.isscalar(direction):
            raise ArgumentError("ExponentialWindInput direction must be a number on this path")
        self.direction = float(direction)
        self.spreading_power = float(spreading_power)
        _integer_spreading_power(self.spreading_power)


class WaveAgeWindInput:
    """rate * max(U cos / c - threshold, 0)^power * cos^spreading_power (Sources.jl:67-95,522-554)."""

    def __init__(self, *, rate=0.0, speed=None, wind=None, direction=None, inverse_wave_age_threshold=0.83,
                 power=1.0, spreading_power=1.0, gravity=9.81):
        speed_value = (10.0 if speed is None else speed) if wind is None else wind
        direction_value = direction if direction is not None else (0.0 if wind is None else wind)
        self.rate = source_parameter(rate, "rate")
        self.speed = source_parameter(speed_value, "speed")
        if not np.isscalar(direction_value):
            raise ArgumentError("WaveAgeWindInput direction must be a number on this path")
        self.direction = float(direction_value)
        self.inverse_wave_age_threshold = float(inverse_wave_age_threshold)
        self.power, self.spreading_power, self.gravity = float(power), float(spreading_power), float(gravity)
        if not self.inverse_wave_age_threshold >= 0:
            raise ArgumentError("wave-age wind-input threshold must be nonnegative")
        if not self.power >= 0:
            raise ArgumentError("wave-age wind-input power must be nonnegative")
        if not self.spreading_power >= 0:
            raise ArgumentError("wave-age wind-input spreading power must be nonnegative")
        if not self.gravity > 0:
            raise ArgumentError("wave-age wind-input gravity must be positive")


class WhitecappingDissipation:
    """rate * max(m0 / threshold - 1, 0)^saturation_power * <kappa^p> / k_ref^p (Sources.jl:105-122,583-598)."""

    def __init__(self, *, rate=0.0, saturation_threshold=1.0, saturation_power=1.0, wavenumber_power=1.0,
                 reference_wavenumber=1.0):
        self.rate = source_parameter(rate, "rate")
        self.saturation_threshold = float(saturation_threshold)
        self.saturation_power = float(saturation_power)
        self.wavenumber_power = float(wavenumber_power)
        self.reference_wavenumber = float(reference_wavenumber)
        if not self.saturation_threshold > 0:
            raise ArgumentError("whitecapping saturation threshold must be positive")
        if not self.reference_wavenumber > 0:
            raise ArgumentError("whitecapping reference wavenumber must be positive")
        if not self.wavenumber_power >= 0:
            raise ArgumentError("wavenumber power must be nonnegative")


class MeanSpectrumWhitecapping:
    """-C_ds (m0 kbar^2)^2 sigmabar (delta1 k/kbar + delta2 (k/kbar)^2) damping with p-th mean wavenumber and
    frequency (mean_spectrum.jl:20-40,90-111); BJA defaults."""

    def __init__(self, *, C_ds=-2.1, δ1=0.4, δ2=0.6, p=0.5, gravity=9.81, delta1=None, delta2=None):
        self.C_ds = float(C_ds)
        self.δ1 = float(δ1 if delta1 is None else delta1)
        self.δ2 = float(δ2 if delta2 is None else delta2)
        self.p, self.gravity = float(p), float(gravity)
        if self.p == 0:
            raise ArgumentError("MeanSpectrumWhitecapping needs a nonzero mean exponent p")


LINEAR_TERMS = (ExponentialWindInput, WaveAgeWindInput, WhitecappingDissipation, MeanSpectrumWhitecapping)


class SourceTermSet:
    """A sum of source terms (Sources.jl:5-11,443-449): here terms whose tendency is linear in the action."""

    def __init__(self, *terms):
        if len(terms) == 1 and isinstance(terms[0], (tuple, list)):
            terms = tuple(terms[0])
        for t in terms:
            if not isinstance(t, LINEAR_TERMS):
                raise ArgumentError(f"source term {type(t).__name__} is outside the B200 path")
        self.terms = tuple(terms)

    def __len__(self):
        return len(self.terms)

    def __iter__(self):
        return iter(self.terms)


def linear_terms(sources):
    """The SourceTermSet terms of a sources argument (a set or one term), or None."""
    if isinstance(sources, SourceTermSet):
        return sources.terms
    if isinstance(sources, LINEAR_TERMS):
        return (sources,)
    return None


def parameter_field(value, grid):
    """A source parameter as (scalar, (Nx, Ny) x-fastest field or None) on the grid's cell centres."""
    if value is None:
        return 0.0, None
    if np.isscalar(value):
        return float(value), None
    if callable(value):
        X, Y = np.meshgrid(grid.xnodes(), grid.ynodes(), indexing="ij")
        value = np.broadcast_to(np.asarray(value(X, Y), dtype=np.float64), (grid.Nx, grid.Ny))
    a = np.asarray(value, dtype=np.float64)
    if a.shape != (grid.Nx, grid.Ny):
        raise ArgumentError(f"source parameter field must have shape {(grid.Nx, grid.Ny)}")
    return 0.0, np.asfortranarray(a).ravel(order="F").copy()


TERM_KIND = {ExponentialWindInput: 1, WaveAgeWindInput: 2, WhitecappingDissipation: 3, MeanSpectrumWhitecapping: 4}


def term_record(t, grid):
    """(kind, rate, rate_field, direction, speed, speed_field, p[4], gravity) of one term."""
    if isinstance(t, ExponentialWindInput):
        rate, rf = parameter_field(t.rate, grid)
        return 1, rate, rf, t.direction, 0.0, None, (t.spreading_power, 0.0, 0.0, 0.0), 9.81
    if isinstance(t, WaveAgeWindInput):
        rate, rf = parameter_field(t.rate, grid)
        speed, sf = parameter_field(t.speed, grid)
        return 2, rate, rf, t.direction, speed, sf, (t.inverse_wave_age_threshold, t.power, t.spreading_power,
                                                    0.0), t.gravity
    if isinstance(t, WhitecappingDissipation):
        rate, rf = parameter_field(t.rate, grid)
        return 3, rate, rf, 0.0, 0.0, None, (t.saturation_threshold, t.saturation_power, t.wavenumber_power,
                                            t.reference_wavenumber), 9.81
    return 4, 0.0, None, 0.0, 0.0, None, (t.C_ds, t.δ1, t.δ2, t.p), t.gravity
