"""SpectralWaveModel on one B200: the drop-in for Ripple.jl's time-step path.

Mirrors SpectralWaveModel / WaveActionField / set! / time_step! / run!
(src/Models/spectral_wave_model.jl:155-211, src/ProductFields/product_field.jl,
src/ProductFields/set.jl, src/Models/time_step.jl:119-170) for the SSP-RK3
timestepper. The wave action lives on the device inside a librpl.so handle; the
Python objects carry grids, parameters and the clock.
"""
import math
import numbers

import numpy as np

from . import _lib
from ._lib import ArgumentError, check, dptr
from .grids import InfiniteDepth, PolarWaveVectorGrid, RectilinearGrid
from .sources import (BulkWindDrag, HollandHurricaneWind, LinearStormTrack, LocalSaturationDissipation,
                      PrecomputedSources, PressureCorrelationInput, evaluate_wind, linear_terms, term_record)


class WENO:
    """Fifth-order WENO advection marker (the only scheme of the fused kernels)."""

    def __init__(self, order=5):
        if order != 5:
            raise ArgumentError("the B200 kernels implement WENO order 5 only")
        self.order = order


class Clock:
    def __init__(self, time=0.0, iteration=0, last_Δt=math.inf):
        self.time = float(time)
        self.iteration = int(iteration)
        self.last_Δt = last_Δt


_UNSET = object()


class SpatialAveraging:
    """Tolman (2002) spatial-averaging GSE alleviation applied after every time step
    (propagation_smoothing.jl:20-56): each bin's field is replaced by the mean of four bilinear samples
    at the corners of a rectangle of half-widths αs·|Δc_g|·Δt along and αn·c_g·Δφ·Δt across its
    propagation direction."""

    def __init__(self, *, αs=0.5, αn=0.5, alpha_s=None, alpha_n=None):
        self.αs = float(alpha_s if alpha_s is not None else αs)
        self.αn = float(alpha_n if alpha_n is not None else αn)
        if not (self.αs >= 0 and self.αn >= 0 and math.isfinite(self.αs) and math.isfinite(self.αn)):
            raise ArgumentError("SpatialAveraging needs finite αs, αn >= 0")


class PseudomomentumVelocities:
    """uᴸ = p: the waves' own pseudomomentum drives their Doppler shift (lagrangian_velocities.jl:55-81).
    The coupling is recomputed from the action before every RK3 stage. Without `q_grid` a Flat wave grid
    needs a finite model depth; the Q grid is then the stretched automatic grid (Nz, surface_spacing,
    vertical_stretching as in automatic_q_grid)."""

    def __init__(self, *, q_grid=None, vertical_grid=None, depth=None, Nz=None, surface_spacing=None,
                 vertical_stretching=2):
        if depth is not None:
            raise ArgumentError("`depth` is a SpectralWaveModel kwarg; pass `SpectralWaveModel(...; depth=...)` "
                                "instead of putting `depth` in `velocities`")
        if q_grid is not None and vertical_grid is not None:
            raise ArgumentError("PseudomomentumVelocities cannot contain both `q_grid` and `vertical_grid`")
        self.q_grid = q_grid if q_grid is not None else vertical_grid
        self.Nz = Nz
        self.surface_spacing = surface_spacing
        self.vertical_stretching = vertical_stretching


class ProductField:
    """4-D field N[i, j, m, n] over (x, y) x (kappa, phi) (product_field.jl:29-34).

    A field owned by a model reads and writes the device state; a free-standing
    field keeps a host array (Fortran order, so memory order is x fastest like
    the reference's flat_data interior).
    """

    def __init__(self, grid, coordinate_grid, *, eltype=np.float64, _model=None):
        self.grid = grid
        self.coordinate_grid = coordinate_grid
        self.eltype = eltype
        self._model = _model
        self._host = None if _model is not None else np.zeros(self.size, dtype=np.float64, order="F")

    @property
    def size(self):
        Nk, Np = self.coordinate_grid.coordinate_size()
        return (self.grid.Nx, self.grid.Ny, Nk, Np)

    shape = size

    def interior(self):
        if self._model is None:
            return self._host.copy(order="F")
        return self._model._get_action()

    def set(self, value):
        set_(self, value)
        return self

    def __getitem__(self, idx):
        return self.interior()[idx]

    def __setitem__(self, idx, value):
        arr = self.interior()
        arr[idx] = value
        set_(self, arr)

    def __repr__(self):
        return f"ProductField{self.size}"


def WaveActionField(grid, coordinate_grid, **kw):
    return ProductField(grid, coordinate_grid, **kw)


def interior(f):
    """Copy of the field's interior as an (Nx, Ny, Nk, Np) array (product_field.jl:453-462)."""
    return f.interior()


def _evaluate(fun, grid, cgrid):
    """set!(f, fun) semantics: fun(x, y, kx, ky) at cell centres (set.jl:32-42)."""
    x, y = grid.xnodes(), grid.ynodes()
    Nk, Np = cgrid.coordinate_size()
    out = np.empty((grid.Nx, grid.Ny, Nk, Np), order="F")
    X, Y = np.meshgrid(x, y, indexing="ij")
    for n in range(Np):
        for m in range(Nk):
            kx, ky = cgrid.k_components(m, n)
            try:
                v = np.asarray(fun(X, Y, kx, ky), dtype=np.float64)
                out[:, :, m, n] = np.broadcast_to(v, X.shape)
            except (TypeError, ValueError):
                out[:, :, m, n] = [[fun(xi, yj, kx, ky) for yj in y] for xi in x]
    return out


def set_(target=None, value=None, *, N=None):
    """set!(field, value) / set!(model; N=value): number, (Nx,Ny,Nk,Np) array, or f(x, y, kx, ky)."""
    if isinstance(target, SpectralWaveModel):
        if N is not None:
            set_(target.action, N)
        return target
    f = target
    if value is None:
        value = N
    if value is None:
        return f
    if isinstance(value, numbers.Number):
        arr = np.full(f.size, float(value), order="F")
    elif callable(value):
        arr = _evaluate(value, f.grid, f.coordinate_grid)
    else:
        arr = np.asarray(value)
        if arr.dtype != np.float32:
            arr = arr.astype(np.float64, copy=False)
        if arr.shape != f.size:
            raise ArgumentError(f"array size {arr.shape} does not match field size {f.size}")
    if f._model is None:
        f._host = np.asfortranarray(arr, dtype=np.float64)
    else:
        f._model._set_action(arr)
    return f


def _xfast(a):
    """(Nx,Ny,...) array -> contiguous float64 buffer with x fastest."""
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def _automatic_q_grid(grid, cgrid, depth_values, Nz=None, surface_spacing=None, vertical_stretching=2):
    """Stretched Q-transform grid for Flat wave grids (lagrangian_velocities.jl:196-225)."""
    H = float(np.max(depth_values))
    kmax = float(np.max(cgrid.κ))
    dz_surface = 1.0 / (20.0 * kmax) if surface_spacing is None else float(surface_spacing)
    if not dz_surface > 0:
        raise ArgumentError("automatic Q-grid `surface_spacing` must be positive")
    stretch = float(vertical_stretching)
    if not stretch > 1:
        raise ArgumentError("automatic Q-grid `vertical_stretching` must be greater than 1")
    if Nz is None:
        Nz = max(16, math.ceil((H / dz_surface) ** (1.0 / stretch)))
    Nz = int(Nz)
    if Nz <= 0:
        raise ArgumentError("automatic Q-grid `Nz` must be positive")
    z = [-H * (1.0 - k / Nz) ** stretch for k in range(Nz + 1)]
    return RectilinearGrid(size=(grid.Nx, grid.Ny, Nz), x=grid.xfaces(), y=grid.yfaces(), z=z,
                           topology=(grid.topology[0], grid.topology[1], "Bounded"))


class SpectralWaveModel:
    """Spectral wave-action model advanced by SSP-RK3 on one B200 (spectral_wave_model.jl:155-211)."""

    def __init__(self, grid, spectral_grid, *, action=None, horizontal_advection=_UNSET,
                 spectral_advection=_UNSET, advection=_UNSET, sources=None, depth=None, velocities=None,
                 coupling=None, propagation_smoothing=None, boundary_conditions=None, timestepper="RK3",
                 clock=None, precision="fp64", device=0, memory_limit_bytes=0):
        if not isinstance(grid, RectilinearGrid):
            raise ArgumentError(f"grid must be a RectilinearGrid; got {type(grid).__name__}")
        if not isinstance(spectral_grid, PolarWaveVectorGrid):
            raise ArgumentError("spectral_grid must be a PolarWaveVectorGrid on this path")
        if coupling is not None:
            raise ArgumentError("pass `velocities`; prebuilt couplings are not supported")
        if propagation_smoothing is not None and not isinstance(propagation_smoothing, SpatialAveraging):
            raise ArgumentError("propagation_smoothing must be nothing or SpatialAveraging()")
        ts = str(timestepper).lstrip(":")
        if ts != "RK3":
            raise ArgumentError(f"unsupported timestepper {timestepper} (the B200 path implements :RK3)")
        if horizontal_advection is _UNSET:
            horizontal_advection = WENO()
        if spectral_advection is _UNSET:
            spectral_advection = WENO()
        if advection is not _UNSET:
            horizontal_advection = advection
            spectral_advection = advection
        for a in (horizontal_advection, spectral_advection):
            if a is not None and not isinstance(a, WENO):
                raise ArgumentError("advection must be nothing or WENO() on the B200 path")
        if precision not in ("fp64", "fp32"):
            raise ArgumentError("precision must be 'fp64' or 'fp32'")
        self.grid = grid
        self.spectral_grid = spectral_grid
        self.depth = InfiniteDepth() if depth is None else depth
        self.horizontal_advection = horizontal_advection
        self.spectral_advection = spectral_advection
        self.sources = sources
        self.velocities = velocities
        self.propagation_smoothing = propagation_smoothing
        self.timestepper = "RK3"
        self.precision = precision
        self.device = device
        self.clock = clock if clock is not None else Clock()
        self.boundary_conditions = boundary_conditions
        Nx, Ny = grid.Nx, grid.Ny
        Nk, Np = spectral_grid.coordinate_size()

        # depth (lagrangian_velocities.jl:114-187)
        if isinstance(self.depth, InfiniteDepth):
            depth_kind, depth_const, depth_field = _lib.RPL_DEPTH_INFINITE, 0.0, None
        elif isinstance(self.depth, numbers.Number):
            if not self.depth > 0:
                raise ArgumentError("model `depth` must be positive")
            depth_kind, depth_const, depth_field = _lib.RPL_DEPTH_CONSTANT, float(self.depth), None
        else:
            if callable(self.depth):
                X, Y = np.meshgrid(grid.xnodes(), grid.ynodes(), indexing="ij")
                dv = np.broadcast_to(np.asarray(self.depth(X, Y), dtype=np.float64), (Nx, Ny))
            else:
                dv = np.asarray(self.depth, dtype=np.float64)
            if dv.shape != (Nx, Ny):
                raise ArgumentError(f"model `depth` must have size {(Nx, Ny)} on the horizontal wave grid")
            if not np.all(dv > 0):
                raise ArgumentError("model `depth` values must be positive")
            depth_kind, depth_const, depth_field = _lib.RPL_DEPTH_FIELD, 0.0, _xfast(dv)
        self._depth_kind, self._depth_const, self._depth_field = depth_kind, depth_const, depth_field

        # transport route (tendencies.jl:18-50,82-101)
        if velocities is not None:
            if spectral_advection is None:
                raise ArgumentError("CWCM coupling with spectral_advection=nothing uses the per-bin "
                                    "Oceananigans path, which is outside the B200 path")
            transport = _lib.RPL_TRANSPORT_REFRACTION
        elif horizontal_advection is not None:
            transport = _lib.RPL_TRANSPORT_INTRINSIC
        else:
            transport = _lib.RPL_TRANSPORT_NONE
        self._transport = transport

        lib = _lib.load()
        self._keep = dict(x=np.ascontiguousarray(grid.xnodes()), y=np.ascontiguousarray(grid.ynodes()),
                          k=spectral_grid.κ.copy(), kf=spectral_grid.κ_faces.copy(),
                          p=spectral_grid.φ.copy(), pf=spectral_grid.φ_faces.copy(),
                          xs=np.ascontiguousarray(grid.xspacings(), dtype=np.float64),
                          ys=np.ascontiguousarray(grid.yspacings(), dtype=np.float64))
        d = _lib.RplDesc()
        d.abi_version = _lib.RPL_ABI_VERSION
        d.precision = _lib.RPL_FP64 if precision == "fp64" else _lib.RPL_FP32
        d.transport = transport
        d.device = int(device)
        d.Nx, d.Ny, d.Nk, d.Np = Nx, Ny, Nk, Np
        d.dx, d.dy = grid.first_spacings()
        d.xnodes, d.ynodes = dptr(self._keep["x"]), dptr(self._keep["y"])
        d.periodic_x = int(grid.topology[0] == "Periodic")
        d.periodic_y = int(grid.topology[1] == "Periodic")
        d.kappa, d.kappa_faces = dptr(self._keep["k"]), dptr(self._keep["kf"])
        d.phi, d.phi_faces = dptr(self._keep["p"]), dptr(self._keep["pf"])
        d.depth_kind, d.depth_constant = depth_kind, depth_const
        d.depth_field = dptr(depth_field)
        d.gravity = 9.81
        d.memory_limit_bytes = int(memory_limit_bytes)
        d.xspacings, d.yspacings = dptr(self._keep["xs"]), dptr(self._keep["ys"])
        h = _lib.ctypes.c_void_p()
        check(lib.rpl_create(_lib.ctypes.byref(d), _lib.ctypes.byref(h)))
        self._h = h
        self._lib = lib
        self.action = ProductField(grid, spectral_grid, _model=self)
        self.tendencies = ProductField(grid, spectral_grid)
        check(lib.rpl_set_clock(h, self.clock.time, self.clock.iteration))

        if velocities is not None:
            self._set_velocities(velocities)
        if propagation_smoothing is not None:
            check(lib.rpl_set_propagation_smoothing(h, 1, propagation_smoothing.αs, propagation_smoothing.αn))
        self._field_wind = None
        if sources is not None:
            self._set_sources(sources)
        if action is not None:
            if not isinstance(action, ProductField):
                raise ArgumentError(f"action must be a ProductField; got {type(action).__name__}")
            if action.size != self.action.size:
                raise ArgumentError("provided action field is not on the model grids")
            self._set_action(action.interior())

    # ------------------------------------------------------------------ coupling
    def _q_depth(self, q_grid):
        """Projection depth of the Q transform: the Q grid's depth for InfiniteDepth, else the model depth
        (lagrangian_velocities.jl:192-194)."""
        if isinstance(self.depth, InfiniteDepth):
            return _lib.RPL_DEPTH_CONSTANT, q_grid.Lz, None
        if self._depth_field is not None:
            return _lib.RPL_DEPTH_FIELD, 0.0, self._depth_field
        return _lib.RPL_DEPTH_CONSTANT, self._depth_const, None

    def _set_pseudomomentum(self, pm):
        """build_coupling(::PseudomomentumVelocities) (lagrangian_velocities.jl:294-311)."""
        grid = self.grid
        q_grid = pm.q_grid
        if q_grid is None:
            if grid.has_flat_vertical():
                if isinstance(self.depth, InfiniteDepth):
                    raise ArgumentError("Flat wave grids require finite model `depth` or `q_grid` for "
                                        "PseudomomentumVelocities")
                dv = self._depth_field if self._depth_field is not None else np.array([self._depth_const])
                q_grid = _automatic_q_grid(grid, self.spectral_grid, dv, Nz=pm.Nz,
                                           surface_spacing=pm.surface_spacing,
                                           vertical_stretching=pm.vertical_stretching)
            else:
                q_grid = grid
        if q_grid.Nx != grid.Nx or q_grid.Ny != grid.Ny or q_grid.has_flat_vertical():
            raise ArgumentError("velocity `q_grid` must match the wave model grid horizontally and resolve z")
        qkind, qconst, qfield = self._q_depth(q_grid)
        self.q_grid = q_grid
        zf = np.ascontiguousarray(q_grid.zfaces())
        check(self._lib.rpl_set_pseudomomentum(self._h, q_grid.Nz, dptr(zf), qkind, qconst, dptr(qfield), 1e-6))
        self._q = dict(zfaces=zf, kind=qkind, const=qconst, field=qfield)

    def update_coupling(self):
        """update_coupling!(model) (current_coupling.jl:127-148): a pseudomomentum coupling is recomputed
        from the current action; prescribed currents are re-read from `velocities` (its "u" and "v" entries,
        arrays or callables of (x, y, z)) and projected again, as the reference re-reads its current fields."""
        if isinstance(self.velocities, dict) and self._transport == _lib.RPL_TRANSPORT_REFRACTION:
            self.update_currents(self.velocities["u"], self.velocities["v"])
        else:
            check(self._lib.rpl_update_coupling(self._h))
        return self

    def _current_arrays(self, u, v):
        q = self.q_grid
        if callable(u) or callable(v):
            X, Y, Z = np.meshgrid(q.xnodes(), q.ynodes(), q.znodes(), indexing="ij")
        uu = np.broadcast_to(np.asarray(u(X, Y, Z), dtype=np.float64), X.shape) if callable(u) else np.asarray(u, np.float64)
        vv = np.broadcast_to(np.asarray(v(X, Y, Z), dtype=np.float64), X.shape) if callable(v) else np.asarray(v, np.float64)
        shape = (self.grid.Nx, self.grid.Ny, q.Nz)
        if uu.shape != shape or vv.shape != shape:
            raise ArgumentError(f"u and v must have size {shape}")
        return _xfast(uu), _xfast(vv)

    def update_currents(self, u, v):
        """New prescribed currents on the Q grid of the model's velocities, applied from the next step on
        without allocating on the device (time-varying currents). u, v: (Nx, Ny, Nz) arrays or callables;
        or float64 CUDA tensors of that shape with x fastest (stride (1, Nx, Nx*Ny)), read in place."""
        if getattr(self, "_u", None) is None:
            raise ArgumentError("update_currents needs prescribed velocities")
        if hasattr(u, "data_ptr") and getattr(u, "is_cuda", False):
            Nx, Ny = self.grid.Nx, self.grid.Ny
            for t in (u, v):
                if (str(t.dtype) != "torch.float64" or tuple(t.shape) != (Nx, Ny, self.q_grid.Nz)
                        or tuple(t.stride()) != (1, Nx, Nx * Ny)):
                    raise ArgumentError("device currents must be float64 (Nx, Ny, Nz) tensors with x fastest")
            check(self._lib.rpl_update_currents_device(self._h, _lib.ctypes.c_void_p(u.data_ptr()),
                                                       _lib.ctypes.c_void_p(v.data_ptr())))
            return self
        self._u, self._v = self._current_arrays(u, v)
        check(self._lib.rpl_update_currents(self._h, dptr(self._u), dptr(self._v)))
        return self

    def _set_velocities(self, velocities):
        grid = self.grid
        if isinstance(velocities, PseudomomentumVelocities):
            self._set_pseudomomentum(velocities)
            return
        if isinstance(velocities, dict):
            u, v = velocities["u"], velocities["v"]
            q_grid = velocities.get("q_grid", velocities.get("vertical_grid"))
            if "depth" in velocities:
                raise ArgumentError("`depth` is a SpectralWaveModel kwarg; pass `SpectralWaveModel(...; depth=...)`")
        else:
            u, v = velocities
            q_grid = None
        if q_grid is None:
            if grid.has_flat_vertical():
                if isinstance(self.depth, InfiniteDepth):
                    raise ArgumentError("Flat wave grids require finite model `depth` or `q_grid` for "
                                        "array-valued prescribed velocities")
                dv = self._depth_field if self._depth_field is not None else np.array([self._depth_const])
                Nz = np.asarray(u).shape[2] if not callable(u) else None
                q_grid = _automatic_q_grid(grid, self.spectral_grid, dv, Nz=Nz)
            else:
                q_grid = grid
        if q_grid.Nx != grid.Nx or q_grid.Ny != grid.Ny or q_grid.has_flat_vertical():
            raise ArgumentError("velocity `q_grid` must match the wave model grid horizontally and resolve z")
        Nz = q_grid.Nz
        X, Y, Z = np.meshgrid(q_grid.xnodes(), q_grid.ynodes(), q_grid.znodes(), indexing="ij")
        uu = np.broadcast_to(np.asarray(u(X, Y, Z), dtype=np.float64), X.shape) if callable(u) else np.asarray(u, np.float64)
        vv = np.broadcast_to(np.asarray(v(X, Y, Z), dtype=np.float64), X.shape) if callable(v) else np.asarray(v, np.float64)
        if uu.shape != (grid.Nx, grid.Ny, Nz) or vv.shape != uu.shape:
            raise ArgumentError(f"u and v must have size {(grid.Nx, grid.Ny, Nz)}")
        qkind, qconst, qfield = self._q_depth(q_grid)
        self.q_grid = q_grid
        zf = np.ascontiguousarray(q_grid.zfaces())
        self._u, self._v = _xfast(uu), _xfast(vv)
        check(self._lib.rpl_set_currents(self._h, Nz, dptr(zf), qkind, qconst, dptr(qfield),
                                         dptr(self._u), dptr(self._v), 1e-6))
        self._q = dict(zfaces=zf, kind=qkind, const=qconst, field=qfield)

    def depth_values(self):
        """The model depth as a scalar (math.inf for InfiniteDepth) or an (Nx, Ny) array."""
        if self._depth_kind == _lib.RPL_DEPTH_INFINITE:
            return math.inf
        if self._depth_kind == _lib.RPL_DEPTH_CONSTANT:
            return self._depth_const
        return np.asarray(self._depth_field).reshape((self.grid.Nx, self.grid.Ny), order="F")

    def coupling_fields(self):
        """Ux, Uy, dUx/dkappa, dUy/dkappa, Ux_x, Ux_y, Uy_x, Uy_y as (Nx, Ny, Nk) arrays."""
        Nk = self.spectral_grid.coordinate_size()[0]
        shape = (self.grid.Nx, self.grid.Ny, Nk)
        outs = [np.empty(shape, order="F") for _ in range(8)]
        check(self._lib.rpl_get_coupling(self._h, *[dptr(o) for o in outs]))
        names = ["Ux", "Uy", "dUxdkappa", "dUydkappa", "Ux_x", "Ux_y", "Uy_x", "Uy_y"]
        return dict(zip(names, outs))

    # ------------------------------------------------------------------ sources
    def _set_sources(self, sources):
        terms = linear_terms(sources)
        if terms is not None:
            # SourceTermSet (or one such term): rates evaluated on the device before every stage
            arr = (_lib.RplSourceTerm * max(1, len(terms)))()
            self._terms_keep = []
            for k, t in enumerate(terms):
                kind, rate, rf, direction, speed, sf, prm, grav = term_record(t, self.grid)
                arr[k].kind, arr[k].rate, arr[k].direction = kind, rate, direction
                arr[k].speed, arr[k].gravity = speed, grav
                for q in range(4):
                    arr[k].p[q] = prm[q]
                if rf is not None:
                    self._terms_keep.append(rf)
                    arr[k].rate_field = dptr(rf)
                if sf is not None:
                    self._terms_keep.append(sf)
                    arr[k].speed_field = dptr(sf)
            check(self._lib.rpl_set_source_terms(self._h, arr, len(terms)))
            return
        wind_input, dissipation, cap = None, None, 0
        if isinstance(sources, PrecomputedSources):
            wind_input, dissipation = sources.wind_input, sources.dissipation
            cap = 1 if wind_input is not None else 0
        elif isinstance(sources, PressureCorrelationInput):
            wind_input = sources
        elif isinstance(sources, LocalSaturationDissipation):
            dissipation = sources
        else:
            raise ArgumentError(f"source term {type(sources).__name__} is outside the B200 path")
        s = _lib.RplSources()
        self._src_keep = []
        if wind_input is not None:
            w = wind_input.wind
            s.stress_cap = cap
            s.drag_form = 0 if wind_input.drag.form == "linear" else 1
            s.beta_max, s.z_alpha, s.p_in = wind_input.β_max, wind_input.z_α, wind_input.p_in
            s.alpha0, s.rho_air, s.rho_water = wind_input.α0, wind_input.ρ_air, wind_input.ρ_water
            s.von_karman, s.wind_gravity = wind_input.von_karman, wind_input.gravity
            if isinstance(w, numbers.Number):
                s.wind_kind = _lib.RPL_WIND_UNIFORM
                s.wind_speed, s.wind_direction = float(w), wind_input.direction
            elif isinstance(w, HollandHurricaneWind):
                s.wind_kind = _lib.RPL_WIND_HOLLAND
                s.vmax, s.rmax, s.radius, s.shape_parameter = w.vmax, w.rmax, w.radius, w.shape_parameter
                s.inflow_angle = w.inflow_angle
                s.background_x, s.background_y = w.background
                s.rotation = w.rotation.sign
                if isinstance(w.center, LinearStormTrack):
                    t = np.array(w.center.times)
                    cx = np.array([c[0] for c in w.center.centers])
                    cy = np.array([c[1] for c in w.center.centers])
                    s.n_track = len(t)
                else:
                    t = np.zeros(1)
                    cx, cy = np.array([float(w.center[0])]), np.array([float(w.center[1])])
                    s.n_track = 0
                self._src_keep += [t, cx, cy]
                s.track_t, s.track_x, s.track_y = dptr(t), dptr(cx), dptr(cy)
            elif callable(w):
                s.wind_kind = _lib.RPL_WIND_FIELD
                self._field_wind = w
            else:
                raise ArgumentError("wind must be a speed, a HollandHurricaneWind or a callable (x, y, t) -> (vx, vy)")
        if dissipation is not None:
            s.has_dissipation = 1
            s.C_ds, s.B_r, s.ds_p = dissipation.C_ds, dissipation.B_r, dissipation.p
            s.sigma_power, s.ds_gravity = dissipation.σ_power, dissipation.gravity
        check(self._lib.rpl_set_sources(self._h, _lib.ctypes.byref(s)))
        self._rpl_sources = s

    def _push_field_wind(self):
        if self._field_wind is not None:
            U, th = evaluate_wind(self._field_wind, self.grid.xnodes(), self.grid.ynodes(), self.clock.time)
            self._wind_keep = (_xfast(U), _xfast(th))
            check(self._lib.rpl_set_wind_field(self._h, dptr(self._wind_keep[0]), dptr(self._wind_keep[1])))

    # ------------------------------------------------------------------ state
    def _set_action(self, arr):
        arr = np.asarray(arr)
        if arr.dtype == np.float32:
            a, code = np.asfortranarray(arr), _lib.RPL_F32
        else:
            a, code = _xfast(arr), _lib.RPL_F64
        if a.shape != self.action.size:
            raise ArgumentError(f"array size {a.shape} does not match field size {self.action.size}")
        check(self._lib.rpl_set_action(self._h, _lib.vptr(a), code, _lib.RPL_LAYOUT_XFAST))

    def _get_action(self):
        out = np.empty(self.action.size, order="F")
        check(self._lib.rpl_get_action(self._h, _lib.vptr(out), _lib.RPL_F64, _lib.RPL_LAYOUT_XFAST))
        return out

    def _sync_clock(self):
        t = _lib.ctypes.c_double()
        it = _lib.ctypes.c_int64()
        check(self._lib.rpl_get_clock(self._h, _lib.ctypes.byref(t), _lib.ctypes.byref(it)))
        self.clock.time, self.clock.iteration = t.value, it.value

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.rpl_destroy(self._h)
            self._h = _lib.ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def device_bytes(self):
        b = _lib.ctypes.c_int64()
        check(self._lib.rpl_device_bytes(self._h, _lib.ctypes.byref(b)))
        return b.value

    def __repr__(self):
        return f"SpectralWaveModel({self.grid!r}, {self.spectral_grid!r}, precision={self.precision})"


def time_step(model, dt, nsteps=1):
    """time_step!(model, dt) for :RK3 (time_step.jl:119-170)."""
    if not dt > 0:
        raise ArgumentError("time step must be positive")
    check(model._lib.rpl_set_clock(model._h, model.clock.time, model.clock.iteration))
    if model._field_wind is not None:
        for _ in range(nsteps):
            model._push_field_wind()
            check(model._lib.rpl_step(model._h, float(dt), 1))
            model._sync_clock()
    else:
        check(model._lib.rpl_step(model._h, float(dt), int(nsteps)))
        model._sync_clock()
    model.clock.last_Δt = dt
    return model


def update_coupling(model):
    """update_coupling!(model) (current_coupling.jl:140-148)."""
    return model.update_coupling()


def compute_tendencies(model):
    """compute_tendencies!(model): fills model.tendencies (tendencies.jl:18-41,82-101)."""
    model._push_field_wind()
    G = np.empty(model.action.size, order="F")
    check(model._lib.rpl_tendency(model._h, dptr(G), _lib.RPL_LAYOUT_XFAST))
    model.tendencies._host = G
    return model.tendencies


class Simulation:
    """Minimal Oceananigans Simulation: run!(sim) calls time_step!(model, Δt) until a stop criterion."""

    def __init__(self, model, *, Δt=None, stop_iteration=None, stop_time=None, callbacks=None, dt=None, **_):
        self.model = model
        self.Δt = Δt if Δt is not None else dt
        if self.Δt is None:
            raise ArgumentError("Simulation needs Δt")
        self.stop_iteration = stop_iteration
        self.stop_time = stop_time
        self.callbacks = list(callbacks or [])

    def _remaining(self):
        m = self.model
        n = math.inf
        if self.stop_iteration is not None:
            n = min(n, self.stop_iteration - m.clock.iteration)
        if self.stop_time is not None:
            n = min(n, math.ceil((self.stop_time - m.clock.time) / self.Δt - 1e-12))
        if n is math.inf:
            raise ArgumentError("Simulation needs stop_iteration or stop_time")
        return max(int(n), 0)


def run_(simulation):
    """run!(simulation)."""
    n = simulation._remaining()
    m = simulation.model
    if simulation.callbacks:
        for _ in range(n):
            time_step(m, simulation.Δt)
            for cb in simulation.callbacks:
                cb(simulation)
    elif n > 0:
        time_step(m, simulation.Δt, nsteps=n)
    return simulation
