"""TEST INFRASTRUCTURE ONLY: ctypes driver of the CPU FP64 oracle (libripple_oracle.so).

Builds an oracle model from a workload's raw inputs (grid coordinates, depth,
currents, sources) with the oracle's own restated set-up functions -- faces,
weights, group velocities, Q-transform Doppler velocity, gradients -- so the
CUDA library's set-up is checked along with its stepping. Only tests/,
__graft_entry__.smoke() and bench.py's CPU baseline may import this module.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libripple_oracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_i64, _i32, _d = ctypes.c_int64, ctypes.c_int32, ctypes.c_double

TRANSPORT_NONE, TRANSPORT_REFRACTION, TRANSPORT_INTRINSIC = 0, 1, 2
WIND_NONE, WIND_UNIFORM, WIND_HOLLAND, WIND_FIELD = 0, 1, 2, 3


class OraHolland(ctypes.Structure):
    _fields_ = [("vmax", _d), ("rmax", _d), ("radius", _d), ("shape_parameter", _d), ("inflow_angle", _d),
                ("background_x", _d), ("background_y", _d), ("rotation", _i32), ("n_track", _i32),
                ("track_t", _dp), ("center_x", _dp), ("center_y", _dp)]


class OraTerm(ctypes.Structure):
    _fields_ = [("kind", _i32), ("pad", _i32), ("rate", _d), ("rate_field", _dp), ("direction", _d), ("speed", _d),
                ("speed_field", _dp), ("p", _d * 4), ("gravity", _d)]


class OraModel(ctypes.Structure):
    _fields_ = [("Nx", _i64), ("Ny", _i64), ("Nk", _i64), ("Np", _i64), ("dx", _d), ("dy", _d),
                ("xnodes", _dp), ("ynodes", _dp), ("kappa", _dp), ("kappa_faces", _dp), ("phi", _dp),
                ("phi_faces", _dp), ("weights", _dp), ("transport", _i32), ("cg_per_cell", _i32),
                ("cg_x", _dp), ("cg_y", _dp), ("Ux", _dp), ("Uy", _dp), ("Uxx", _dp), ("Uxy", _dp),
                ("Uyx", _dp), ("Uyy", _dp), ("wind_kind", _i32), ("wind_speed", _d), ("wind_direction", _d),
                ("holland", OraHolland), ("wind_U10", _dp), ("wind_theta", _dp), ("beta_max", _d),
                ("z_alpha", _d), ("p_in", _d), ("alpha0", _d), ("rho_air", _d), ("rho_water", _d),
                ("von_karman", _d), ("gravity", _d), ("has_dissipation", _i32), ("C_ds", _d), ("B_r", _d),
                ("ds_p", _d), ("sigma_power", _d), ("ds_gravity", _d), ("pm_mode", _i32), ("pm_per_cell", _i32),
                ("pm_overlap", _dp), ("pm_kx", _dp), ("pm_ky", _dp), ("gse", _i32), ("periodic_x", _i32),
                ("periodic_y", _i32), ("gse_alpha_s", _d), ("gse_alpha_n", _d), ("xspacings", _dp),
                ("yspacings", _dp), ("n_terms", _i32), ("terms", ctypes.POINTER(OraTerm))]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        for name in ("ora_q_value", "ora_q_cdf", "ora_q_cell_integral", "ora_q_cdf_kappa_derivative",
                     "ora_q_cell_integral_kappa_derivative", "ora_q_cdf_kernel", "ora_q_cell_integral_kernel",
                     "ora_q_cell_integral_kappa_derivative_kernel"):
            f = getattr(L, name)
            f.restype = _d
            f.argtypes = [_d] * (4 if name in ("ora_q_value", "ora_q_cdf", "ora_q_cdf_kappa_derivative",
                                               "ora_q_cdf_kernel") else 5)
        L.ora_doppler_velocity.argtypes = [_i64, _i64, _i64, _i64, _dp, _dp, _dp, _d, _dp, _dp, _d, _i32, _dp, _dp]
        L.ora_current_gradients.argtypes = [_i64, _i64, _i64, _dp, _dp, _d, _d, _dp, _dp, _dp, _dp]
        L.ora_lower_bounded_faces.argtypes = [_i64, _dp, _d, _dp]
        L.ora_uniform_periodic_faces.argtypes = [_i64, _dp, _dp]
        L.ora_polar_weights.argtypes = [_i64, _i64, _dp, _dp, _dp]
        L.ora_group_velocity_deep.argtypes = [_i64, _i64, _dp, _dp, _dp, _d, _dp, _dp]
        L.ora_group_velocity_finite.argtypes = [_i64, _i64, _i64, _i64, _dp, _dp, _dp, _d, _d, _dp, _dp]
        L.ora_friction_velocity_linear.restype = _d
        L.ora_friction_velocity_linear.argtypes = [_d]
        L.ora_holland_velocity.argtypes = [ctypes.POINTER(OraHolland), _d, _d, _d, _dp, _dp]
        L.ora_storm_center.argtypes = [ctypes.POINTER(OraHolland), _d, _dp, _dp]
        L.ora_wind_fields.argtypes = [ctypes.POINTER(OraModel), _d, _dp, _dp, _dp]
        L.ora_tendency.argtypes = [ctypes.POINTER(OraModel), _dp, _d, _i32, _dp]
        L.ora_stress_factor.argtypes = [ctypes.POINTER(OraModel), _dp, _d, _dp]
        L.ora_rk3_step.argtypes = [ctypes.POINTER(OraModel), _dp, _d, _i64, _dp]
        L.ora_diagnostics.argtypes = [ctypes.POINTER(OraModel), _dp, _dp, _dp, _dp, _dp, _dp]
        L.ora_first_moment_measures.argtypes = [_i64, _i64, _dp, _dp, _dp, _dp]
        L.ora_pm_overlap_tables.argtypes = [_i64, _i64, _i64, _dp, _i64, _dp, _dp, _d, _d, _dp, _dp]
        L.ora_pm_doppler_velocity.argtypes = [_i64, _i64, _i64, _i64, _dp, _i32, _dp, _dp, _dp, _dp,
                                              _dp, _dp, _dp, _dp]
        L.ora_pm_cells.argtypes = [_i64, _i64, _i64, _i64, _dp, _i64, _dp, _dp, _d, _dp, _dp, _dp, _d, _i32,
                                   _dp, _dp]
        L.ora_spatial_averaging.argtypes = [ctypes.POINTER(OraModel), _dp, _d]
        L.ora_spatial_averaging_at.argtypes = [ctypes.POINTER(OraModel), _dp, _d, ctypes.c_int64]
        L.ora_num_threads.restype = ctypes.c_int
        L.ora_set_num_threads.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def f64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def xfast(a):
    return np.asfortranarray(np.asarray(a, dtype=np.float64))


def lower_bounded_faces(centers, lower=0.0):
    c = f64(centers)
    out = np.empty(len(c) + 1)
    lib().ora_lower_bounded_faces(len(c), p(c), lower, p(out))
    return out


def uniform_periodic_faces(centers):
    c = f64(centers)
    out = np.empty(len(c) + 1)
    lib().ora_uniform_periodic_faces(len(c), p(c), p(out))
    return out


def holland_struct(w, keep):
    h = OraHolland()
    h.vmax, h.rmax, h.radius, h.shape_parameter = w.vmax, w.rmax, w.radius, w.shape_parameter
    h.inflow_angle = w.inflow_angle
    h.background_x, h.background_y = w.background
    h.rotation = w.rotation.sign
    c = w.center
    if hasattr(c, "times"):
        t, cx, cy = f64(c.times), f64([q[0] for q in c.centers]), f64([q[1] for q in c.centers])
        h.n_track = len(t)
    else:
        t, cx, cy = f64([0.0]), f64([c[0]]), f64([c[1]])
        h.n_track = 0
    keep += [t, cx, cy]
    h.track_t, h.center_x, h.center_y = p(t), p(cx), p(cy)
    return h


class Oracle:
    """CPU FP64 model built from a workload (ripple_b200.workloads.Workload or the same fields)."""

    def __init__(self, w, explicit_spectral_faces=None):
        L = lib()
        g = w.grid
        sg = w.spectral_grid
        self.w = w
        self.Nx, self.Ny = g.Nx, g.Ny
        self.Nk, self.Np = len(sg.κ), len(sg.φ)
        k = self._k = f64(sg.κ)
        ph = self._p = f64(sg.φ)
        # faces: restated defaults, unless the workload's grid was built with explicit faces
        if explicit_spectral_faces:
            self._kf, self._pf = f64(sg.κ_faces), f64(sg.φ_faces)
        else:
            self._kf, self._pf = lower_bounded_faces(k), uniform_periodic_faces(ph)
        nb = self.Nk * self.Np
        self._w = np.empty(nb)
        L.ora_polar_weights(self.Nk, self.Np, p(self._kf), p(self._pf), p(self._w))
        self._x, self._y = f64(g.xnodes()), f64(g.ynodes())
        m = self.m = OraModel()
        m.Nx, m.Ny, m.Nk, m.Np = self.Nx, self.Ny, self.Nk, self.Np
        m.dx, m.dy = g.first_spacings() if hasattr(g, "first_spacings") else (float(g.xspacings()[0]),
                                                                              float(g.yspacings()[0]))
        m.xnodes, m.ynodes = p(self._x), p(self._y)
        self._xsp, self._ysp = f64(g.xspacings()), f64(g.yspacings())
        m.xspacings, m.yspacings = p(self._xsp), p(self._ysp)
        m.kappa, m.kappa_faces, m.phi, m.phi_faces, m.weights = p(k), p(self._kf), p(ph), p(self._pf), p(self._w)
        depth = w.depth
        infinite = type(depth).__name__ == "InfiniteDepth"
        self._keep = []
        if infinite:
            cgx, cgy = np.empty(nb), np.empty(nb)
            L.ora_group_velocity_deep(self.Nk, self.Np, p(self._kf), p(self._pf), p(self._w), 9.81, p(cgx), p(cgy))
            m.cg_per_cell = 0
        elif np.isscalar(depth):
            cgx, cgy = np.empty(nb), np.empty(nb)
            L.ora_group_velocity_finite(self.Nx, self.Ny, self.Nk, self.Np, p(k), p(ph), None, float(depth),
                                        9.81, p(cgx), p(cgy))
            m.cg_per_cell = 0
        else:
            dfield = xfast(depth)
            self._keep.append(dfield)
            n = self.Nx * self.Ny * nb
            cgx, cgy = np.empty(n), np.empty(n)
            L.ora_group_velocity_finite(self.Nx, self.Ny, self.Nk, self.Np, p(k), p(ph), p(dfield), 0.0, 9.81,
                                        p(cgx), p(cgy))
            m.cg_per_cell = 1
        self._cg = (cgx, cgy)
        m.cg_x, m.cg_y = p(cgx), p(cgy)
        if w.velocities is not None:
            m.transport = TRANSPORT_REFRACTION
            if type(w.velocities).__name__ == "PseudomomentumVelocities":
                self._set_pseudomomentum(w)
            else:
                self._set_currents(w)
        elif w.horizontal_advection is not None:
            m.transport = TRANSPORT_INTRINSIC
        else:
            m.transport = TRANSPORT_NONE
        self._set_sources(w.sources)
        m.periodic_x = int(g.topology[0] == "Periodic")
        m.periodic_y = int(g.topology[1] == "Periodic")
        ps = getattr(w, "propagation_smoothing", None)
        if ps is not None:
            m.gse, m.gse_alpha_s, m.gse_alpha_n = 1, float(ps.αs), float(ps.αn)

    def _set_currents(self, w, u=None, v=None):
        L = lib()
        g = w.grid
        q_grid = w.velocities.get("q_grid", g)
        if u is None:
            u, v = w.velocities["u"], w.velocities["v"]
        u, v = xfast(u), xfast(v)
        zf = f64(q_grid.zfaces())
        Nz = len(zf) - 1
        depth = w.depth
        if type(depth).__name__ == "InfiniteDepth":
            dfield, dconst = None, float(zf[-1] - zf[0])
        elif np.isscalar(depth):
            dfield, dconst = None, float(depth)
        else:
            dfield, dconst = xfast(depth), 0.0
        n3 = self.Nx * self.Ny * self.Nk
        self.U = {k: np.empty(n3) for k in ("Ux", "Uy", "dUxdkappa", "dUydkappa", "Ux_x", "Ux_y", "Uy_x", "Uy_y")}
        L.ora_doppler_velocity(self.Nx, self.Ny, Nz, self.Nk, p(u), p(v), p(dfield), dconst, p(self._k), p(zf),
                               1e-6, 0, p(self.U["Ux"]), p(self.U["Uy"]))
        L.ora_doppler_velocity(self.Nx, self.Ny, Nz, self.Nk, p(u), p(v), p(dfield), dconst, p(self._k), p(zf),
                               1e-6, 1, p(self.U["dUxdkappa"]), p(self.U["dUydkappa"]))
        m = self.m
        L.ora_current_gradients(self.Nx, self.Ny, self.Nk, p(self.U["Ux"]), p(self.U["Uy"]), 1.0 / m.dx, 1.0 / m.dy,
                                p(self.U["Ux_x"]), p(self.U["Ux_y"]), p(self.U["Uy_x"]), p(self.U["Uy_y"]))
        m.Ux, m.Uy = p(self.U["Ux"]), p(self.U["Uy"])
        m.Uxx, m.Uxy, m.Uyx, m.Uyy = p(self.U["Ux_x"]), p(self.U["Ux_y"]), p(self.U["Uy_x"]), p(self.U["Uy_y"])

    def update_currents(self, u, v):
        """New currents on the same Q grid: update_coupling!(::CWCMPrescribedCurrentCoupling)
        (current_coupling.jl:127-138)."""
        self._set_currents(self.w, u, v)

    def _q_faces_and_depth(self, w, q_grid, Nz=None, surface_spacing=None, stretch=2.0):
        """Q-transform z faces and projection depth (lagrangian_velocities.jl:192-225,294-311)."""
        g = w.grid
        depth = w.depth
        infinite = type(depth).__name__ == "InfiniteDepth"
        if q_grid is None and not g.has_flat_vertical():
            q_grid = g
        if q_grid is not None:
            zf = f64(q_grid.zfaces())
        else:
            if infinite:
                raise ValueError("Flat wave grids need a finite depth or a q_grid")
            H = float(depth) if np.isscalar(depth) else float(np.max(depth))
            dz = 1.0 / (20.0 * float(np.max(self._k))) if surface_spacing is None else float(surface_spacing)
            if Nz is None:
                Nz = max(16, math.ceil((H / dz) ** (1.0 / stretch)))
            zf = f64([-H * (1.0 - k / Nz) ** stretch for k in range(Nz + 1)])
        if infinite:
            return zf, None, float(zf[-1] - zf[0])
        if np.isscalar(depth):
            return zf, None, float(depth)
        return zf, xfast(depth), 0.0

    def _set_pseudomomentum(self, w):
        """PseudomomentumVelocities: overlap and moment tables (current_coupling.jl:93-118); the velocity
        itself is recomputed from the action inside every tendency."""
        L = lib()
        v = w.velocities
        zf, dfield, dconst = self._q_faces_and_depth(w, v.q_grid, v.Nz, v.surface_spacing,
                                                     float(v.vertical_stretching))
        Nk, Np = self.Nk, self.Np
        kx, ky = np.empty(Nk * Np), np.empty(Nk * Np)
        L.ora_first_moment_measures(Nk, Np, p(self._kf), p(self._pf), p(kx), p(ky))
        cols = 1 if dfield is None else self.Nx * self.Ny
        ov, dov = np.empty(cols * Nk * Nk), np.empty(cols * Nk * Nk)
        L.ora_pm_overlap_tables(self.Nx, self.Ny, Nk, p(self._k), len(zf) - 1, p(zf), p(dfield), dconst, 1e-6,
                                p(ov), p(dov))
        self.pm = dict(zfaces=zf, depth_field=dfield, depth=dconst, kx=kx, ky=ky, overlap=ov,
                       derivative_overlap=dov, per_cell=int(dfield is not None))
        m = self.m
        m.pm_mode, m.pm_per_cell = 1, self.pm["per_cell"]
        m.pm_overlap, m.pm_kx, m.pm_ky = p(ov), p(kx), p(ky)

    def pm_velocity(self, N):
        """Pseudomomentum Doppler velocity of the action N (pseudomomentum.jl:123-138,316-342):
        Ux, Uy, dUxdkappa, dUydkappa as (Nx, Ny, Nk) arrays."""
        q = self.pm
        N = xfast(N)
        shape = (self.Nx, self.Ny, self.Nk)
        outs = [np.empty(shape, order="F") for _ in range(4)]
        lib().ora_pm_doppler_velocity(self.Nx, self.Ny, self.Nk, self.Np, p(N), q["per_cell"], p(q["overlap"]),
                                      p(q["derivative_overlap"]), p(q["kx"]), p(q["ky"]), *[p(o) for o in outs])
        return dict(zip(("Ux", "Uy", "dUxdkappa", "dUydkappa"), outs))

    def pm_cells(self, N, cell_average=True):
        """Pseudomomentum per Q-grid cell (pseudomomentum.jl:173-210,380-410): px, py as (Nx, Ny, Nz)."""
        q = self.pm
        N = xfast(N)
        Nz = len(q["zfaces"]) - 1
        px, py = np.empty((self.Nx, self.Ny, Nz), order="F"), np.empty((self.Nx, self.Ny, Nz), order="F")
        lib().ora_pm_cells(self.Nx, self.Ny, self.Nk, self.Np, p(N), Nz, p(q["zfaces"]), p(q["depth_field"]),
                           q["depth"], p(self._k), p(q["kx"]), p(q["ky"]), 1e-6, int(cell_average), p(px), p(py))
        return px, py

    def doppler_of(self, u, v):
        """Q-transform Doppler velocity of a current profile (u, v) on the pseudomomentum Q grid
        (doppler_velocity.jl:45-82): Ux, Uy, dUxdkappa, dUydkappa."""
        q = self.pm
        L = lib()
        Nz = len(q["zfaces"]) - 1
        u, v = xfast(u), xfast(v)
        shape = (self.Nx, self.Ny, self.Nk)
        outs = [np.empty(shape, order="F") for _ in range(4)]
        L.ora_doppler_velocity(self.Nx, self.Ny, Nz, self.Nk, p(u), p(v), p(q["depth_field"]), q["depth"], p(self._k),
                               p(q["zfaces"]), 1e-6, 0, p(outs[0]), p(outs[1]))
        L.ora_doppler_velocity(self.Nx, self.Ny, Nz, self.Nk, p(u), p(v), p(q["depth_field"]), q["depth"], p(self._k),
                               p(q["zfaces"]), 1e-6, 1, p(outs[2]), p(outs[3]))
        return dict(zip(("Ux", "Uy", "dUxdkappa", "dUydkappa"), outs))

    def _set_sources(self, s):
        m = self.m
        m.wind_kind = WIND_NONE
        m.has_dissipation = 0
        m.n_terms = 0
        if s is None:
            return
        from ripple_b200.sources import linear_terms, term_record
        terms = linear_terms(s)
        if terms is not None:
            arr = (OraTerm * max(1, len(terms)))()
            for k, t in enumerate(terms):
                kind, rate, rf, direction, speed, sf, prm, grav = term_record(t, self.w.grid)
                arr[k].kind, arr[k].rate, arr[k].direction, arr[k].speed, arr[k].gravity = kind, rate, direction, speed, grav
                for q in range(4):
                    arr[k].p[q] = prm[q]
                if rf is not None:
                    self._keep.append(rf)
                    arr[k].rate_field = p(rf)
                if sf is not None:
                    self._keep.append(sf)
                    arr[k].speed_field = p(sf)
            self._keep.append(arr)
            m.n_terms, m.terms = len(terms), arr
            return
        name = type(s).__name__
        wind_input = dissipation = None
        if name == "PrecomputedSources":
            wind_input, dissipation = s.wind_input, s.dissipation
            self.stress_cap = wind_input is not None
        elif name == "PressureCorrelationInput":
            wind_input = s
            self.stress_cap = False
        elif name == "LocalSaturationDissipation":
            dissipation = s
        if wind_input is not None:
            if not getattr(self, "stress_cap", False):
                raise NotImplementedError("the oracle restates the bundled (stress-capped) wind input only")
            if wind_input.drag.form != "linear":
                raise NotImplementedError("the oracle restates BulkWindDrag(:linear)")
            wnd = wind_input.wind
            if np.isscalar(wnd):
                m.wind_kind = WIND_UNIFORM
                m.wind_speed, m.wind_direction = float(wnd), wind_input.direction
            else:
                m.wind_kind = WIND_HOLLAND
                m.holland = holland_struct(wnd, self._keep)
            m.beta_max, m.z_alpha, m.p_in, m.alpha0 = wind_input.β_max, wind_input.z_α, wind_input.p_in, wind_input.α0
            m.rho_air, m.rho_water, m.von_karman, m.gravity = (wind_input.ρ_air, wind_input.ρ_water,
                                                              wind_input.von_karman, wind_input.gravity)
        if dissipation is not None:
            m.has_dissipation = 1
            m.C_ds, m.B_r, m.ds_p = dissipation.C_ds, dissipation.B_r, dissipation.p
            m.sigma_power, m.ds_gravity = dissipation.σ_power, dissipation.gravity

    # -------------------------------------------------------------- operations
    def tendency(self, N, t=0.0, with_sources=True):
        N = xfast(N)
        G = np.empty_like(N, order="F")
        lib().ora_tendency(ctypes.byref(self.m), p(N), float(t), int(with_sources), p(G))
        return G

    def step(self, N, dt, nsteps=1, t=0.0):
        N = xfast(N).copy(order="F")
        tt = np.array([float(t)])
        lib().ora_rk3_step(ctypes.byref(self.m), p(N), float(dt), int(nsteps), p(tt))
        return N, float(tt[0])

    def spatial_averaging(self, N, dt, y_offset=0):
        """SpatialAveraging applied once (propagation_smoothing.jl:60-199); y_offset: the model's rows are
        rows y_offset + 1 .. y_offset + Ny of a larger grid (a decomposition slab), whose row indices
        the corner positions are computed at."""
        N = xfast(N).copy(order="F")
        lib().ora_spatial_averaging_at(ctypes.byref(self.m), p(N), float(dt), int(y_offset))
        return N

    def stress_factor(self, N, t=0.0):
        out = np.empty((self.Nx, self.Ny), order="F")
        lib().ora_stress_factor(ctypes.byref(self.m), p(xfast(N)), float(t), p(out))
        return out

    def wind_fields(self, t=0.0):
        outs = [np.empty((self.Nx, self.Ny), order="F") for _ in range(3)]
        lib().ora_wind_fields(ctypes.byref(self.m), float(t), *[p(o) for o in outs])
        return outs

    def diagnostics(self, N):
        outs = [np.empty((self.Nx, self.Ny), order="F") for _ in range(4)]
        tot = np.zeros(1)
        lib().ora_diagnostics(ctypes.byref(self.m), p(xfast(N)), *[p(o) for o in outs], p(tot))
        return dict(m0=outs[0], Hs=outs[1], kappa_rms=outs[2], mean_direction=outs[3], total_action=float(tot[0]))

    def coupling(self, shape):
        return {k: v.reshape(shape, order="F") for k, v in self.U.items()}


def set_threads(n):
    lib().ora_set_num_threads(int(n))


def num_threads():
    return lib().ora_num_threads()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    den = math.sqrt(float(np.dot(b, b)))
    return math.sqrt(float(np.dot(a - b, a - b))) / (den if den > 0 else 1.0)
