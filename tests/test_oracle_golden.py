"""The CPU oracle against the reference's own known answers (CPU only).

Each case restates a reference test: test/coupling/q_transform.jl:21-70,126-143,
test/integration/transport.jl:43-97, test/forcing/winds.jl, test/physics/shared.jl,
test/physics/st3.jl:34-55, plus an analytic SSP-RK3 column.
"""
import math

import numpy as np
import pytest

from ripple_b200.grids import InfiniteDepth, PolarWaveVectorGrid, RectilinearGrid
from ripple_b200.model import WENO
from ripple_b200.sources import (BulkWindDrag, Clockwise, HollandHurricaneWind, LinearStormTrack,
                                 LocalSaturationDissipation, PrecomputedSources, PressureCorrelationInput)
from ripple_b200.workloads import Workload

ZF = [-1.0, -0.73, -0.31, -0.08, 0.0]


def test_q_integrals(oracle_mod):
    L = oracle_mod.lib()
    for kappa in (1e-8, 0.5, 5.0):
        s = sum(L.ora_q_cell_integral(kappa, ZF[k], ZF[k + 1], 1.0, 1e-6) for k in range(4))
        ds = sum(L.ora_q_cell_integral_kappa_derivative(kappa, ZF[k], ZF[k + 1], 1.0, 1e-6) for k in range(4))
        assert abs(s - 1) <= 1e-14
        assert abs(ds) <= 1e-12
        sk = sum(L.ora_q_cell_integral_kernel(kappa, ZF[k], ZF[k + 1], 1.0, 1e-6) for k in range(4))
        assert abs(sk - 1) <= 1e-14
    assert L.ora_q_value(1e-10, -0.3, 2.0, 1e-6) == pytest.approx(0.5, rel=1.5e-8)
    assert abs(L.ora_q_cell_integral(0.7, -10.0, 10.0, 1.0, 1e-6) - 1) <= 1e-14
    assert abs(L.ora_q_cell_integral(0.7, 10.0, -10.0, 1.0, 1e-6) - 1) <= 1e-14
    assert abs(L.ora_q_cell_integral(0.7, -2.0, -1.0, 1.0, 1e-6)) <= 1e-14
    assert abs(L.ora_q_cell_integral(0.7, 0.0, 2.0, 1.0, 1e-6)) <= 1e-14
    assert abs(L.ora_q_cell_integral_kappa_derivative(0.7, -10.0, 10.0, 1.0, 1e-6)) <= 1e-14
    assert math.isnan(L.ora_q_cdf(0.5, -0.5, 0.0, 1e-6))  # depth <= 0 is an error in the reference


def test_doppler_explicit_sums(oracle_mod):
    L = oracle_mod.lib()
    p = oracle_mod.p
    u = np.array([0.1, -0.4, 0.8, 1.6])
    v = np.array([1.2, 0.7, -0.5, 0.3])
    kappa = np.array([0.2, 1.0])
    zf = np.array(ZF)
    Ux, Uy, dUx, dUy = (np.zeros(2) for _ in range(4))
    L.ora_doppler_velocity(1, 1, 4, 2, p(u), p(v), None, 1.0, p(kappa), p(zf), 1e-6, 0, p(Ux), p(Uy))
    L.ora_doppler_velocity(1, 1, 4, 2, p(u), p(v), None, 1.0, p(kappa), p(zf), 1e-6, 1, p(dUx), p(dUy))
    eUx = sum(u[k] * L.ora_q_cell_integral(0.2, ZF[k], ZF[k + 1], 1.0, 1e-6) for k in range(4))
    eUy = sum(v[k] * L.ora_q_cell_integral(1.0, ZF[k], ZF[k + 1], 1.0, 1e-6) for k in range(4))
    edx = sum(u[k] * L.ora_q_cell_integral_kappa_derivative(0.2, ZF[k], ZF[k + 1], 1.0, 1e-6) for k in range(4))
    edy = sum(v[k] * L.ora_q_cell_integral_kappa_derivative(1.0, ZF[k], ZF[k + 1], 1.0, 1e-6) for k in range(4))
    assert abs(Ux[0] - eUx) <= 1e-14 and abs(Uy[1] - eUy) <= 1e-14
    assert abs(dUx[0] - edx) <= 1e-14 and abs(dUy[1] - edy) <= 1e-14


def barotropic_workload():
    g = RectilinearGrid(size=(2, 2, 32), x=(0, 2), y=(0, 2), z=(-1, 0))
    sg = PolarWaveVectorGrid(κ=[0.5, 1.0], φ=[0.0, math.pi / 2, math.pi, 3 * math.pi / 2])
    u = np.ones((2, 2, 32), order="F")
    v = 2 * np.ones((2, 2, 32), order="F")
    N0 = np.ones((2, 2, 2, 4), order="F")
    return Workload("barotropic", g, sg, InfiniteDepth(), N0, 0.001, 1, velocities={"u": u, "v": v},
                    horizontal_advection=None)


def test_barotropic_current(oracle_mod):
    o = oracle_mod.Oracle(barotropic_workload())
    assert np.max(np.abs(o.U["Ux"] - 1)) <= 1e-12
    assert np.max(np.abs(o.U["Uy"] - 2)) <= 1e-12
    assert np.max(np.abs(o.U["dUxdkappa"])) < 1e-10


def sinusoid_workload(axis="x"):
    N, L = 64, 64.0
    g = RectilinearGrid(size=(N, N, 1), x=(0, L), y=(0, L), z=(-1, 0))
    if axis == "x":
        sg = PolarWaveVectorGrid(κ=[1.0], φ=[0.0], φ_faces=[-math.pi / 32, math.pi / 32])
        prof = 1 + 0.1 * np.sin(2 * math.pi * g.xnodes() / L)
        N0 = np.broadcast_to(prof[:, None, None, None], (N, N, 1, 1))
    else:
        sg = PolarWaveVectorGrid(κ=[1.0], φ=[math.pi / 2], φ_faces=[math.pi / 2 - math.pi / 32, math.pi / 2 + math.pi / 32])
        prof = 1 + 0.1 * np.sin(2 * math.pi * g.ynodes() / L)
        N0 = np.broadcast_to(prof[None, :, None, None], (N, N, 1, 1))
    return Workload("sinusoid", g, sg, InfiniteDepth(), np.asfortranarray(N0), 0.1, 1)


@pytest.mark.parametrize("axis", ["x", "y"])
def test_weno_sinusoid_transport(oracle_mod, axis):
    w = sinusoid_workload(axis)
    o = oracle_mod.Oracle(w, explicit_spectral_faces=True)
    G = o.tendency(w.N0)
    L = 64.0
    if axis == "x":
        u = o._cg[0][0]
        exp = -u * 0.1 * 2 * math.pi / L * np.cos(2 * math.pi * w.grid.xnodes() / L)[:, None]
        assert abs(o._cg[1][0]) < 1e-15
    else:
        u = o._cg[1][0]
        exp = -u * 0.1 * 2 * math.pi / L * np.cos(2 * math.pi * w.grid.ynodes() / L)[None, :]
        assert abs(o._cg[0][0]) <= 10 * np.finfo(float).eps
    assert np.max(np.abs(G[:, :, 0, 0] - exp)) < 1e-7
    tot0 = o.diagnostics(w.N0)["total_action"]
    N1, _ = o.step(w.N0, 0.1)
    assert abs(o.diagnostics(N1)["total_action"] - tot0) <= 1e-10
    assert N1.min() > 0


def linear_damping_workload(N0val=50.0):
    """Source-only column whose whitecapping rate is constant (p = 0, overshoot > 0 throughout)."""
    g = RectilinearGrid(size=(1, 1, 1), x=(0, 1), y=(0, 1), z=(0, 1))
    sg = PolarWaveVectorGrid(κ=[0.5, 1.0], φ=[0.0, math.pi])
    diss = LocalSaturationDissipation(C_ds=-0.4, B_r=1e-3, p=0.0, σ_power=1.0)
    N0 = np.full((1, 1, 2, 2), N0val, order="F")
    return Workload("damping", g, sg, InfiniteDepth(), N0, 0.1, 3, sources=diss, horizontal_advection=None)


def test_rk3_linear_column(oracle_mod):
    w = linear_damping_workload()
    o = oracle_mod.Oracle(w)
    dt = 0.1
    N, _ = o.step(w.N0, dt, nsteps=3)
    for m, k in enumerate((0.5, 1.0)):
        lam = 0.4 * math.sqrt(9.81 * k)
        z = lam * dt
        amp = 1 - z + z * z / 2 - z ** 3 / 6
        assert N[0, 0, m, 0] == pytest.approx(50.0 * amp ** 3, rel=1e-14)


def test_drag_and_winds(oracle_mod):
    L = oracle_mod.lib()
    assert L.ora_friction_velocity_linear(10.0) == pytest.approx(10.0 * math.sqrt(1.45e-3), rel=1e-12)
    assert BulkWindDrag("linear").drag_coefficient(10.0) == pytest.approx(1.45e-3, rel=1e-12)
    assert BulkWindDrag("capped").drag_coefficient(60.0) >= 4e-4
    keep = []
    track = LinearStormTrack([0.0, 1.0, 3.0], [(0.0, 0.0), (2.0, 1.0), (4.0, -1.0)])
    assert track(-1.0) == (0.0, 0.0) and track(0.5) == (1.0, 0.5)
    assert track(2.0) == (3.0, 0.0) and track(4.0) == (4.0, -1.0)
    h = oracle_mod.holland_struct(HollandHurricaneWind(center=track, vmax=0.3, rmax=1.0, radius=4.0), keep)
    cx, cy = oracle_mod.ctypes.c_double(), oracle_mod.ctypes.c_double()
    for t, c in ((-1.0, (0.0, 0.0)), (0.5, (1.0, 0.5)), (2.0, (3.0, 0.0)), (4.0, (4.0, -1.0))):
        L.ora_storm_center(oracle_mod.ctypes.byref(h), t, oracle_mod.ctypes.byref(cx), oracle_mod.ctypes.byref(cy))
        assert (cx.value, cy.value) == c

    def speed_angle(w, x, y, t):
        hs = oracle_mod.holland_struct(w, keep)
        vx, vy = oracle_mod.ctypes.c_double(), oracle_mod.ctypes.c_double()
        L.ora_holland_velocity(oracle_mod.ctypes.byref(hs), x, y, t, oracle_mod.ctypes.byref(vx), oracle_mod.ctypes.byref(vy))
        return math.hypot(vx.value, vy.value), math.atan2(vy.value, vx.value)

    moving = HollandHurricaneWind(center=LinearStormTrack([0.0, 2.0], [(0.0, 0.0), (2.0, 0.0)]), vmax=0.3,
                                  rmax=1.0, radius=4.0, shape_parameter=1.5)
    assert speed_angle(moving, 1.0, 0.0, 0.0)[0] == pytest.approx(0.3)
    assert speed_angle(moving, 2.0, 0.0, 1.0)[0] == pytest.approx(0.3)
    assert speed_angle(moving, 0.0, 0.0, 0.0)[0] == 0
    assert speed_angle(moving, 3.0, 0.0, 0.0)[0] < 0.3
    assert speed_angle(moving, 1.0, 0.0, 0.0)[1] == pytest.approx(math.pi / 2)
    cw = HollandHurricaneWind(vmax=0.3, rmax=1.0, radius=4.0, rotation=Clockwise)
    assert speed_angle(cw, 1.0, 0.0, 0.0)[1] == pytest.approx(-math.pi / 2)
    inflow = HollandHurricaneWind(vmax=0.3, rmax=1.0, radius=4.0, inflow_angle=math.pi / 12, background=(0.05, 0.0))
    s, a = speed_angle(inflow, 2.0, 0.0, 0.0)
    assert math.isfinite(s) and math.isfinite(a) and s > 0
    tracked = HollandHurricaneWind(center=track, vmax=0.3, rmax=1.0, radius=4.0)
    assert speed_angle(tracked, 3.0, 1.0, 1.0)[0] == pytest.approx(0.3)


def wind_column_workload(U10=15.0):
    """Wind input on a 1x1 column: frequencies 0.1..0.3 Hz as deep-water wavenumbers, 8 directions."""
    g = RectilinearGrid(size=(1, 1, 1), x=(0, 1), y=(0, 1), z=(0, 1))
    f = np.linspace(0.1, 0.3, 4)
    kappa = (2 * math.pi * f) ** 2 / 9.81
    phi = np.linspace(0, 2 * math.pi * 7 / 8, 8)
    sg = PolarWaveVectorGrid(κ=kappa, φ=phi)
    src = PrecomputedSources(wind_input=PressureCorrelationInput(drag=BulkWindDrag("linear"), wind=U10))
    N0 = np.full((1, 1, 4, 8), 1e-3, order="F")
    return Workload("wind", g, sg, InfiniteDepth(), N0, 1.0, 1, sources=src, horizontal_advection=None)


def test_wind_input_signs(oracle_mod):
    w = wind_column_workload(15.0)
    G = oracle_mod.Oracle(w).tendency(w.N0)
    assert G.max() > 0 and G.min() >= 0
    calm = wind_column_workload(0.0)
    assert np.all(oracle_mod.Oracle(calm).tendency(calm.N0) == 0)


def test_spectral_grid_defaults_match_oracle(oracle_mod):
    kappa = np.geomspace(0.002, 0.5, 32)
    phi = np.arange(36) * (2 * math.pi / 36)
    sg = PolarWaveVectorGrid(κ=kappa, φ=phi)
    assert np.array_equal(sg.κ_faces, oracle_mod.lower_bounded_faces(kappa))
    assert np.array_equal(sg.φ_faces, oracle_mod.uniform_periodic_faces(phi))
    w = np.empty(32 * 36)
    oracle_mod.lib().ora_polar_weights(32, 36, oracle_mod.p(sg.κ_faces), oracle_mod.p(sg.φ_faces), oracle_mod.p(w))
    assert np.array_equal(sg.weights, w.reshape(32, 36, order="F"))


def stretched_workload():
    """A small model on a stretched horizontal grid (x faces growing geometrically, y faces ragged):
    the total action must weight every column by its own Δx(i)·Δy(j)."""
    xf = np.cumsum(np.concatenate([[0.0], 1.0 * 1.3 ** np.arange(9)]))
    yf = np.array([0.0, 0.5, 2.0, 2.25, 4.0, 7.5, 8.0, 11.0])
    g = RectilinearGrid(size=(9, 7, 2), x=xf, y=yf, z=(-1.0, 0.0))
    sg = PolarWaveVectorGrid(κ=np.linspace(0.3, 0.9, 5), φ=np.arange(6) * 2 * math.pi / 6)
    N0 = np.asfortranarray(np.random.default_rng(3).uniform(0.0, 1.0, (9, 7, 5, 6)))
    return Workload("stretched", g, sg, 2.0, N0, 0.05, 1, horizontal_advection=None)


def test_total_action_stretched_grid(oracle_mod):
    """total_action sums density(i,j)·Δx(i)·Δy(j) per cell (diagnostic_operations.jl:492-503,
    bulk_statistics.jl:87-91), not m0 times the first cell's area."""
    w = stretched_workload()
    d = oracle_mod.Oracle(w).diagnostics(w.N0)
    dx, dy = w.grid.xspacings(), w.grid.yspacings()
    expect = float(np.sum(d["m0"] * dx[:, None] * dy[None, :]))
    assert d["total_action"] == pytest.approx(expect, rel=1e-14)
    assert abs(d["total_action"] - float(np.sum(d["m0"])) * dx[0] * dy[0]) > 0.1 * expect
