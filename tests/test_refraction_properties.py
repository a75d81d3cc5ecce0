"""Pins of the refraction terms (wave_current_refraction.jl:74-151) that do not come from the oracle.

The reference holds no vectors for the fused kernel's kappa and phi fluxes, so these tests check
properties that follow from the scheme itself. Each runs on the CPU oracle and, marked gpu, on the
FP64 library path through the C-ABI:

* a spatially uniform current has zero gradients, so c_kappa = c_phi = 0 (:94-95). On an action that is
  uniform in x and y, every WENO5 face equals its cell value and the tendency is exactly zero;
* mirror symmetry. Reflecting y (j -> Ny-1-j) maps phi -> -phi and v -> -v, hence U_y -> -U_y,
  U_x,y -> -U_x,y and U_y,x -> -U_y,x. Then c_kappa is unchanged and c_phi changes sign, as do c_g,y and
  the y velocity. The upwinded WENO5 stencils mirror with them, so the tendency of the mirrored input is
  the mirrored tendency. The same holds for x (i -> Nx-1-i, phi -> pi - phi, u -> -u);
* direction of the kappa flux. A converging current (dU_x/dx < 0, no other gradient) gives
  c_kappa = -kappa cos^2(phi) U_x,x >= 0, which moves action to larger kappa. On an action that is
  uniform in x, y and phi only the kappa flux acts: the kappa-weighted moment of the tendency is
  positive where the flow converges and negative where it diverges;
* the reference's own FP32 agreement check (scripts/gpu/run_metal_smoke.jl:152-226), restated against
  the FP64 oracle: on its 6 x 5 grid with 4 kappa x 6 directions and its analytic currents and action,
  the FP32 fused tendency is within 2e-4 and the action after one step within 2e-5 (max abs).
"""
import math

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import workloads
from ripple_b200.grids import InfiniteDepth, PolarWaveVectorGrid, RectilinearGrid


def refraction_workload(Nx=12, Ny=10, Nk=6, Np=8, seed=1, uniform_action=False, isotropic=False, u=None, v=None):
    """A small refraction model: barotropic currents (random smooth fields unless given), random
    positive action (or uniform in x and y, optionally also in phi)."""
    rng = np.random.default_rng(seed)
    Lx, Ly = 2.0 * Nx, 2.0 * Ny
    g = RectilinearGrid(size=(Nx, Ny, 4), x=(0.0, Lx), y=(0.0, Ly), z=(-1.0, 0.0))
    sg = PolarWaveVectorGrid(κ=np.linspace(0.3, 0.9, Nk), φ=np.arange(Np) * 2 * math.pi / Np)
    X, Y = np.meshgrid(g.xnodes(), g.ynodes(), indexing="ij")
    if u is None:
        a = rng.uniform(-0.3, 0.3, 4)
        u = a[0] * np.sin(2 * math.pi * X / Lx + a[1]) + a[2] * np.cos(4 * math.pi * Y / Ly + a[3])
        b = rng.uniform(-0.3, 0.3, 4)
        v = b[0] * np.cos(2 * math.pi * X / Lx + b[1]) + b[2] * np.sin(2 * math.pi * Y / Ly + b[3])
    u3 = np.asfortranarray(np.repeat(np.asarray(u, dtype=np.float64)[:, :, None], 4, axis=2))
    v3 = np.asfortranarray(np.repeat(np.asarray(v, dtype=np.float64)[:, :, None], 4, axis=2))
    if uniform_action:
        spec = rng.uniform(0.2, 1.0, (Nk, 1 if isotropic else Np))
        N0 = np.asfortranarray(np.broadcast_to(spec[None, None], (Nx, Ny, Nk, Np)).copy())
    else:
        N0 = np.asfortranarray(rng.uniform(0.1, 1.0, (Nx, Ny, Nk, Np)))
    return workloads.Workload("refraction_props", g, sg, InfiniteDepth(), N0, 0.05, 1,
                              velocities={"u": u3, "v": v3}, horizontal_advection=None)


def oracle_tendency(oracle_mod):
    return lambda w: oracle_mod.Oracle(w).tendency(w.N0)


def gpu_tendency(w):
    m = w.model("fp64")
    G = rp.interior(rp.compute_tendencies(m))
    m.close()
    return G


def mirrored(w, axis):
    """The workload reflected in x (axis 0) or y (axis 1), with directions and currents reflected."""
    Np = w.N0.shape[3]
    n = np.arange(Np)
    perm = (-n) % Np if axis == 1 else (Np // 2 - n) % Np
    N0 = np.asfortranarray(np.flip(w.N0, axis=axis)[:, :, :, perm])
    u, v = np.flip(w.velocities["u"], axis=axis), np.flip(w.velocities["v"], axis=axis)
    if axis == 0:
        u = -u
    else:
        v = -v
    return workloads.Workload(w.name, w.grid, w.spectral_grid, w.depth, N0, w.dt, w.nsteps,
                              velocities={"u": np.asfortranarray(u), "v": np.asfortranarray(v)},
                              horizontal_advection=None), perm


def check_uniform_current(tend):
    Nx, Ny = 12, 10
    w = refraction_workload(uniform_action=True, u=np.full((Nx, Ny), 0.25), v=np.full((Nx, Ny), -0.15))
    G = tend(w)
    assert np.max(np.abs(G)) == 0.0


def check_mirror(tend, axis):
    w = refraction_workload(seed=3 + axis)
    wm, perm = mirrored(w, axis)
    G, Gm = tend(w), tend(wm)
    back = np.flip(Gm, axis=axis)[:, :, :, np.argsort(perm)]
    scale = np.max(np.abs(G))
    assert scale > 1e-3
    assert np.max(np.abs(back - G)) <= 1e-12 * scale


def check_converging_current(tend):
    Nx, Ny = 16, 6
    L = 2.0 * Nx
    x = (np.arange(Nx) + 0.5) * L / Nx
    u = np.broadcast_to((0.3 * np.sin(2 * math.pi * x / L))[:, None], (Nx, Ny))
    w = refraction_workload(Nx=Nx, Ny=Ny, uniform_action=True, isotropic=True, u=u, v=np.zeros((Nx, Ny)))
    G = tend(w)
    kappa = np.asarray(w.spectral_grid.κ)
    moment = np.einsum("ijmn,m->ij", G, kappa)[:, 0]
    dudx = np.cos(2 * math.pi * x / L)           # sign of dU_x/dx
    assert np.all(moment[dudx < -0.1] > 0) and np.all(moment[dudx > 0.1] < 0)


def test_uniform_current_gives_zero_tendency(oracle_mod):
    check_uniform_current(oracle_tendency(oracle_mod))


@pytest.mark.parametrize("axis", [0, 1])
def test_mirror_equivariance(oracle_mod, axis):
    check_mirror(oracle_tendency(oracle_mod), axis)


def test_converging_current_moves_action_to_larger_kappa(oracle_mod):
    check_converging_current(oracle_tendency(oracle_mod))


@pytest.mark.gpu
def test_uniform_current_gives_zero_tendency_gpu():
    check_uniform_current(gpu_tendency)


@pytest.mark.gpu
@pytest.mark.parametrize("axis", [0, 1])
def test_mirror_equivariance_gpu(axis):
    check_mirror(gpu_tendency, axis)


@pytest.mark.gpu
def test_converging_current_moves_action_to_larger_kappa_gpu():
    check_converging_current(gpu_tendency)


def metal_smoke_workload():
    """The reference's FP32 refraction check (run_metal_smoke.jl:55-86,152-176): 6 x 5 x 1 grid on
    [0,6) x [0,5) x [-1,0], kappa = range(0.45, 1.20; length=4), 6 directions, u = 0.04 sin(2 pi x/Lx)
    + 0.01 cos(2 pi y/Ly), v = 0.03 cos(2 pi x/Lx) - 0.02 sin(2 pi y/Ly), action 0.6 + 0.04 sin(2 pi i/Nx)
    + 0.03 cos(2 pi j/Ny) + 0.02 m + 0.01 cos(2 pi n/Nphi) with 1-based indices."""
    Nx, Ny, Nk, Np = 6, 5, 4, 6
    g = RectilinearGrid(size=(Nx, Ny, 1), x=(0.0, 6.0), y=(0.0, 5.0), z=(-1.0, 0.0))
    sg = PolarWaveVectorGrid(κ=np.linspace(0.45, 1.20, Nk), φ=np.arange(Np) * 2 * math.pi / Np)
    X, Y = np.meshgrid(g.xnodes(), g.ynodes(), indexing="ij")
    u = 0.04 * np.sin(2 * math.pi * X / Nx) + 0.01 * np.cos(2 * math.pi * Y / Ny)
    v = 0.03 * np.cos(2 * math.pi * X / Nx) - 0.02 * np.sin(2 * math.pi * Y / Ny)
    i, j, m, n = np.meshgrid(np.arange(1, Nx + 1), np.arange(1, Ny + 1), np.arange(1, Nk + 1),
                             np.arange(1, Np + 1), indexing="ij")
    N0 = np.asfortranarray(0.6 + 0.04 * np.sin(2 * math.pi * i / Nx) + 0.03 * np.cos(2 * math.pi * j / Ny)
                           + 0.02 * m + 0.01 * np.cos(2 * math.pi * n / Np))
    return workloads.Workload("metal_smoke_refraction", g, sg, InfiniteDepth(), N0, 0.01, 1,
                              velocities={"u": np.asfortranarray(u[:, :, None]), "v": np.asfortranarray(v[:, :, None])})


@pytest.mark.gpu
@pytest.mark.parametrize("column_kernel", ["0", "1"])
def test_reference_fp32_refraction_agreement(oracle_mod, monkeypatch, column_kernel):
    """FP32 fused refraction tendency within 2e-4 and the action after one step within 2e-5 of the FP64
    oracle (the reference's tolerances; its step is forward Euler, this path's SSP-RK3)."""
    monkeypatch.setenv("RPL_FORCE_COLUMN_KERNEL", column_kernel)
    w = metal_smoke_workload()
    o = oracle_mod.Oracle(w)
    m = w.model("fp32")
    G = rp.interior(rp.compute_tendencies(m))
    assert np.max(np.abs(G - o.tendency(w.N0))) <= 2e-4
    rp.time_step(m, w.dt)
    No, _ = o.step(w.N0, w.dt, 1)
    assert np.max(np.abs(m.action.interior() - No)) <= 2e-5
    m.close()
