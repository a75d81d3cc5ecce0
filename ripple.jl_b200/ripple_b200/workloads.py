"""Synthetic workloads: the benchmark configurations built on the host as seeded FP64 inputs.

vortex_refraction  -- 64x64x16 periodic [0,80)^2, z in [-1,0], kappa = range(0.30, 0.50, 4),
                      16 directions, barotropic Gaussian-core vortex (U0 = 0.4, a = 10) at (40, 40),
                      N0 = exp(-((kappa-0.4)/0.05)^2 - sin^2(phi/2)/0.3^2), dt = 0.05, 400 steps
                      (the reference README's vortex-refraction example).
seamount_eddies    -- 1024^2 x 32 levels at 5 km, periodic; depth 4000 m minus three seeded Gaussian
                      seamounts (heights 3000-3900 m, widths 50-150 km, clamped >= 100 m); 32 log-spaced
                      kappa in 0.002-0.5 x 36 directions; current = 8 seeded Gaussian eddies (peak
                      0.5 m/s, radius 30-120 km, random sign) times exp(z/200); JONSWAP-like N0; 200 steps.
self_coupled_swell -- PseudomomentumVelocities: a swell packet Doppler-shifted by its own pseudomomentum
                      (Flat periodic grid, finite depth, automatic Q grid).
hurricane_swell    -- 768^2 at 10 km, depth 4000 m, 32 log kappa 0.003-0.3 x 36 directions, no current;
                      translating Holland hurricane (Vmax 50, Rmax 30 km, B 1.5) with wind input and
                      local-saturation whitecapping; N0 = 1e-6; 1000 steps.
Every builder takes the grid size so tests can run the same physics on a reduced grid.
"""
import math
from dataclasses import dataclass, field

import numpy as np

from .grids import InfiniteDepth, PolarWaveVectorGrid, RectilinearGrid
from .model import SpectralWaveModel, WENO
from .sources import (BulkWindDrag, HollandHurricaneWind, LinearStormTrack, LocalSaturationDissipation,
                      PrecomputedSources, PressureCorrelationInput)

G = 9.81


@dataclass
class Workload:
    name: str
    grid: RectilinearGrid
    spectral_grid: PolarWaveVectorGrid
    depth: object
    N0: np.ndarray                      # (Nx, Ny, Nk, Np), Fortran order
    dt: float
    nsteps: int
    velocities: dict = None             # {"u": (Nx,Ny,Nz), "v": ..., "q_grid": grid}
    sources: object = None
    horizontal_advection: object = field(default_factory=WENO)
    notes: dict = field(default_factory=dict)
    propagation_smoothing: object = None

    @property
    def units(self):
        return int(np.prod(self.N0.shape))

    def model(self, precision="fp64", **kw):
        m = SpectralWaveModel(self.grid, self.spectral_grid, depth=self.depth, velocities=self.velocities,
                              sources=self.sources, horizontal_advection=self.horizontal_advection,
                              propagation_smoothing=self.propagation_smoothing,
                              timestepper="RK3", precision=precision, **kw)
        m.action.set(self.N0)
        return m


def vortex_refraction(N=64, Nz=16, nsteps=400):
    L = 80.0
    grid = RectilinearGrid(size=(N, N, Nz), x=(0.0, L), y=(0.0, L), z=(-1.0, 0.0), halo=(3, 3, 3),
                           topology=("Periodic", "Periodic", "Bounded"))
    kappa = [(9.0 + 2.0 * k) / 30.0 for k in range(4)]           # range(0.30, 0.50; length=4)
    step = 2.0 * math.pi / 16.0
    phi = [k * step for k in range(16)]                           # range(0, 2pi; length=17)[1:16]
    sg = PolarWaveVectorGrid(κ=kappa, φ=phi)
    xc = yc = L / 2.0
    a, U0 = L / 8.0, 0.4
    x, y, z = grid.xnodes(), grid.ynodes(), grid.znodes()
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    r = np.hypot(X - xc, Y - yc)
    ut = np.where(r == 0, 0.0, U0 * (r / a) * np.exp(0.5 - 0.5 * (r / a) ** 2))
    rr = np.maximum(r, np.finfo(np.float64).eps)
    u = -ut * (Y - yc) / rr
    v = ut * (X - xc) / rr
    K, P = np.meshgrid(sg.κ, sg.φ, indexing="ij")
    spec = np.exp(-((K - 0.4) / 0.05) ** 2 - (np.sin(P / 2.0) ** 2) / 0.3 ** 2)
    N0 = np.asfortranarray(np.broadcast_to(spec[None, None], (N, N) + spec.shape))
    return Workload("vortex_refraction", grid, sg, InfiniteDepth(), N0, 0.05, nsteps,
                    velocities={"u": np.asfortranarray(u), "v": np.asfortranarray(v)},
                    horizontal_advection=None,
                    notes={"N0": "exp(-((kappa-0.4)/0.05)^2 - sin^2(phi/2)/0.3^2) at cell centres"})


def _periodic_delta(a, b, L):
    d = a - b
    return d - L * np.round(d / L)


def jonswap_spectrum(kappa, phi, kp=0.03, gamma=3.3, s=10, phi0=math.pi / 4):
    """Deep-water JONSWAP shape in kappa with cos^{2s}((phi-phi0)/2) spreading, peak value 1."""
    sig = np.sqrt(G * np.asarray(kappa))
    sp = math.sqrt(G * kp)
    width = np.where(sig <= sp, 0.07, 0.09)
    E = sig ** -5.0 * np.exp(-1.25 * (sp / sig) ** 4) * gamma ** np.exp(-((sig - sp) ** 2) / (2 * width ** 2 * sp ** 2))
    E = E / E.max()
    D = np.cos((np.asarray(phi) - phi0) / 2.0) ** (2 * s)
    return np.outer(E, D)


def seamount_eddies(N=1024, Nz=32, Nk=32, Np=36, nsteps=200, seed=2, L=1024 * 5000.0, cfl=0.4,
                    n0_dtype=np.float64, peak_current=0.5, n_eddies=8):
    """Reduced N keeps the 5120 km domain (coarser cells), so seamounts and eddies keep their extent.
    peak_current / n_eddies change the eddy field (the ensemble members use them)."""
    dx = L / N
    grid = RectilinearGrid(size=(N, N, Nz), x=(0.0, L), y=(0.0, L), z=(-4000.0, 0.0),
                           topology=("Periodic", "Periodic", "Bounded"))
    kappa = np.geomspace(0.002, 0.5, Nk)
    phi = np.arange(Np) * (2.0 * math.pi / Np)
    sg = PolarWaveVectorGrid(κ=kappa, φ=phi)
    rng = np.random.default_rng(seed)
    x, y, z = grid.xnodes(), grid.ynodes(), grid.znodes()
    X, Y = np.meshgrid(x, y, indexing="ij")
    depth = np.full((N, N), 4000.0)
    for _ in range(3):
        h = rng.uniform(3000.0, 3900.0)
        sgm = rng.uniform(50e3, 150e3)
        cx, cy = rng.uniform(0, L), rng.uniform(0, L)
        dX, dY = _periodic_delta(X, cx, L), _periodic_delta(Y, cy, L)
        depth -= h * np.exp(-(dX ** 2 + dY ** 2) / (2 * sgm ** 2))
    depth = np.maximum(depth, 100.0)
    us = np.zeros((N, N))
    vs = np.zeros((N, N))
    for _ in range(n_eddies):
        R = rng.uniform(30e3, 120e3)
        cx, cy = rng.uniform(0, L), rng.uniform(0, L)
        sgn = 1.0 if rng.uniform() < 0.5 else -1.0
        A = peak_current * R * math.exp(0.5) / math.sqrt(2.0)   # peak azimuthal speed at r = R/sqrt(2)
        dX, dY = _periodic_delta(X, cx, L), _periodic_delta(Y, cy, L)
        e = np.exp(-(dX ** 2 + dY ** 2) / R ** 2)
        us += sgn * A * (2 * dY / R ** 2) * e
        vs += -sgn * A * (2 * dX / R ** 2) * e
    decay = np.exp(z / 200.0)
    u = np.asfortranarray(us[:, :, None] * decay[None, None, :])
    v = np.asfortranarray(vs[:, :, None] * decay[None, None, :])
    spec = jonswap_spectrum(kappa, phi)
    env = 1.0 + 0.3 * np.sin(2 * math.pi * X / L) * np.cos(4 * math.pi * Y / L)
    N0 = np.empty((N, N, Nk, Np), dtype=n0_dtype, order="F")
    for n in range(Np):
        for m in range(Nk):
            N0[:, :, m, n] = env * spec[m, n]
    # time step from the CFL sum with deep-water c_g, surface currents and the first kappa spacing
    cg_max = 0.5 * math.sqrt(G / kappa[0]) + float(np.max(np.hypot(us, vs)))
    grads = max(np.max(np.abs(np.gradient(us, dx, axis=a))) for a in (0, 1))
    grads = max(grads, max(np.max(np.abs(np.gradient(vs, dx, axis=a))) for a in (0, 1)))
    dk = sg.κ_faces[1] - sg.κ_faces[0]
    dphi = 2 * math.pi / Np
    rate = 2 * cg_max / dx + kappa[-1] * 2 * grads / dk + 2 * grads / dphi
    dt = cfl / rate
    return Workload("seamount_eddies", grid, sg, depth, N0, dt, nsteps,
                    velocities={"u": u, "v": v},
                    notes={"seed": seed, "dt_rule": f"CFL sum {cfl}", "amplitude": "peak N = 1.3",
                           "N0": "JONSWAP kp=0.03 gamma=3.3, cos^20((phi-pi/4)/2), x-y envelope 1+0.3 sin cos"})


def hurricane_swell(N=768, Nk=32, Np=36, nsteps=1000, L=768 * 10000.0, cfl=0.4, translation=5.0, Nz=24,
                    vmax=50.0, start=(0.5, 0.2), n0_dtype=np.float64):
    """Reduced N keeps the 7680 km domain (coarser cells). vmax, start (fractions of the domain) and
    translation (m/s along +y) vary the storm (the learned source's training runs use other storms)."""
    dx = L / N
    grid = RectilinearGrid(size=(N, N, Nz), x=(0.0, L), y=(0.0, L), z=(-4000.0, 0.0),
                           topology=("Periodic", "Periodic", "Bounded"))
    kappa = np.geomspace(0.003, 0.3, Nk)
    phi = np.arange(Np) * (2.0 * math.pi / Np)
    sg = PolarWaveVectorGrid(κ=kappa, φ=phi)
    depth = 4000.0
    mu = kappa[0] * depth
    cg0 = 0.5 * (1 + 2 * mu / math.sinh(2 * mu)) * math.sqrt(G * math.tanh(mu) / kappa[0])
    dt = cfl / (2 * cg0 / dx)
    T = nsteps * dt
    start = (start[0] * L, start[1] * L)
    track = LinearStormTrack([0.0, T], [start, (start[0], start[1] + translation * T)])
    hurricane = HollandHurricaneWind(center=track, vmax=vmax, rmax=30e3, radius=500e3, shape_parameter=1.5,
                                     inflow_angle=math.radians(20.0))
    sources = PrecomputedSources(
        wind_input=PressureCorrelationInput(drag=BulkWindDrag("linear"), wind=hurricane, direction=0.0),
        dissipation=LocalSaturationDissipation(B_r=1.05e-2, σ_power=1.0))
    N0 = np.full((N, N, Nk, Np), 1e-6, dtype=n0_dtype, order="F")
    return Workload("hurricane_swell", grid, sg, depth, N0, dt, nsteps, sources=sources,
                    notes={"track": "start (Lx/2, 0.2 Ly), +y at 5 m/s", "radius": 500e3,
                           "inflow_angle_deg": 20.0, "dt_rule": f"CFL {cfl}"})


def self_coupled_swell(N=64, Nk=16, Np=24, nsteps=200, dx=2000.0, depth=50.0, depth_field=False, amplitude=4e4,
                       seed=7, cfl=0.4, peak_velocity=0.3, n0_dtype=np.float64):
    """PseudomomentumVelocities: a swell packet whose own pseudomomentum Doppler-shifts it. Flat periodic
    N x N grid at dx; 16 log kappa 0.01-0.3 x 24 directions; finite depth (50 m, or with depth_field a
    seeded 30-80 m bathymetry) so the Q grid is the automatic stretched one; N0 = amplitude x Gaussian
    packet (width L/6) x exp(-(ln(kappa/0.05)/0.3)^2) cos^20((phi-0.5)/2) plus a 1e-3 floor. The default
    amplitude gives a peak Doppler velocity near peak_velocity m/s, which sizes dt with the CFL sum."""
    from .model import PseudomomentumVelocities
    L = N * dx
    grid = RectilinearGrid(size=(N, N), x=(0.0, L), y=(0.0, L), topology=("Periodic", "Periodic", "Flat"))
    kappa = np.geomspace(0.01, 0.3, Nk)
    phi = np.arange(Np) * (2.0 * math.pi / Np)
    sg = PolarWaveVectorGrid(κ=kappa, φ=phi)
    X, Y = np.meshgrid(grid.xnodes(), grid.ynodes(), indexing="ij")
    if depth_field:
        rng = np.random.default_rng(seed)
        d = np.full((N, N), 80.0)
        for _ in range(3):
            cx, cy, w = rng.uniform(0, L), rng.uniform(0, L), rng.uniform(L / 10, L / 4)
            dX, dY = _periodic_delta(X, cx, L), _periodic_delta(Y, cy, L)
            d -= rng.uniform(10.0, 25.0) * np.exp(-(dX ** 2 + dY ** 2) / (2 * w ** 2))
        depth = np.maximum(d, 30.0)
    K, P = np.meshgrid(kappa, phi, indexing="ij")
    spec = np.exp(-((np.log(K / 0.05)) / 0.3) ** 2) * np.cos((P - 0.5) / 2) ** 20
    env = np.exp(-((X - L / 2) ** 2 + (Y - L / 2) ** 2) / (2 * (L / 6) ** 2))
    N0 = np.empty((N, N, Nk, Np), dtype=n0_dtype, order="F")
    for n in range(Np):
        for m in range(Nk):
            N0[:, :, m, n] = amplitude * spec[m, n] * env + 1e-3
    hmax = float(np.max(depth))
    cg_max = max(0.5 * math.sqrt(G * math.tanh(k * hmax) / k) for k in kappa) + peak_velocity
    grad = 2.0 * peak_velocity / (L / 6)
    dk = sg.κ_faces[1] - sg.κ_faces[0]
    rate = 2 * cg_max / dx + kappa[-1] * 2 * grad / dk + 2 * grad / (2 * math.pi / Np)
    return Workload("self_coupled_swell", grid, sg, depth, N0, cfl / rate, nsteps,
                    velocities=PseudomomentumVelocities(),
                    notes={"amplitude": amplitude, "depth": "field 30-80 m" if depth_field else depth,
                           "dt_rule": f"CFL sum {cfl}"})


ENSEMBLE_SIZES = (64, 128, 256, 384)
ENSEMBLE_SPECTRA = ((16, 24), (24, 36), (32, 36))


def ensemble_members(count=64, seed=4, nsteps=500, sizes=ENSEMBLE_SIZES, spectra=ENSEMBLE_SPECTRA, dx=5000.0,
                     Nz=16, n0_dtype=np.float32):
    """The batching-form ensemble: `count` independent members, each drawn with one seeded generator:
    grid N x N x Nz (N uniform from `sizes`, dx = 5 km, periodic), spectral grid uniform from `spectra`
    (32/24/16 log kappa 0.002-0.5 x 36/24 directions), depth 4000 m minus three seeded seamounts, and
    either one vortex or 8 eddies (even odds) with peak current U0 uniform in [0.1, 0.8] m/s decaying as
    exp(z/200 m); JONSWAP-like N0; dt from each member's own CFL. A generator yields the members one at a
    time so the caller can build a model and drop the host arrays before the next one."""
    rng = np.random.default_rng(seed)
    for i in range(count):
        N = int(sizes[int(rng.integers(len(sizes)))])
        Nk, Np = spectra[int(rng.integers(len(spectra)))]
        U0 = float(rng.uniform(0.1, 0.8))
        vortex = bool(rng.uniform() < 0.5)
        member_seed = int(rng.integers(2 ** 31))
        w = seamount_eddies(N=N, Nz=Nz, Nk=Nk, Np=Np, nsteps=nsteps, seed=member_seed, L=N * dx,
                            n0_dtype=n0_dtype, peak_current=U0, n_eddies=1 if vortex else 8)
        w.name = f"ensemble_member_{i}"
        w.notes.update({"member": i, "U0": U0, "currents": "vortex" if vortex else "8 eddies",
                        "member_seed": member_seed})
        yield w
