"""SpatialAveraging (Tolman 2002 GSE alleviation) after every RK3 step
(src/Models/propagation_smoothing.jl:20-199, time_step.jl:168).

The reference has no test of its own for it (the translating-hurricane example uses it). The oracle is
pinned by properties of the averaging: zero widths leave the field unchanged, a constant stays constant,
the total of every periodic plane is conserved, and with a rectangle of half-width exactly half a cell
along x the average is the (1, 2, 1)/4 stencil. GPU tests compare librpl.so with the oracle: FP64 at
rel-L2 <= 1e-12 (1e-14 for a lone averaging), FP32 at <= 1e-5 (1e-6 for a lone averaging).
"""
import math

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import workloads
from ripple_b200.workloads import Workload


def rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def still_field(Nx=20, Ny=14, kappa=(0.05, 0.08, 0.12), Np=8, topology=("Periodic", "Periodic"), seed=3,
                alpha=(0.5, 0.5), dt=400.0, dx=2000.0):
    """No transport, no sources: the RK3 step leaves N unchanged, so a step is one averaging."""
    grid = rp.RectilinearGrid(size=(Nx, Ny), x=(0.0, Nx * dx), y=(0.0, Ny * dx),
                              topology=(topology[0], topology[1], "Flat"))
    phi = np.arange(Np) * (2 * math.pi / Np)
    sg = rp.PolarWaveVectorGrid(κ=list(kappa), φ=phi)
    rng = np.random.default_rng(seed)
    N0 = np.asfortranarray(rng.uniform(0.5, 1.5, (Nx, Ny, len(kappa), Np)))
    return Workload("still", grid, sg, rp.InfiniteDepth(), N0, dt, 1, horizontal_advection=None,
                    propagation_smoothing=rp.SpatialAveraging(αs=alpha[0], αn=alpha[1]))


# ---------------------------------------------------------------- oracle pins (CPU)

def test_oracle_zero_widths_are_identity(oracle_mod):
    w = still_field(alpha=(0.0, 0.0))
    out = oracle_mod.Oracle(w).spatial_averaging(w.N0, w.dt)
    assert np.array_equal(out, w.N0)


def test_oracle_constant_stays_constant(oracle_mod):
    w = still_field()
    w.N0 = np.asfortranarray(np.full(w.N0.shape, 2.5))
    out = oracle_mod.Oracle(w).spatial_averaging(w.N0, w.dt)
    assert np.max(np.abs(out - 2.5)) <= 4e-16 * 2.5


def test_oracle_conserves_periodic_planes(oracle_mod):
    w = still_field()
    out = oracle_mod.Oracle(w).spatial_averaging(w.N0, w.dt)
    s_in, s_out = w.N0.sum(axis=(0, 1)), out.sum(axis=(0, 1))
    assert np.max(np.abs(s_out - s_in) / s_in) <= 1e-13
    assert rel_l2(out, w.N0) > 1e-3                       # it did average


def test_oracle_half_cell_rectangle_is_121_stencil(oracle_mod):
    """Two rings have the same |dc_g| (one-sided differences at both ends); alpha_n = 0 and a dt giving
    L_s = dx / 2 put the corners at i -/+ 1/2 along the bin's direction."""
    kappa = (0.05, 0.09)
    cg = [0.5 * math.sqrt(9.81 / k) for k in kappa]
    dcg = abs(cg[0] - cg[1]) / 2
    dx = 2000.0
    w = still_field(kappa=kappa, Np=4, alpha=(1.0, 0.0), dt=0.5 * dx / dcg, dx=dx)
    out = oracle_mod.Oracle(w).spatial_averaging(w.N0, w.dt)
    f = w.N0
    along_x = (np.roll(f, 1, 0) + 2 * f + np.roll(f, -1, 0)) / 4     # directions 0 and pi
    along_y = (np.roll(f, 1, 1) + 2 * f + np.roll(f, -1, 1)) / 4     # directions pi/2 and 3pi/2
    for n, ref in ((0, along_x), (2, along_x), (1, along_y), (3, along_y)):
        assert np.max(np.abs(out[:, :, :, n] - ref[:, :, :, n])) <= 1e-14, n


def test_oracle_step_applies_the_averaging_after_rk3(oracle_mod):
    w = workloads.hurricane_swell(N=16, Nk=8, Np=12, nsteps=1)
    o_plain = oracle_mod.Oracle(w)
    w.propagation_smoothing = rp.SpatialAveraging()
    o_gse = oracle_mod.Oracle(w)
    N1, _ = o_plain.step(w.N0, w.dt, 1)
    N2, _ = o_gse.step(w.N0, w.dt, 1)
    assert np.array_equal(N2, o_gse.spatial_averaging(N1, w.dt))


def test_spatial_averaging_arguments():
    with pytest.raises(rp.ArgumentError):
        rp.SpatialAveraging(αs=-1.0)
    s = rp.SpatialAveraging()
    assert (s.αs, s.αn) == (0.5, 0.5)


# ---------------------------------------------------------------- CUDA path (GPU)

@pytest.mark.gpu
@pytest.mark.parametrize("topology", [("Periodic", "Periodic"), ("Bounded", "Periodic"), ("Bounded", "Bounded")])
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("fp32", 1e-6)])
def test_lone_averaging_matches_oracle(oracle_mod, topology, precision, tol):
    w = still_field(topology=topology, alpha=(0.9, 0.7))
    m = w.model(precision)
    rp.time_step(m, w.dt, 1)
    ref = oracle_mod.Oracle(w).spatial_averaging(w.N0, w.dt)
    assert rel_l2(m.action.interior(), ref) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-14), ("fp32", 1e-6)])
def test_far_corners_take_the_bilinear_path(oracle_mod, precision, tol):
    """A dt whose rectangle reaches beyond one cell: every bin takes the per-corner path."""
    w = still_field(alpha=(1.5, 1.5), dt=1500.0)   # corners 1-6 cells out, within one period
    m = w.model(precision)
    rp.time_step(m, w.dt, 1)
    ref = oracle_mod.Oracle(w).spatial_averaging(w.N0, w.dt)
    assert rel_l2(m.action.interior(), ref) <= tol


@pytest.mark.gpu
def test_hurricane_with_averaging_fp64(oracle_mod):
    w = workloads.hurricane_swell(N=24, Nk=8, Np=12, nsteps=3)
    w.N0 = np.asfortranarray(np.full(w.N0.shape, 1e-3))
    w.propagation_smoothing = rp.SpatialAveraging()
    m = w.model("fp64")
    rp.time_step(m, w.dt, 3)
    No, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 3)
    assert rel_l2(m.action.interior(), No) <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("column_kernel", [False, True])
def test_hurricane_with_averaging_fp32(oracle_mod, monkeypatch, column_kernel):
    if column_kernel:
        monkeypatch.setenv("RPL_FORCE_COLUMN_KERNEL", "1")
    w = workloads.hurricane_swell(N=24, Nk=16, Np=12, nsteps=3)
    w.N0 = np.asfortranarray(np.full(w.N0.shape, 1e-3))
    w.propagation_smoothing = rp.SpatialAveraging(αs=1.0, αn=1.0)
    m = w.model("fp32")
    rp.time_step(m, w.dt, 3)
    No, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 3)
    assert rel_l2(m.action.interior(), No) <= 1e-5


@pytest.mark.gpu
def test_refraction_with_averaging_fp64(oracle_mod):
    w = workloads.seamount_eddies(N=24, Nz=8, Nk=8, Np=12, nsteps=3)
    w.propagation_smoothing = rp.SpatialAveraging()
    m = w.model("fp64")
    rp.time_step(m, w.dt, 3)
    No, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 3)
    assert rel_l2(m.action.interior(), No) <= 1e-12
    m2 = workloads.seamount_eddies(N=24, Nz=8, Nk=8, Np=12, nsteps=3).model("fp64")
    rp.time_step(m2, w.dt, 3)
    assert rel_l2(m.action.interior(), m2.action.interior()) > 1e-6    # the averaging acted
