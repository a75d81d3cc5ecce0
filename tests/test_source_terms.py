"""SourceTermSet terms whose tendency is linear in the action (ExponentialWindInput, WaveAgeWindInput,
WhitecappingDissipation, MeanSpectrumWhitecapping).

The oracle is pinned by the reference's own tests, restated: the whitecapping radial-power ratio and
the weak-threshold zero (test/sources/source_terms.jl:236-262), and the fetch-limited source balance
(src/Validation/Validation.jl:248-287, equilibrium m0* = 0.5 (1 + 1.2 / 4.8)). Further pins come from
closed forms: the directional weight of a power-2 spreading integrates to pi/2 over a full ring, and a
wave-age term vanishes below its threshold. The library (FP64 <= 1e-12, FP32 <= 1e-5) is checked
against the oracle on a randomised model with every term (gpu tests).
"""
import math

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200.grids import InfiniteDepth, PolarWaveVectorGrid, RectilinearGrid
from ripple_b200.sources import (ExponentialWindInput, MeanSpectrumWhitecapping, SourceTermSet, WaveAgeWindInput,
                                 WhitecappingDissipation)
from ripple_b200.workloads import Workload

UNIT_GRID = dict(size=(1, 1, 1), x=(0, 1), y=(0, 1), z=(0, 1))


def column(kappa, phi, sources, N0):
    g = RectilinearGrid(**UNIT_GRID)
    sg = PolarWaveVectorGrid(κ=kappa, φ=phi)
    N0 = np.asfortranarray(np.broadcast_to(np.asarray(N0, dtype=np.float64), (1, 1, len(kappa), len(phi))).copy())
    return Workload("column", g, sg, InfiniteDepth(), N0, 0.02, 1, sources=sources, horizontal_advection=None)


def test_whitecapping_radial_power_ratio(oracle_mod):
    """test/sources/source_terms.jl:236-256: N = 1 on kappa = [0.5, 1, 2], one direction; damping grows
    with kappa and the tendency ratio of bins 3 and 2 is the ratio of their kappa^2 cell averages."""
    wc = WhitecappingDissipation(rate=0.2, saturation_threshold=0.1, saturation_power=1.0, wavenumber_power=2.0,
                                 reference_wavenumber=1.0)
    w = column([0.5, 1.0, 2.0], [0.0], wc, 1.0)
    G = oracle_mod.Oracle(w).tendency(w.N0).ravel()
    kf = w.spectral_grid.κ_faces
    factor = [(kf[m + 1] ** 2 + kf[m] ** 2) / 2 for m in range(3)]   # annular average of kappa^2
    assert G[0] < 0 and G[1] < G[0] and G[2] < G[1]
    assert G[2] / G[1] == pytest.approx(factor[2] / factor[1], rel=1e-14)


def test_whitecapping_weak_threshold_is_zero(oracle_mod):
    """test/sources/source_terms.jl:258-261: below the saturation threshold nothing is dissipated."""
    w = column([0.5, 1.0, 2.0], [0.0], WhitecappingDissipation(rate=0.2, saturation_threshold=100.0), 1.0)
    assert np.max(np.abs(oracle_mod.Oracle(w).tendency(w.N0))) < 1e-14


def balance_sources():
    """Validation.jl:248-267: exponential growth 1.2 against whitecapping 4.8 (threshold 0.5)."""
    sg = PolarWaveVectorGrid(κ=[1.0], φ=[0.0])
    weight = float(sg.weights[0, 0])
    kf, pf = sg.κ_faces, sg.φ_faces
    # cell average of max(cos, 0)^2 over the one direction cell [-pi, pi]: (pi/2) / (2 pi)
    directional_weight = (math.pi / 2) / (pf[1] - pf[0])
    src = SourceTermSet(ExponentialWindInput(rate=1.2 / directional_weight, direction=0.0, spreading_power=2),
                        WhitecappingDissipation(rate=4.8, saturation_threshold=0.5, saturation_power=1.0,
                                                wavenumber_power=0.0))
    return src, weight


def test_fetch_limited_equilibrium_tendency(oracle_mod):
    """The tendency vanishes at m0* = 0.5 (1 + 1.2 / 4.8) to 1e-12 (Validation.jl:269-286)."""
    src, weight = balance_sources()
    m0_eq = 0.5 * (1 + 1.2 / 4.8)
    w = column([1.0], [0.0], src, m0_eq / weight)
    assert abs(float(oracle_mod.Oracle(w).tendency(w.N0).ravel()[0])) <= 1e-12


def test_fetch_limited_growth_is_monotone_to_equilibrium(oracle_mod):
    """From m0 = 0.5 / 20 the column grows monotonically to m0* (the reference's 240 steps of 0.02 with its
    semi-implicit stepper reach it within 1e-2; SSP-RK3 here)."""
    src, weight = balance_sources()
    w = column([1.0], [0.0], src, 0.5 / (20 * weight))
    o = oracle_mod.Oracle(w)
    N = w.N0
    moments = [float(N.ravel()[0]) * weight]
    for _ in range(240):
        N, _ = o.step(N, 0.02, 1)
        moments.append(float(N.ravel()[0]) * weight)
    assert abs(moments[-1] - 0.5 * (1 + 1.2 / 4.8)) <= 1e-2
    assert min(np.diff(moments)) >= -1e-12


def test_exponential_wind_direction_weights(oracle_mod):
    """On a full ring of 8 directions the power-2 cell averages sum to (pi/2) / (2 pi / 8) (the closed-form
    integral of max(cos, 0)^2), and the growth is rate * N * weight."""
    phi = np.arange(8) * 2 * math.pi / 8
    w = column([0.5], phi, ExponentialWindInput(rate=0.3, direction=0.4, spreading_power=2), 1.0)
    G = oracle_mod.Oracle(w).tendency(w.N0).ravel()
    assert float(np.sum(G)) / 0.3 == pytest.approx((math.pi / 2) / (2 * math.pi / 8), rel=1e-13)
    assert np.all(G >= 0) and G[0] > G[4]


def test_wave_age_threshold(oracle_mod):
    """Below the inverse wave-age threshold (U cos / c < 0.83) no energy is added; above it the rate is
    rate * excess^power * alignment^spreading_power (Sources.jl:522-554)."""
    kappa = [0.01, 0.5]                      # c = 31.3 and 4.4 m/s
    phi = [0.0, math.pi]
    w = column(kappa, phi, WaveAgeWindInput(rate=0.5, speed=10.0, direction=0.0, power=1.0, spreading_power=1.0),
               2.0)
    G = oracle_mod.Oracle(w).tendency(w.N0)[0, 0]
    c = math.sqrt(9.81 / 0.5)
    assert G[0, 0] == 0.0 and G[0, 1] == 0.0 and G[1, 1] == 0.0
    assert G[1, 0] == pytest.approx(0.5 * (10.0 / c - 0.83) * 2.0, rel=1e-13)


def test_mean_spectrum_whitecapping_closed_form(oracle_mod):
    """One direction, two bins: the damping rate -C_ds (m0 kbar^2)^2 sigmabar (d1 k/kbar + d2 (k/kbar)^2)
    with kbar, sigmabar the p-th means (mean_spectrum.jl:43-111), evaluated by hand."""
    kappa, N = [0.2, 0.6], [3.0, 1.0]
    ms = MeanSpectrumWhitecapping()
    w = column(kappa, [0.0], ms, 0.0)
    w.N0[0, 0, :, 0] = N
    G = oracle_mod.Oracle(w).tendency(w.N0)[0, 0, :, 0]
    wts = w.spectral_grid.weights[:, 0]
    m0 = float(np.sum(np.array(N) * wts))
    p = 0.5
    kbar = (np.sum(np.array(N) * wts * np.array(kappa) ** p) / m0) ** (1 / p)
    sbar = (np.sum(np.array(N) * wts * np.sqrt(9.81 * np.array(kappa)) ** p) / m0) ** (1 / p)
    for m in range(2):
        r = kappa[m] / kbar
        rate = 2.1 * (m0 * kbar ** 2) ** 2 * sbar * (0.4 * r + 0.6 * r * r)
        assert G[m] == pytest.approx(-rate * N[m], rel=1e-12)


def test_source_term_validation():
    with pytest.raises(rp.ArgumentError):
        ExponentialWindInput(rate=1.0, spreading_power=1.5)
    with pytest.raises(rp.ArgumentError):
        WhitecappingDissipation(saturation_threshold=0.0)
    with pytest.raises(rp.ArgumentError):
        WaveAgeWindInput(gravity=0.0)
    with pytest.raises(rp.ArgumentError):
        SourceTermSet(rp.LocalSaturationDissipation())


def random_terms_workload(N=20, Nk=16, Np=24, seed=9):
    """A periodic model with intrinsic transport and every linear term at once, one rate as a field."""
    rng = np.random.default_rng(seed)
    L = N * 1000.0
    g = RectilinearGrid(size=(N, N, 4), x=(0.0, L), y=(0.0, L), z=(-100.0, 0.0))
    sg = PolarWaveVectorGrid(κ=np.geomspace(0.01, 0.5, Nk), φ=np.arange(Np) * 2 * math.pi / Np)
    rate_field = rng.uniform(1e-5, 3e-5, (N, N))
    src = SourceTermSet(
        ExponentialWindInput(rate=rate_field, direction=0.7, spreading_power=2),
        WaveAgeWindInput(rate=2e-5, speed=15.0, direction=0.5, power=1.0, spreading_power=2.0),
        WhitecappingDissipation(rate=3e-5, saturation_threshold=0.05, saturation_power=2.0, wavenumber_power=1.0,
                                reference_wavenumber=0.1),
        MeanSpectrumWhitecapping(C_ds=-2.1))
    N0 = np.asfortranarray(rng.uniform(0.5, 1.5, (N, N, Nk, Np)))
    return Workload("linear_terms", g, sg, 50.0, N0, 20.0, 4, sources=src)


def test_random_terms_oracle_runs(oracle_mod):
    w = random_terms_workload(N=6, Nk=8, Np=12)
    G = oracle_mod.Oracle(w).tendency(w.N0)
    Gt = oracle_mod.Oracle(w).tendency(w.N0, with_sources=False)
    assert np.max(np.abs(G - Gt)) > 0 and np.all(np.isfinite(G))


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_linear_terms_match_oracle(oracle_mod, precision, tol):
    w = random_terms_workload()
    m = w.model(precision)
    G = rp.interior(rp.compute_tendencies(m))
    Go = oracle_mod.Oracle(w).tendency(w.N0)
    assert np.linalg.norm(G - Go) <= tol * np.linalg.norm(Go)
    rp.time_step(m, w.dt, w.nsteps)
    No, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, w.nsteps)
    assert np.linalg.norm(m.action.interior() - No) <= tol * np.linalg.norm(No)
    m.close()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32", 1e-5)])
def test_five_terms_match_oracle(oracle_mod, precision, tol):
    """More than four terms take the one-kernel form of the rates (one warp per column for both passes)."""
    w = random_terms_workload(N=16, Nk=16, Np=24, seed=4)
    w.sources = SourceTermSet(*w.sources.terms, ExponentialWindInput(rate=1e-5, direction=-1.2, spreading_power=4))
    m = w.model(precision)
    G = rp.interior(rp.compute_tendencies(m))
    Go = oracle_mod.Oracle(w).tendency(w.N0)
    assert np.linalg.norm(G - Go) <= tol * np.linalg.norm(Go)
    m.close()


@pytest.mark.gpu
def test_reference_source_tests_on_gpu(oracle_mod):
    """The whitecapping ratio and the equilibrium tendency through the library (FP64)."""
    wc = WhitecappingDissipation(rate=0.2, saturation_threshold=0.1, saturation_power=1.0, wavenumber_power=2.0,
                                 reference_wavenumber=1.0)
    w = column([0.5, 1.0, 2.0], [0.0], wc, 1.0)
    m = w.model("fp64")
    G = rp.interior(rp.compute_tendencies(m)).ravel()
    assert np.max(np.abs(G - oracle_mod.Oracle(w).tendency(w.N0).ravel())) <= 1e-13 * np.max(np.abs(G))
    m.close()
    src, weight = balance_sources()
    w = column([1.0], [0.0], src, 0.5 * (1 + 1.2 / 4.8) / weight)
    m = w.model("fp64")
    assert abs(float(rp.interior(rp.compute_tendencies(m)).ravel()[0])) <= 1e-12
    m.close()
