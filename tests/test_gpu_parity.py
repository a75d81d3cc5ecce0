"""Parity of the CUDA path (librpl.so through the C-ABI) with the CPU FP64 oracle.

Tolerances: the FP64 path must match the oracle to rel-L2 <= 1e-12 on the action after
the run; the FP32 precision form to rel-L2 <= 1e-5 (both stated by the benchmark
contract). Tendencies and set-up fields are compared at 1e-13 of their maximum.
"""
import ctypes
import math
import os
import sys

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import _lib, workloads

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

FP64_TOL = 1e-12
FP32_TOL = 1e-5


def rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def run_both(oracle_mod, w, nsteps, precision="fp64", **kw):
    m = w.model(precision, **kw)
    rp.time_step(m, w.dt, nsteps)
    Ng = m.action.interior()
    No, t = oracle_mod.Oracle(w).step(w.N0, w.dt, nsteps)
    assert m.clock.time == pytest.approx(t, rel=1e-15)
    assert m.clock.iteration == nsteps
    return m, Ng, No


def test_kat_tendency_matches_golden(oracle_mod):
    from make_golden import kat_workload
    ref = np.load(os.path.join(GOLDEN, "kat_tendency_8x7x4x6.npz"))
    k = kat_workload()
    m = k.model("fp64")
    G = rp.interior(rp.compute_tendencies(m))
    assert np.max(np.abs(G - ref["G"])) <= 1e-13 * np.max(np.abs(ref["G"]))


def test_coupling_fields_match_oracle(oracle_mod):
    from make_golden import kat_workload
    for w in (kat_workload(), workloads.seamount_eddies(N=24, Nz=32, Nk=8, Np=12, nsteps=1)):
        m = w.model("fp64")
        got = m.coupling_fields()
        o = oracle_mod.Oracle(w)
        ref = o.coupling(got["Ux"].shape)
        for name in ("Ux", "Uy", "dUxdkappa", "dUydkappa", "Ux_x", "Ux_y", "Uy_x", "Uy_y"):
            scale = max(np.max(np.abs(ref[name])), np.max(np.abs(ref["Ux"])))
            assert np.max(np.abs(got[name] - ref[name])) <= 1e-13 * scale, name


def test_vortex_refraction_reduced_fp64(oracle_mod):
    w = workloads.vortex_refraction(N=16, nsteps=40)
    m, Ng, No = run_both(oracle_mod, w, 40)
    assert rel_l2(Ng, No) <= FP64_TOL
    assert Ng.min() >= 0


@pytest.mark.slow
def test_vortex_refraction_full_run_matches_golden(oracle_mod):
    """The full vortex-refraction configuration (400 steps) against the oracle's golden output."""
    ref = np.load(os.path.join(GOLDEN, "c1_vortex_refraction.npz"))
    w = workloads.vortex_refraction()
    m = w.model("fp64")
    sim = rp.Simulation(m, Δt=w.dt, stop_iteration=w.nsteps)
    rp.run_(sim)
    N = m.action.interior().ravel(order="F")
    assert rel_l2(N[::97], ref["sample"]) <= FP64_TOL
    assert abs(N.sum() - float(ref["sum"])) <= FP64_TOL * abs(float(ref["sum"]))
    d = rp.diagnostics(m.action)
    assert rel_l2(d["m0"], ref["m0"]) <= FP64_TOL
    assert rel_l2(d["kappa_rms"], ref["kappa_rms"]) <= FP64_TOL
    assert np.max(np.abs(d["mean_direction"] - ref["mean_direction"])) <= 1e-10
    assert d["total_action"] == pytest.approx(float(ref["total_action"]), rel=FP64_TOL)
    # and against a fresh oracle run of the same configuration
    No, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, w.nsteps)
    assert rel_l2(N, No.ravel(order="F")) <= FP64_TOL


def test_vortex_refraction_fp32(oracle_mod):
    w = workloads.vortex_refraction(N=32, nsteps=40)
    m, Ng, No = run_both(oracle_mod, w, 40, precision="fp32")
    assert rel_l2(Ng, No) <= FP32_TOL


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_seamount_eddies_reduced(oracle_mod, precision, tol):
    w = workloads.seamount_eddies(N=40, Nz=32, Nk=32, Np=36, nsteps=4)
    m, Ng, No = run_both(oracle_mod, w, 4, precision=precision)
    assert rel_l2(Ng, No) <= tol


@pytest.mark.parametrize("precision,tol", [("fp64", FP64_TOL), ("fp32", FP32_TOL)])
def test_hurricane_sources_reduced(oracle_mod, precision, tol):
    w = workloads.hurricane_swell(N=48, Nk=32, Np=36, nsteps=4)
    m, Ng, No = run_both(oracle_mod, w, 4, precision=precision)
    assert rel_l2(Ng, No) <= tol
    assert np.max(np.abs(Ng - No)) > 0 or precision == "fp64"


@pytest.mark.parametrize("column_kernel", ["0", "1"])
def test_hurricane_fp32_sources_both_kernels(oracle_mod, monkeypatch, column_kernel):
    """FP32 source path (tile kernel: per-cell/per-kappa FP32 constants and the warp-per-column FP32
    stress cap; column kernel: FP64 per-unit sources) on a ragged action field with the cap active.
    Three steps: from this random start the wind input grows the action by up to ~e^1.3 per step, a
    stiff regime in which rounding differences grow (after 12 steps FP32 and FP64 runs differ by
    ~1e-3 rel-L2 with either source path)."""
    monkeypatch.setenv("RPL_FORCE_COLUMN_KERNEL", column_kernel)
    w = workloads.hurricane_swell(N=48, Nk=32, Np=36, nsteps=3)
    rng = np.random.default_rng(11)
    w.N0 = np.asfortranarray(rng.uniform(0.5e-6, 1.5e-6, w.N0.shape))
    f = oracle_mod.Oracle(w).stress_factor(w.N0)
    assert np.min(f) < 0.5 and np.mean(f < 1.0) > 0.05      # the cap binds in part of the domain
    m, Ng, No = run_both(oracle_mod, w, 3, precision="fp32")
    assert rel_l2(Ng, No) <= FP32_TOL
    assert np.max(np.abs(Ng - No)) > 0


@pytest.mark.slow
def test_hurricane_full_run_fp32_against_fp64():
    """The translating-hurricane configuration at full size (768^2 x 32 x 36, 1000 steps): the FP32
    precision form against the FP64 path (itself pinned to the oracle above) on the action, Hs, the
    mean period and the total action. Measured on B200: rel-L2(N) 4.1e-6, Hs 1.3e-6 (max 1.2e-5
    where Hs > 1% of its maximum), mean period 8.8e-8, total action 2.2e-6."""
    w = workloads.hurricane_swell()
    res = {}
    for prec in ("fp64", "fp32"):
        m = w.model(prec)
        rp.time_step(m, w.dt, w.nsteps)
        d = rp.diagnostics(m.action)
        res[prec] = (np.asarray(m.action.interior(), dtype=np.float64), d["Hs"], d["total_action"],
                     rp.mean_period(m.action))
        m.close()
    (N32, H32, T32, P32), (N64, H64, T64, P64) = res["fp32"], res["fp64"]
    assert rel_l2(N32, N64) <= FP32_TOL
    assert rel_l2(H32, H64) <= FP32_TOL
    mask = H64 > 0.01 * H64.max()
    assert np.max(np.abs(H32 - H64)[mask] / H64[mask]) <= 1e-4
    assert rel_l2(P32, P64) <= FP32_TOL
    assert abs(T32 - T64) <= FP32_TOL * T64
    assert H64.max() > 1.0                                   # the storm has raised a sea


def test_stress_factor_and_wind_match_oracle(oracle_mod):
    w = workloads.hurricane_swell(N=24, Nk=16, Np=24, nsteps=2)
    rng = np.random.default_rng(5)
    w.N0 = np.asfortranarray(rng.uniform(0.0, 2.0, w.N0.shape))
    m = w.model("fp64")
    G = rp.interior(rp.compute_tendencies(m))
    Go = oracle_mod.Oracle(w).tendency(w.N0)
    assert np.max(np.abs(G - Go)) <= 1e-12 * np.max(np.abs(Go))


@pytest.mark.parametrize("axis", ["x", "y"])
def test_weno_sinusoid_on_gpu(axis):
    from test_oracle_golden import sinusoid_workload
    w = sinusoid_workload(axis)
    m = w.model("fp64")
    G = rp.interior(rp.compute_tendencies(m))
    L = 64.0
    import oracle as O
    o = O.Oracle(w, explicit_spectral_faces=True)
    if axis == "x":
        o_u = o._cg[0][0]
        exp = -o_u * 0.1 * 2 * math.pi / L * np.cos(2 * math.pi * w.grid.xnodes() / L)[:, None]
    else:
        o_u = o._cg[1][0]
        exp = -o_u * 0.1 * 2 * math.pi / L * np.cos(2 * math.pi * w.grid.ynodes() / L)[None, :]
    assert np.max(np.abs(G[:, :, 0, 0] - exp)) < 1e-7
    tot0 = rp.total_action(m.action)
    rp.time_step(m, 0.1)
    assert abs(rp.total_action(m.action) - tot0) <= 1e-10
    assert m.action.interior().min() > 0


def test_rk3_linear_column_on_gpu():
    from test_oracle_golden import linear_damping_workload
    w = linear_damping_workload()
    m = w.model("fp64")
    rp.time_step(m, 0.1, nsteps=3)
    N = m.action.interior()
    for mm, k in enumerate((0.5, 1.0)):
        z = 0.4 * math.sqrt(9.81 * k) * 0.1
        amp = 1 - z + z * z / 2 - z ** 3 / 6
        assert N[0, 0, mm, 0] == pytest.approx(50.0 * amp ** 3, rel=1e-14)


def test_wind_input_signs_on_gpu():
    from test_oracle_golden import wind_column_workload
    w = wind_column_workload(15.0)
    G = rp.interior(rp.compute_tendencies(w.model("fp64")))
    assert G.max() > 0 and G.min() >= 0
    calm = wind_column_workload(0.0)
    assert np.all(rp.interior(rp.compute_tendencies(calm.model("fp64"))) == 0)


def test_diagnostics_match_oracle(oracle_mod):
    w = workloads.seamount_eddies(N=24, Nz=8, Nk=32, Np=36, nsteps=1)
    m = w.model("fp64")
    d = rp.diagnostics(m.action)
    do = oracle_mod.Oracle(w).diagnostics(w.N0)
    for k in ("m0", "Hs", "kappa_rms"):
        assert rel_l2(d[k], do[k]) <= 1e-14, k
    assert np.max(np.abs(d["mean_direction"] - do["mean_direction"])) <= 1e-13
    assert d["total_action"] == pytest.approx(do["total_action"], rel=1e-14)


@pytest.mark.parametrize("shape", [(3, 5, 1, 3), (37, 29, 5, 7), (33, 3, 2, 4)])
def test_edge_sizes_refraction(oracle_mod, shape):
    Nx, Ny, Nk, Np = shape
    rng = np.random.default_rng(sum(shape))
    g = rp.RectilinearGrid(size=(Nx, Ny, 4), x=(0.0, Nx * 2.0), y=(0.0, Ny * 2.0), z=(-3.0, 0.0))
    sg = rp.PolarWaveVectorGrid(κ=np.linspace(0.3, 0.9, Nk), φ=np.arange(Np) * 2 * math.pi / Np)
    u = np.asfortranarray(rng.uniform(-0.3, 0.3, (Nx, Ny, 4)))
    v = np.asfortranarray(rng.uniform(-0.3, 0.3, (Nx, Ny, 4)))
    N0 = np.asfortranarray(rng.uniform(0.0, 1.0, shape))
    w = workloads.Workload("edge", g, sg, 2.0, N0, 0.05, 3, velocities={"u": u, "v": v})
    m, Ng, No = run_both(oracle_mod, w, 3)
    assert rel_l2(Ng, No) <= FP64_TOL


@pytest.mark.parametrize("column_kernel", ["0", "1"])
@pytest.mark.parametrize("shape", [(3, 5, 4, 3), (37, 29, 8, 7), (20, 9, 24, 12), (17, 11, 32, 36)])
def test_fp32_kernels_edge_sizes(oracle_mod, monkeypatch, shape, column_kernel):
    """FP32 tile kernel (default) and column kernel on grids that leave partial tiles."""
    monkeypatch.setenv("RPL_FORCE_COLUMN_KERNEL", column_kernel)
    Nx, Ny, Nk, Np = shape
    rng = np.random.default_rng(3 * sum(shape))
    g = rp.RectilinearGrid(size=(Nx, Ny, 4), x=(0.0, Nx * 2.0), y=(0.0, Ny * 2.0), z=(-3.0, 0.0))
    sg = rp.PolarWaveVectorGrid(κ=np.linspace(0.3, 0.9, Nk), φ=np.arange(Np) * 2 * math.pi / Np)
    u = np.asfortranarray(rng.uniform(-0.3, 0.3, (Nx, Ny, 4)))
    v = np.asfortranarray(rng.uniform(-0.3, 0.3, (Nx, Ny, 4)))
    N0 = np.asfortranarray(rng.uniform(0.5, 1.0, shape))
    w = workloads.Workload("edge32", g, sg, 2.0, N0, 0.05, 3, velocities={"u": u, "v": v})
    m, Ng, No = run_both(oracle_mod, w, 3, precision="fp32")
    assert rel_l2(Ng, No) <= FP32_TOL


def pass_a_workload(shape, current, seed, depth_field=False):
    Nx, Ny, Nk, Np = shape
    rng = np.random.default_rng(seed)
    if depth_field:
        w = workloads.seamount_eddies(N=Nx, Nz=4, Nk=Nk, Np=Np, nsteps=3)
        return w
    g = rp.RectilinearGrid(size=(Nx, Ny, 4), x=(0.0, Nx * 2.0), y=(0.0, Ny * 2.0), z=(-3.0, 0.0))
    sg = rp.PolarWaveVectorGrid(κ=np.linspace(0.3, 0.9, Nk), φ=np.arange(Np) * 2 * math.pi / Np)
    u = np.asfortranarray(rng.uniform(-current, current, (Nx, Ny, 4)))
    v = np.asfortranarray(rng.uniform(-current, current, (Nx, Ny, 4)))
    N0 = np.asfortranarray(rng.uniform(0.5, 1.0, shape))
    return workloads.Workload("pass_a", g, sg, 2.0, N0, 0.05, 3, velocities={"u": u, "v": v})


@pytest.mark.gpu
@pytest.mark.parametrize("shape,current,depth_field", [
    ((3, 5, 4, 3), 0.3, False), ((37, 29, 8, 7), 0.3, False), ((20, 9, 24, 12), 0.3, False),
    ((17, 11, 32, 36), 0.3, False), ((33, 300, 16, 8), 0.05, False), ((70, 140, 32, 12), 3.0, False),
    ((40, 40, 32, 24), 0.0, False), ((48, 48, 32, 36), 0.0, True)])
def test_fp32_pass_a_forms_agree_bitwise(monkeypatch, shape, current, depth_field):
    """The y-walk pass A (one reconstruction per face, uniform-sign CTAs without selects) and the tile
    form give the same FP32 state bit for bit after three SSP-RK3 steps: partial x tiles, several
    128-row segments, weak, strong and no currents (uniform and mixed upwind CTAs), c_g per cell."""
    w = pass_a_workload(shape, current, 11 + sum(shape), depth_field)
    out = {}
    for form in ("", "tiles"):
        monkeypatch.setenv("RPL_PASS_A", form)
        m = w.model("fp32")
        rp.time_step(m, w.dt, 3)
        out[form] = m.action.interior()
        m.close()
    assert np.all(np.isfinite(out[""])) and np.max(np.abs(out[""])) > 0
    assert np.array_equal(out[""], out["tiles"])


@pytest.mark.gpu
@pytest.mark.parametrize("shape,current,depth_field,terms", [
    ((3, 5, 4, 3), 0.3, False, False), ((37, 29, 8, 7), 0.3, False, False), ((20, 9, 24, 12), 0.3, False, True),
    ((17, 11, 32, 36), 0.3, False, False), ((70, 40, 32, 12), 3.0, False, True), ((48, 48, 32, 36), 0.0, True, False)])
def test_fp32_pass_b_forms_agree_bitwise(monkeypatch, shape, current, depth_field, terms):
    """Pass B with four kappa bins per lane (the default for stages without bundle or learned sources)
    and with two (RPL_PASS_B=pairs) give the same FP32 state bit for bit after three SSP-RK3 steps:
    few and many kappa bins (the clamped stencil at both ends), mixed kappa and phi upwind signs, c_g per
    cell, and the SourceTermSet rates."""
    from ripple_b200.sources import ExponentialWindInput, SourceTermSet, WhitecappingDissipation
    w = pass_a_workload(shape, current, 5 + sum(shape), depth_field)
    if terms:
        w.sources = SourceTermSet(ExponentialWindInput(rate=2e-3, direction=0.6, spreading_power=2),
                                  WhitecappingDissipation(rate=1e-3, saturation_threshold=0.05))
    out = {}
    for form in ("", "pairs"):
        monkeypatch.setenv("RPL_PASS_B", form)
        m = w.model("fp32")
        rp.time_step(m, w.dt, 3)
        out[form] = m.action.interior()
        m.close()
    assert np.all(np.isfinite(out[""])) and np.max(np.abs(out[""])) > 0
    assert np.array_equal(out[""], out["pairs"])


def intrinsic_workloads():
    from test_source_terms import random_terms_workload
    plain = workloads.seamount_eddies(N=40, Nz=8, Nk=16, Np=24, nsteps=3)
    plain.velocities = None                           # intrinsic transport, c_g per cell (depth field)
    return {"depth_field": plain,
            "hurricane": workloads.hurricane_swell(N=48, Nk=32, Np=36, nsteps=3),     # bundle, stress cap
            "hurricane_small_k": workloads.hurricane_swell(N=33, Nk=8, Np=12, nsteps=3),
            "terms": random_terms_workload(N=37, Nk=16, Np=24)}                       # SourceTermSet rates


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["depth_field", "hurricane", "hurricane_small_k", "terms"])
def test_fp32_intrinsic_forms_agree_bitwise(monkeypatch, name):
    """The y-walk stage of intrinsic transport (one reconstruction per x and y face, the SourceTermSet rates
    and the stage update in the same kernel) and the fused tile kernel (RPL_PASS_A=tiles) give the same
    FP32 state bit for bit after three SSP-RK3 steps; the bundle sources (hurricane) take the tile kernel
    in both."""
    w = intrinsic_workloads()[name]
    out = {}
    for form in ("", "tiles"):
        monkeypatch.setenv("RPL_PASS_A", form)
        m = w.model("fp32")
        rp.time_step(m, w.dt, 3)
        out[form] = m.action.interior()
        m.close()
    assert np.all(np.isfinite(out[""])) and np.max(np.abs(out[""])) > 0
    assert np.array_equal(out[""], out["tiles"])


@pytest.mark.parametrize("column_kernel", ["0", "1"])
def test_fp32_kernels_intrinsic_and_depth_field(oracle_mod, monkeypatch, column_kernel):
    monkeypatch.setenv("RPL_FORCE_COLUMN_KERNEL", column_kernel)
    w = workloads.seamount_eddies(N=40, Nz=8, Nk=16, Np=24, nsteps=3)
    w.velocities = None                     # intrinsic transport with a depth field (c_g per cell)
    m, Ng, No = run_both(oracle_mod, w, 3, precision="fp32")
    assert rel_l2(Ng, No) <= FP32_TOL


def test_set_get_roundtrip_and_clock():
    w = workloads.seamount_eddies(N=16, Nz=4, Nk=4, Np=6, nsteps=1)
    for precision in ("fp64", "fp32"):
        m = w.model(precision)
        got = m.action.interior()
        if precision == "fp64":
            assert np.array_equal(got, w.N0)
        else:
            assert np.array_equal(got, w.N0.astype(np.float32).astype(np.float64))
        m.clock.time = 12.5
        rp.time_step(m, 0.5)
        assert m.clock.time == 13.0 and m.clock.iteration == 1


def test_error_paths():
    w = workloads.seamount_eddies(N=16, Nz=4, Nk=4, Np=6, nsteps=1)
    m = w.model("fp64")
    with pytest.raises(rp.ArgumentError):
        rp.time_step(m, 0.0)
    with pytest.raises(rp.ArgumentError):
        rp.time_step(m, -1.0)
    bad = w.N0.copy(order="F")
    bad[3, 2, 1, 0] = np.nan
    with pytest.raises(rp.RplError) as e:
        m.action.set(bad)
    assert e.value.code == _lib.RPL_ERR_NONFINITE
    # a huge step drives the action to overflow; the kernels' error word reports it
    m.action.set(w.N0 * 1e300)
    with pytest.raises(rp.RplError) as e:
        rp.time_step(m, 1e12)
    assert e.value.code == _lib.RPL_ERR_DEVICE
    # the handle stays usable afterwards
    m.action.set(w.N0)
    rp.time_step(m, w.dt)
    assert np.all(np.isfinite(m.action.interior()))
    # refraction transport without currents is refused
    lib = _lib.load()
    d = _lib.RplDesc()
    keep = dict(x=np.arange(4.0) + 0.5, k=np.array([0.5]), kf=np.array([0.4, 0.6]), p=np.array([0.0, 2.0, 4.0]),
                pf=np.array([-1.0, 1.0, 3.0, 5.0]))
    d.abi_version, d.precision, d.transport = _lib.RPL_ABI_VERSION, _lib.RPL_FP64, _lib.RPL_TRANSPORT_REFRACTION
    d.Nx = d.Ny = 4
    d.Nk, d.Np = 1, 3
    d.dx = d.dy = 1.0
    d.xnodes = d.ynodes = _lib.dptr(keep["x"])
    d.periodic_x = d.periodic_y = 1
    d.kappa, d.kappa_faces, d.phi, d.phi_faces = (_lib.dptr(keep[k]) for k in ("k", "kf", "p", "pf"))
    d.gravity = 9.81
    h = ctypes.c_void_p()
    assert lib.rpl_create(ctypes.byref(d), ctypes.byref(h)) == _lib.RPL_OK
    assert lib.rpl_step(h, 0.1, 1) == _lib.RPL_ERR_STATE
    assert lib.rpl_stage_async(h, 0.1, 4) == _lib.RPL_ERR_STATE
    assert lib.rpl_destroy(h) == _lib.RPL_OK


def test_diagnostics_stretched_grid(oracle_mod):
    """Total action on a stretched grid: every column weighted by its own cell area, as the oracle."""
    from test_oracle_golden import stretched_workload
    w = stretched_workload()
    for precision in ("fp64", "fp32"):
        m = w.model(precision)
        d = rp.diagnostics(m.action)
        do = oracle_mod.Oracle(w).diagnostics(m.action.interior().astype(np.float64))
        assert d["total_action"] == pytest.approx(do["total_action"], rel=1e-14), precision
        assert rel_l2(d["m0"], do["m0"]) <= 1e-14
        m.close()


def test_seamount_eddies_128_fp64_against_oracle(oracle_mod):
    """The seamount-eddies physics (32 log kappa x 36 directions, 32 levels, seamount depth field, eight
    eddies) on a 128^2 grid of the same 5120 km domain: the FP64 GPU path against the CPU oracle after
    20 RK3 steps, rel-L2 <= 1e-12. This pins the FP64 path that the full-size FP32 comparison below
    takes as its reference."""
    w = workloads.seamount_eddies(N=128, Nz=32, Nk=32, Np=36, nsteps=20)
    m, Ng, No = run_both(oracle_mod, w, 20)
    assert rel_l2(Ng, No) <= FP64_TOL
    d, do = rp.diagnostics(m.action), oracle_mod.Oracle(w).diagnostics(No)
    assert rel_l2(d["Hs"], do["Hs"]) <= FP64_TOL
    assert d["total_action"] == pytest.approx(do["total_action"], rel=FP64_TOL)
    m.close()


def device_state(m, precision):
    """The model's action as a CUDA tensor in the caller layout (x fastest)."""
    import torch
    Nx, Ny = m.grid.Nx, m.grid.Ny
    Nk, Np = m.spectral_grid.coordinate_size()
    t = torch.empty(Nx * Ny * Nk * Np, dtype=torch.float64 if precision == "fp64" else torch.float32,
                    device=f"cuda:{m.device}")
    _lib.check(m._lib.rpl_get_action_device(m.handle, ctypes.c_void_p(t.data_ptr()),
                                            _lib.RPL_F64 if precision == "fp64" else _lib.RPL_F32, 0))
    return t


def rel_l2_device(a, b, chunk=1 << 27):
    """rel-L2 of two equal-length CUDA tensors in FP64, chunked (no full-size temporaries)."""
    import torch
    num = den = 0.0
    for s in range(0, a.numel(), chunk):
        x, y = a[s:s + chunk].double(), b[s:s + chunk].double()
        num += float(torch.sum((x - y) ** 2))
        den += float(torch.sum(y * y))
    return math.sqrt(num / den)


@pytest.mark.slow
def test_seamount_full_run_fp32_against_fp64():
    """The seamount-eddies configuration at full size (1024^2 x 32 levels x 32 kappa x 36 directions,
    200 RK3 steps): the FP32 precision form against the FP64 path (pinned to the oracle above) from the
    same initial action, rel-L2 <= 1e-5 on the action and on Hs, the total action within 1e-5, and the
    same action-budget drift (change of the total action over the run) to 1e-5 of the total."""
    import torch
    w = workloads.seamount_eddies(n0_dtype=np.float32)
    res = {}
    for prec in ("fp64", "fp32"):
        m = w.model(prec)
        t0 = rp.total_action(m.action)
        rp.time_step(m, w.dt, w.nsteps)
        d = rp.diagnostics(m.action)
        res[prec] = (device_state(m, prec), d["Hs"], d["total_action"], t0)
        m.close()
    (N32, H32, T32, S32), (N64, H64, T64, S64) = res["fp32"], res["fp64"]
    assert rel_l2_device(N32, N64) <= FP32_TOL
    assert rel_l2(H32, H64) <= FP32_TOL
    assert abs(T32 - T64) <= FP32_TOL * T64
    assert S32 == pytest.approx(S64, rel=1e-7)                       # same initial action
    assert abs((T32 - S32) - (T64 - S64)) <= FP32_TOL * T64           # action-budget drift
    assert float(torch.min(N32)) >= 0.0
