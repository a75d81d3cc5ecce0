"""PseudomomentumVelocities: the waves' own pseudomomentum as the Doppler-shifting current
(src/Coupling/pseudomomentum.jl, current_coupling.jl:41-143, lagrangian_velocities.jl:55-81,294-311).

CPU tests pin the oracle with the identities the reference's own tests use
(test/integration/model_api.jl:200-237): the pseudomomentum Doppler velocity equals the Q-transform
Doppler velocity of the pseudomomentum cell averages, and it is linear in the action. GPU tests compare
librpl.so with the oracle: the coupling fields at 1e-12 of their maximum, the FP64 RK3 state (the
coupling recomputed from every stage's action) at rel-L2 <= 1e-12, the FP32 state at <= 1e-5.
"""
import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import workloads

FP64_TOL = 1e-12
FP32_TOL = 1e-5
NAMES = ("Ux", "Uy", "dUxdkappa", "dUydkappa")


def rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def max_rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


# ---------------------------------------------------------------- oracle pins (CPU)

@pytest.mark.parametrize("depth_field", [False, True])
def test_oracle_velocity_is_doppler_of_cell_averages(oracle_mod, depth_field):
    w = workloads.self_coupled_swell(N=12, Nk=8, Np=12, depth_field=depth_field)
    o = oracle_mod.Oracle(w)
    U = o.pm_velocity(w.N0)
    px, py = o.pm_cells(w.N0, cell_average=True)
    D = o.doppler_of(px, py)
    for k in NAMES:
        assert max_rel(U[k], D[k]) <= 1e-12, k
    assert np.max(np.abs(U["Ux"])) > 0.05   # a current that matters


def test_oracle_velocity_is_linear_in_action(oracle_mod):
    w = workloads.self_coupled_swell(N=12, Nk=8, Np=12)
    o = oracle_mod.Oracle(w)
    U1, U2 = o.pm_velocity(w.N0), o.pm_velocity(2.0 * w.N0)
    for k in NAMES:
        assert max_rel(U2[k], 2.0 * U1[k]) <= 1e-14, k


def test_oracle_per_column_tables_equal_shared_tables(oracle_mod):
    w = workloads.self_coupled_swell(N=10, Nk=6, Np=8)
    o1 = oracle_mod.Oracle(w)
    w.depth = np.full((10, 10), float(w.depth))
    o2 = oracle_mod.Oracle(w)
    assert o1.pm["per_cell"] == 0 and o2.pm["per_cell"] == 1
    P = 100
    ov2 = o2.pm["overlap"].reshape(P, -1, order="F")
    assert np.array_equal(ov2, np.broadcast_to(o1.pm["overlap"], ov2.shape))
    U1, U2 = o1.pm_velocity(w.N0), o2.pm_velocity(w.N0)
    for k in NAMES:
        assert np.array_equal(U1[k], U2[k]), k


def test_oracle_tendency_uses_the_stage_action(oracle_mod):
    """The pseudomomentum coupling is recomputed inside the tendency: scaling the action changes the
    Doppler shift, so G(2N) != 2 G(N) (a prescribed current would give exact linearity)."""
    w = workloads.self_coupled_swell(N=12, Nk=8, Np=12)
    o = oracle_mod.Oracle(w)
    G1 = o.tendency(w.N0, with_sources=False)
    G2 = o.tendency(2.0 * w.N0, with_sources=False)
    assert rel_l2(G2, 2.0 * G1) > 1e-3


def test_pseudomomentum_arguments():
    with pytest.raises(rp.ArgumentError):
        rp.PseudomomentumVelocities(depth=2.0, Nz=6)
    g = rp.RectilinearGrid(size=(4, 3, 2), x=(0, 4), y=(0, 3), z=(-1, 0))
    with pytest.raises(rp.ArgumentError):
        rp.PseudomomentumVelocities(q_grid=g, vertical_grid=g)
    v = rp.PseudomomentumVelocities(Nz=7)
    assert v.q_grid is None and v.Nz == 7 and v.vertical_stretching == 2


# ---------------------------------------------------------------- CUDA path (GPU)

@pytest.mark.gpu
@pytest.mark.parametrize("depth_field", [False, True])
def test_coupling_fields_match_oracle(oracle_mod, depth_field):
    w = workloads.self_coupled_swell(N=20, Nk=12, Np=16, depth_field=depth_field)
    m = w.model("fp64")
    before = m.coupling_fields()
    assert all(np.all(before[k] == 0.0) for k in before)        # the caches start at zero
    m.update_coupling()
    got = m.coupling_fields()
    o = oracle_mod.Oracle(w)
    ref = o.pm_velocity(w.N0)
    for k in NAMES:
        assert max_rel(got[k], ref[k]) <= FP64_TOL, k
    g = [np.empty_like(ref["Ux"], order="F") for _ in range(4)]
    oracle_mod.lib().ora_current_gradients(20, 20, 12, oracle_mod.p(np.asfortranarray(ref["Ux"])),
                                           oracle_mod.p(np.asfortranarray(ref["Uy"])), 1.0 / 2000.0, 1.0 / 2000.0,
                                           *[oracle_mod.p(a) for a in g])
    for k, r in zip(("Ux_x", "Ux_y", "Uy_x", "Uy_y"), g):
        assert max_rel(got[k], r) <= FP64_TOL, k
    # linear in the action (model_api.jl:234-237)
    m.action.set(2.0 * w.N0)
    m.update_coupling()
    got2 = m.coupling_fields()
    assert max_rel(got2["Ux"], 2.0 * got["Ux"]) <= 1e-14


@pytest.mark.gpu
def test_tendency_matches_oracle(oracle_mod):
    w = workloads.self_coupled_swell(N=20, Nk=12, Np=16)
    m = w.model("fp64")
    G = rp.interior(rp.compute_tendencies(m))
    ref = oracle_mod.Oracle(w).tendency(w.N0, with_sources=False)
    assert max_rel(G, ref) <= 1e-12
    # compute_tendencies refreshed the coupling from the action (tendencies.jl:103-107)
    U = m.coupling_fields()["Ux"]
    assert max_rel(U, oracle_mod.Oracle(w).pm_velocity(w.N0)["Ux"]) <= FP64_TOL


@pytest.mark.gpu
@pytest.mark.parametrize("depth_field", [False, True])
def test_rk3_fp64_matches_oracle(oracle_mod, depth_field):
    w = workloads.self_coupled_swell(N=24, Nk=12, Np=16, depth_field=depth_field)
    nsteps = 6
    m = w.model("fp64")
    rp.time_step(m, w.dt, nsteps)
    No, t = oracle_mod.Oracle(w).step(w.N0, w.dt, nsteps)
    assert rel_l2(m.action.interior(), No) <= FP64_TOL
    assert rel_l2(No, w.N0) > 1e-2                               # the packet moved
    # after the step the coupling holds the third stage's velocity, as the reference's caches do
    assert m.clock.iteration == nsteps


@pytest.mark.gpu
@pytest.mark.parametrize("column_kernel", [False, True])
def test_rk3_fp32_matches_oracle(oracle_mod, monkeypatch, column_kernel):
    if column_kernel:
        monkeypatch.setenv("RPL_FORCE_COLUMN_KERNEL", "1")
    w = workloads.self_coupled_swell(N=24, Nk=16, Np=24)
    m = w.model("fp32")
    rp.time_step(m, w.dt, 6)
    No, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 6)
    assert rel_l2(m.action.interior(), No) <= FP32_TOL


@pytest.mark.gpu
def test_self_coupling_changes_the_solution(oracle_mod):
    """The same packet without velocities (intrinsic transport only) ends elsewhere."""
    w = workloads.self_coupled_swell(N=24, Nk=12, Np=16)
    m = w.model("fp64")
    rp.time_step(m, w.dt, 10)
    w.velocities = None
    m0 = w.model("fp64")
    rp.time_step(m0, w.dt, 10)
    assert rel_l2(m.action.interior(), m0.action.interior()) > 1e-3


@pytest.mark.gpu
def test_prescribed_currents_replace_pseudomomentum(oracle_mod):
    w = workloads.self_coupled_swell(N=20, Nk=12, Np=16)
    m = w.model("fp64")
    m.update_coupling()
    Nz = 8
    g3 = rp.RectilinearGrid(size=(20, 20, Nz), x=(0.0, 40000.0), y=(0.0, 40000.0), z=(-50.0, 0.0))
    u = np.full((20, 20, Nz), 0.2)
    m._set_velocities({"u": u, "v": np.zeros_like(u), "q_grid": g3})
    got = m.coupling_fields()
    assert np.allclose(got["Ux"], 0.2, rtol=0, atol=1e-12)      # barotropic current: U = u for every ring
    assert np.all(got["Uy"] == 0.0)
    m.update_coupling()                                          # static currents: nothing changes
    assert np.array_equal(m.coupling_fields()["Ux"], got["Ux"])
