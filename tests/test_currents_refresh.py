"""Time-varying prescribed currents: the Q-transform Doppler velocity, its gradients and the stage
coefficients refreshed between steps without allocating (rpl_update_currents / _device), the
B200 form of update_coupling!(::CWCMPrescribedCurrentCoupling) (current_coupling.jl:127-138).

Parity with the oracle: coupling fields at 1e-13 of their maximum, the FP64 state at rel-L2 <= 1e-12
after steps whose currents change every step.
"""
import math

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import workloads

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
NAMES = ("Ux", "Uy", "dUxdkappa", "dUydkappa", "Ux_x", "Ux_y", "Uy_x", "Uy_y")


def rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def small_cases():
    return [workloads.seamount_eddies(N=24, Nz=16, Nk=8, Np=12, nsteps=4),      # depth field: per-column Q weights
            workloads.vortex_refraction(N=24, Nz=8, nsteps=4)]                   # InfiniteDepth: Q weight tables


def other_currents(w, k):
    """A second current field: the workload's own, rotated by k radians and scaled by 1 + 0.3 sin k."""
    u, v = np.asarray(w.velocities["u"]), np.asarray(w.velocities["v"])
    c, s, a = math.cos(k), math.sin(k), 1.0 + 0.3 * math.sin(k)
    return np.asfortranarray(a * (c * u - s * v)), np.asfortranarray(a * (s * u + c * v))


@pytest.mark.parametrize("case", [0, 1])
def test_update_currents_matches_oracle(oracle_mod, case):
    w = small_cases()[case]
    m = w.model("fp64")
    u2, v2 = other_currents(w, 1.1)
    m.update_currents(u2, v2)
    got = m.coupling_fields()
    o = oracle_mod.Oracle(w)
    o.update_currents(u2, v2)
    ref = o.coupling(got["Ux"].shape)
    for k in NAMES:
        # a barotropic current has dU/dkappa = 0 up to rounding: scale by the velocity too
        scale = max(np.max(np.abs(ref[k])), np.max(np.abs(ref["Ux"])))
        assert np.max(np.abs(got[k] - ref[k])) <= 1e-13 * scale, k
    rp.time_step(m, w.dt, 2)
    No, _ = o.step(w.N0, w.dt, 2)
    assert rel_l2(m.action.interior(), No) <= FP64_TOL


@pytest.mark.parametrize("case", [0, 1])
def test_currents_changing_every_step(oracle_mod, case):
    w = small_cases()[case]
    m = w.model("fp64")
    o = oracle_mod.Oracle(w)
    N, t = w.N0, 0.0
    for k in range(4):
        u, v = other_currents(w, 0.4 * k)
        m.update_currents(u, v)
        rp.time_step(m, w.dt, 1)
        o.update_currents(u, v)
        N, t = o.step(N, w.dt, 1, t)
    assert rel_l2(m.action.interior(), N) <= FP64_TOL
    assert rel_l2(N, oracle_mod.Oracle(w).step(w.N0, w.dt, 4)[0]) > 1e-6   # the currents mattered


def test_device_currents_equal_host_currents():
    import torch
    w = small_cases()[0]
    m1, m2 = w.model("fp64"), w.model("fp64")
    u, v = other_currents(w, 0.7)
    m1.update_currents(u, v)
    Nx, Ny, Nz = u.shape

    def dev(a):
        return torch.from_numpy(np.ravel(a, order="F").copy()).cuda().view(Nz, Ny, Nx).permute(2, 1, 0)

    du, dv = dev(u), dev(v)
    assert du.stride() == (1, Nx, Nx * Ny)
    torch.cuda.synchronize()
    m2.update_currents(du, dv)
    a, b = m1.coupling_fields(), m2.coupling_fields()
    for k in NAMES:
        assert np.array_equal(a[k], b[k]), k
    rp.time_step(m1, w.dt, 2)
    rp.time_step(m2, w.dt, 2)
    assert np.array_equal(m1.action.interior(), m2.action.interior())
    with pytest.raises(rp.ArgumentError):
        m2.update_currents(du.contiguous(), dv.contiguous())          # z fastest: wrong layout


def test_update_coupling_rereads_the_velocities(oracle_mod):
    w = small_cases()[1]
    m = w.model("fp64")
    u2, v2 = other_currents(w, 2.0)
    m.velocities["u"], m.velocities["v"] = u2, v2
    rp.update_coupling(m)
    o = oracle_mod.Oracle(w)
    o.update_currents(u2, v2)
    got = m.coupling_fields()
    ref = o.coupling(got["Ux"].shape)
    assert np.max(np.abs(got["Ux"] - ref["Ux"])) <= 1e-13 * np.max(np.abs(ref["Ux"]))


def test_update_currents_needs_prescribed_currents():
    w = workloads.self_coupled_swell(N=12, Nk=8, Np=12)
    m = w.model("fp64")
    u = np.zeros((12, 12, 4))
    with pytest.raises(rp.ArgumentError):
        m.update_currents(u, u)
    with pytest.raises(rp.RplError):
        rp._lib.check(m._lib.rpl_update_currents(m.handle, rp._lib.dptr(u), rp._lib.dptr(u)))
