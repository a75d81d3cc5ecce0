"""rpl_diagnostics_static: the diagnostics entry point that allocates nothing.

It serves callers that must not allocate device memory when they ask for diagnostics (a host
framework whose device memory belongs to its own pool allocator, or work enqueued during a stream
capture); its only scratch is a fixed array inside librpl.so. This checks it through the C-ABI
against the handle-based rpl_diagnostics on two calls in a row (the second call reuses the scratch
the first one left behind), at the tolerances the other diagnostics tests use, and that a grid above
its stated limit is refused. The file name keeps it last in collection order.
"""
import ctypes
import math

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


def spectral_measures(sg):
    """weights, first-moment x/y and second-moment trace per bin, kappa fastest (4*Nk*Np)."""
    kf, pf = sg.κ_faces, sg.φ_faces
    Nk, Np = sg.coordinate_size()
    out = np.empty((4, Np, Nk))
    for n in range(Np):
        for m in range(Nk):
            k1, k2, p1, p2 = kf[m], kf[m + 1], pf[n], pf[n + 1]
            r1 = (k2 * k2 * k2 - k1 * k1 * k1) / 3.0
            r2 = (k2 ** 4 - k1 ** 4) / 4.0
            dp, s2 = p2 - p1, math.sin(2 * p2) - math.sin(2 * p1)
            out[0, n, m] = ((k2 * k2 - k1 * k1) / 2.0) * (p2 - p1)
            out[1, n, m] = r1 * (math.sin(p2) - math.sin(p1))
            out[2, n, m] = r1 * (math.cos(p1) - math.cos(p2))
            out[3, n, m] = r2 * (dp / 2.0 + s2 / 4.0) + r2 * (dp / 2.0 - s2 / 4.0)
    return out.ravel()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_static_diagnostics_match_handle_diagnostics(precision):
    import torch
    w = workloads.seamount_eddies(N=48, Nz=8, Nk=32, Np=36, nsteps=1)
    m = w.model(precision)
    rp.time_step(m, w.dt)                      # a state that is not the initial condition
    ref = rp.diagnostics(m.action)
    lib = _lib.load()
    Nx, Ny = w.grid.Nx, w.grid.Ny
    Nk, Np = w.spectral_grid.coordinate_size()
    tdtype = torch.float64 if precision == "fp64" else torch.float32
    code = _lib.RPL_F64 if precision == "fp64" else _lib.RPL_F32
    N_dev = torch.empty(Nx * Ny * Nk * Np, dtype=tdtype, device="cuda")
    _lib.check(lib.rpl_get_action_device(m.handle, ctypes.c_void_p(N_dev.data_ptr()), code, 0))
    meas = torch.tensor(spectral_measures(w.spectral_grid), dtype=torch.float64, device="cuda")
    out = torch.full((4, Nx * Ny), float("nan"), dtype=torch.float64, device="cuda")
    total = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    dx, dy = float(w.grid.xspacings()[0]), float(w.grid.yspacings()[0])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):
        out.fill_(float("nan"))
        total.fill_(float("nan"))
        st = lib.rpl_diagnostics_static(ctypes.c_void_p(N_dev.data_ptr()), code, Nx, Ny, Nk, Np,
                                        ctypes.c_void_p(meas.data_ptr()), dx, dy,
                                        *[ctypes.c_void_p(out[k].data_ptr()) for k in range(4)],
                                        ctypes.c_void_p(total.data_ptr()), stream)
        assert st == _lib.RPL_OK, lib.rpl_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(4, Ny, Nx).transpose(0, 2, 1)
        for k, name in enumerate(("m0", "Hs", "kappa_rms")):
            r = ref[name]
            assert np.linalg.norm(got[k] - r) <= 1e-14 * np.linalg.norm(r), (call, name)
        assert np.max(np.abs(got[3] - ref["mean_direction"])) <= 1e-13, call
        assert float(total.item()) == pytest.approx(ref["total_action"], rel=1e-14), call
    m.close()


def test_static_diagnostics_rejects_grids_above_its_limit():
    import torch
    lib = _lib.load()
    dummy = torch.zeros(8, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    st = lib.rpl_diagnostics_static(p, _lib.RPL_F64, 4096, 2048, 1, 1, p, 1.0, 1.0, None, None, None, None,
                                    None, None)
    assert st == _lib.RPL_ERR_ARGUMENT
    assert b"at most 4194304" in lib.rpl_last_error()
    # sizes whose product wraps around in 64 bits are refused too, not accepted as a small grid
    st = lib.rpl_diagnostics_static(p, _lib.RPL_F64, 1 << 33, 1 << 31, 1, 1, p, 1.0, 1.0, None, None, None,
                                    None, None, None)
    assert st == _lib.RPL_ERR_ARGUMENT
    assert b"at most 4194304" in lib.rpl_last_error()
