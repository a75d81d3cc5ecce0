"""Spectral diagnostics of a model's wave action, computed on the device in FP64 with
compensated sums: m0 (src/Diagnostics/moments.jl:33-37), significant_wave_height
(bulk_statistics.jl:9), root_mean_square_wavenumber (moments.jl:100-111),
mean_direction (moments.jl:117-123) and total_action (bulk_statistics.jl:87-91).
"""
import numpy as np

from . import _lib
from ._lib import ArgumentError, check, dptr


def _model_of(N):
    m = getattr(N, "_model", None)
    if m is None:
        raise ArgumentError("diagnostics run on a model's action (model.action); this field is not on a device")
    return m


def diagnostics(N):
    """All per-(i,j) diagnostics and the total action in one device pass."""
    m = _model_of(N)
    shape = (m.grid.Nx, m.grid.Ny)
    outs = [np.empty(shape, order="F") for _ in range(4)]
    total = np.zeros(1)
    check(m._lib.rpl_diagnostics(m._h, *[dptr(o) for o in outs], dptr(total)))
    return dict(m0=outs[0], Hs=outs[1], kappa_rms=outs[2], mean_direction=outs[3], total_action=float(total[0]))


def m0(N):
    return diagnostics(N)["m0"]


def significant_wave_height(N):
    return diagnostics(N)["Hs"]


def root_mean_square_wavenumber(N):
    return diagnostics(N)["kappa_rms"]


def mean_direction(N):
    return diagnostics(N)["mean_direction"]


def total_action(N):
    return diagnostics(N)["total_action"]


def mean_period(N, gravity=9.81):
    """Mean wave period per (i,j), T = 2 pi m0 / m_sigma with m_sigma = sum N sigma(kappa, d) w over the
    spectral cells, sigma = sqrt(g kappa tanh(kappa d)) (deep water when d is infinite). The reference
    defines mean_period only on frequency-direction grids (src/Diagnostics/moments.jl:362-370); this is
    its analogue on the polar wavenumber grid, computed on the host from the interior (FP64)."""
    m = _model_of(N)
    A = np.asarray(N.interior(), dtype=np.float64)             # (Nx, Ny, Nk, Np)
    sg = m.spectral_grid
    w = np.asarray(sg.weights, dtype=np.float64)               # (Nk, Np)
    k = np.asarray(sg.kappa, dtype=np.float64)
    d = m.depth_values()                                       # scalar, inf or (Nx, Ny)
    if np.isscalar(d):
        sig = np.sqrt(gravity * k * (np.tanh(k * d) if np.isfinite(d) else 1.0))
        m_s = np.einsum("ijmn,mn->ij", A, w * sig[:, None])
    else:
        sig = np.sqrt(gravity * k[None, None, :] * np.tanh(k[None, None, :] * np.asarray(d)[:, :, None]))
        m_s = np.einsum("ijmn,mn,ijm->ij", A, w, sig)
    m0v = np.einsum("ijmn,mn->ij", A, w)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(m_s > 0, 2.0 * np.pi * m0v / m_s, 0.0)
