"""Host-side checks that need no GPU: the C-ABI library's exports and argument validation,
the Python mirror of the reference interface, the workload builders, and the oracle
against its committed golden fixtures."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import _lib, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def header_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^\s*(?:int|const char\*)\s+(rpl_\w+)\s*\(", txt, re.M))
    return names


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in sorted(syms):
        assert hasattr(lib, s), s
    assert lib.rpl_abi_version() == _lib.RPL_ABI_VERSION


def _desc(**kw):
    x = np.arange(4, dtype=float) + 0.5
    k = np.array([0.3, 0.4])
    kf = np.array([0.25, 0.35, 0.45])
    p = np.array([0.0, 2.0, 4.0])
    pf = np.array([-1.0, 1.0, 3.0, 5.0])
    keep = [x, k, kf, p, pf]
    d = _lib.RplDesc()
    d.abi_version = _lib.RPL_ABI_VERSION
    d.precision, d.transport = _lib.RPL_FP64, _lib.RPL_TRANSPORT_INTRINSIC
    d.Nx = d.Ny = 4
    d.Nk, d.Np = 2, 3
    d.dx = d.dy = 1.0
    d.xnodes = d.ynodes = _lib.dptr(x)
    d.periodic_x = d.periodic_y = 1
    d.kappa, d.kappa_faces, d.phi, d.phi_faces = (_lib.dptr(a) for a in (k, kf, p, pf))
    d.depth_kind = _lib.RPL_DEPTH_INFINITE
    d.gravity = 9.81
    for name, val in kw.items():
        setattr(d, name, val)
    return d, keep


@pytest.mark.parametrize("field,value,code", [
    ("abi_version", 99, _lib.RPL_ERR_ARGUMENT),
    ("Nx", 0, _lib.RPL_ERR_ARGUMENT),
    ("dx", -1.0, _lib.RPL_ERR_ARGUMENT),
    ("periodic_x", 0, _lib.RPL_ERR_UNSUPPORTED),
    ("depth_kind", _lib.RPL_DEPTH_CONSTANT, _lib.RPL_ERR_ARGUMENT),   # depth_constant 0
    ("precision", 7, _lib.RPL_ERR_ARGUMENT),
    ("memory_limit_bytes", 1024, _lib.RPL_ERR_OOM),
])
def test_create_rejects_bad_descriptors_before_touching_the_device(field, value, code):
    lib = _lib.load()
    d, keep = _desc(**{field: value})
    h = ctypes.c_void_p()
    assert lib.rpl_create(ctypes.byref(d), ctypes.byref(h)) == code
    assert not h.value
    assert len(lib.rpl_last_error()) > 0


def test_create_rejects_bad_spectral_faces():
    lib = _lib.load()
    kf = np.array([0.35, 0.36, 0.45])  # centre 0.3 outside its faces
    d, keep = _desc()
    d.kappa_faces = _lib.dptr(kf)
    h = ctypes.c_void_p()
    assert lib.rpl_create(ctypes.byref(d), ctypes.byref(h)) == _lib.RPL_ERR_ARGUMENT
    assert b"inside its cell faces" in lib.rpl_last_error()
    assert lib.rpl_create(None, ctypes.byref(h)) == _lib.RPL_ERR_ARGUMENT
    assert lib.rpl_step(None, 1.0, 1) == _lib.RPL_ERR_ARGUMENT
    assert lib.rpl_destroy(None) == _lib.RPL_OK


def test_python_api_validation():
    g = rp.RectilinearGrid(size=(8, 8, 2), x=(0, 8), y=(0, 8), z=(-1, 0))
    sg = rp.PolarWaveVectorGrid(κ=[0.5, 1.0], φ=[0.0, 2.0, 4.0])
    with pytest.raises(rp.ArgumentError):
        rp.SpectralWaveModel(g, sg, timestepper="AB2")
    with pytest.raises(rp.ArgumentError):
        rp.SpectralWaveModel(g, sg, horizontal_advection="Centered")
    with pytest.raises(rp.ArgumentError):
        rp.SpectralWaveModel(g, sg, depth=-3.0)
    with pytest.raises(rp.ArgumentError):
        rp.PolarWaveVectorGrid(κ=[1.0, 0.5], φ=[0.0])
    with pytest.raises(rp.ArgumentError):
        rp.PolarWaveVectorGrid(κ=[-1.0], φ=[0.0])
    with pytest.raises(rp.ArgumentError):
        rp.PolarWaveVectorGrid(φ=[0.0])
    with pytest.raises(rp.ArgumentError):
        rp.HollandHurricaneWind(rmax=2.0, radius=1.0)
    with pytest.raises(rp.ArgumentError):
        rp.LinearStormTrack([1.0, 0.5], [(0, 0), (1, 1)])
    with pytest.raises(rp.ArgumentError):
        rp.WENO(order=3)
    f = rp.WaveActionField(g, sg)
    rp.set_(f, lambda x, y, kx, ky: 1 + 0.1 * x + 0.02 * np.hypot(kx, ky))
    a = rp.interior(f)
    assert a.shape == (8, 8, 2, 3)
    assert a[3, 0, 1, 2] == pytest.approx(1 + 0.1 * 3.5 + 0.02 * 1.0)
    with pytest.raises(rp.ArgumentError):
        rp.set_(f, np.zeros((2, 2, 2, 2)))


def test_polar_grid_defaults():
    sg = rp.PolarWaveVectorGrid(κ=[(9.0 + 2 * k) / 30 for k in range(4)], φ=[k * 2 * math.pi / 16 for k in range(16)])
    assert sg.κ_faces[0] == pytest.approx(0.3 - 1 / 30)
    assert np.all(np.diff(sg.φ_faces) > 0)
    w = sg.weights
    assert w.shape == (4, 16)
    assert w[1, 0] == pytest.approx(((sg.κ_faces[2] ** 2 - sg.κ_faces[1] ** 2) / 2) * (2 * math.pi / 16))


def test_workloads_are_seeded_and_sane():
    a = workloads.seamount_eddies(N=32, Nz=8, Nk=8, Np=12, nsteps=2)
    b = workloads.seamount_eddies(N=32, Nz=8, Nk=8, Np=12, nsteps=2)
    assert np.array_equal(a.N0, b.N0) and np.array_equal(a.velocities["u"], b.velocities["u"])
    assert np.all(a.depth >= 100.0) and np.all(a.depth <= 4000.0)
    assert a.dt > 0 and np.all(a.N0 > 0)
    c = workloads.hurricane_swell(N=16, Nk=8, Np=12, nsteps=3)
    assert c.dt > 0 and c.N0.shape == (16, 16, 8, 12)
    v = workloads.vortex_refraction(N=16)
    u = v.velocities["u"]
    assert u.shape == (16, 16, 16) and np.max(np.hypot(u, v.velocities["v"])) <= 0.4 + 1e-12


def test_oracle_reproduces_golden_c1(oracle_mod):
    ref = np.load(os.path.join(GOLDEN, "c1_vortex_refraction.npz"))
    w = workloads.vortex_refraction()
    o = oracle_mod.Oracle(w)
    N, t = o.step(w.N0, w.dt, w.nsteps)
    d = o.diagnostics(N)
    flat = N.ravel(order="F")
    assert np.array_equal(flat[::97], ref["sample"])
    assert d["total_action"] == pytest.approx(float(ref["total_action"]), rel=1e-14)
    assert np.array_equal(d["m0"], ref["m0"])


def test_oracle_reproduces_golden_kat(oracle_mod):
    ref = np.load(os.path.join(GOLDEN, "kat_tendency_8x7x4x6.npz"))
    import sys
    sys.path.insert(0, GOLDEN)
    from make_golden import kat_workload
    k = kat_workload()
    assert np.array_equal(k.N0, ref["N0"])
    G = oracle_mod.Oracle(k).tendency(k.N0)
    assert np.array_equal(G, ref["G"])
