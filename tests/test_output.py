"""Output during a run: asynchronous snapshots (fetch_output(::ProductField) = interior(field),
src/OceananigansIntegration.jl:7-9), the SnapshotWriter callback, device-side diagnostics.

A snapshot must equal interior(model.action) at the moment it was taken, bit for bit in the model's own
dtype, even when later steps run before the copy is waited for.
"""
import json
import os

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import workloads

pytestmark = pytest.mark.gpu


def small(precision):
    w = workloads.seamount_eddies(N=32, Nz=8, Nk=8, Np=12, nsteps=6)
    return w, w.model(precision)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_snapshot_equals_interior_at_its_time(precision):
    w, m = small(precision)
    rp.time_step(m, w.dt, 2)
    ref = m.action.interior()
    buf = rp.snapshot_async(m)
    rp.time_step(m, w.dt, 3)              # later steps before the copy is waited for
    rp.snapshot_wait(m)
    dt = np.float32 if precision == "fp32" else np.float64
    assert buf.array.dtype == dt
    assert np.array_equal(buf.array, ref.astype(dt))
    assert not np.array_equal(m.action.interior(), ref)
    buf.close()


def test_snapshot_dtype_conversion_and_fetch_output():
    w, m = small("fp64")
    rp.time_step(m, w.dt, 1)
    b32 = rp.snapshot_async(m, rp.HostBuffer(m.action.size, np.float32))
    rp.snapshot_wait(m)
    ref = rp.fetch_output(m.action, m)
    assert np.array_equal(ref, m.action.interior())
    assert np.array_equal(b32.array, ref.astype(np.float32))
    with pytest.raises(rp.ArgumentError):
        rp.snapshot_async(m, rp.HostBuffer((2, 2, 2, 2), np.float64))


def test_snapshot_writer_files_match_the_run(tmp_path):
    w, m = small("fp32")
    _, m2 = small("fp32")
    writer = rp.SnapshotWriter(m, 2, str(tmp_path), prefix="N")
    sim = rp.Simulation(m, Δt=w.dt, stop_iteration=6, callbacks=[writer])
    rp.run_(sim)
    writer.close()
    index = json.load(open(os.path.join(tmp_path, "N_index.json")))
    assert [e["iteration"] for e in index] == [2, 4, 6]
    for e in index:
        rp.time_step(m2, w.dt, e["iteration"] - m2.clock.iteration)
        got = np.load(os.path.join(tmp_path, e["file"]))
        assert got.shape == tuple(m2.action.size)
        assert np.array_equal(got, m2.action.interior().astype(np.float32))
        assert e["time"] == pytest.approx(m2.clock.time, rel=1e-15)


def test_diagnostics_device_equal_host_diagnostics():
    import torch
    w, m = small("fp64")
    rp.time_step(m, w.dt, 2)
    d = rp.diagnostics(m.action)
    Nx, Ny = m.grid.Nx, m.grid.Ny
    fields = [torch.empty(Nx * Ny, dtype=torch.float64, device="cuda") for _ in range(4)]
    series = torch.zeros(3, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rp.diagnostics_device(m, *fields, total_action=series[1:2])
    rp._lib.check(m._lib.rpl_sync(m.handle))
    for k, f in zip(("m0", "Hs", "kappa_rms", "mean_direction"), fields):
        assert np.array_equal(f.cpu().numpy().reshape((Nx, Ny), order="F"), d[k]), k
    assert series[1].item() == d["total_action"] and series[0].item() == 0.0


def test_total_only_diagnostics_equal_the_full_call():
    """A call that asks for m0 and the total action alone takes the m0-only kernel: same values, bit for
    bit, as the full call."""
    w, m = small("fp32")
    rp.time_step(m, w.dt, 2)
    full = rp.diagnostics(m.action)
    m0 = np.empty((m.grid.Nx, m.grid.Ny), order="F")
    tot = np.zeros(1)
    rp._lib.check(m._lib.rpl_diagnostics(m.handle, rp._lib.dptr(m0), None, None, None, rp._lib.dptr(tot)))
    assert np.array_equal(m0, full["m0"])
    assert tot[0] == full["total_action"]
