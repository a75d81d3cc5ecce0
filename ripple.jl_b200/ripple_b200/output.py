"""Output during a run without stalling the time stepping.

fetch_output(field, model) is Oceananigans' hook for output writers, which the reference defines as
interior(field) for a ProductField (src/OceananigansIntegration.jl:7-9). Here a snapshot of the action
is converted to the caller's layout on the GPU and copied to page-locked host memory on a second
stream while the following steps run (rpl_snapshot_async); SnapshotWriter is a Simulation callback
that writes those snapshots to .npy files from a worker thread, double-buffered. Per-step diagnostics
can stay in device memory (diagnostics_device) so a time series needs no host round trip.
The reference's JLD2 writer is not reproduced: the image has no HDF5 library, so files are NumPy's
.npy (the array is interior(field) itself, (Nx, Ny, Nk, Np) in Fortran order).
"""
import ctypes
import json
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import _lib
from ._lib import ArgumentError, check
from .model import interior


def fetch_output(field, model=None):
    """fetch_output(::ProductField, model) = interior(field) (OceananigansIntegration.jl:7-9)."""
    return interior(field)


class HostBuffer:
    """Page-locked host memory (rpl_host_alloc) viewed as a Fortran-ordered NumPy array."""

    def __init__(self, shape, dtype=np.float64):
        self._lib = _lib.load()
        self.dtype = np.dtype(dtype)
        self.shape = tuple(int(s) for s in shape)
        nbytes = int(np.prod(self.shape)) * self.dtype.itemsize
        p = ctypes.c_void_p()
        check(self._lib.rpl_host_alloc(nbytes, ctypes.byref(p)))
        self._p = p
        raw = (ctypes.c_char * max(nbytes, 1)).from_address(p.value)
        self.array = np.frombuffer(raw, dtype=self.dtype, count=int(np.prod(self.shape))).reshape(
            self.shape, order="F")

    @property
    def ptr(self):
        return self._p

    def close(self):
        if getattr(self, "_p", None) is not None and self._p.value:
            self.array = None
            self._lib.rpl_host_free(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _dtype_code(dtype):
    dt = np.dtype(dtype)
    if dt == np.float64:
        return _lib.RPL_F64
    if dt == np.float32:
        return _lib.RPL_F32
    raise ArgumentError("snapshots are float64 or float32")


def snapshot_async(model, out=None, dtype=None):
    """Enqueue a copy of model.action (interior layout) into `out` (a HostBuffer; allocated when None)
    and return it at once; the data is there after snapshot_wait(model)."""
    if dtype is None:
        dtype = np.float32 if model.precision == "fp32" else np.float64
    if out is None:
        out = HostBuffer(model.action.size, dtype)
    if tuple(out.shape) != tuple(model.action.size):
        raise ArgumentError("snapshot buffer does not match the action field")
    check(model._lib.rpl_snapshot_async(model.handle, out.ptr, _dtype_code(out.dtype)))
    return out


def snapshot_wait(model):
    check(model._lib.rpl_snapshot_wait(model.handle))


def diagnostics_device(model, m0=None, hs=None, kappa_rms=None, mean_direction=None, total_action=None):
    """Enqueue the diagnostics of the current action into CUDA float64 tensors (any may be None): (Nx, Ny)
    fields with x fastest, total_action a one-element tensor (e.g. a slot of a time series)."""
    def ptr(t):
        return None if t is None else ctypes.c_void_p(t.data_ptr())
    check(model._lib.rpl_diagnostics_device(model.handle, ptr(m0), ptr(hs), ptr(kappa_rms), ptr(mean_direction),
                                            ptr(total_action)))


class SnapshotWriter:
    """Simulation callback: every `schedule` iterations a snapshot of the action is taken asynchronously
    into one of two page-locked buffers; the previous one is written to
    `<directory>/<prefix>_<iteration>.npy` by a worker thread. close() flushes the last snapshot and
    writes `<prefix>_index.json` (iteration, time, file of each snapshot)."""

    def __init__(self, model, schedule, directory, prefix="action", dtype=None):
        if int(schedule) < 1:
            raise ArgumentError("schedule must be a positive iteration interval")
        self.model, self.schedule = model, int(schedule)
        self.directory, self.prefix = directory, prefix
        os.makedirs(directory, exist_ok=True)
        dtype = dtype or (np.float32 if model.precision == "fp32" else np.float64)
        self.buffers = [HostBuffer(model.action.size, dtype) for _ in range(2)]
        self.busy = [None, None]          # worker future writing each buffer
        self.pending = None               # (buffer index, iteration, time) copying to the host
        self.index = []
        self.k = 0
        self.pool = ThreadPoolExecutor(max_workers=1)

    def _flush_pending(self):
        if self.pending is None:
            return
        snapshot_wait(self.model)
        b, it, t = self.pending
        name = f"{self.prefix}_{it:08d}.npy"
        path = os.path.join(self.directory, name)
        self.busy[b] = self.pool.submit(np.save, path, self.buffers[b].array)
        self.index.append({"iteration": it, "time": t, "file": name})
        self.pending = None

    def __call__(self, simulation):
        m = self.model
        if m.clock.iteration % self.schedule:
            return
        self._flush_pending()
        b = self.k % 2
        if self.busy[b] is not None:
            self.busy[b].result()
            self.busy[b] = None
        snapshot_async(m, self.buffers[b])
        self.pending = (b, m.clock.iteration, m.clock.time)
        self.k += 1

    def close(self):
        self._flush_pending()
        self.pool.shutdown(wait=True)
        for f in self.busy:
            if f is not None:
                f.result()
        with open(os.path.join(self.directory, f"{self.prefix}_index.json"), "w") as f:
            json.dump(self.index, f, indent=1)
        for b in self.buffers:
            b.close()
