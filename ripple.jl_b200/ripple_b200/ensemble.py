"""Batching form: an ensemble of independent FP32 SpectralWaveModels advanced together.

The reference advances one model per `time_step!` call (src/Models/time_step.jl:119-170); a Julia
caller with many members loops over them. `Ensemble` keeps that meaning -- each `time_step` is one
SSP-RK3 step of every member with its own dt -- but runs it as three persistent launches in total
(one per stage, all members' tiles taken from one work counter), replayed from a CUDA graph, with
tile shapes from the library's autotuner (rpl_ensemble_* in include/rpl.h).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError, check


class Ensemble:
    """Members: SpectralWaveModels with precision="fp32", one device, one transport kind, no sources.

    dts: one time step per member. use_graph: replay a captured CUDA graph per step. autotune: time the
    candidate tile shapes of every size class at creation (cached in `autotune_cache` if given).
    """

    def __init__(self, models, dts, use_graph=True, autotune=False, autotune_cache=None, direct_cells=0):
        models = list(models)
        dts = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, dtype=np.float64), (len(models),)))
        if not models:
            raise ArgumentError("an ensemble needs at least one model")
        self._lib = _lib.load()
        self.models = models
        self.dts = dts
        handles = (ctypes.c_void_p * len(models))(*[m.handle.value for m in models])
        self._cache = autotune_cache.encode() if autotune_cache else None
        opts = _lib.RplEnsembleOptions(_lib.RPL_ABI_VERSION, 1 if use_graph else 0, 1 if autotune else 0,
                                       int(direct_cells), self._cache)
        h = ctypes.c_void_p()
        for m in models:
            check(self._lib.rpl_set_clock(m.handle, m.clock.time, m.clock.iteration))
        check(self._lib.rpl_ensemble_create(handles, _lib.dptr(dts), len(models), ctypes.byref(opts),
                                            ctypes.byref(h)))
        self._h = h

    def _sync_clocks(self):
        for m in self.models:
            m._sync_clock()

    def time_step(self, nsteps=1):
        """nsteps SSP-RK3 steps of every member (persistent launches, graph replay)."""
        check(self._lib.rpl_ensemble_step(self._h, int(nsteps)))
        self._sync_clocks()
        return self

    def time_step_sequential(self, nsteps=1):
        """The same steps as per-member sequential launches of the single-model kernels (the baseline)."""
        check(self._lib.rpl_ensemble_step_sequential_async(self._h, int(nsteps)))
        check(self._lib.rpl_ensemble_sync(self._h))
        self._sync_clocks()
        return self

    def autotune(self, force=False):
        check(self._lib.rpl_ensemble_autotune(self._h, 1 if force else 0))

    def shapes(self):
        """(lanes, tile_x, tile_y) used for each member."""
        out = []
        for i in range(len(self.models)):
            L, tx, ty = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
            check(self._lib.rpl_ensemble_shape(self._h, i, ctypes.byref(L), ctypes.byref(tx), ctypes.byref(ty)))
            out.append((L.value, tx.value, ty.value))
        return out

    @property
    def handle(self):
        return self._h

    @property
    def units(self):
        return int(sum(int(np.prod(m.action.size)) for m in self.models))

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.rpl_ensemble_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
