"""Y-slab domain decomposition (ripple_b200.decomposition): slabs with 3 halo rows whose halos are
refreshed before every RK3 stage reproduce the undecomposed run exactly.

CPU: the oracle advanced slab by slab (its tendency on each halo-extended slab, the RK3 combinations
of time_step.jl:138-152 stage by stage) with the halo exchange of the library's driver, in one process
and across 2 and 3 gloo ranks, equals the global oracle run bit for bit. GPU: librpl.so slabs on one
GPU, exchanged in turn by one process (no kernel waits for another), equal the global model bit for
bit in FP64 and FP32; a one-rank DecomposedModel too.
"""
import os
import socket

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import decomposition as dc
from ripple_b200 import workloads


def relu(x):
    return np.where(x > 0.0, x, 0.0)


class OracleBackend:
    """A slab advanced by the oracle: N, A, B like the library's three state buffers."""

    def __init__(self, oracle_mod, w):
        import torch  # noqa: F401
        self.o = oracle_mod.Oracle(w)
        self.smooth = w.propagation_smoothing is not None   # stage 3 into A, then the averaging A -> N
        self.N = np.asfortranarray(np.array(w.N0, dtype=np.float64))
        self.A = np.zeros_like(self.N, order="F")
        self.B = np.zeros_like(self.N, order="F")
        self.t = 0.0

    def _arr(self, which):
        return (self.N, self.A, self.B)[which]

    def rows_get(self, which, first, count, buf):
        import torch
        a = self._arr(which)[:, first:first + count]
        buf.copy_(torch.from_numpy(np.ascontiguousarray(np.transpose(a, (3, 1, 0, 2))).ravel()))

    def rows_set(self, which, first, count, buf):
        Nx, _, Nk, Np = self.N.shape
        self._arr(which)[:, first:first + count] = buf.numpy().reshape(Np, count, Nx, Nk).transpose(2, 1, 3, 0)

    def stage(self, dt, s, defer_smooth=False):
        Ny = self.N.shape[1]
        self.stage_rows(dt, s, 0, Ny, True, True, defer_smooth)

    def stage_rows(self, dt, s, first, count, prepare, finish, defer_smooth=False):
        """The stage for rows [first, first + count) only, from the buffers as they are now (halo rows
        included, refreshed or not), like rpl_stage_rows_async."""
        if count > 0:
            r = slice(first, first + count)
            if s == 1:
                self.A[:, r] = relu(self.N + dt * self.o.tendency(self.N, self.t))[:, r]
            elif s == 2:
                st = relu(self.A + dt * self.o.tendency(self.A, self.t))
                self.B[:, r] = relu(0.75 * self.N + 0.25 * st)[:, r]
            else:
                st = relu(self.B + dt * self.o.tendency(self.B, self.t))
                out = self.A if self.smooth else self.N
                out[:, r] = relu((1.0 / 3.0) * self.N + (2.0 / 3.0) * st)[:, r]
        if finish and s == 3:
            if self.smooth and not defer_smooth:
                self.smooth_rows(dt, 0, self.N.shape[1])
            self.t += dt

    def smooth_rows(self, dt, first, count, y_offset=0):
        """SpatialAveraging A -> N for rows [first, first + count), like rpl_smooth_rows_async."""
        r = slice(first, first + count)
        self.N[:, r] = self.o.spatial_averaging(self.A, dt, y_offset)[:, r]

    def mark_input(self):
        pass

    def begin_exchange(self):
        pass

    def end_exchange(self):
        pass

    def sync(self):
        pass


def cases():
    from test_source_terms import random_terms_workload
    smoothed = workloads.seamount_eddies(N=24, Nz=8, Nk=8, Np=12, nsteps=3)
    smoothed.propagation_smoothing = rp.SpatialAveraging(αs=0.5, αn=0.5)
    return [workloads.seamount_eddies(N=24, Nz=8, Nk=8, Np=12, nsteps=3),   # currents, depth field
            workloads.hurricane_swell(N=24, Nk=8, Np=12, nsteps=3),          # sources, moving storm
            random_terms_workload(N=12, Nk=8, Np=12),                        # SourceTermSet, a rate field
            smoothed]                                                        # SpatialAveraging after every step


def smoothing_slabs(w, slabs):
    """The slabs argument of rk3_steps for models with SpatialAveraging, else None."""
    return slabs if w.propagation_smoothing is not None else None


def _buffers(slab, w):
    import torch
    Nk, Np = w.spectral_grid.coordinate_size()
    n = Np * slab.halo * w.grid.Nx * Nk
    return {k: torch.zeros(n, dtype=torch.float64) for k in ("send_low", "send_high", "recv_low", "recv_high")}


# ---------------------------------------------------------------- bookkeeping (CPU)

def test_slabs_cover_the_rows_once():
    for Ny, world in ((24, 1), (24, 2), (25, 3), (30, 7)):
        rows = np.concatenate([np.arange(*dc.slab_rows(Ny, world, r)) for r in range(world)])
        assert np.array_equal(rows, np.arange(Ny))
        s = dc.Slab(Ny, world, world - 1)
        g = s.global_rows()
        assert len(g) == s.rows and g[-1] == 2 and g[s.halo] == s.start
    with pytest.raises(rp.ArgumentError):
        dc.Slab(8, 4, 0)                      # 2 rows per rank < 3 halo rows


def test_local_grid_keeps_the_parent_geometry():
    w = cases()[0]
    s = dc.Slab(24, 3, 1)
    lw = dc.local_workload(w, s)
    assert lw.grid.first_spacings() == w.grid.first_spacings()
    assert np.array_equal(lw.grid.yfaces()[s.halo:s.halo + s.ny + 1], w.grid.yfaces()[s.start:s.stop + 1])
    assert np.array_equal(lw.N0, w.N0[:, (np.arange(s.start - 3, s.stop + 3) % 24)])
    assert lw.velocities["u"].shape == (24, s.rows, 8)


def test_local_workload_rejects_what_is_not_decomposed():
    s = dc.Slab(24, 2, 0)
    w = workloads.self_coupled_swell(N=24, Nk=8, Np=12)
    with pytest.raises(rp.ArgumentError):
        dc.local_workload(w, s)                       # pseudomomentum coupling
    w = cases()[1]
    g = w.grid
    w.grid = rp.RectilinearGrid(size=(g.Nx, g.Ny, g.Nz), x=g.xfaces(), y=g.yfaces(), z=g.zfaces(),
                                topology=("Periodic", "Bounded", "Bounded"))
    with pytest.raises(rp.ArgumentError):
        dc.local_workload(w, s)                       # a bounded y axis


def test_smoothing_reach_limits_the_step():
    """The averaging's corners must stay within the 3 halo rows: at the workload's dt they reach a small
    fraction of a row; a dt that takes them 3 rows or further is refused."""
    w = cases()[3]
    dy = (w.grid.yfaces()[-1] - w.grid.yfaces()[0]) / w.grid.Ny
    r = dc.smoothing_reach_rows(w.spectral_grid, w.propagation_smoothing, w.dt, dy)
    assert 0 < r < 1
    dc.check_smoothing_reach(w, w.dt)
    with pytest.raises(rp.ArgumentError):
        dc.check_smoothing_reach(w, w.dt * 3.01 / r)


@pytest.mark.parametrize("case", [0, 1, 3])
@pytest.mark.parametrize("world", [2, 3])
def test_oracle_slabs_in_one_process_equal_the_global_run(oracle_mod, case, world):
    w = cases()[case]
    slabs = [dc.Slab(w.grid.Ny, world, r) for r in range(world)]
    backs = [OracleBackend(oracle_mod, dc.local_workload(w, s)) for s in slabs]
    bufs = [_buffers(s, w) for s in slabs]
    dc.rk3_steps(backs, lambda which: dc.exchange_local(backs, slabs, which, bufs), w.dt, 3,
                 slabs=smoothing_slabs(w, slabs))
    got = np.concatenate([b.N[:, s.owned()] for b, s in zip(backs, slabs)], axis=1)
    ref, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 3)
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("case", [0, 1, 2, 3])
@pytest.mark.parametrize("world", [1, 2, 3])
def test_oracle_overlapped_slabs_equal_the_global_run(oracle_mod, case, world):
    """Interior rows computed before the exchange (their halo rows still hold the previous stage's
    values), boundary rows after it: a row that read a halo in the interior launch would differ."""
    w = cases()[case]
    slabs = [dc.Slab(w.grid.Ny, world, r) for r in range(world)]
    backs = [OracleBackend(oracle_mod, dc.local_workload(w, s)) for s in slabs]
    for b in backs:                                   # halos start wrong: only exchanges may fill them
        for arr in (b.N, b.A, b.B):
            arr[:, :3] = -7.0
            arr[:, -3:] = -7.0
    bufs = [_buffers(s, w) for s in slabs]
    dc.rk3_steps_overlapped(backs, slabs, lambda which: dc.exchange_local(backs, slabs, which, bufs), w.dt, 3,
                            smooth=w.propagation_smoothing is not None)
    got = np.concatenate([b.N[:, s.owned()] for b, s in zip(backs, slabs)], axis=1)
    ref, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 3)
    assert np.array_equal(got, ref)


def test_interior_and_boundary_rows_cover_the_owned_rows_once():
    for Ny, world in ((24, 2), (9, 3), (40, 4), (12, 1)):
        for r in range(world):
            s = dc.Slab(Ny, world, r)
            (l0, l1), (h0, h1) = dc.boundary_rows(s)
            i0, i1 = dc.interior_rows(s)
            rows = list(range(l0, l1)) + list(range(i0, i1)) + list(range(h0, h1))
            assert rows == list(range(s.halo, s.halo + s.ny))
            assert all(r - 3 >= s.halo and r + 3 < s.halo + s.ny for r in range(i0, i1))


def _gloo_rank(rank, world, port, case, out, overlap=False):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import oracle as oracle_mod
        w = cases()[case]
        slab = dc.Slab(w.grid.Ny, world, rank)
        back = OracleBackend(oracle_mod, dc.local_workload(w, slab))
        bufs = _buffers(slab, w)
        smooth = w.propagation_smoothing is not None
        if overlap:
            dc.rk3_steps_overlapped([back], [slab], lambda which: dc.exchange_dist(back, slab, which, bufs),
                                    w.dt, 3, smooth=smooth)
        else:
            dc.rk3_steps([back], lambda which: dc.exchange_dist(back, slab, which, bufs), w.dt, 3,
                         slabs=[slab] if smooth else None)
        parts = [None] * world
        dist.all_gather_object(parts, (slab.start, back.N[:, slab.owned()]))
        if rank == 0:
            np.save(out, np.concatenate([p for _, p in sorted(parts, key=lambda t: t[0])], axis=1))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world,case,overlap", [(2, 0, False), (3, 0, False), (2, 1, False), (2, 0, True),
                                                 (3, 1, True), (2, 3, False), (3, 3, True)])
def test_oracle_slabs_across_gloo_ranks_equal_the_global_run(oracle_mod, tmp_path, world, case, overlap):
    import torch.multiprocessing as mp
    out = str(tmp_path / "global.npy")
    mp.start_processes(_gloo_rank, args=(world, _free_port(), case, out, overlap), nprocs=world, join=True,
                       start_method="spawn")
    w = cases()[case]
    ref, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 3)
    assert np.array_equal(np.load(out), ref)


# ---------------------------------------------------------------- CUDA path (GPU)

@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 1, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("world", [2, 3])
def test_library_slabs_on_one_gpu_equal_the_global_model(case, precision, world):
    import torch
    w = cases()[case]
    if precision == "fp32":
        w.N0 = w.N0.astype(np.float32, order="F")
    slabs = [dc.Slab(w.grid.Ny, world, r) for r in range(world)]
    models = [dc.local_workload(w, s).model(precision) for s in slabs]
    st = torch.cuda.Stream()                       # kernels, row copies and exchange copies in one order
    for m in models:
        rp._lib.check(m._lib.rpl_set_stream(m.handle, rp._lib.ctypes.c_void_p(st.cuda_stream)))
    backs = [dc.LibBackend(m) for m in models]
    Nk, Np = w.spectral_grid.coordinate_size()
    dt_t = torch.float32 if precision == "fp32" else torch.float64
    bufs = [{k: torch.zeros(Np * 3 * w.grid.Nx * Nk, dtype=dt_t, device="cuda")
             for k in ("send_low", "send_high", "recv_low", "recv_high")} for _ in slabs]

    with torch.cuda.stream(st):
        dc.rk3_steps(backs, lambda which: dc.exchange_local(backs, slabs, which, bufs), w.dt, 3,
                     slabs=smoothing_slabs(w, slabs))
    got = np.concatenate([m.action.interior()[:, s.owned()] for m, s in zip(models, slabs)], axis=1)
    g = w.model(precision)
    rp.time_step(g, w.dt, 3)
    assert np.array_equal(got, g.action.interior())
    assert all(m.clock.iteration == 3 for m in models)


@pytest.mark.gpu
@pytest.mark.parametrize("case", [0, 3])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_library_overlapped_slabs_on_one_gpu_equal_the_global_model(case, precision):
    """Row-range stage launches (interior rows, then the two boundary ranges) on one compute stream, the
    exchange copies on a second stream ordered by events, halo rows never recomputed; with
    SpatialAveraging (case 3) the averaging after the exchange of stage 3's result."""
    import torch
    w = cases()[case]
    if precision == "fp32":
        w.N0 = w.N0.astype(np.float32, order="F")
    world = 2
    slabs = [dc.Slab(w.grid.Ny, world, r) for r in range(world)]
    models = [dc.local_workload(w, s).model(precision) for s in slabs]
    st, xs = torch.cuda.Stream(), torch.cuda.Stream()
    for m in models:
        rp._lib.check(m._lib.rpl_set_stream(m.handle, rp._lib.ctypes.c_void_p(st.cuda_stream)))
    backs = [dc.LibBackend(m, st, xs) for m in models]
    Nk, Np = w.spectral_grid.coordinate_size()
    dt_t = torch.float32 if precision == "fp32" else torch.float64
    bufs = [{k: torch.zeros(Np * 3 * w.grid.Nx * Nk, dtype=dt_t, device="cuda")
             for k in ("send_low", "send_high", "recv_low", "recv_high")} for _ in slabs]

    def exchange(which):
        with torch.cuda.stream(xs):
            dc.exchange_local(backs, slabs, which, bufs)

    with torch.cuda.stream(st):
        dc.rk3_steps_overlapped(backs, slabs, exchange, w.dt, 3, smooth=w.propagation_smoothing is not None)
    got = np.concatenate([m.action.interior()[:, s.owned()] for m, s in zip(models, slabs)], axis=1)
    g = w.model(precision)
    rp.time_step(g, w.dt, 3)
    assert np.array_equal(got, g.action.interior())
    assert all(m.clock.iteration == 3 for m in models)


@pytest.mark.gpu
@pytest.mark.parametrize("case", [1, 3])
def test_one_rank_decomposed_model_equals_the_global_model(case):
    import datetime
    import torch.distributed as dist
    w = cases()[case]
    store = dist.TCPStore("127.0.0.1", _free_port(), 1, True)
    dist.init_process_group("gloo", store=store, rank=0, world_size=1, timeout=datetime.timedelta(seconds=60))
    try:
        dm = dc.DecomposedModel(w, "fp64")
        dm.step(w.dt, 3)
        got = dm.gather()
    finally:
        dist.destroy_process_group()
    g = w.model("fp64")
    rp.time_step(g, w.dt, 3)
    assert np.array_equal(got, g.action.interior())
