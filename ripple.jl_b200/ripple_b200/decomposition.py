"""Y-slab domain decomposition of the SSP-RK3 step across ranks, one GPU each, for domains larger than
one GPU's memory. The reference runs one domain per architecture; this module has no counterpart there.

Rank r owns rows [start, stop) of the global grid and keeps HALO = 3 rows on either side (the reach of
the WENO5 stencils in y: the update of row j reads rows j-3 .. j+3). Its local model is an ordinary
periodic model on stop - start + 6 rows: the stage kernels wrap around at the local array's edges,
which only corrupts halo rows, and every stage's input has its halo rows refreshed from the neighbouring
slabs (periodic in y) before the stage runs. Everything else on the path is column- or cell-local
(Q transform, stress cap, wind, coefficient records; the current gradients at the interior rows read
halo rows only), so the owned rows evolve exactly as in the undecomposed model: the interior faces,
nodes and spacings are the parent grid's own values, and the arithmetic per cell is the same.

The exchange per stage: rows are copied out of the stage's input buffer into packed device buffers
(rpl_rows_get), sent upward then downward with torch.distributed point-to-point operations (NCCL between
GPUs; gloo between CPU processes in the tests), and copied into the halo rows (rpl_rows_set).
SpatialAveraging (propagation_smoothing.jl:60-199) averages each bin's field over the corners of a
rectangle around every cell, after stage 3: stage 3 finishes without it (RPL_STAGE_DEFER_SMOOTH, its
result stays in buffer A), A's halo rows are exchanged, and the owned rows are averaged
(rpl_smooth_rows_async). The corners must stay within the 3 halo rows in y (smoothing_reach_rows < 3
for the step's dt), which holds well inside the CFL limit. Pseudomomentum coupling is not decomposed.

Overlap (rk3_steps_overlapped): an owned row r reads rows r-3 .. r+3, so the owned rows at least 3
rows from either slab edge (local rows [6, ny)) read no halo row. Each stage first launches those
rows, then exchanges the stage input's halos on a stream of its own beside that launch, then launches
the 3 + 3 boundary rows once the halos have arrived. Halo rows are not updated (their values come from
the neighbours before every use).
"""
import copy

import numpy as np

from ._lib import ArgumentError, check
from . import _lib
from .grids import RectilinearGrid
from .sources import SourceTermSet, linear_terms
from .workloads import Workload

HALO = 3


def slab_rows(Ny, world, rank):
    """Rows [start, stop) of rank `rank` in a balanced split of Ny rows."""
    return rank * Ny // world, (rank + 1) * Ny // world


class Slab:
    """Row bookkeeping of one rank: owned rows, local (halo-extended) rows, neighbours."""

    def __init__(self, Ny, world, rank, halo=HALO):
        if not 0 <= rank < world:
            raise ArgumentError("rank out of range")
        self.Ny, self.world, self.rank, self.halo = Ny, world, rank, halo
        self.start, self.stop = slab_rows(Ny, world, rank)
        self.ny = self.stop - self.start
        if self.ny < halo:
            raise ArgumentError(f"each rank needs at least {halo} rows (Ny = {Ny}, {world} ranks)")
        self.rows = self.ny + 2 * halo
        self.prev, self.next = (rank - 1) % world, (rank + 1) % world

    def global_rows(self):
        """Global row index (periodic) of every local row."""
        return np.arange(self.start - self.halo, self.stop + self.halo) % self.Ny

    # local row ranges: (first, count)
    def send_low(self):
        return self.halo, self.halo                  # lowest owned rows -> the previous rank's top halo

    def send_high(self):
        return self.ny, self.halo                    # highest owned rows -> the next rank's bottom halo

    def halo_low(self):
        return 0, self.halo

    def halo_high(self):
        return self.halo + self.ny, self.halo

    def owned(self):
        return slice(self.halo, self.halo + self.ny)


def _local_grid(grid, slab):
    """The slab's grid: the parent's x faces, y faces a + k d of the parent's uniform y axis extended past
    its ends (so interior faces are the parent's own values), the parent's spacings and z."""
    yf = grid.yfaces()
    Ny = grid.Ny
    d = (yf[-1] - yf[0]) / Ny
    if not np.allclose(np.diff(yf), d, rtol=1e-12, atol=0.0):
        raise ArgumentError("the decomposition needs a uniform y axis")
    k = np.arange(slab.start - slab.halo, slab.stop + slab.halo + 1)
    inside = (k >= 0) & (k <= Ny)
    faces = np.where(inside, yf[np.clip(k, 0, Ny)], yf[0] + k * d)
    size = (grid.Nx, slab.rows) if grid.Nz == 0 else (grid.Nx, slab.rows, grid.Nz)
    kw = dict(size=size, x=grid.xfaces(), y=faces, topology=(grid.topology[0], "Periodic", grid.topology[2]),
              first_spacings=grid.first_spacings())
    if grid.Nz:
        kw["z"] = grid.zfaces()
    return RectilinearGrid(**kw)


def local_workload(w, slab):
    """The slab's part of workload `w` (N0, depth, currents on the halo-extended rows)."""
    g = w.grid
    if g.topology[1] != "Periodic":
        raise ArgumentError("the y-slab decomposition needs a periodic y axis")
    if w.velocities is not None and not isinstance(w.velocities, dict):
        raise ArgumentError("only prescribed currents are decomposed")
    rows = slab.global_rows()
    grid = _local_grid(g, slab)
    N0 = np.asfortranarray(np.take(w.N0, rows, axis=1))
    depth = w.depth
    if not np.isscalar(depth) and type(depth).__name__ != "InfiniteDepth":
        depth = np.asfortranarray(np.take(np.asarray(depth), rows, axis=1))
    vel = None
    if w.velocities is not None:
        vel = {k: (np.asfortranarray(np.take(np.asarray(v), rows, axis=1)) if k in ("u", "v") else v)
               for k, v in w.velocities.items()}
        if "q_grid" in vel:
            raise ArgumentError("give the currents on the wave grid's own vertical grid")
    sources = w.sources
    terms = linear_terms(sources)
    if terms is not None:
        # (Nx, Ny) rate and speed arrays of SourceTermSet terms: the slab's rows (callables of (x, y) are
        # evaluated on the slab grid, whose owned rows have the parent's nodes)
        local = []
        for t in terms:
            t = copy.copy(t)
            for name in ("rate", "speed"):
                v = getattr(t, name, None)
                if isinstance(v, np.ndarray):
                    setattr(t, name, np.take(v, rows, axis=1))
            local.append(t)
        sources = SourceTermSet(*local)
    return Workload(f"{w.name}[rows {slab.start}:{slab.stop}]", grid, w.spectral_grid, depth, N0, w.dt, w.nsteps,
                    velocities=vel, sources=sources, horizontal_advection=w.horizontal_advection,
                    notes=dict(w.notes, slab=(slab.start, slab.stop)),
                    propagation_smoothing=w.propagation_smoothing)


def smoothing_reach_rows(spectral_grid, smoothing, dt, dy):
    """Largest |y offset| in rows of a SpatialAveraging corner for step dt (propagation_smoothing.jl:72-86,
    117-158): |L_s sin(phi)| + |L_n cos(phi)| over dy, L_s = alpha_s |dc_g| dt, L_n = alpha_n c_g dphi dt,
    with the deep-water c_g = sqrt(9.81 / kappa) / 2 and dc_g half its difference to the neighbouring rings."""
    kappa = np.asarray(spectral_grid.κ, dtype=np.float64)
    phi = np.asarray(spectral_grid.φ, dtype=np.float64)
    pf = np.asarray(spectral_grid.φ_faces, dtype=np.float64)
    cg = 0.5 * np.sqrt(9.81 / kappa)
    lo = np.concatenate([cg[:1], cg[:-1]])
    hi = np.concatenate([cg[1:], cg[-1:]])
    dcg = np.abs(lo - hi) / 2.0
    Ls = smoothing.αs * dcg * dt
    Ln = smoothing.αn * cg * (pf[1] - pf[0]) * dt
    reach = np.abs(Ls[:, None] * np.sin(phi)[None, :]) + np.abs(Ln[:, None] * np.cos(phi)[None, :])
    return float(np.max(reach)) / float(dy)


def check_smoothing_reach(w, dt, halo=HALO):
    """ArgumentError when the averaging's corners would read beyond the halo rows for step dt."""
    if w.propagation_smoothing is None:
        return
    yf = w.grid.yfaces()
    dy = (yf[-1] - yf[0]) / w.grid.Ny
    r = smoothing_reach_rows(w.spectral_grid, w.propagation_smoothing, dt, dy)
    if not r < halo:
        raise ArgumentError(f"SpatialAveraging corners reach {r:.3g} rows at dt = {dt}, beyond the {halo} halo rows "
                            "of the y-slab decomposition")


def interior_rows(slab):
    """Local rows [first, stop) whose update reads no halo row (may be empty)."""
    h, ny = slab.halo, slab.ny
    lo = min(2 * h, h + ny)
    return lo, max(ny, lo)


def boundary_rows(slab):
    """The two local row ranges [first, stop) of owned rows that read the low and the high halo."""
    h, ny = slab.halo, slab.ny
    lo, hi = interior_rows(slab)
    return (h, lo), (hi, h + ny)


class LibBackend:
    """The slab's model in librpl.so: row copies and (partial) stages on the handle's stream; with an
    exchange stream, the row copies of an exchange run on it between begin_exchange and end_exchange."""

    def __init__(self, model, compute_stream=None, exchange_stream=None):
        self.model = model
        self.lib, self.h = model._lib, model.handle
        self.compute, self.xstream = compute_stream, exchange_stream
        if exchange_stream is not None:
            import torch
            self.ev_in = torch.cuda.Event()
            self.ev_x = torch.cuda.Event()

    def _stream_arg(self):
        return _lib.ctypes.c_void_p(self.xstream.cuda_stream)

    def rows_get(self, which, first, count, buf):
        ptr = _lib.ctypes.c_void_p(buf.data_ptr())
        if self.xstream is not None:
            check(self.lib.rpl_rows_get_on(self.h, which, first, count, ptr, self._stream_arg()))
        else:
            check(self.lib.rpl_rows_get(self.h, which, first, count, ptr))

    def rows_set(self, which, first, count, buf):
        ptr = _lib.ctypes.c_void_p(buf.data_ptr())
        if self.xstream is not None:
            check(self.lib.rpl_rows_set_on(self.h, which, first, count, ptr, self._stream_arg()))
        else:
            check(self.lib.rpl_rows_set(self.h, which, first, count, ptr))

    def stage(self, dt, s, defer_smooth=False):
        if defer_smooth:
            flags = _lib.RPL_STAGE_PREPARE | _lib.RPL_STAGE_FINISH | _lib.RPL_STAGE_DEFER_SMOOTH
            check(self.lib.rpl_stage_rows_async(self.h, float(dt), int(s), 0, int(self.model.grid.Ny), flags))
        else:
            check(self.lib.rpl_stage_async(self.h, float(dt), int(s)))

    def stage_rows(self, dt, s, first, count, prepare, finish, defer_smooth=False):
        flags = ((_lib.RPL_STAGE_PREPARE if prepare else 0) | (_lib.RPL_STAGE_FINISH if finish else 0) |
                 (_lib.RPL_STAGE_DEFER_SMOOTH if defer_smooth else 0))
        check(self.lib.rpl_stage_rows_async(self.h, float(dt), int(s), int(first), int(count), flags))

    def smooth_rows(self, dt, first, count, y_offset=0):
        check(self.lib.rpl_smooth_rows_async(self.h, float(dt), int(first), int(count), int(y_offset)))

    def mark_input(self):
        """The stage's input is final on the compute stream (before the interior launch)."""
        if self.xstream is not None:
            self.ev_in.record(self.compute)

    def begin_exchange(self):
        if self.xstream is not None:
            self.xstream.wait_event(self.ev_in)

    def end_exchange(self):
        if self.xstream is not None:
            self.ev_x.record(self.xstream)
            self.compute.wait_event(self.ev_x)

    def sync(self):
        check(self.lib.rpl_sync(self.h))
        self.model._sync_clock()


def _buffers(slab, Nx, Nk, Np, dtype, device):
    import torch
    n = Np * slab.halo * Nx * Nk
    return {k: torch.empty(n, dtype=dtype, device=device) for k in ("send_low", "send_high", "recv_low", "recv_high")}


def exchange_dist(backend, slab, which, bufs, group=None, stream=None):
    """Refresh the halo rows of buffer `which` from the neighbouring ranks: owned high rows go up to the
    next rank's bottom halo, then owned low rows go down to the previous rank's top halo. Each phase is
    one send and one receive per rank, so ranks that are each other's previous and next (two ranks) pair
    their messages unambiguously. With `stream` (a torch CUDA stream) the copies and the point-to-point
    operations are enqueued on it."""
    if stream is not None:
        import torch
        with torch.cuda.stream(stream):
            return exchange_dist(backend, slab, which, bufs, group)
    import torch.distributed as dist
    backend.rows_get(which, *slab.send_low(), bufs["send_low"])
    backend.rows_get(which, *slab.send_high(), bufs["send_high"])
    if slab.world == 1:
        bufs["recv_low"].copy_(bufs["send_high"])
        bufs["recv_high"].copy_(bufs["send_low"])
    else:
        for send, dst, recv, src in ((bufs["send_high"], slab.next, bufs["recv_low"], slab.prev),
                                     (bufs["send_low"], slab.prev, bufs["recv_high"], slab.next)):
            ops = [dist.P2POp(dist.isend, send, dst, group), dist.P2POp(dist.irecv, recv, src, group)]
            for r in dist.batch_isend_irecv(ops):
                r.wait()
    backend.rows_set(which, *slab.halo_low(), bufs["recv_low"])
    backend.rows_set(which, *slab.halo_high(), bufs["recv_high"])


def exchange_local(backends, slabs, which, bufs):
    """The same exchange for all slabs held by one process (one GPU emulating the ranks in turn; no
    kernel waits for another)."""
    for b, s, q in zip(backends, slabs, bufs):
        b.rows_get(which, *s.send_low(), q["send_low"])
        b.rows_get(which, *s.send_high(), q["send_high"])
    for b, s, q in zip(backends, slabs, bufs):
        q["recv_low"].copy_(bufs[s.prev]["send_high"])
        q["recv_high"].copy_(bufs[s.next]["send_low"])
    for b, s, q in zip(backends, slabs, bufs):
        b.rows_set(which, *s.halo_low(), q["recv_low"])
        b.rows_set(which, *s.halo_high(), q["recv_high"])


def _smooth(backends, slabs, exchange, dt):
    """SpatialAveraging of a decomposed step: stage 3's result (buffer A) gets its halo rows from the
    neighbours, then every slab averages its owned rows into N."""
    for b in backends:
        b.mark_input()
        b.begin_exchange()
    exchange(1)
    for b, sl in zip(backends, slabs):
        b.end_exchange()
        b.smooth_rows(dt, sl.halo, sl.ny, sl.start - sl.halo)


def rk3_steps_overlapped(backends, slabs, exchange, dt, nsteps, before_step=None, smooth=False):
    """nsteps decomposed SSP-RK3 steps with the exchange beside the interior rows: per stage every slab
    launches its interior rows (with the stage's preparation kernels), the halos of the stage's input
    are exchanged (exchange(which), between the backends' begin_exchange and end_exchange), then every
    slab launches its two boundary row ranges (the last one finishes the stage). smooth: the models have
    SpatialAveraging, applied after stage 3 (see _smooth)."""
    for _ in range(nsteps):
        if before_step is not None:
            before_step()
        for s, which in ((1, 0), (2, 1), (3, 2)):
            for b, sl in zip(backends, slabs):
                b.mark_input()
                lo, hi = interior_rows(sl)
                b.stage_rows(dt, s, lo, hi - lo, True, False)
            for b in backends:
                b.begin_exchange()
            exchange(which)
            for b, sl in zip(backends, slabs):
                b.end_exchange()
                (l0, l1), (h0, h1) = boundary_rows(sl)
                b.stage_rows(dt, s, l0, l1 - l0, False, False)
                b.stage_rows(dt, s, h0, h1 - h0, False, True, defer_smooth=smooth and s == 3)
        if smooth:
            _smooth(backends, slabs, exchange, dt)
    for b in backends:
        b.sync()


def rk3_steps(backends, exchange, dt, nsteps, before_step=None, slabs=None):
    """nsteps decomposed SSP-RK3 steps: before stage s the halo rows of its input buffer (N, A, B) are
    exchanged, then every slab runs the stage. slabs (given for models with SpatialAveraging): the
    averaging after stage 3 (see _smooth)."""
    for _ in range(nsteps):
        if before_step is not None:
            before_step()
        for s, which in ((1, 0), (2, 1), (3, 2)):
            exchange(which)
            for b in backends:
                b.stage(dt, s, defer_smooth=slabs is not None and s == 3)
        if slabs is not None:
            _smooth(backends, slabs, exchange, dt)
    for b in backends:
        b.sync()


class DecomposedModel:
    """This rank's slab of a workload, advanced with halo exchanges over torch.distributed (one process
    per GPU, NCCL). interior() is the owned rows' action; gather() assembles the global field on rank 0."""

    def __init__(self, w, precision="fp64", group=None, device=0, overlap=True):
        import torch
        import torch.distributed as dist
        self.group = group
        world, rank = dist.get_world_size(group), dist.get_rank(group)
        self.slab = Slab(w.grid.Ny, world, rank)
        self.local = local_workload(w, self.slab)
        self.model = self.local.model(precision, device=device)
        # a stream for the library's kernels (of its own: the legacy default stream does not order against
        # the library's non-blocking streams); with overlap, the exchange runs on a second stream
        self.stream = torch.cuda.Stream(device)
        check(self.model._lib.rpl_set_stream(self.model.handle, _lib.ctypes.c_void_p(self.stream.cuda_stream)))
        self.overlap = overlap
        self.xstream = torch.cuda.Stream(device) if overlap else None
        self.backend = LibBackend(self.model, self.stream, self.xstream)
        Nk, Np = w.spectral_grid.coordinate_size()
        self.bufs = _buffers(self.slab, w.grid.Nx, Nk, Np, torch.float32 if precision == "fp32" else torch.float64,
                             f"cuda:{device}")

    def step(self, dt, nsteps=1):
        import torch
        m = self.model
        check(m._lib.rpl_set_clock(m.handle, m.clock.time, m.clock.iteration))
        before = m._push_field_wind if m._field_wind is not None else None
        check_smoothing_reach(self.local, dt)
        smooth = self.local.propagation_smoothing is not None
        with torch.cuda.stream(self.stream):
            if self.overlap:
                rk3_steps_overlapped([self.backend], [self.slab],
                                     lambda which: exchange_dist(self.backend, self.slab, which, self.bufs,
                                                                 self.group, self.xstream),
                                     dt, nsteps, before_step=before, smooth=smooth)
            else:
                rk3_steps([self.backend],
                          lambda which: exchange_dist(self.backend, self.slab, which, self.bufs, self.group),
                          dt, nsteps, before_step=before, slabs=[self.slab] if smooth else None)
        m.clock.last_Δt = dt
        return self

    def interior(self):
        return self.model.action.interior()[:, self.slab.owned()]

    def gather(self):
        import torch.distributed as dist
        parts = [None] * self.slab.world
        dist.all_gather_object(parts, (self.slab.start, self.interior()), group=self.group)
        return np.concatenate([p for _, p in sorted(parts, key=lambda t: t[0])], axis=1)
