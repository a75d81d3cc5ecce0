"""Benchmark: cell-bin SSP-RK3 updates per second of the seamount-eddies (default) or hurricane-swell
workload on B200.

Default workload: 1024^2 grid (5 km, periodic), 32 vertical levels for the Q-transform,
32 log-spaced kappa x 36 directions, seeded seamount depth and eddy currents, FP32
state with FP64 tables (the precision form). One step = one SSP-RK3 step over all
1.21e9 cell-bins. `value` is device-timed with the state resident in HBM; `e2e` runs
the same steps through the public API (set!, time_step!, a per-step total-action
read, interior) with pinned host buffers. --impl reference times the reference's CPU
path (the FP64 C++ restatement) on the host cores instead.

--workload hurricane: 768^2 grid (10 km), 32 kappa x 36 directions, 4000 m depth, moving Holland
hurricane with Janssen wind input (wave-supported stress cap) and local-saturation whitecapping.

--workload selfcoupled: PseudomomentumVelocities on a 1024^2 grid (2 km, Flat, periodic), 32 kappa x
36 directions, 50 m depth: a swell packet whose Doppler velocity is recomputed from every stage's
action (overlap moments + gradients, then the fused refraction stage).

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision fp32|fp64]
               [--workload seamount|hurricane] [--size N]
Under torchrun each rank advances its own copy of the workload (independent replicas).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ripple.jl_b200"))

import numpy as np  # noqa: E402

METRIC = "cell·bin RK3 updates/s on 1 B200, FP32/learned vs plain FP64, at stated rel-L2"
UNIT = "cell·bin updates/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--workload", default="seamount", choices=["seamount", "hurricane", "ensemble", "learned",
                                                                       "selfcoupled", "mlp"])
    ap.add_argument("--rows", type=int, default=65536,
                    help="network rows per forward pass (--workload mlp: the learned source's GEMMs alone)")
    ap.add_argument("--train-steps", type=int, default=40000, help="Adam steps (--workload learned)")
    ap.add_argument("--snapshots", type=int, default=40, help="training snapshots per storm run (--workload learned)")
    ap.add_argument("--dagger", type=int, default=0,
                    help="rounds of rows collected along learned-source runs, labelled by the plain sources (--workload learned)")
    ap.add_argument("--feature-pad", type=float, default=0.25,
                    help="absolute widening of the per-bin log-action input bounds beyond the training rows, in "
                         "feature units (x 4 in log N); a cell outside the bounds uses the plain sources "
                         "(--workload learned)")
    ap.add_argument("--learned-gate", type=float, default=0.02,
                    help="trust gate of the learned source: cells whose network rates exceed this fraction of "
                         "the action per step use the plain sources (0: off; --workload learned)")
    ap.add_argument("--calm-fraction", type=float, default=0.05,
                    help="share of cells without source activity kept as training rows (--workload learned)")
    ap.add_argument("--members", type=int, default=64, help="ensemble members (--workload ensemble)")
    ap.add_argument("--autotune-cache", default="", help="tile-shape cache file (--workload ensemble)")
    ap.add_argument("--direct-cells", type=int, default=65536,
                    help="ensemble members of at least this many cells take their own single-model stage launches "
                         "inside the captured step; 0: all members in the persistent launches (--workload ensemble)")
    ap.add_argument("--member-sizes", default="64,128,256,384",
                    help="grid sizes the ensemble members are drawn from (--workload ensemble)")
    ap.add_argument("--size", type=int, default=0, help="grid points per side (default 1024 / 768)")
    ap.add_argument("--refresh-currents", action="store_true",
                    help="time-varying currents (--workload seamount): new u, v every step, projected again "
                         "(rpl_update_currents_device in the timed region; from pinned host buffers in e2e)")
    ap.add_argument("--output-every", type=int, default=0,
                    help="output during the timed steps: diagnostics into a device time series every step and an "
                         "asynchronous snapshot of the action to pinned host memory every K steps")
    ap.add_argument("--smoothing", action="store_true",
                    help="propagation_smoothing = SpatialAveraging() after every step (the reference's hurricane example)")
    ap.add_argument("--decompose", action="store_true",
                    help="one domain split into y slabs over the --gpus ranks with halo exchanges before every RK3 "
                         "stage (strong scaling); on one GPU it measures the exchange machinery's cost")
    ap.add_argument("--accuracy-steps", type=int, default=-1,
                    help="FP32 precision form: steps of the accuracy arm (FP32 and FP64 runs from the same start, "
                         "compared on the device); -1: the configuration's own step count, 0: off")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.size <= 0:
        args.size = 1024 if args.workload in ("seamount", "ensemble", "selfcoupled") else 768
    return args


CONFIG_STEPS = {"seamount": 200, "hurricane": 1000, "selfcoupled": 200}   # RK3 steps of each configuration
WORKLOAD_NAMES = {"seamount": "seamount_eddies", "hurricane": "hurricane_swell", "ensemble": "ensemble_members",
                  "learned": "hurricane_swell (learned source)", "selfcoupled": "self_coupled_swell"}
TRAFFIC_SUFFIX = {"seamount": "", "hurricane": "_hurricane", "selfcoupled": "_selfcoupled"}
# the FP32 stage kernels each workload runs (refraction: two passes per stage; intrinsic: one fused kernel)
STAGE_KERNELS = {"seamount": "xyw_kernel+kq_kernel", "hurricane": "xyw_kernel+ks_kernel",
                 "selfcoupled": "xyw_kernel+kq_kernel"}
DATA = {"seamount": "synthetic (seeded seamount depth, eddy currents, JONSWAP-like N0)",
        "hurricane": "synthetic (Holland hurricane on a linear track, uniform N0 = 1e-6)",
        "selfcoupled": "synthetic (Gaussian swell packet, 50 m depth, pseudomomentum self-coupling)"}


def make_workload(name, n, nsteps, n0_dtype=np.float64):
    from ripple_b200 import workloads
    if name == "ensemble":
        # the CPU sample of the ensemble: its 32 kappa x 36 direction physics on an n^2 member grid
        return workloads.seamount_eddies(N=n, Nz=16, Nk=32, Np=36, nsteps=nsteps, seed=4, L=n * 5000.0,
                                         n0_dtype=n0_dtype)
    if name == "seamount":
        return workloads.seamount_eddies(N=n, Nz=32, Nk=32, Np=36, nsteps=nsteps, n0_dtype=n0_dtype)
    if name == "selfcoupled":
        return workloads.self_coupled_swell(N=n, Nk=32, Np=36, nsteps=nsteps, n0_dtype=n0_dtype)
    w = workloads.hurricane_swell(N=n, Nk=32, Np=36, nsteps=nsteps)
    if n0_dtype != np.float64:
        w.N0 = w.N0.astype(n0_dtype, order="F")
    return w


def launches_per_step(name, precision="fp32"):
    """Our kernels per RK3 step. A stage is two launches in FP32 (refraction: the x/y flux pass, then the
    kappa/phi pass with the stage update; the hurricane's intrinsic transport with the bundle sources: the
    x/y pass, then the sources and the update) and one fused launch in FP64; the hurricane adds 1 wind + 3
    stress-cap kernels; the self-coupled swell adds 2 coupling kernels per stage, and in FP32 the refresh
    of the velocity planes of the x/y pass."""
    per_stage = 2 if precision == "fp32" else 1
    coupling = 3 if precision == "fp32" else 2
    return {"seamount": 3 * per_stage, "selfcoupled": 3 * (per_stage + coupling)}.get(name, 3 * per_stage + 4)


def current_launches(precision):
    """Kernels of one update of time-varying currents: Q transform, gradients, coefficient records, and
    in FP32 the velocity planes of the x/y pass."""
    return 4 if precision == "fp32" else 3


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            with open(self.f.name) as f:
                for line in f:
                    parts = [x.strip() for x in line.split(",")]
                    if len(parts) >= 9:
                        rows.append(parts)
        finally:
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        busy = [s for s in sm if mx and s > 0.5 * max(mx)] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(w, precision):
    """Per RK3 step: 8 state words per unit (N0->N1; N1,N0->N2; N2,N0->N3) + per stage the FP64
    per-(i,j,kappa) tables (Ux, Uy, 4 gradients, and c_g when depth varies) amortised over phi.
    With a stress-capped wind source, each stage also reads its input once for the cap (one state
    word per unit) and the per-(i,j) wind record (32 bytes, amortised over kappa and phi)."""
    s = 4 if precision == "fp32" else 8
    Nk, Np = w.spectral_grid.coordinate_size()
    c_d = 0 if np.isscalar(w.depth) or type(w.depth).__name__ == "InfiniteDepth" else 1
    tables = 3 * (6 + c_d) * 8 * (w.units // Np) if w.velocities is not None else 3 * c_d * 8 * (w.units // Np)
    extra = 0
    if w.sources is not None:
        cols = w.units // (Nk * Np)
        extra = 3 * (s * w.units + 2 * 32 * cols)
    if type(w.velocities).__name__ == "PseudomomentumVelocities":
        # per stage the coupling refresh reads the state once and writes/reads the velocity (32 B) and
        # rewrites six coefficient fields (48 B) per (i,j,kappa)
        extra += 3 * (s * w.units + 96 * (w.units // Np))
    return 8 * s * w.units + tables + extra


CPU_GRID = 96          # CPU sample grid: the workload's physics and spectral grid on 96^2 cells


def cpu_sample(name, steps, warmup=1, threads=None, n=CPU_GRID):
    """The reference CPU path (the oracle: FP64 C++ restatement, OpenMP over columns) on a bounded
    sample of the workload: `warmup` untimed then `steps` timed RK3 steps on an n^2 grid with the same
    physics and spectral grid. threads=None: every host thread OpenMP offers. Returns (units/s, s,
    threads used, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    full = oracle.num_threads()
    oracle.set_threads(threads or full)
    try:
        w = make_workload(name, n, steps)
        o = oracle.Oracle(w)
        N = w.N0
        for _ in range(warmup):
            N, _ = o.step(N, w.dt, 1)
        t = time.perf_counter()
        for _ in range(steps):
            N, _ = o.step(N, w.dt, 1)
        el = time.perf_counter() - t
        used = oracle.num_threads()
    finally:
        oracle.set_threads(full)
    sample = (f"{WORKLOAD_NAMES[name]} at {n}^2 x 32 kappa x 36 phi (same physics, reduced grid), "
              f"{steps} FP64 RK3 steps after {warmup} warm-up, {used} thread(s), {el:.1f} s")
    return w.units * steps / el, el, used, sample


def cpu_baseline(name, steps):
    """cpu_baseline of the GPU line: the same sample as the --impl reference arm (same grid, same step
    count) on all host threads, plus a shorter 1-thread sample."""
    v, el, used, sample = cpu_sample(name, steps)
    v1, el1, _, sample1 = cpu_sample(name, max(1, min(2, steps)), threads=1)
    return {"value": v, "unit": UNIT, "cores": used, "kind": "port", "sample": sample,
            "one_thread": {"value": v1, "unit": UNIT, "cores": 1, "sample": sample1}}


def run_reference(args, rank):
    if rank != 0:
        return
    value, el, used, sample = cpu_sample(args.workload, args.steps, warmup=args.warmup)
    sample += f" ({args.size}^2 does not fit a bounded CPU sample); per-unit throughput"
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference",
            "config": {"workload": WORKLOAD_NAMES[args.workload], "grid": [CPU_GRID, CPU_GRID], "spectral": [32, 36],
                       "precision": "fp64", "path": "reference CPU path restated in C++ (oracle/), OpenMP"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": used, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def device_state(m, precision, torch, _lib):
    """The model's action as a CUDA tensor, caller layout (x fastest)."""
    t = torch.empty(m.action.size if isinstance(m.action.size, int) else int(np.prod(m.action.size)),
                    dtype=torch.float32 if precision == "fp32" else torch.float64, device=f"cuda:{m.device}")
    _lib.check(m._lib.rpl_get_action_device(m.handle, _lib.ctypes.c_void_p(t.data_ptr()),
                                            _lib.RPL_F32 if precision == "fp32" else _lib.RPL_F64, 0))
    return t


def rel_l2_device(a, b, torch, chunk=1 << 27):
    num = den = 0.0
    for s in range(0, a.numel(), chunk):
        x, y = a[s:s + chunk].double(), b[s:s + chunk].double()
        num += float(torch.sum((x - y) ** 2))
        den += float(torch.sum(y * y))
    return math.sqrt(num / den)


def accuracy_arm(w, steps, local_rank):
    """The precision form against the plain FP64 GPU path (pinned to the CPU oracle on reduced grids):
    FP32 and FP64 models run `steps` RK3 steps from the same initial action; the last steps - 3 of each
    are device-timed (CUDA events on the model's stream); final actions, Hs and total actions are
    compared on the device. Drift = change of the total action over the run / its initial value."""
    import torch
    import ripple_b200 as rp
    from ripple_b200 import _lib
    warm = min(3, max(0, steps - 1))
    res = {}
    for prec in ("fp32", "fp64"):
        m = w.model(prec, device=local_rank)
        stream = torch.cuda.Stream(device=local_rank)
        _lib.check(m._lib.rpl_set_stream(m.handle, _lib.ctypes.c_void_p(stream.cuda_stream)))
        t0 = rp.total_action(m.action)
        _lib.check(m._lib.rpl_step_async(m.handle, w.dt, warm))
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        _lib.check(m._lib.rpl_step_async(m.handle, w.dt, steps - warm))
        b.record(stream)
        stream.synchronize()
        _lib.check(m._lib.rpl_sync(m.handle))
        m._sync_clock()
        d = rp.diagnostics(m.action)
        res[prec] = dict(ms=a.elapsed_time(b) / (steps - warm), N=device_state(m, prec, torch, _lib), Hs=d["Hs"],
                         t0=t0, t1=d["total_action"])
        m.close()
    f, g = res["fp32"], res["fp64"]
    out = {"steps": steps, "timed_steps": steps - warm,
           "rel_l2_vs_fp64": rel_l2_device(f["N"], g["N"], torch),
           "hs_rel_l2_vs_fp64": float(np.linalg.norm(f["Hs"] - g["Hs"]) / np.linalg.norm(g["Hs"])),
           "total_action_rel_diff_vs_fp64": abs(f["t1"] - g["t1"]) / abs(g["t1"]),
           "action_drift": (f["t1"] - f["t0"]) / f["t0"], "action_drift_fp64": (g["t1"] - g["t0"]) / g["t0"],
           "fp32_ms_per_step": f["ms"], "fp64_ms_per_step": g["ms"],
           "reference": "plain FP64 GPU path, pinned to the CPU FP64 oracle at <= 1e-12 (128^2, 20 steps)"}
    del res
    torch.cuda.empty_cache()
    return out


def run_ours(args, rank, world, local_rank):
    import torch
    import ripple_b200 as rp
    from ripple_b200 import _lib

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    try:
        smi_id = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        smi_id = str(local_rank)
    w = make_workload(args.workload, args.size, args.steps,
                      n0_dtype=np.float32 if args.precision == "fp32" else np.float64)
    if args.smoothing:
        w.propagation_smoothing = rp.SpatialAveraging()
    m = w.model(args.precision, device=local_rank)
    lib, h = m._lib, m.handle
    torch_stream = torch.cuda.Stream(device=local_rank)
    _lib.check(lib.rpl_set_stream(h, _lib.ctypes.c_void_p(torch_stream.cuda_stream)))
    dt = w.dt

    # time-varying currents: two current fields (the workload's and a rotated, rescaled copy), device
    # resident with x fastest, alternated step by step
    cur = None
    if args.refresh_currents:
        if not isinstance(w.velocities, dict):
            raise SystemExit("--refresh-currents needs a workload with prescribed currents")
        Nx, Ny, Nz = np.shape(w.velocities["u"])
        host_cur = []
        for k in range(2):
            c, sn, a = math.cos(0.5 * k), math.sin(0.5 * k), 1.0 + 0.2 * k
            u0, v0 = np.asarray(w.velocities["u"]), np.asarray(w.velocities["v"])
            pair = []
            for arr in (a * (c * u0 - sn * v0), a * (sn * u0 + c * v0)):
                t = torch.empty(arr.size, dtype=torch.float64, pin_memory=True)
                t.numpy()[:] = np.ravel(arr, order="F")
                pair.append(t)
            host_cur.append(pair)
        cur = [[t.to(f"cuda:{local_rank}") for t in pair] for pair in host_cur]
        torch.cuda.synchronize()

    def refresh(k):
        _lib.check(lib.rpl_update_currents_device(h, _lib.ctypes.c_void_p(cur[k % 2][0].data_ptr()),
                                                  _lib.ctypes.c_void_p(cur[k % 2][1].data_ptr())))

    # output: two pinned snapshot buffers used in turn, a device time series of the total action
    snap_bufs, series = None, None
    if args.output_every > 0:
        snap_bufs = [rp.HostBuffer(m.action.size, np.float32 if args.precision == "fp32" else np.float64)
                     for _ in range(2)]
        series = torch.zeros(max(args.steps, 1), dtype=torch.float64, device=f"cuda:{local_rank}")
        torch.cuda.synchronize()

    def output(k):
        _lib.check(lib.rpl_diagnostics_device(h, None, None, None, None,
                                              _lib.ctypes.c_void_p(series[k:k + 1].data_ptr())))
        if (k + 1) % args.output_every == 0:
            buf = snap_bufs[(k // args.output_every) % 2]
            _lib.check(lib.rpl_snapshot_async(h, buf.ptr, _lib.RPL_F32 if args.precision == "fp32" else _lib.RPL_F64))

    # warm-up
    for k in range(args.warmup):
        if cur is not None:
            refresh(k)
        _lib.check(lib.rpl_step_async(h, dt, 1))
        if snap_bufs is not None:
            output(0)
    _lib.check(lib.rpl_sync(h))
    if snap_bufs is not None:
        _lib.check(lib.rpl_snapshot_wait(h))
    barrier()

    # device-timed region: K steps, events around each stage launch on the launching stream
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    rev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(smi_id) as clk:
        barrier()
        with torch.cuda.stream(torch_stream):
            start.record(torch_stream)
            for k in range(args.steps):
                if cur is not None:
                    rev[k].record(torch_stream)
                    refresh(k)
                ev[k][0].record(torch_stream)
                for s in (1, 2, 3):
                    _lib.check(lib.rpl_stage_async(h, dt, s))
                    ev[k][s].record(torch_stream)
                if snap_bufs is not None:
                    output(k)
            end.record(torch_stream)
        torch_stream.synchronize()
        _lib.check(lib.rpl_sync(h))
        if snap_bufs is not None:
            t_wait = time.perf_counter()
            _lib.check(lib.rpl_snapshot_wait(h))
            snap_tail_ms = 1e3 * (time.perf_counter() - t_wait)
        barrier()
    ms = start.elapsed_time(end)
    stage_ms = [ev[k][s].elapsed_time(ev[k][s + 1]) for k in range(args.steps) for s in range(3)]
    refresh_ms = statistics.mean(rev[k].elapsed_time(ev[k][0]) for k in range(args.steps)) if cur else None
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    clocks = clk.summary()
    value = world * w.units * args.steps / (ms / 1e3)

    # roofline of the dominant kernel (the fused stage kernel: one launch per RK3 stage)
    peak, peak_kind = peaks()
    launch_ms = statistics.mean(stage_ms)
    bytes_per_launch = algorithmic_bytes(w, args.precision) / 3.0
    achieved = bytes_per_launch / (launch_ms / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "stage_traffic.json")
    if os.path.exists(tp):
        try:
            key = f"{args.precision}_{args.size}" + TRAFFIC_SUFFIX[args.workload]
            traffic = json.load(open(tp)).get(key)
        except Exception:
            traffic = None

    # end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        host = torch.empty(w.units, dtype=torch.float32 if args.precision == "fp32" else torch.float64,
                           pin_memory=True)
        hv = host.numpy()
        hv[:] = np.ravel(w.N0, order="F")
        tot = np.zeros(1)
        barrier()
        t0 = time.perf_counter()
        _lib.check(lib.rpl_set_action(h, _lib.ctypes.c_void_p(host.data_ptr()),
                                      _lib.RPL_F32 if args.precision == "fp32" else _lib.RPL_F64, 0))
        for k in range(args.steps):
            if cur is not None:
                _lib.check(lib.rpl_update_currents(h, _lib.dptr(host_cur[k % 2][0].numpy()),
                                                   _lib.dptr(host_cur[k % 2][1].numpy())))
            _lib.check(lib.rpl_step(h, dt, 1))
            _lib.check(lib.rpl_diagnostics(h, None, None, None, None, _lib.dptr(tot)))
        _lib.check(lib.rpl_get_action(h, _lib.ctypes.c_void_p(host.data_ptr()),
                                      _lib.RPL_F32 if args.precision == "fp32" else _lib.RPL_F64, 0))
        el = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        nbytes = host.numel() * host.element_size()
        cur_bytes = 2 * host_cur[0][0].numel() * 8 if cur is not None else 0
        e2e = {"value": world * w.units * args.steps / el, "unit": UNIT,
               "h2d_bytes_per_step": nbytes / args.steps + cur_bytes,
               "d2h_bytes_per_step": (nbytes + 8 * args.steps) / args.steps,
               "includes": "set! from pinned host, K x (" + ("new currents from pinned host + " if cur else "") +
                           "time_step! + total_action read), interior to pinned host"}

    m.close()
    acc = None
    acc_steps = CONFIG_STEPS.get(args.workload, 0) if args.accuracy_steps < 0 else args.accuracy_steps
    if args.precision == "fp32" and acc_steps > 0 and not (cur or snap_bufs or args.smoothing):
        acc = accuracy_arm(w, acc_steps, local_rank)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args.workload, args.steps)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": DATA[args.workload],
            "config": {"workload": WORKLOAD_NAMES[args.workload], "grid": [args.size, args.size],
                       "spectral": [32, 36],
                       "precision": args.precision, "units_per_step": w.units, "dt": dt,
                       "l2": "state (%.1f GB per buffer) larger than L2; no flush" % (w.units * (4 if args.precision == "fp32" else 8) / 1e9),
                       "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU",
                       **({"currents": "time-varying: new u, v every step (Q transform + gradients + coefficients "
                                       "in the timed region)", "currents_refresh_ms": refresh_ms} if cur else {}),
                       **({"propagation_smoothing": "SpatialAveraging(αs=0.5, αn=0.5) after every step"}
                          if args.smoothing else {}),
                       **({"output": {"diagnostics": "total action into a device time series every step",
                                      "snapshot_every": args.output_every,
                                      "snapshot_bytes": snap_bufs[0].array.nbytes,
                                      "snapshot_copy_after_timed_region_ms": snap_tail_ms}}
                          if snap_bufs is not None else {})},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": STAGE_KERNELS[args.workload] if args.precision == "fp32" else "column_kernel",
                         "launch_ms": launch_ms, "algorithmic_bytes_per_launch": bytes_per_launch,
                         "launch_interval": "one RK3 stage" + {"seamount": "",
                                                               "selfcoupled": " incl. its coupling refresh"}.get(
                                                                   args.workload, " incl. its wind/stress-cap kernels")},
            "cpu_baseline": cpu, "e2e": e2e,
            **({"rel_l2_vs_fp64": acc["rel_l2_vs_fp64"], "action_drift": acc["action_drift"],
                "fp64_ms_per_step": acc["fp64_ms_per_step"],
                "speedup_vs_fp64": acc["fp64_ms_per_step"] / (ms / args.steps), "accuracy": acc} if acc else {}),
            "gpu_launches": (launches_per_step(args.workload, args.precision) + (current_launches(args.precision) if cur else 0) + (2 if snap_bufs else 0)
                             + (1 if args.smoothing else 0)) * args.steps
                            + (args.steps // args.output_every if snap_bufs else 0),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_ensemble(args, rank, world, local_rank):
    """The batching form: `--members` seeded members of uneven grids, one persistent launch per stage,
    one CUDA graph per RK3 step; timed beside the same steps as per-member sequential launches."""
    import torch
    import ripple_b200 as rp
    from ripple_b200 import _lib, workloads

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    try:
        smi_id = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        smi_id = str(local_rank)
    models, dts, nbytes_alg, shapes_info = [], [], 0.0, []
    t_build = time.perf_counter()
    sizes = tuple(int(x) for x in args.member_sizes.split(","))
    for w in workloads.ensemble_members(count=args.members, seed=4, nsteps=args.steps, sizes=sizes):
        m = w.model("fp32", device=local_rank)
        models.append(m)
        dts.append(w.dt)
        nbytes_alg += algorithmic_bytes(w, "fp32")
        shapes_info.append((w.grid.Nx, w.spectral_grid.coordinate_size()))
        w.N0 = None
    t_build = time.perf_counter() - t_build
    cache = args.autotune_cache or None
    t_tune = time.perf_counter()
    ens = rp.Ensemble(models, dts, use_graph=True, autotune=True, autotune_cache=cache, direct_cells=args.direct_cells)
    t_tune = time.perf_counter() - t_tune
    lib, h = ens._lib, ens.handle
    units = ens.units
    stream = torch.cuda.Stream(device=local_rank)
    _lib.check(lib.rpl_ensemble_set_stream(h, _lib.ctypes.c_void_p(stream.cuda_stream)))

    def timed(step_fn, k):
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        with torch.cuda.stream(stream):
            start.record(stream)
            _lib.check(step_fn(h, k))
            end.record(stream)
        stream.synchronize()
        _lib.check(lib.rpl_ensemble_sync(h))
        barrier()
        ms = start.elapsed_time(end)
        if dist is not None:
            t = torch.tensor([ms], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    _lib.check(lib.rpl_ensemble_step_async(h, args.warmup))
    _lib.check(lib.rpl_ensemble_sync(h))
    with ClockSampler(smi_id) as clk:
        ms = timed(lib.rpl_ensemble_step_async, args.steps)
    clocks = clk.summary()
    _lib.check(lib.rpl_ensemble_step_sequential_async(h, args.warmup))
    _lib.check(lib.rpl_ensemble_sync(h))
    ms_seq = timed(lib.rpl_ensemble_step_sequential_async, args.steps)
    value = world * units * args.steps / (ms / 1e3)
    peak, peak_kind = peaks()
    launch_ms = ms / args.steps / 3.0
    achieved = nbytes_alg / 3.0 / (launch_ms / 1e3) / 1e9

    e2e = None
    if not args.no_e2e:
        # one pinned buffer holding every member's state back to back (filled untimed from the devices)
        host = torch.empty(units, dtype=torch.float32, pin_memory=True)
        offs = np.cumsum([0] + [int(np.prod(m.action.size)) for m in models])
        ptr = lambda i: _lib.ctypes.c_void_p(host.data_ptr() + 4 * int(offs[i]))
        for i, m in enumerate(models):
            _lib.check(m._lib.rpl_get_action(m.handle, ptr(i), _lib.RPL_F32, 0))
        tot = np.zeros(1)
        barrier()
        t0 = time.perf_counter()
        for i, m in enumerate(models):       # every member's state from pinned host memory
            _lib.check(m._lib.rpl_set_action(m.handle, ptr(i), _lib.RPL_F32, 0))
        for _ in range(args.steps):
            _lib.check(lib.rpl_ensemble_step(h, 1))
            for m in models:
                _lib.check(m._lib.rpl_diagnostics(m.handle, None, None, None, None, _lib.dptr(tot)))
        for i, m in enumerate(models):
            _lib.check(m._lib.rpl_get_action(m.handle, ptr(i), _lib.RPL_F32, 0))
        el = time.perf_counter() - t0
        if dist is not None:
            t = torch.tensor([el], device="cuda", dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            el = float(t.item())
        e2e = {"value": world * units * args.steps / el, "unit": UNIT,
               "h2d_bytes_per_step": 4 * units / args.steps,
               "d2h_bytes_per_step": (4 * units + 8 * len(models) * args.steps) / args.steps,
               "includes": "set! of every member from pinned host, K x (ensemble step + per-member total_action "
                           "read), interior of every member to pinned host"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline("ensemble", args.steps)
    if rank == 0:
        classes = {}
        for (N, (Nk, Np)), shp in zip(shapes_info, ens.shapes()):
            classes.setdefault(f"{N}^2x{Nk}x{Np}", [0, shp])[0] += 1
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded members: seamount depth, vortex or eddy currents U0 0.1-0.8 m/s, JONSWAP N0)",
            "config": {"workload": "ensemble_members", "members": len(models), "seed": 4, "member_sizes": sizes,
                       "units_per_step": units, "classes": {k: {"count": v[0], "tile": v[1]} for k, v in classes.items()},
                       "direct_cells": args.direct_cells,
                       "sequential_ms_per_step": ms_seq / args.steps,
                       "speedup_vs_sequential": ms_seq / ms,
                       "build_s": t_build, "autotune_s": t_tune,
                       "l2": "state (%.1f GB per buffer set) larger than L2; no flush" % (4 * units / 1e9),
                       "parallelism": f"{world} independent replicas" if world > 1 else "1 GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": peak_kind, "kernel": "ensemble_kernel",
                         "launch_ms": launch_ms, "algorithmic_bytes_per_launch": nbytes_alg / 3.0,
                         "launch_interval": "one RK3 stage of every member (graph replay: counter reset + 3 launches per step)"},
            "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": 3 * args.steps, "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    ens.close()
    for m in models:
        m.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def run_learned(args, rank, world, local_rank):
    """The learned form on the translating-hurricane configuration (--size^2 x 32 kappa x 36 directions,
    --steps RK3 steps): training rows from two plain FP32 runs (this storm and a second seeded storm:
    Vmax 40 m/s, start (0.3 L, 0.3 L), 7 m/s), the library's own training, then the same run with the
    learned source and with the plain FP32 sources from the same start, both device-timed; the learned
    run's Hs, spectra and total action against the plain run's."""
    import torch
    import ripple_b200 as rp
    from ripple_b200 import _lib, learned, workloads

    torch.cuda.set_device(local_rank)
    try:
        smi_id = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    except Exception:
        smi_id = str(local_rank)
    n, K = args.size, args.steps
    nb, hd = 32 * 36, 512
    net = learned.SourceNetwork(nbins=nb, hidden=hd, rows=65536, seed=5, device=local_rank)
    # 1. training rows from the plain sources
    t0 = time.perf_counter()
    storms = [dict(), dict(vmax=40.0, start=(0.3, 0.3), translation=7.0)]
    every = max(1, K // max(1, args.snapshots))
    gen = torch.Generator(device="cuda").manual_seed(7)
    def collect(bounds=None):
        """Rows of both storms' runs every `every` steps: plain-source runs, or (with bounds) runs driven by
        the current network; the targets are always the plain sources' rates at the visited states."""
        Xs, Es, Ts = [], [], []
        for st in storms:
            w = workloads.hurricane_swell(N=n, nsteps=K, n0_dtype=np.float32, **st)
            m = w.model("fp32", device=local_rank)
            if bounds is not None:
                learned.use_learned_source(m, net, *bounds)
            for k in range(0, K, every):
                X, E, T = learned.sample(m, net)
                peak = T.abs().amax(1)
                act = peak > 0.5
                calm = (~act) & (torch.rand(peak.shape, device=peak.device, generator=gen) < args.calm_fraction)
                keep = (act | calm).nonzero().squeeze(1)
                Xs.append(X[keep])
                Es.append(E[keep])
                Ts.append(T[keep])
                del X, E, T, peak, act, calm, keep
                rp.time_step(m, w.dt, min(every, K - k))
            m.close()
        return torch.cat(Xs), torch.cat(Es), torch.cat(Ts)

    X, E, T = collect()
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    # out-of-distribution bounds and output clamps from the plain-source rows only
    lo, hi = learned.input_bounds(X, E, feature_pad=args.feature_pad)
    ylo, yhi = learned.output_bounds(T)
    # 2. training (the library's forward/backward/Adam kernels), then rounds of rows gathered along the
    #    network's own trajectories (labelled by the plain sources) and more training
    t0 = time.perf_counter()
    losses = learned.train(net, X, E, T, steps=args.train_steps, batch=16384, lr=1e-3,
                           weights=learned.row_weights(T), log_every=max(1, args.train_steps // 4))
    for r in range(args.dagger):
        X2, E2, T2 = collect((lo, hi, ylo, yhi))
        X, E, T = torch.cat([X, X2]), torch.cat([E, E2]), torch.cat([T, T2])
        del X2, E2, T2
        losses += learned.train(net, X, E, T, steps=args.train_steps // 2, batch=16384, lr=5e-4, seed=r + 1,
                                weights=learned.row_weights(T), log_every=max(1, args.train_steps // 4))
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    rows = int(X.shape[0])
    del X, E, T
    # 3. the evaluation run, plain FP32 and learned, from the same start
    w = workloads.hurricane_swell(N=n, nsteps=K, n0_dtype=np.float32)
    res = {}
    for mode in ("plain", "learned"):
        warm = w.model("fp32", device=local_rank)     # warm-up on a throwaway copy
        if mode == "learned":
            learned.use_learned_source(warm, net, lo, hi, ylo, yhi, gate=args.learned_gate)
        rp.time_step(warm, w.dt, args.warmup)
        warm.close()
        m = w.model("fp32", device=local_rank)
        if mode == "learned":
            learned.use_learned_source(m, net, lo, hi, ylo, yhi, gate=args.learned_gate)
        lib, h = m._lib, m.handle
        stream = torch.cuda.Stream(device=local_rank)
        _lib.check(lib.rpl_set_stream(h, _lib.ctypes.c_void_p(stream.cuda_stream)))
        _lib.check(lib.rpl_set_clock(h, 0.0, 0))
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with ClockSampler(smi_id) as clk:
            with torch.cuda.stream(stream):
                start.record(stream)
                _lib.check(lib.rpl_step_async(h, w.dt, K))
                end.record(stream)
            stream.synchronize()
            _lib.check(lib.rpl_sync(h))
        m._sync_clock()
        ms = start.elapsed_time(end)
        state = torch.empty(w.units, dtype=torch.float32, device="cuda")
        _lib.check(lib.rpl_get_action_device(h, _lib.ctypes.c_void_p(state.data_ptr()), _lib.RPL_F32, 0))
        d = rp.diagnostics(m.action)
        res[mode] = dict(ms=ms, clocks=clk.summary(), N=state, Hs=d["Hs"], total=d["total_action"],
                         fallback=learned.fallback_cells(m) if mode == "learned" else 0,
                         totals=learned.fallback_totals(m) if mode == "learned" else (0, 1))
        m.close()
    a, b = res["learned"], res["plain"]
    dN = float(torch.linalg.vector_norm((a["N"] - b["N"]).double()) / torch.linalg.vector_norm(b["N"].double()))
    Nk, Np = 32, 36
    spec = lambda v: v.double().reshape(Np, Nk, n * n).sum(2)   # device layout: bins (m, n) of all cells
    dS = float(torch.linalg.vector_norm(spec(a["N"]) - spec(b["N"])) / torch.linalg.vector_norm(spec(b["N"])))
    mask = b["Hs"] > 0.01 * b["Hs"].max()
    dH = float(np.linalg.norm(a["Hs"] - b["Hs"]) / np.linalg.norm(b["Hs"]))
    dHmax = float(np.max(np.abs(a["Hs"] - b["Hs"])[mask] / b["Hs"][mask]))
    # 4. the network's forward GEMMs alone on one stage's rows, against the BF16 tensor-core peak
    P = n * n
    prow = (P + 127) // 128 * 128
    Xf = torch.zeros((prow, nb), dtype=torch.bfloat16, device="cuda")
    Ef = torch.zeros((prow, 4), device="cuda")
    net.forward(Xf, Ef)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        net.forward(Xf, Ef)
    e1.record()
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1) / 3
    flops = 2.0 * prow * (nb * hd + 2 * hd * hd + hd * nb)
    try:
        bf16_peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
        peak_kind = "measured"
    except Exception:
        bf16_peak, peak_kind = 1590.0, "fallback"
    peak, hbm_kind = peaks()
    value = w.units * K / (a["ms"] / 1e3)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": K, "warmup": args.warmup,
            "ms_per_step": a["ms"] / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 state, bf16 network", "impl": "learned",
            "data": "synthetic (Holland hurricane on a linear track, uniform N0 = 1e-6)",
            "config": {"workload": "hurricane_swell with the learned source", "grid": [n, n], "spectral": [Nk, Np],
                       "network": f"{nb}+4 -> 3 x {hd} GELU -> {nb}, bf16 weights, fp32 accumulate",
                       "plain_fp32_ms_per_step": b["ms"] / K, "speedup_vs_plain_fp32": b["ms"] / a["ms"],
                       "Hs_relL2_vs_plain": dH, "Hs_max_rel_err_vs_plain": dHmax, "N_relL2_vs_plain": dN,
                       "mean_spectrum_relL2_vs_plain": dS,
                       "total_action_rel_diff": abs(a["total"] - b["total"]) / b["total"],
                       "fallback_cells_last_stage": a["fallback"], "cells": P,
                       "fallback_cell_stage_fraction": a["totals"][0] / max(1, a["totals"][1]),
                       "training_rows": rows, "training_steps": args.train_steps * (2 + args.dagger) // 2,
                       "dagger_rounds": args.dagger, "feature_pad": args.feature_pad, "learned_gate": args.learned_gate, "training_s": t_train,
                       "data_generation_s": t_data, "losses": losses,
                       "mlp_forward_ms_per_stage": fwd_ms, "mlp_forward_tflops": flops / fwd_ms / 1e9,
                       "mlp_tensor_frac": flops / fwd_ms / 1e9 / bf16_peak, "bf16_peak_tflops": bf16_peak,
                       "bf16_peak_kind": peak_kind},
            "clocks": a["clocks"], "gpu_launches": None,
        }
        print(json.dumps(line), flush=True)
    net.close()


def run_mlp(args, rank, world, local_rank):
    """The learned source network's forward pass alone (1152 + 4 -> 3 x 512 GELU -> 1152, BF16 tcgen05
    GEMMs with FP32 accumulation) on --rows random rows: --warmup untimed passes, then --steps timed
    passes (CUDA events); FLOP/s against the measured BF16 tensor-core peak."""
    import torch
    from ripple_b200 import learned

    torch.cuda.set_device(local_rank)
    nb, hd, n = 32 * 36, 512, args.rows
    net = learned.SourceNetwork(nbins=nb, hidden=hd, rows=min(n, 65536), seed=5, device=local_rank)
    g = torch.Generator(device="cuda").manual_seed(3)
    X = torch.randn((n, nb), device="cuda", generator=g).to(torch.bfloat16)
    E = torch.randn((n, 4), device="cuda", generator=g)
    for _ in range(args.warmup):
        net.forward(X, E)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(args.steps):
        net.forward(X, E)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(1, args.steps)
    flops = 2.0 * n * (nb * hd + 2 * hd * hd + hd * nb)
    try:
        peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops"])
        kind = "measured"
    except Exception:
        peak, kind = 1590.0, "fallback"
    if rank == 0:
        tf = flops / ms / 1e9
        print(json.dumps({"metric": "MLP forward TFLOP/s (learned source network)", "value": tf, "unit": "TFLOP/s",
                          "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16",
                          "data": "synthetic (random rows)",
                          "config": {"workload": "learned-source MLP forward", "rows": n,
                                     "network": f"{nb}+4 -> 3 x {hd} GELU -> {nb}"},
                          "roofline": {"bound": "tensor", "achieved": tf, "peak": peak, "unit": "TFLOP/s",
                                       "frac": tf / peak, "peak_kind": kind, "kernel": "gemm_kernel"},
                          "gpu_launches": 4 * args.steps}), flush=True)
    net.close()


def run_decomposed(args, rank, world, local_rank):
    """The workload's one domain split into y slabs, one per rank (ripple_b200.decomposition): halo rows
    exchanged before every stage (NCCL point-to-point between GPUs; local copies on one rank)."""
    import datetime
    import torch
    import torch.distributed as dist
    from ripple_b200 import _lib, decomposition

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        store = dist.TCPStore("127.0.0.1", 0, 1, True)
        dist.init_process_group("gloo", store=store, rank=0, world_size=1)
    w = make_workload(args.workload, args.size, args.steps,
                      n0_dtype=np.float32 if args.precision == "fp32" else np.float64)
    dm = decomposition.DecomposedModel(w, args.precision, device=local_rank)
    del w.N0
    dm.step(w.dt, args.warmup)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    smi_id = "GPU-" + str(torch.cuda.get_device_properties(local_rank).uuid)
    with ClockSampler(smi_id) as clk:
        dist.barrier()
        torch.cuda.synchronize()
        start.record(dm.stream)
        dm.step(w.dt, args.steps)
        end.record(dm.stream)
        torch.cuda.synchronize()
        dist.barrier()
    ms = start.elapsed_time(end)
    t = torch.tensor([ms], dtype=torch.float64)
    if world > 1:
        t = t.cuda()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms = float(t.item())
    units = w.grid.Nx * w.grid.Ny * dm.model.spectral_grid.coordinate_size()[0] * \
        dm.model.spectral_grid.coordinate_size()[1]
    if rank == 0:
        line = {
            "metric": METRIC, "value": units * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32" if args.precision == "fp32" else "f64",
            "data": DATA.get(args.workload, "synthetic"),
            "config": {"workload": WORKLOAD_NAMES[args.workload] + " (y-slab decomposition)",
                       "grid": [args.size, args.size], "spectral": [32, 36], "precision": args.precision,
                       "units_per_step": units, "parallelism": f"{world} y slabs, 3 halo rows, exchange before "
                                                              "every stage",
                       "rows_per_rank": dm.slab.ny},
            "roofline": None, "cpu_baseline": None, "e2e": None,
            # every stage runs as three row ranges (interior, then the two boundary ranges after the exchange)
            "gpu_launches": 3 * launches_per_step(args.workload, args.precision) * args.steps,
            "clocks": clk.summary(),
        }
        print(json.dumps(line), flush=True)
    dm.model.close()
    dist.destroy_process_group()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.workload == "ensemble":
        run_ensemble(args, rank, world, local_rank)
        return
    if args.workload == "learned":
        run_learned(args, rank, world, local_rank)
        return
    if args.workload == "mlp":
        run_mlp(args, rank, world, local_rank)
        return
    if args.decompose:
        run_decomposed(args, rank, world, local_rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
