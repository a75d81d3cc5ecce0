"""Regenerates the golden fixtures in this directory from the CPU FP64 oracle.

c1_vortex_refraction.npz -- the vortex-refraction configuration (64x64, 4x16 bins, dt 0.05,
    400 SSP-RK3 steps): m0, kappa_rms and mean direction fields, total action, and the
    action on a strided subsample plus whole-field checksums.
kat_tendency_8x7x4x6.npz -- a seeded random action and current on an 8x7 grid with 4x6
    bins and the fused refraction tendency of that state.
The reference publishes no output for the fused kernel or for RK3 trajectories, so these
fixtures pin the oracle (and through it the CUDA path) against its own FP64 result;
the oracle's pieces are pinned to the reference's known answers in test_oracle_golden.py.

Usage: python tests/golden/make_golden.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "ripple.jl_b200"), os.path.join(ROOT, "oracle")]

import oracle  # noqa: E402
from ripple_b200 import workloads  # noqa: E402
from ripple_b200.grids import InfiniteDepth, PolarWaveVectorGrid, RectilinearGrid  # noqa: E402


def kat_workload():
    rng = np.random.default_rng(20241203)
    g = RectilinearGrid(size=(8, 7, 5), x=(0.0, 8.0), y=(0.0, 7.0), z=(-2.0, 0.0))
    sg = PolarWaveVectorGrid(κ=[0.4, 0.6, 0.9, 1.3], φ=np.arange(6) * (2 * math.pi / 6))
    u = np.asfortranarray(rng.uniform(-0.5, 0.5, (8, 7, 5)))
    v = np.asfortranarray(rng.uniform(-0.5, 0.5, (8, 7, 5)))
    N0 = np.asfortranarray(rng.uniform(0.0, 1.0, (8, 7, 4, 6)))
    return workloads.Workload("kat", g, sg, 1.5, N0, 0.01, 1, velocities={"u": u, "v": v},
                              horizontal_advection=None)


def main():
    w = workloads.vortex_refraction()
    o = oracle.Oracle(w)
    N, t = o.step(w.N0, w.dt, w.nsteps)
    d = o.diagnostics(N)
    flat = N.ravel(order="F")
    np.savez_compressed(os.path.join(HERE, "c1_vortex_refraction.npz"),
                        m0=d["m0"], kappa_rms=d["kappa_rms"], mean_direction=d["mean_direction"],
                        total_action=d["total_action"], sample=flat[::97], sum=flat.sum(),
                        sumsq=(flat * flat).sum(), time=t)
    k = kat_workload()
    ok = oracle.Oracle(k)
    G = ok.tendency(k.N0)
    np.savez_compressed(os.path.join(HERE, "kat_tendency_8x7x4x6.npz"), N0=k.N0, u=k.velocities["u"],
                        v=k.velocities["v"], G=G)
    print("wrote fixtures; total action", d["total_action"])


if __name__ == "__main__":
    main()
