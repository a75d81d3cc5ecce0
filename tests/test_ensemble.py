"""Batching form (rpl_ensemble_*): an ensemble of uneven FP32 members advanced by one persistent
launch per stage must give each member the result of advancing it alone (single-model kernels), and
the FP64 oracle's result within the FP32 tolerance."""
import os

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import workloads

pytestmark = pytest.mark.gpu

FP32_TOL = 1e-5


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


# (N, Nk, Np, peak current, vortex?) -- every lane count (Nk 8 -> 4 lanes, 16 -> 8, 24 and 32 -> 16),
# grids that leave partial tiles for every tile shape, and the 36-direction ring
MEMBERS = [(20, 8, 12, 0.3, True), (37, 16, 24, 0.6, False), (24, 24, 36, 0.1, True),
           (19, 32, 36, 0.8, False), (64, 16, 24, 0.5, False), (13, 24, 12, 0.4, True)]


def member_workloads(nsteps=3):
    out = []
    for k, (N, Nk, Np, U0, vortex) in enumerate(MEMBERS):
        w = workloads.seamount_eddies(N=N, Nz=8, Nk=Nk, Np=Np, nsteps=nsteps, seed=40 + k, L=N * 20e3,
                                      peak_current=U0, n_eddies=1 if vortex else 8)
        out.append(w)
    return out


def test_ensemble_matches_members_run_alone_and_oracle(oracle_mod):
    ws = member_workloads()
    models = [w.model("fp32") for w in ws]
    ens = rp.Ensemble(models, [w.dt for w in ws])
    ens.time_step(3)
    alone = []
    for w in ws:
        m = w.model("fp32")
        rp.time_step(m, w.dt, 3)
        alone.append(m.action.interior())
        m.close()
    for w, m, a in zip(ws, models, alone):
        got = m.action.interior()
        assert m.clock.iteration == 3 and m.clock.time == pytest.approx(3 * w.dt, rel=1e-15)
        assert np.max(np.abs(got - a)) <= 1e-6 * np.max(np.abs(a))
        No, _ = oracle_mod.Oracle(w).step(w.N0, w.dt, 3)
        assert rel_l2(got, No) <= FP32_TOL
    ens.close()


@pytest.mark.parametrize("direct_cells", [1000, 1])
def test_direct_members_equal_their_own_runs(direct_cells):
    """Members of at least direct_cells cells take their own single-model stage launches inside the
    captured step (bit-identical to running alone); the others share the persistent launches (1: all
    members direct, no persistent launch)."""
    ws = member_workloads(nsteps=2)
    models = [w.model("fp32") for w in ws]
    ens = rp.Ensemble(models, [w.dt for w in ws], direct_cells=direct_cells)
    ens.time_step(2)
    for w, m in zip(ws, models):
        a = w.model("fp32")
        rp.time_step(a, w.dt, 2)
        ref = a.action.interior()
        if w.grid.Nx * w.grid.Ny >= direct_cells:
            assert np.array_equal(m.action.interior(), ref)
        else:
            assert np.max(np.abs(m.action.interior() - ref)) <= 1e-6 * np.max(np.abs(ref))
        assert m.clock.iteration == 2
        a.close()
    ens.close()


def test_ensemble_graph_plain_and_sequential_agree():
    ws = member_workloads(nsteps=2)
    results = []
    for mode in ("graph", "plain", "sequential"):
        models = [w.model("fp32") for w in ws]
        ens = rp.Ensemble(models, [w.dt for w in ws], use_graph=(mode == "graph"))
        if mode == "sequential":
            ens.time_step_sequential(2)
        else:
            ens.time_step(1)
            ens.time_step(1)
        results.append([m.action.interior() for m in models])
        ens.close()
        for m in models:
            m.close()
    for a, b, c in zip(*results):
        assert np.array_equal(a, b)
        assert np.max(np.abs(a - c)) <= 1e-6 * np.max(np.abs(c))


def test_ensemble_autotune_cache_and_every_shape(tmp_path):
    ws = member_workloads(nsteps=1)
    cache = str(tmp_path / "tiles.txt")
    models = [w.model("fp32") for w in ws]
    ens = rp.Ensemble(models, [w.dt for w in ws], autotune=True, autotune_cache=cache)
    shapes = ens.shapes()
    for (N, Nk, Np, _, _), (L, tx, ty) in zip(MEMBERS, shapes):
        assert L == (4 if Nk <= 8 else 8 if Nk <= 16 else 16) and L * tx * ty == 512
    lines = open(cache).read().splitlines()
    assert len(lines) == len({(N, Nk, Np) for N, Nk, Np, _, _ in MEMBERS})
    ens.time_step(1)
    tuned = [m.action.interior() for m in models]
    ens.close()
    # a second ensemble reads the cache (no timing) and gets the same shapes
    models2 = [w.model("fp32") for w in ws]
    ens2 = rp.Ensemble(models2, [w.dt for w in ws], autotune_cache=cache)
    assert ens2.shapes() == shapes
    ens2.close()
    # every candidate shape gives the same result: pin each shape through a hand-written cache
    table = [(16, 8, 4), (16, 4, 8), (16, 16, 2), (8, 8, 8), (8, 16, 4), (8, 4, 16), (4, 16, 8), (4, 8, 16),
             (4, 32, 4)]
    for pick in range(3):
        forced = []
        for line in lines:
            key = line[len("rpl-tile "):line.index(" | ")]
            Nk = int(key.split()[3])
            lanes = 4 if Nk <= 8 else 8 if Nk <= 16 else 16
            v = [i for i, t in enumerate(table) if t[0] == lanes][pick]
            forced.append(f"rpl-tile {key} | {v} {table[v][0]} {table[v][1]} {table[v][2]} 1.0")
        path = str(tmp_path / f"forced{pick}.txt")
        open(path, "w").write("\n".join(forced) + "\n")
        models3 = [w.model("fp32") for w in ws]
        ens3 = rp.Ensemble(models3, [w.dt for w in ws], autotune_cache=path)
        assert all(s == table[[i for i, t in enumerate(table) if t[0] == s[0]][pick]] for s in ens3.shapes())
        ens3.time_step(1)
        for m, t in zip(models3, tuned):
            assert np.max(np.abs(m.action.interior() - t)) <= 1e-6 * np.max(np.abs(t))
        ens3.close()
        for m in models3:
            m.close()
    for m in models + models2:
        m.close()


def test_ensemble_rejects_bad_members():
    ws = member_workloads(nsteps=1)
    m32 = ws[0].model("fp32")
    m64 = ws[1].model("fp64")
    with pytest.raises((rp.RplError, rp.ArgumentError)):
        rp.Ensemble([m32, m64], [ws[0].dt, ws[1].dt])
    with pytest.raises((rp.RplError, rp.ArgumentError)):
        rp.Ensemble([m32, m32], [ws[0].dt, ws[0].dt])
    with pytest.raises((rp.RplError, rp.ArgumentError)):
        rp.Ensemble([m32], [0.0])
    h = workloads.hurricane_swell(N=16, Nk=8, Np=12, nsteps=1)
    mh = h.model("fp32")
    with pytest.raises((rp.RplError, rp.ArgumentError)):
        rp.Ensemble([m32, mh], [ws[0].dt, h.dt])   # sources / other transport
    for m in (m32, m64, mh):
        m.close()
