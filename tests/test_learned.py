"""Learned form: the tcgen05 BF16 GEMM, the MLP's forward/backward against the CPU oracle, training, and
the learned source inside the RK3 step (fallback, out-of-distribution cells, gain over no sources)."""
import copy
import os
import sys

import numpy as np
import pytest

import ripple_b200 as rp
from ripple_b200 import learned, workloads

pytestmark = pytest.mark.gpu

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))


@pytest.fixture(scope="module")
def torch():
    import torch as t
    return t


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (256, 384, 1152), (19200, 512, 128)])
def test_gemm_matches_fp32_product(torch, M, N, K):
    """C = A B^T on the tensor cores (BN 128, and BN 256 for the 19200-row case) against FP64 products of
    the same BF16 values (FP32 accumulation: tolerance 1e-5 of the row norms)."""
    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.empty(M, N, device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    lib = rp.load_library()
    rp._lib.check(lib.rpl_gemm_bf16(learned._ptr(A), learned._ptr(B), learned._ptr(C), M, N, K, None))
    ref = A.double() @ B.double().T
    scale = (A.double().norm(dim=1)[:, None] * B.double().norm(dim=1)[None, :])
    assert float(((C.double() - ref).abs() / scale).max()) <= 1e-5


def test_gemm_rejects_bad_shapes(torch):
    A = torch.zeros(100, 64, device="cuda", dtype=torch.bfloat16)
    C = torch.zeros(100, 128, device="cuda")
    lib = rp.load_library()
    assert lib.rpl_gemm_bf16(learned._ptr(A), learned._ptr(A), learned._ptr(C), 100, 128, 64, None) != 0


def test_gemm_bounded_wait_runs_out_and_recovers(torch):
    """A poll limit of one makes the first barrier wait give up (a TMA load takes far longer than one
    poll): the kernel drains its loads and MMAs, frees its tensor memory and returns; the call reports
    RPL_ERR_DEVICE with error bit 4, and the next GEMM with the default limit on the same context is
    correct."""
    M, N, K = 1024, 512, 1152
    g = torch.Generator(device="cuda").manual_seed(3)
    A = torch.randn(M, K, device="cuda", generator=g).to(torch.bfloat16)
    B = torch.randn(N, K, device="cuda", generator=g).to(torch.bfloat16)
    C = torch.zeros(M, N, device="cuda", dtype=torch.float32)
    torch.cuda.synchronize()
    lib = rp.load_library()
    st = lib.rpl_gemm_bf16_bounded(learned._ptr(A), learned._ptr(B), learned._ptr(C), M, N, K, 1, None)
    assert st == rp._lib.RPL_ERR_DEVICE
    assert b"bounded wait ran out" in lib.rpl_last_error()
    torch.cuda.synchronize()                                  # no sticky CUDA error
    rp._lib.check(lib.rpl_gemm_bf16_bounded(learned._ptr(A), learned._ptr(B), learned._ptr(C), M, N, K, 0, None))
    ref = A.double() @ B.double().T
    scale = (A.double().norm(dim=1)[:, None] * B.double().norm(dim=1)[None, :])
    assert float(((C.double() - ref).abs() / scale).max()) <= 1e-5


def small_net_and_batch(torch, nbins=256, hidden=256, B=256, seed=1):
    net = learned.SourceNetwork(nbins=nbins, hidden=hidden, rows=256, seed=seed)
    g = torch.Generator(device="cuda").manual_seed(seed)
    X = torch.randn(B, nbins, device="cuda", generator=g).to(torch.bfloat16)
    E = torch.randn(B, 4, device="cuda", generator=g)
    T = torch.randn(B, nbins, device="cuda", generator=g)
    rows = torch.arange(B, device="cuda", dtype=torch.int32)
    return net, X, E, T, rows


def test_mlp_gradients_match_cpu_oracle(torch):
    import mlp_oracle as mo
    nb, hd = 256, 256
    net, X, E, T, rows = small_net_and_batch(torch, nb, hd)
    # give the biases and the output layer non-trivial values
    rng = np.random.default_rng(2)
    p = net.get_params()
    p += rng.normal(0.0, 0.02, p.size).astype(np.float32)
    net.set_params(p)
    g_gpu, loss_gpu = net.gradients(X, E, T, rows)
    loss_cpu, g_cpu, _ = mo.forward_backward(p, X.float().cpu().numpy(), E.cpu().numpy(), T.cpu().numpy(), nb, hd)
    assert loss_gpu == pytest.approx(loss_cpu, rel=1e-4)
    bg, bc = mo.blocks(g_gpu, nb, hd), mo.blocks(g_cpu, nb, hd)
    for k in bc:
        err = np.linalg.norm(bg[k] - bc[k]) / np.linalg.norm(bc[k])
        assert err <= 2e-2, (k, err)
    # the forward output itself
    Y = net.forward(X, E).double().cpu().numpy()
    _, _, y_cpu = mo.forward_backward(p, X.float().cpu().numpy(), E.cpu().numpy(), T.cpu().numpy(), nb, hd)
    assert np.linalg.norm(Y - y_cpu) / np.linalg.norm(y_cpu) <= 1e-2
    net.close()


def test_mlp_training_reduces_loss(torch):
    """A smooth synthetic map (targets a fixed random linear function of the inputs, squashed)."""
    nb, hd, n = 256, 256, 4096
    net = learned.SourceNetwork(nbins=nb, hidden=hd, rows=512, seed=3)
    g = torch.Generator(device="cuda").manual_seed(4)
    X = torch.randn(n, nb, device="cuda", generator=g)
    E = torch.randn(n, 4, device="cuda", generator=g)
    Wm = torch.randn(nb, nb, device="cuda", generator=g) / nb ** 0.5
    T = torch.tanh(X @ Wm.T + E[:, :1])
    X = X.to(torch.bfloat16)
    first = learned.train(net, X, E, T, steps=1, batch=512, lr=1e-3, log_every=1)[0][1]
    losses = learned.train(net, X, E, T, steps=400, batch=512, lr=2e-3, log_every=100)
    assert losses[-1][1] < 0.2 * first
    net.close()


def hurricane(N=24, Nk=16, Np=24, nsteps=6):
    return workloads.hurricane_swell(N=N, Nk=Nk, Np=Np, nsteps=nsteps)


def small_storm(nsteps=40):
    """48 x 48 cells of 10 km (the full configuration's spacing, so its CFL time step of ~70 s) under the
    translating hurricane, 16 kappa x 24 directions."""
    return workloads.hurricane_swell(N=48, Nk=16, Np=24, nsteps=nsteps, L=48 * 10e3)


def test_learned_source_with_all_cells_falling_back_equals_plain(torch):
    """Bounds that no input satisfies: every cell takes the plain FP32 sources, bit for bit."""
    w = hurricane()
    net = learned.SourceNetwork(nbins=16 * 24, hidden=256, rows=256, seed=1)
    plain = w.model("fp32")
    rp.time_step(plain, w.dt, 4)
    m = w.model("fp32")
    nb = 16 * 24
    learned.use_learned_source(m, net, np.full(nb + 4, 1e9, np.float32), np.full(nb + 4, 2e9, np.float32))
    rp.time_step(m, w.dt, 4)
    assert learned.fallback_cells(m) == w.grid.Nx * w.grid.Ny
    assert np.array_equal(m.action.interior(), plain.action.interior())
    learned.use_learned_source(m, None)
    net.close()


def test_learned_sample_targets_are_the_plain_rates(torch, oracle_mod):
    """rpl_learned_sample's targets times N equal the plain sources' tendency (the FP64 oracle's sources)."""
    w = hurricane(nsteps=1)
    rng = np.random.default_rng(8)
    w.N0 = np.asfortranarray(rng.uniform(0.5e-6, 1.5e-6, w.N0.shape))
    net = learned.SourceNetwork(nbins=16 * 24, hidden=256, rows=256, seed=1, target_scale=1e-5)
    m = w.model("fp32")
    X, E, T = learned.sample(m, net)
    Nx, Ny, Nk, Np = w.N0.shape
    rate = np.sinh(T.double().cpu().numpy()) * 1e-5            # (cells, bins), cell = i + Nx j, bin = m + Nk n
    N32 = w.N0.astype(np.float32).astype(np.float64)
    S_gpu = rate.reshape(Ny, Nx, Np, Nk).transpose(1, 0, 3, 2) * N32
    o = oracle_mod.Oracle(w)
    w2 = copy.copy(w)
    w2.sources = None
    S_ref = o.tendency(w.N0) - oracle_mod.Oracle(w2).tendency(w.N0)
    assert np.linalg.norm(S_gpu - S_ref) / np.linalg.norm(S_ref) <= 1e-4
    feats = X.float().cpu().numpy().reshape(Ny, Nx, Np, Nk).transpose(1, 0, 3, 2)
    assert np.allclose(feats, (np.log(N32) + 6.0) / 4.0, atol=2e-2)
    assert np.allclose(E[:, 0].cpu().numpy(), o.wind_fields(0.0)[0].ravel(order="F") / 30.0, rtol=1e-6, atol=1e-6)
    net.close()


def test_learned_stage_outputs_are_the_network_on_the_stage_input(torch):
    """The stage's network rows (features of the stage input) give exactly the network's output on the
    rows rpl_learned_sample writes for the same state."""
    w = small_storm(nsteps=1)
    nb = 16 * 24
    net = learned.SourceNetwork(nbins=nb, hidden=256, rows=2048, seed=2)
    m = w.model("fp32")
    rp.time_step(m, w.dt, 5)
    X, E, _ = learned.sample(m, net)
    P = X.shape[0]
    n128 = (P + 127) // 128 * 128
    Xp = torch.zeros((n128, nb), dtype=torch.bfloat16, device="cuda")
    Ep = torch.zeros((n128, 4), device="cuda")
    Xp[:P] = X
    Ep[:P] = E
    Yf = net.forward(Xp, Ep)[:P].cpu().numpy()
    m.action.set(m.action.interior().astype(np.float32))
    learned.use_learned_source(m, net, np.full(nb + 4, -1e9, np.float32), np.full(nb + 4, 1e9, np.float32))
    rp._lib.check(m._lib.rpl_set_clock(m.handle, m.clock.time, m.clock.iteration))
    rp._lib.check(m._lib.rpl_stage_async(m.handle, w.dt, 1))
    rp._lib.check(m._lib.rpl_sync(m.handle))
    assert np.array_equal(learned.outputs(m, nb), Yf)
    assert learned.fallback_cells(m) == 0
    net.close()


LEARNED_HS_TOL = 0.45


def test_learned_source_error_against_the_plain_sources(torch):
    """Train on plain-source states of a small hurricane (16 kappa x 24 directions, 4000 Adam steps), run
    40 steps with the learned source: its Hs stays within rel-L2 LEARNED_HS_TOL of the plain-source run
    (measured on B200: 0.33; without sources or with the untrained network the error is 1.0), and cells
    with an out-of-range wind fall back to the plain sources."""
    w = small_storm()
    nb = 16 * 24
    net = learned.SourceNetwork(nbins=nb, hidden=256, rows=2048, seed=2)
    P = w.grid.Nx * w.grid.Ny
    # training rows: states of the plain FP32 run every 2 steps
    m = w.model("fp32")
    chunks = []
    for k in range(20):
        chunks.append([t.clone() for t in learned.sample(m, net)])
        rp.time_step(m, w.dt, 2)
    X = torch.cat([c[0] for c in chunks])
    E = torch.cat([c[1] for c in chunks])
    T = torch.cat([c[2] for c in chunks])
    lo, hi = learned.input_bounds(X, E)
    untrained = learned.SourceNetwork(nbins=nb, hidden=256, rows=2048, seed=2)
    learned.train(net, X, E, T, steps=4000, batch=2048, lr=2e-3, weights=learned.row_weights(T))
    Hs = {}
    for mode in ("plain", "learned", "untrained", "none"):
        if mode == "none":
            w2 = small_storm()
            w2.sources = None
            mm = w2.model("fp32")
        else:
            mm = w.model("fp32")
        if mode in ("learned", "untrained"):
            learned.use_learned_source(mm, net if mode == "learned" else untrained, lo, hi)
        rp.time_step(mm, w.dt, 40)
        Hs[mode] = rp.diagnostics(mm.action)["Hs"]
        if mode == "learned":
            assert learned.fallback_cells(mm) < P // 4
    err = {k: np.linalg.norm(Hs[k] - Hs["plain"]) / np.linalg.norm(Hs["plain"]) for k in Hs}
    print("Hs rel-L2 errors vs plain:", err)
    assert err["learned"] <= LEARNED_HS_TOL, err
    assert err["learned"] < 0.5 * err["none"] and err["learned"] < 0.5 * err["untrained"], err
    # out of distribution: a wind-speed band no cell has sends every cell to the plain path
    lo2, hi2 = lo.copy(), hi.copy()
    lo2[nb] = hi2[nb] = -1.0
    mm = w.model("fp32")
    learned.use_learned_source(mm, net, lo2, hi2)
    rp.time_step(mm, w.dt, 1)
    assert learned.fallback_cells(mm) == P
    untrained.close()
    net.close()


def test_learned_trust_gate(torch):
    """The trust gate: with a gate no rate reaches the run equals the ungated learned run bit for bit; a
    small gate sends the cells with stiff network rates to the plain sources."""
    w = small_storm(nsteps=1)
    nb = 16 * 24
    net = learned.SourceNetwork(nbins=nb, hidden=256, rows=2048, seed=2)
    lo, hi = np.full(nb + 4, -1e9, np.float32), np.full(nb + 4, 1e9, np.float32)
    res = {}
    for name, gate in (("none", 0.0), ("huge", 1e30), ("small", 1e-6)):
        m = w.model("fp32")
        rp.time_step(m, w.dt, 3)
        learned.use_learned_source(m, net, lo, hi, gate=gate)
        rp.time_step(m, w.dt, 2)
        res[name] = (m.action.interior().copy(), learned.fallback_cells(m), learned.fallback_totals(m))
        m.close()
    P = w.grid.Nx * w.grid.Ny
    assert np.array_equal(res["none"][0], res["huge"][0]) and res["none"][1] == res["huge"][1] == 0
    assert res["none"][2] == (0, 6 * P)                       # 2 steps x 3 stages, no cell fell back
    assert res["small"][1] > 0 and 0 < res["small"][2][0] <= 6 * P
    assert not np.array_equal(res["small"][0], res["none"][0])
    net.close()
