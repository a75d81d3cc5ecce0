"""CPU oracle of the learned-source MLP (test infrastructure; only tests/ use it).

The network has no counterpart in the reference, so this file states the GPU network's arithmetic
(ripple.jl_b200/csrc/rpl_mlp.cu, rpl_gemm.cu) in NumPy: the same layers, the same BF16 rounding points
(weights, activations, output and hidden gradients) with FP64 accumulation in place of the tensor cores'
FP32. Its exact-arithmetic form (rounding=False) is pinned by finite differences in
tests/test_mlp_oracle.py.

Parameter layout (one FP32 vector): W1 (H x B), W1e (H x 4), b1 (H), W2 (H x H), b2, W3 (H x H), b3,
W4 (B x H), b4 (B); B = nbins, H = hidden.
"""
import numpy as np


def bf16(x):
    """Round to the nearest BF16 value (ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) & 0xFFFF0000).astype(np.uint32).view(np.float32)


GELU_C, GELU_A = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    """GELU in its tanh form, the network's activation: 0.5 z (1 + tanh(c (z + a z^3)))."""
    return 0.5 * z * (1.0 + np.tanh(GELU_C * (z + GELU_A * z ** 3)))


def gelu_grad(z):
    t = np.tanh(GELU_C * (z + GELU_A * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * z * z)


def unpack(p, nbins, hidden):
    B, H = nbins, hidden
    sizes = [("W1", (H, B)), ("W1e", (H, 4)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
             ("b3", (H,)), ("W4", (B, H)), ("b4", (B,))]
    out, o = {}, 0
    for name, shp in sizes:
        n = int(np.prod(shp))
        out[name] = np.asarray(p[o:o + n], dtype=np.float64).reshape(shp)
        o += n
    assert o == p.size
    return out


def pack(d):
    return np.concatenate([np.ravel(d[k]) for k in ("W1", "W1e", "b1", "W2", "b2", "W3", "b3", "W4", "b4")])


def forward_backward(p, X, E, T, nbins, hidden, rounding=True):
    """Loss (mean squared error), gradient (parameter layout) and output of the batch X, E, T."""
    q = unpack(p, nbins, hidden)
    r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
    W1, W2, W3, W4 = (r(q[k]).astype(np.float64) for k in ("W1", "W2", "W3", "W4"))
    X = r(X).astype(np.float64)
    E = np.asarray(E, dtype=np.float64)
    z1 = X @ W1.T + q["b1"] + E @ q["W1e"].T
    h1 = r(gelu(z1)).astype(np.float64)
    z2 = h1 @ W2.T + q["b2"]
    h2 = r(gelu(z2)).astype(np.float64)
    z3 = h2 @ W3.T + q["b3"]
    h3 = r(gelu(z3)).astype(np.float64)
    y = h3 @ W4.T + q["b4"]
    d = y - np.asarray(T, dtype=np.float64)
    n = d.size
    loss = float(np.sum(d * d) / n)
    dY = r(2.0 * d / n).astype(np.float64)
    g = {"W4": dY.T @ h3, "b4": dY.sum(0)}
    dZ3 = r((dY @ W4) * gelu_grad(z3)).astype(np.float64)
    g.update(W3=dZ3.T @ h2, b3=dZ3.sum(0))
    dZ2 = r((dZ3 @ W3) * gelu_grad(z2)).astype(np.float64)
    g.update(W2=dZ2.T @ h1, b2=dZ2.sum(0))
    dZ1 = r((dZ2 @ W2) * gelu_grad(z1)).astype(np.float64)
    g.update(W1=dZ1.T @ X, b1=dZ1.sum(0), W1e=dZ1.T @ E)
    return loss, pack(g), y


def blocks(v, nbins, hidden):
    """The parameter vector split into its named blocks (for per-block comparisons)."""
    return unpack(np.asarray(v, dtype=np.float64), nbins, hidden)
