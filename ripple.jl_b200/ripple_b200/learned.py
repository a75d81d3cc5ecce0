"""Learned form: an MLP that stands in for the per-cell source-term tendency of PrecomputedSources
(src/Sources/precomputed_sources.jl:396-439 with PressureCorrelationInput and
LocalSaturationDissipation), trained on tendencies the plain sources generate.

All network arithmetic runs in librpl.so (rpl_mlp_*: tcgen05 BF16 GEMMs with FP32 accumulation, the
library's own backward pass and Adam); PyTorch only holds the device buffers of the training set.
Per cell the inputs are the Nk*Np-bin log action spectrum and (U10 / 30, sin, cos of the wind
direction, log10(depth) / 4); the outputs are y = asinh(rate / target_scale) for the per-bin source
rates S / N (the compressed form keeps the relative accuracy from 1e-6 /s growth to 1 /s damping).
"""
import ctypes

import numpy as np

from . import _lib
from ._lib import ArgumentError, check


def _torch():
    import torch
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


class SourceNetwork:
    """nbins -> 3 x hidden GELU -> nbins; `rows` = training batch capacity and inference chunk."""

    def __init__(self, nbins=1152, hidden=512, rows=16384, seed=5, feature_shift=-6.0, feature_scale=4.0,
                 log_floor=1e-12, target_scale=1e-5, device=0):
        self._lib = _lib.load()
        d = _lib.RplMlpDesc(_lib.RPL_ABI_VERSION, nbins, hidden, rows, device, 0, seed, feature_shift,
                            feature_scale, log_floor, target_scale)
        h = ctypes.c_void_p()
        check(self._lib.rpl_mlp_create(ctypes.byref(d), ctypes.byref(h)))
        self._h = h
        # the training and inference arrays are PyTorch tensors: run in PyTorch's stream order
        torch = _torch()
        check(self._lib.rpl_mlp_set_stream(h, ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)))
        self.nbins, self.hidden, self.rows, self.device = nbins, hidden, rows, device
        self.target_scale = target_scale
        self.feature_shift, self.feature_scale, self.log_floor = feature_shift, feature_scale, log_floor

    @property
    def handle(self):
        return self._h

    def param_count(self):
        n = ctypes.c_int64()
        check(self._lib.rpl_mlp_param_count(self._h, ctypes.byref(n)))
        return n.value

    def get_params(self):
        p = np.empty(self.param_count(), dtype=np.float32)
        check(self._lib.rpl_mlp_get_params(self._h, ctypes.c_void_p(p.ctypes.data)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.param_count():
            raise ArgumentError("parameter vector has the wrong length")
        check(self._lib.rpl_mlp_set_params(self._h, ctypes.c_void_p(p.ctypes.data)))

    def train_step(self, X, E, T, rows, lr):
        """One Adam step on rows `rows` (int32 CUDA tensor) of the CUDA tensors X (bf16), E, T (float32)."""
        loss = np.zeros(1)
        check(self._lib.rpl_mlp_train_step(self._h, _ptr(X), _ptr(E), _ptr(T), _ptr(rows), int(rows.numel()),
                                           float(lr), _lib.dptr(loss)))
        return float(loss[0])

    def gradients(self, X, E, T, rows):
        g = np.empty(self.param_count(), dtype=np.float32)
        loss = np.zeros(1)
        check(self._lib.rpl_mlp_gradients(self._h, _ptr(X), _ptr(E), _ptr(T), _ptr(rows), int(rows.numel()),
                                          ctypes.c_void_p(g.ctypes.data), _lib.dptr(loss)))
        return g, float(loss[0])

    def forward(self, X, E):
        """Outputs y for the rows of X (bf16) and E; the row count must be a multiple of 128."""
        torch = _torch()
        n = X.shape[0]
        Y = torch.empty((n, self.nbins), dtype=torch.float32, device=X.device)
        check(self._lib.rpl_mlp_forward(self._h, _ptr(X), _ptr(E), int(n), _ptr(Y)))
        return Y

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.rpl_mlp_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample(model, net, out=None):
    """(X, E, T) training rows of the FP32 model's current state from its plain sources (one row per cell,
    cell c = i + Nx j). `out` = preallocated (X, E, T) views to fill."""
    torch = _torch()
    P = model.grid.Nx * model.grid.Ny
    dev = torch.device("cuda", model.device)
    if out is None:
        out = (torch.empty((P, net.nbins), dtype=torch.bfloat16, device=dev),
               torch.empty((P, 4), dtype=torch.float32, device=dev),
               torch.empty((P, net.nbins), dtype=torch.float32, device=dev))
    X, E, T = out
    torch.cuda.synchronize(dev)   # the library writes these from the model's own stream
    check(model._lib.rpl_set_clock(model.handle, model.clock.time, model.clock.iteration))
    check(model._lib.rpl_learned_sample(model.handle, net.handle, _ptr(X), _ptr(E), _ptr(T)))
    return X, E, T


def use_learned_source(model, net, lo=None, hi=None, ylo=None, yhi=None, gate=0.0):
    """Replace the model's plain sources by `net` (None: back to the plain sources). lo, hi: input bounds
    (nbins + 4 values); a cell with any input outside them uses the plain sources. ylo, yhi (optional,
    nbins values): the network's outputs are clamped to them (see output_bounds). gate > 0: a cell whose
    network rates would change a bin by more than `gate` of itself in one step uses the plain sources too."""
    if net is None:
        check(model._lib.rpl_set_learned_source(model.handle, None, None, None, None, None))
        return
    lo = np.ascontiguousarray(lo, dtype=np.float32)
    hi = np.ascontiguousarray(hi, dtype=np.float32)
    if lo.size != net.nbins + 4 or hi.size != net.nbins + 4:
        raise ArgumentError("bounds need nbins + 4 values")
    yp = [None, None]
    if ylo is not None:
        ylo = np.ascontiguousarray(ylo, dtype=np.float32)
        yhi = np.ascontiguousarray(yhi, dtype=np.float32)
        if ylo.size != net.nbins or yhi.size != net.nbins:
            raise ArgumentError("output bounds need nbins values")
        yp = [ctypes.c_void_p(ylo.ctypes.data), ctypes.c_void_p(yhi.ctypes.data)]
    check(model._lib.rpl_set_learned_source(model.handle, net.handle, ctypes.c_void_p(lo.ctypes.data),
                                            ctypes.c_void_p(hi.ctypes.data), *yp))
    check(model._lib.rpl_set_learned_gate(model.handle, float(gate)))
    model._learned_keep = (net, lo, hi, ylo, yhi)


def output_bounds(T, margin=0.1):
    """Per-output [lo, hi] of the training targets T (network output units), widened by `margin` of the
    range."""
    lo, hi = T.amin(0), T.amax(0)
    pad = margin * (hi - lo)
    return (lo - pad).cpu().numpy(), (hi + pad).cpu().numpy()


def outputs(model, nbins):
    """Network outputs y of the model's most recent stage, (cells, nbins) with cell = i + Nx j."""
    Y = np.empty((model.grid.Nx * model.grid.Ny, nbins), dtype=np.float32)
    check(model._lib.rpl_learned_outputs(model.handle, ctypes.c_void_p(Y.ctypes.data)))
    return Y


def fallback_cells(model):
    n = ctypes.c_int64()
    check(model._lib.rpl_learned_fallback_cells(model.handle, ctypes.byref(n)))
    return n.value


def fallback_totals(model):
    """(cell-stages that took the plain sources, all cell-stages) since the learned source was set."""
    f, t = ctypes.c_int64(), ctypes.c_int64()
    check(model._lib.rpl_learned_fallback_totals(model.handle, ctypes.byref(f), ctypes.byref(t)))
    return f.value, t.value


def input_bounds(X, E, margin=0.05, feature_pad=0.25, extra_pad=0.02):
    """Per-input [lo, hi] of a training set (X bf16 rows, E rows), widened by `margin` of each input's range
    plus an absolute pad: `feature_pad` for the log-action features (0.25 = a factor e^(0.25 feature_scale)
    in N beyond anything seen), `extra_pad` for the extras (U10 / 30, sin, cos, log10(d) / 4). Inputs
    that never varied in training (a calm cell's constant floor) keep a usable band this way."""
    torch = _torch()
    xs = X.float()
    lo = torch.cat([xs.amin(0), E.amin(0)])
    hi = torch.cat([xs.amax(0), E.amax(0)])
    nb = X.shape[1]
    pad = margin * (hi - lo)
    pad[:nb] += feature_pad
    pad[nb:] += extra_pad
    return (lo - pad).cpu().numpy(), (hi + pad).cpu().numpy()


def row_weights(T, floor=0.05):
    """Sampling weights of training rows: the row's largest |target| plus `floor` times the mean of those.
    Source rates are sparse (calm cells and bins facing away from the wind have none), so uniform
    batches would be nearly all zeros; these weights put the active cells in most batches."""
    peak = T.abs().amax(1)
    return peak + floor * peak.mean()


def train(net, X, E, T, steps, batch, lr=1e-3, lr_final=None, seed=0, log_every=0, weights=None):
    """Adam on random batches of the training rows (CUDA tensors); cosine decay to lr_final. With
    `weights` (one per row) the batches are drawn in proportion to them, with replacement."""
    torch = _torch()
    g = torch.Generator(device=X.device)
    g.manual_seed(seed)
    n = X.shape[0]
    lr_final = lr * 0.05 if lr_final is None else lr_final
    losses = []
    for k in range(steps):
        if weights is None:
            rows = torch.randint(0, n, (batch,), device=X.device, generator=g, dtype=torch.int32)
        else:
            rows = torch.multinomial(weights, batch, replacement=True, generator=g).to(torch.int32)
        a = lr_final + 0.5 * (lr - lr_final) * (1 + np.cos(np.pi * k / max(1, steps)))
        want = log_every and (k % log_every == 0 or k == steps - 1)
        if want:
            losses.append((k, net.train_step(X, E, T, rows, a)))
        else:
            check(net._lib.rpl_mlp_train_step(net.handle, _ptr(X), _ptr(E), _ptr(T), _ptr(rows), batch,
                                              float(a), None))
    return losses
