"""Gradients of the stage-2 coherence through the CUDA library.

The differentiable map (K given, no trial search) is the one topofit scores
for a fixed K (crates/pystamps-core/src/native_stage2.rs:1257-1303) after
the binning (:888-903), CLAP filter (:904-1184) and resampling:

    grid  = sum over each cell of ph * exp(-j K bperp) * w
    filt  = CLAP(grid; alpha, beta) + pyramid overlap-add
    p     = filt[cell] / |filt[cell]|
    coh   = |sum_c conj(p_c) ph_c exp(-j K bperp_c)| / sum_c |conj(p_c) ph_c|

`coherence(...)` is a torch.autograd.Function whose forward and backward are
ps2_coherence_forward / ps2_coherence_backward: hand-written adjoints of the
coherence, the resample, the bin sum and CLAP (window spectra recomputed in
the backward pass). Complex gradients follow torch's convention for a real
loss, dL/dRe + j dL/dIm. `calibrate_clap` tunes clap_alpha / clap_beta by
gradient steps on a loss of the coherences.
"""
from __future__ import annotations

import ctypes
import math
from typing import Callable

import torch

from . import _lib
from ._lib import check
from .stage2 import PRECISION_FP32, PRECISION_FP64, PreparedPatch, Stage2Context

_vp = ctypes.c_void_p
_d = ctypes.c_double


class CoherenceMap:
    """A loaded context that evaluates and differentiates the coherence map on
    its patch geometry (cells, bperp, low-pass, CLAP window).

    precision "fp32" runs forward and adjoint kernels in FP32 (gradients with
    respect to alpha / beta agree with FP64 to ~1e-7; those with respect to ph
    and K carry the FP32 conditioning of p = f / |f|, ~3e-3 in norm on the
    100k-PS differentiation shape, like torch's own FP32 autograd); "fp64"
    runs the same kernels in FP64 on the same float inputs and outputs."""

    def __init__(self, prepared: PreparedPatch, device: int = 0, precision: str = "fp32"):
        if precision not in ("fp32", "fp64"):
            raise ValueError(f"precision must be 'fp32' or 'fp64', got {precision!r}")
        self.prepared = prepared
        self.precision = precision
        self.device = torch.device("cuda", device)
        self.ctx = Stage2Context(device)
        self.ctx.load(prepared, PRECISION_FP64 if precision == "fp64" else PRECISION_FP32)
        self.n_ps, self.n_ifg = prepared.n_ps, prepared.n_ifg

    def close(self) -> None:
        self.ctx.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, ph: torch.Tensor, K: torch.Tensor, w: torch.Tensor) -> None:
        if ph.dtype != torch.complex64 or tuple(ph.shape) != (self.n_ps, self.n_ifg):
            raise ValueError(f"ph must be complex64 [{self.n_ps}, {self.n_ifg}], got {ph.dtype} {tuple(ph.shape)}")
        for name, t in (("K", K), ("w", w)):
            if t.dtype != torch.float32 or tuple(t.shape) != (self.n_ps,):
                raise ValueError(f"{name} must be float32 [{self.n_ps}], got {t.dtype} {tuple(t.shape)}")
        for name, t in (("ph", ph), ("K", K), ("w", w)):
            if t.device != self.device or not t.is_contiguous():
                raise ValueError(f"{name} must be a contiguous tensor on {self.device}")

    def forward(self, ph, K, w, alpha: float, beta: float) -> torch.Tensor:
        self._check(ph, K, w)
        coh = torch.empty(self.n_ps, dtype=torch.float32, device=self.device)
        st = torch.cuda.current_stream(self.device).cuda_stream
        check(_lib.lib().ps2_coherence_forward(
            self.ctx._ctx, _vp(ph.data_ptr()), _vp(K.data_ptr()), _vp(w.data_ptr()), _d(alpha), _d(beta),
            _vp(coh.data_ptr()), _vp(st)))
        return coh

    def backward(self, ph, K, w, alpha: float, beta: float, gcoh: torch.Tensor):
        self._check(ph, K, w)
        gcoh = gcoh.to(torch.float32).contiguous()
        gph = torch.empty_like(ph)
        gK = torch.empty_like(K)
        gab = torch.empty(2, dtype=torch.float64, device=self.device)
        st = torch.cuda.current_stream(self.device).cuda_stream
        check(_lib.lib().ps2_coherence_backward(
            self.ctx._ctx, _vp(ph.data_ptr()), _vp(K.data_ptr()), _vp(w.data_ptr()), _d(alpha), _d(beta),
            _vp(gcoh.data_ptr()), _vp(gph.data_ptr()), _vp(gK.data_ptr()), _vp(gab.data_ptr()), _vp(st)))
        return gph, gK, gab

    def launch_count(self) -> int:
        return int(self.ctx.launch_count())


class _Coherence(torch.autograd.Function):
    @staticmethod
    def forward(ctx, ph, K, alpha, beta, w, cmap: CoherenceMap):
        a, b = float(alpha), float(beta)
        coh = cmap.forward(ph.detach().contiguous(), K.detach().contiguous(), w.detach().contiguous(), a, b)
        ctx.save_for_backward(ph, K, w)
        ctx.cmap, ctx.a, ctx.b = cmap, a, b
        ctx.alpha_like = (alpha.dtype, alpha.device) if torch.is_tensor(alpha) else None
        ctx.beta_like = (beta.dtype, beta.device) if torch.is_tensor(beta) else None
        return coh

    @staticmethod
    def backward(ctx, gcoh):
        ph, K, w = ctx.saved_tensors
        gph, gK, gab = ctx.cmap.backward(ph.detach().contiguous(), K.detach().contiguous(), w.detach().contiguous(),
                                         ctx.a, ctx.b, gcoh)
        ga = gab[0].to(*ctx.alpha_like[::-1]) if ctx.alpha_like is not None else None
        gb = gab[1].to(*ctx.beta_like[::-1]) if ctx.beta_like is not None else None
        return gph, gK, ga, gb, None, None


def coherence(cmap: CoherenceMap, ph: torch.Tensor, K: torch.Tensor, alpha, beta,
              w: torch.Tensor | None = None) -> torch.Tensor:
    """Per-PS coherence [n_ps] (float32), differentiable in ph, K, alpha and
    beta (alpha / beta as 0-dim tensors to get their gradients). w is the
    per-PS bin weight (default 1)."""
    if w is None:
        w = torch.ones(cmap.n_ps, dtype=torch.float32, device=cmap.device)
    return _Coherence.apply(ph, K, alpha, beta, w, cmap)


def calibrate_clap(cmap: CoherenceMap, ph: torch.Tensor, K: torch.Tensor, *, alpha0: float = 1.0,
                   beta0: float = 0.3, steps: int = 20, lr: float = 0.05, w: torch.Tensor | None = None,
                   loss_fn: Callable[[torch.Tensor], torch.Tensor] | None = None) -> dict:
    """CLAP parameter calibration: Adam steps on (log alpha, log beta) to
    minimise loss_fn(coh) (default: minus the mean coherence). Returns the
    final parameters and the loss / parameter history."""
    loss_fn = loss_fn or (lambda coh: -coh.double().mean())
    la = torch.tensor(math.log(alpha0), dtype=torch.float64, device=cmap.device, requires_grad=True)
    lb = torch.tensor(math.log(beta0), dtype=torch.float64, device=cmap.device, requires_grad=True)
    opt = torch.optim.Adam([la, lb], lr=lr)
    hist = []
    for _ in range(steps):
        opt.zero_grad()
        alpha, beta = la.exp(), lb.exp()
        loss = loss_fn(coherence(cmap, ph, K, alpha, beta, w))
        loss.backward()
        hist.append({"alpha": float(alpha.detach()), "beta": float(beta.detach()), "loss": float(loss.detach())})
        opt.step()
    with torch.no_grad():
        alpha, beta = float(la.exp()), float(lb.exp())
        final = float(loss_fn(coherence(cmap, ph, K, torch.tensor(alpha), torch.tensor(beta), w)))
    hist.append({"alpha": alpha, "beta": beta, "loss": final})
    return {"alpha": alpha, "beta": beta, "loss": final, "history": hist}
