"""FP64 torch-ops restatement of the differentiable stage-2 coherence map
(test infrastructure: the checker for the CUDA adjoints).

bin ph * exp(-j K bperp) * w per cell; CLAP filter of the grid
(crates/pystamps-core/src/native_stage2.rs:904-1184: 32-point FFT of each
zero-padded window, |H| smoothed by the 7x7 gausswin(7, 2.5) product in
fftshifted coordinates, median of the 1,024 values, max((H/med)^alpha-1, 0)
* beta + low-pass, inverse FFT, pyramid weight / 1024, overlap-add);
resample and normalise; coherence as in topofit's refine step (:1257-1303).
Differentiated by torch autograd in complex128 / float64.
"""
import math

import numpy as np


def _window_weight(nw):
    h = nw // 2
    out = np.zeros((nw, nw))
    for r in range(h):
        for c in range(h):
            out[r, c] = r + c + 1e-6
            out[r, h + c] = r + (h - 1 - c) + 1e-6
    for r in range(h):
        out[h + r] = out[h - 1 - r]
    return out / 1024.0


def clap_geometry(n_i, n_j, nw, low_pass, dev):
    """Window cells, pyramid weights (shifted for clamped edge windows),
    smoothing kernel and low-pass for a CLAP over an n_i x n_j grid."""
    import torch

    n_inc = max(nw // 4, 1)
    nwi = math.ceil(n_i / n_inc) - 3
    nwj = math.ceil(n_j / n_inc) - 3

    def axis(n, count):
        idx, shift = [], []
        for k in range(count):
            s = k * n_inc
            r = max(0, s + nw - n)
            idx.append(np.arange(s - r, s - r + nw))
            shift.append(r)
        return np.array(idx), np.array(shift)

    ri, rs = axis(n_i, nwi)
    cj, cs = axis(n_j, nwj)
    wt = _window_weight(nw)
    W = np.zeros((nwi, nwj, nw, nw))
    for a in range(nwi):
        for b in range(nwj):
            W[a, b, rs[a]:, cs[b]:] = wt[: nw - rs[a], : nw - cs[b]]
    cells = ri[:, None, :, None] * n_j + cj[None, :, None, :]
    sd = (7 - 1) / (2 * 2.5)
    g7 = np.exp(-0.5 * ((np.arange(7) - 3) / sd) ** 2)
    return {
        "n_i": n_i, "n_j": n_j, "nw": nw,
        "win_cells": torch.from_numpy(np.broadcast_to(cells, (nwi, nwj, nw, nw)).copy()).to(dev),
        "win_weight": torch.from_numpy(W).to(dev),
        "kern": torch.from_numpy(np.outer(g7, g7)).to(dev),
        "lp": torch.from_numpy(np.asarray(low_pass, dtype=np.float64).reshape(32, 32)).to(dev),
    }


def geometry(prep, dev):
    """clap_geometry plus the rows' cells and bperp of a prepared patch."""
    import torch

    geo = clap_geometry(prep.n_i, prep.n_j, prep.clap_window, prep.low_pass, dev)
    bp = np.asarray(prep.bperp, dtype=np.float64)
    geo.update({
        "cell": torch.from_numpy(np.asarray(prep.grid_lin, dtype=np.int64)).to(dev),
        "bp": torch.from_numpy(bp if bp.ndim == 2 else bp[None, :]).to(dev),
        "bp_max": float(np.abs(bp).max()),
    })
    return geo


def torch_clap(geo, grid, kinks=None):
    """CLAP of a grid [n_i * n_j, M] (complex) with the window geometry of geo.
    If `kinks` is a list, the non-smooth decisions are appended to it: the
    positions of the 512th / 513th order statistics of each window's smoothed
    spectrum and the active set of max((H/med)^alpha - 1, 0)."""
    import torch
    import torch.nn.functional as F

    alpha, beta = geo["alpha"], geo["beta"]
    G, M = grid.shape
    nw = geo["nw"]
    wc = geo["win_cells"]
    nwi, nwj = wc.shape[:2]
    x = grid[wc.reshape(-1)].reshape(nwi, nwj, nw, nw, M).permute(0, 1, 4, 2, 3)
    xp = torch.zeros(nwi, nwj, M, 32, 32, dtype=grid.dtype, device=grid.device)
    xp[..., :nw, :nw] = x
    X = torch.fft.fft2(xp)
    H = torch.fft.fftshift(X.abs(), dim=(-2, -1))
    Hs = F.conv2d(H.reshape(-1, 1, 32, 32), geo["kern"][None, None], padding=3).reshape(H.shape)
    Hs = torch.fft.ifftshift(Hs, dim=(-2, -1))
    srt, order = Hs.reshape(nwi, nwj, M, 1024).sort(dim=-1)
    med = 0.5 * (srt[..., 511] + srt[..., 512])
    Hn = Hs / med[..., None, None]
    if kinks is not None:
        kinks.append(order[..., 511:513].sort(dim=-1).values.detach().clone())
        kinks.append((Hn.detach() ** alpha > 1.0).clone())
    Gf = torch.relu(Hn ** alpha - 1.0) * beta + geo["lp"]
    y = torch.fft.ifft2(X * Gf) * 1024.0
    y = y[..., :nw, :nw] * geo["win_weight"][:, :, None]
    return torch.zeros(G, M, dtype=grid.dtype, device=grid.device).index_add(
        0, wc.reshape(-1), y.permute(0, 1, 3, 4, 2).reshape(-1, M))


def torch_coherence(geo, ph, K, w, alpha, beta, kinks=None):
    """The differentiable map in torch ops (complex128 / float64)."""
    import torch

    N, M = ph.shape
    kb = K[:, None] * geo["bp"]
    e = torch.complex(torch.cos(kb), -torch.sin(kb))
    G = geo["n_i"] * geo["n_j"]
    grid = torch.zeros(G, M, dtype=ph.dtype, device=ph.device).index_add(0, geo["cell"], ph * e * w[:, None])
    filt = torch_clap(dict(geo, alpha=alpha, beta=beta), grid, kinks)
    p = filt[geo["cell"]]
    mag = p.abs()
    pn = torch.where(mag > 0, p / torch.where(mag > 0, mag, torch.ones_like(mag)), torch.zeros_like(p))
    z = pn.conj() * ph
    S = (z * e).sum(1)
    D = z.abs().sum(1)
    return S.abs() / torch.where(D > 0, D, torch.ones_like(D))


def same_kinks(a, b):
    """True when two kink records (torch_clap's `kinks`) take every
    non-smooth decision the same way."""
    import torch

    return len(a) == len(b) and all(torch.equal(x, y) for x, y in zip(a, b))
