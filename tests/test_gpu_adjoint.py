"""Adjoints of the stage-2 coherence (ps2_coherence_forward / _backward)
against an FP64 torch-ops restatement of the same map and FP64 central
finite differences, on the differentiation shape (100,000 PS, 40
interferograms, 96 x 96 grid).

The map (K given): bin ph * exp(-j K bperp) * w per cell, CLAP-filter the
grid (crates/pystamps-core/src/native_stage2.rs:904-1184), resample and
normalise, coherence of conj(p) ph exp(-j K bperp) (:1257-1303). The loss is
the mean coherence over the stable 30% of the synthetic PS; gradients are
taken with respect to ph (complex64), K (float32), clap_alpha and clap_beta.

Finite differences: central, step 1e-4, 64 random directions cycling over
ph-only, K-only, alpha-only, beta-only and all-at-once. The map has kinks
(the median's order statistics, the (.)+ clamp); a direction is used only if
the FP64 map takes every kink decision the same way at -h, 0 and +h, and is
redrawn otherwise (at most 4 times). Direction blocks are Gaussian with norm
0.1 (ph), 1e-4 (K: the step then moves no phase by more than ~1e-8 rad) and
1 (alpha, beta), so that most draws stay between kinks.

Two adjoint precisions run through the same kernels: a context loaded FP64
gives FP64 arithmetic, FP32 gives FP32. Tolerances: forward |d coh| <= 2e-5
(FP32) and <= 1e-9 (FP64) against the FP64 torch map; the FP64 adjoint within
1e-6 relative of the FP64 autograd gradient and every directional derivative
within 1e-3 relative of the FP64 central difference; the FP32 adjoint within
1e-3 relative for alpha and beta (also against central differences) and, for
ph and K, in norm no more than twice the error torch's own FP32 autograd
makes on the same map (the FP32 conditioning of the normalisation p = f/|f|).
"""
import math

import numpy as np
import pytest

from torch_coherence_ref import geometry, same_kinks, torch_coherence

pytestmark = pytest.mark.gpu

FD_STEP = 1e-4
FD_REL_TOL = 1e-3
GRAD_REL_TOL = 1e-3
N_DIRECTIONS = 64
SCALES = {"ph": 0.1, "K": 1e-4, "a": 1.0, "b": 1.0}


@pytest.fixture(scope="module")
def env(cuda_lib):
    import torch

    from pystamps_b200 import autograd as AG
    from pystamps_b200 import stage2 as S
    from pystamps_b200 import synth

    patch = synth.make_workload("D")
    stable = np.asarray(patch["truth"]["stable"], dtype=bool)
    prep = S.prepare_patch(patch)
    dev = torch.device("cuda", 0)
    # a realistic K: the first gamma iteration's estimate (invalid rows -> 0)
    with S.Stage2Context(0) as c:
        c.load(prep, "fp32")
        c.iterate(1)
        K = c.download(["K_ps"])["K_ps"]
    K = np.nan_to_num(K.astype(np.float32), nan=0.0)
    cmap = AG.CoherenceMap(prep, 0)
    cmap64 = AG.CoherenceMap(prep, 0, "fp64")
    ph = torch.from_numpy(np.ascontiguousarray(prep.ph_nm, dtype=np.complex64)).to(dev)
    Kt = torch.from_numpy(K).to(dev)
    w = torch.from_numpy(np.asarray(prep.weight0, dtype=np.float32)).to(dev)
    geo = geometry(prep, dev)
    gcoh = torch.from_numpy(stable.astype(np.float64) / stable.sum()).to(dev)
    yield {"AG": AG, "S": S, "prep": prep, "cmap": cmap, "cmap64": cmap64, "ph": ph, "K": Kt, "w": w, "geo": geo,
           "torch": torch, "gcoh": gcoh}
    cmap.close()
    cmap64.close()


def _cuda_grads(env, alpha, beta, gcoh, cmap="cmap"):
    torch = env["torch"]
    ph = env["ph"].clone().requires_grad_(True)
    K = env["K"].clone().requires_grad_(True)
    a = torch.tensor(alpha, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(beta, dtype=torch.float64, requires_grad=True)
    coh = env["AG"].coherence(env[cmap], ph, K, a, b, env["w"])
    (coh.double() * gcoh).sum().backward()
    torch.cuda.synchronize()
    return coh.detach(), ph.grad, K.grad, float(a.grad), float(b.grad)


def _ref_grads(env, alpha, beta, gcoh, fp32=False):
    torch = env["torch"]
    if fp32:
        geo = {k: (v.float() if torch.is_tensor(v) and v.dtype == torch.float64 else v) for k, v in env["geo"].items()}
        ph, K, w, dt = env["ph"].clone(), env["K"].clone(), env["w"], torch.float32
    else:
        geo = env["geo"]
        ph, K, w, dt = env["ph"].to(torch.complex128), env["K"].double(), env["w"].double(), torch.float64
    ph.requires_grad_(True)
    K.requires_grad_(True)
    a = torch.tensor(alpha, dtype=dt, device=ph.device, requires_grad=True)
    b = torch.tensor(beta, dtype=dt, device=ph.device, requires_grad=True)
    coh = torch_coherence(geo, ph, K, w, a, b)
    (coh.double() * gcoh).sum().backward()
    return coh.detach(), ph.grad, K.grad, float(a.grad), float(b.grad)


def _rel(a, b):
    torch = __import__("torch")
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    return float((a - b).abs().norm() / b.abs().norm())


PARAMS = [(1.0, 0.3), (0.8, 0.5)]


@pytest.mark.parametrize("alpha,beta", PARAMS)
def test_forward_matches_fp64(env, alpha, beta):
    torch = env["torch"]
    ref = torch_coherence(env["geo"], env["ph"].to(torch.complex128), env["K"].double(), env["w"].double(),
                          alpha, beta)
    assert 0.05 < float(ref.mean()) < 0.99
    for name, tol in (("cmap", 2e-5), ("cmap64", 1e-6)):
        coh = env[name].forward(env["ph"], env["K"], env["w"], alpha, beta)
        # the FP64 path returns float32 coherences: its bound is float rounding
        d = (coh.double() - ref).abs()
        assert float(d.max()) <= tol, (name, float(d.max()))


@pytest.mark.parametrize("alpha,beta", PARAMS)
def test_fp64_adjoint_matches_fp64_autograd(env, alpha, beta):
    g = env["gcoh"]
    _, gph, gK, ga, gb = _cuda_grads(env, alpha, beta, g, "cmap64")
    _, rph, rK, ra, rb = _ref_grads(env, alpha, beta, g)
    e = (_rel(gph, rph), _rel(gK, rK), abs(ga - ra) / abs(ra), abs(gb - rb) / abs(rb))
    print(f"fp64 adjoint alpha {alpha} beta {beta}: e_ph {e[0]:.2e} e_K {e[1]:.2e} e_a {e[2]:.2e} e_b {e[3]:.2e}")
    assert max(e) <= 1e-6, e


@pytest.mark.parametrize("alpha,beta", PARAMS)
def test_gradients_match_fp64_autograd(env, alpha, beta):
    g = env["gcoh"]
    _, gph, gK, ga, gb = _cuda_grads(env, alpha, beta, g)
    _, rph, rK, ra, rb = _ref_grads(env, alpha, beta, g)
    _, fph, fK, _, _ = _ref_grads(env, alpha, beta, g, fp32=True)
    e_ph, e_K = _rel(gph, rph), _rel(gK, rK)
    f_ph, f_K = _rel(fph, rph), _rel(fK, rK)
    print(f"alpha {alpha} beta {beta}: cuda e_ph {e_ph:.2e} e_K {e_K:.2e} (torch fp32: {f_ph:.2e}, {f_K:.2e}); "
          f"e_alpha {abs(ga - ra) / abs(ra):.2e} e_beta {abs(gb - rb) / abs(rb):.2e}")
    assert abs(ga - ra) <= GRAD_REL_TOL * abs(ra), (ga, ra)
    assert abs(gb - rb) <= GRAD_REL_TOL * abs(rb), (gb, rb)
    assert e_ph <= max(2 * f_ph, GRAD_REL_TOL), (e_ph, f_ph)
    assert e_K <= max(2 * f_K, GRAD_REL_TOL), (e_K, f_K)


def test_directional_derivatives_match_central_differences(env):
    torch = env["torch"]
    alpha, beta = 1.0, 0.3
    gcoh = env["gcoh"]
    _, gph, gK, ga, gb = _cuda_grads(env, alpha, beta, gcoh, "cmap64")
    _, _, _, ga32, gb32 = _cuda_grads(env, alpha, beta, gcoh, "cmap")
    _, rph, rK, ra, rb = _ref_grads(env, alpha, beta, gcoh)
    geo = env["geo"]
    ph0 = env["ph"].to(torch.complex128)
    K0 = env["K"].double()
    w = env["w"].double()
    gen = torch.Generator(device="cuda").manual_seed(11)

    def L(t, v, kinks=None):
        vph, vK, va, vb = v
        coh = torch_coherence(geo, ph0 + t * vph, K0 + t * vK, w, alpha + t * va, beta + t * vb, kinks)
        return float((coh * gcoh).sum())

    def draw(pat):
        vph = torch.complex(torch.randn(ph0.shape, dtype=torch.float64, device="cuda", generator=gen),
                            torch.randn(ph0.shape, dtype=torch.float64, device="cuda", generator=gen))
        vK = torch.randn(K0.shape, dtype=torch.float64, device="cuda", generator=gen)
        s = torch.randn(2, dtype=torch.float64, device="cuda", generator=gen).sign()
        vph = vph * (SCALES["ph"] / float(vph.abs().norm())) if pat in (0, 4) else torch.zeros_like(vph)
        vK = vK * (SCALES["K"] / float(vK.norm())) if pat in (1, 4) else torch.zeros_like(vK)
        va = float(s[0]) * SCALES["a"] if pat in (2, 4) else 0.0
        vb = float(s[1]) * SCALES["b"] if pat in (3, 4) else 0.0
        return vph, vK, va, vb

    def dot(G, v):
        vph, vK, va, vb = v
        return (float((G[0].real.double() * vph.real + G[0].imag.double() * vph.imag).sum())
                + float((G[1].double() * vK).sum()) + G[2] * va + G[3] * vb)

    base = []
    L(0.0, draw(0), base)
    h = FD_STEP
    worst, worst_ref, worst32, redrawn = 0.0, 0.0, 0.0, 0
    for i in range(N_DIRECTIONS):
        pat = i % 5  # 0 ph, 1 K, 2 alpha, 3 beta, 4 all together
        for attempt in range(5):
            v = draw(pat)
            kp, km = [], []
            fp, fm = L(h, v, kp), L(-h, v, km)
            if same_kinks(base, kp) and same_kinks(base, km):
                break
            redrawn += 1
        else:
            pytest.fail(f"direction {i} (pattern {pat}) crossed a kink in 5 draws")
        fd = (fp - fm) / (2 * h)
        ad = dot((gph, gK, ga, gb), v)
        rd = dot((rph, rK, ra, rb), v)
        err = abs(ad - fd) / abs(fd)
        worst = max(worst, err)
        worst_ref = max(worst_ref, abs(rd - fd) / abs(fd))
        assert err <= FD_REL_TOL, (i, pat, ad, fd, rd)
        if pat in (2, 3):
            ad32 = ga32 * v[2] + gb32 * v[3]
            worst32 = max(worst32, abs(ad32 - fd) / abs(fd))
            assert abs(ad32 - fd) <= FD_REL_TOL * abs(fd), (i, pat, ad32, fd)
    print(f"{N_DIRECTIONS} directions ({redrawn} redrawn for kinks): max relative error fp64 adjoint {worst:.2e}, "
          f"fp32 adjoint (alpha, beta) {worst32:.2e}, fp64 torch autograd {worst_ref:.2e}")


def test_gradients_deterministic_and_launch_count(env):
    g = env["gcoh"]
    a1 = _cuda_grads(env, 1.0, 0.3, g)
    n = env["cmap"].launch_count()
    a2 = _cuda_grads(env, 1.0, 0.3, g)
    torch = env["torch"]
    assert torch.equal(a1[1], a2[1]) and torch.equal(a1[2], a2[2])
    assert a1[3] == a2[3] and a1[4] == a2[4]
    assert n == 15  # 6 recompute + gather, coherence, cell sum, CLAP, overlap, reduce, bin, 2 scatters


def test_clap_calibration_lowers_loss(env):
    AG = env["AG"]
    g = env["gcoh"]
    out = AG.calibrate_clap(env["cmap"], env["ph"], env["K"], alpha0=1.0, beta0=0.3, steps=6, lr=0.1, w=env["w"],
                            loss_fn=lambda coh: -(coh.double() * g).sum())
    assert out["loss"] < out["history"][0]["loss"]
    assert out["alpha"] > 0 and out["beta"] > 0


def test_bad_arguments_rejected(env):
    from pystamps_b200._lib import Stage2CudaError

    with pytest.raises(Stage2CudaError):
        env["cmap"].forward(env["ph"], env["K"], env["w"], -1.0, 0.3)
    with pytest.raises(Stage2CudaError):
        env["cmap"].backward(env["ph"], env["K"], env["w"], 1.0, float("nan"), env["gcoh"])
    with pytest.raises(ValueError):
        env["cmap"].forward(env["ph"][:10], env["K"], env["w"], 1.0, 0.3)
    with pytest.raises(ValueError):
        env["cmap"].forward(env["ph"], env["K"].double(), env["w"], 1.0, 0.3)
