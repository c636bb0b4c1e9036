"""The FP64 torch restatement used to check the CUDA adjoints, pinned on CPU
against the oracle's FP64 CLAP (clap_filter_grid_stack) and against torch's
own finite differences of itself."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from torch_coherence_ref import clap_geometry, torch_clap  # noqa: E402


@pytest.mark.parametrize("n_i,n_j,m,alpha,beta", [(40, 50, 3, 1.0, 0.3), (30, 37, 2, 1.7, 0.45), (24, 24, 1, 0.8, 0.5)])
def test_torch_clap_matches_oracle_fp64(oracle, n_i, n_j, m, alpha, beta):
    rng = np.random.default_rng(n_i * 100 + n_j)
    g = rng.standard_normal((n_i, n_j, m)) + 1j * rng.standard_normal((n_i, n_j, m))
    g[rng.random((n_i, n_j)) < 0.2] = 0  # empty cells
    lp = oracle.build_low_pass(32)
    ref = oracle.clap_filter_grid_stack(g, alpha, beta, lp, 24, fp64=True)
    geo = dict(clap_geometry(n_i, n_j, 24, lp, "cpu"), alpha=alpha, beta=beta)
    out = torch_clap(geo, torch.from_numpy(g.reshape(-1, m).astype(np.complex128))).numpy().reshape(n_i, n_j, m)
    err = np.abs(out - ref).max() / np.abs(ref).max()
    assert err <= 1e-12, err


def test_torch_clap_alpha_beta_gradients_match_differences():
    rng = np.random.default_rng(3)
    n_i, n_j, m = 30, 30, 2
    g = torch.from_numpy(rng.standard_normal((n_i * n_j, m)) + 1j * rng.standard_normal((n_i * n_j, m)))
    lp = np.zeros((32, 32))
    lp[:4, :4] = 1.0
    gw = torch.from_numpy(rng.standard_normal((n_i * n_j, m)) + 1j * rng.standard_normal((n_i * n_j, m)))

    def L(a, b):
        geo = dict(clap_geometry(n_i, n_j, 24, lp, "cpu"), alpha=a, beta=b)
        return (torch_clap(geo, g) * gw.conj()).real.sum()

    a = torch.tensor(1.3, dtype=torch.float64, requires_grad=True)
    b = torch.tensor(0.4, dtype=torch.float64, requires_grad=True)
    L(a, b).backward()
    h = 1e-6
    fa = (L(1.3 + h, 0.4) - L(1.3 - h, 0.4)) / (2 * h)
    fb = (L(1.3, 0.4 + h) - L(1.3, 0.4 - h)) / (2 * h)
    assert abs(float(a.grad) - float(fa)) <= 1e-6 * abs(float(fa))
    assert abs(float(b.grad) - float(fb)) <= 1e-6 * abs(float(fb))
