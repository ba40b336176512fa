"""The CPU oracle of the learned preconditioner: its analytic gradient against
central finite differences (directional, step 1e-7 to stay clear of ReLU
kinks), and the Kaporin loss's minimiser being the FSAI factor. CPU only."""
from __future__ import annotations

import numpy as np
import pytest

from clsparse_b200 import matgen
from oracle import gnn_oracle as go


@pytest.fixture(scope="module")
def small_graph():
    rp, c, v = matgen.diffusion2d_grf(5, corr_len=0.3, sigma=1.0, seed=2)
    return go.Graph(rp, c, v)


@pytest.mark.parametrize("lam", [0.0, 0.5])
def test_oracle_gradient_matches_finite_differences(small_graph, lam):
    rng = np.random.default_rng(1)
    p = rng.normal(0, 0.05, go.TOTAL)
    p[go.OFF["b_d"][0]] = 0.5413
    probes = [rng.normal(size=small_graph.n) for _ in range(2)] if lam else ()
    L, g = go.loss_grad(p, small_graph, probes, lam)
    for name in ("w_in", "U0", "V1", "c2", "w3", "P", "Q", "r", "w_o", "b_o", "w_d", "b_d"):
        o, s = go.OFF[name]
        d = np.zeros(go.TOTAL)
        d[o:o + s] = rng.normal(size=s)
        eps = 1e-7
        Lp, _ = go.loss_grad(p + eps * d, small_graph, probes, lam)
        Lm, _ = go.loss_grad(p - eps * d, small_graph, probes, lam)
        fd = (Lp - Lm) / (2 * eps)
        an = g @ d
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (name, fd, an)


def test_kaporin_loss_is_lowest_at_fsai(small_graph):
    """Among factors on the tril pattern, FSAI (rows solving B_i g_i = e_i,
    scaled to unit G A G^T diagonal) minimises the Kaporin term."""
    gr = small_graph
    g = np.zeros(len(gr.Lrow))
    for i in range(gr.n):
        k0, k1 = gr.Lrp[i], gr.Lrp[i + 1]
        e = np.zeros(k1 - k0)
        e[-1] = 1.0
        gi = np.linalg.solve(gr.blocks[i], e)
        g[k0:k1] = gi / np.sqrt(gi[-1])
    L0, dg = go.loss_and_dg(g, gr)
    assert np.abs(dg).max() < 1e-10
    rng = np.random.default_rng(3)
    for _ in range(5):
        L1, _ = go.loss_and_dg(g + 1e-3 * rng.normal(size=g.size), gr)
        assert L1 > L0


def test_bf16_round_matches_torch():
    """The oracle's BF16 rounding (ties to even through FP32) against torch's
    float32 -> bfloat16 conversion."""
    import torch
    rng = np.random.default_rng(3)
    x = np.concatenate([rng.normal(size=4000) * 10.0 ** rng.integers(-6, 6, 4000),
                        [1.0, 1.0 + 2.0 ** -8, 1.0 + 3 * 2.0 ** -8, -1.0 - 2.0 ** -8, 0.0]]).astype(np.float32)
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(go.bf16_round(x), ref)
    assert go.bf16_round(np.float32(1.0 + 2.0 ** -8)) == 1.0  # tie to even
