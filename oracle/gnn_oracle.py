"""CPU oracle of the learned factorized sparse approximate inverse -- TEST
INFRASTRUCTURE ONLY.

A float64 numpy restatement of the network, loss and gradients that
clsparse_b200/csrc/gnn.cu computes on the GPU (no reference counterpart: the
learned preconditioner is a project extension). Used by the tests to check the
GPU forward pass, loss and gradients, and checked itself against central
finite differences. The parameter layout matches the library's flat vector.
"""
from __future__ import annotations

import numpy as np

H, HO, NF, NL = 64, 32, 4, 4


def layout():
    off = {}
    k = 0

    def take(name, size):
        nonlocal k
        off[name] = (k, size)
        k += size

    take("w_in", H * NF)
    take("b_in", H)
    for l in range(NL):
        take(f"U{l}", H * H)
        take(f"w{l}", H)
        take(f"c{l}", H)
        take(f"V{l}", H * 2 * H)
        take(f"d{l}", H)
    take("P", HO * H)
    take("Q", HO * H)
    take("r", HO)
    take("t", HO)
    take("w_o", HO)
    take("b_o", 1)
    take("w_d", H)
    take("b_d", 1)
    return off, k


OFF, TOTAL = layout()


def unpack(p):
    out = {}
    for name, (o, s) in OFF.items():
        out[name] = np.asarray(p[o:o + s], dtype=np.float64)
    out["w_in"] = out["w_in"].reshape(H, NF)
    for l in range(NL):
        out[f"U{l}"] = out[f"U{l}"].reshape(H, H)
        out[f"V{l}"] = out[f"V{l}"].reshape(H, 2 * H)
    out["P"] = out["P"].reshape(HO, H)
    out["Q"] = out["Q"].reshape(HO, H)
    return out


def pack(d):
    p = np.zeros(TOTAL)
    for name, (o, s) in OFF.items():
        p[o:o + s] = np.asarray(d[name]).ravel()
    return p


class Graph:
    """Scaled operator, tril pattern, local loss blocks and node features of an
    SPD CSR matrix (sorted columns)."""

    def __init__(self, rp, col, val, with_blocks=True):
        rp = np.asarray(rp, dtype=np.int64)
        col = np.asarray(col, dtype=np.int64)
        val = np.asarray(val, dtype=np.float64)
        n = len(rp) - 1
        self.n = n
        rows = np.repeat(np.arange(n), np.diff(rp))
        diag = np.zeros(n)
        diag[rows[col == rows]] = val[col == rows]
        self.dinv = 1.0 / np.sqrt(diag)
        self.rows, self.cols = rows, col
        self.ehat = val * self.dinv[rows] * self.dinv[col]
        self.offdiag = col != rows
        keep = col <= rows
        self.Lrow, self.Lcol = rows[keep], col[keep]
        self.Le = self.ehat[keep]
        self.Lrp = np.concatenate([[0], np.cumsum(np.bincount(self.Lrow, minlength=n))])
        self.isdiag = self.Lrow == self.Lcol
        import scipy.sparse as sp
        self.Ahat = sp.csr_matrix((self.ehat, col, rp), shape=(n, n))
        absum = np.bincount(rows[self.offdiag], weights=np.abs(self.ehat[self.offdiag]), minlength=n)
        deg = np.bincount(rows[self.offdiag], minlength=n)
        self.F = np.stack([np.ones(n), absum, deg / 8.0, np.zeros(n)], axis=1)
        Ad = self.Ahat.toarray() if n <= 4000 and with_blocks else None
        self.blocks = []  # loss blocks; not needed for the forward pass alone
        for i in range(n if with_blocks else 0):
            P = self.Lcol[self.Lrp[i]:self.Lrp[i + 1]]
            if Ad is not None:
                self.blocks.append(Ad[np.ix_(P, P)])
            else:
                self.blocks.append(self.Ahat[P][:, P].toarray())

    def G_hat(self, g):
        import scipy.sparse as sp
        return sp.csr_matrix((g, (self.Lrow, self.Lcol)), shape=(self.n, self.n))


def relu(z):
    return np.maximum(z, 0.0)


def softplus(z):
    return np.where(z > 20, z, np.log1p(np.exp(np.minimum(z, 20))))


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


def bf16_round(x):
    """Round to the nearest BF16 value (ties to even) through FP32, as
    __float2bfloat16_rn does; returned as float64."""
    u = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32)
    u = (u + (((u >> 16) & 1) + 0x7FFF)) & 0xFFFF0000
    return u.view(np.float32).astype(np.float64)


def forward(p, gr: Graph, bf16=False):
    """The network's forward pass. bf16=True restates the library's BF16
    inference: every weight is rounded to BF16, and the four dense layers that
    run on tensor cores (U, V, P, Q) also round their inputs (FP32 activations)
    to BF16; accumulation stays wide."""
    W = unpack(p)
    if bf16:
        W = {k: bf16_round(v) for k, v in W.items()}
    rx = bf16_round if bf16 else (lambda v: v)
    c = {}
    h = relu(gr.F @ W["w_in"].T + W["b_in"])
    c["H0"] = h
    Hs = [h]
    for l in range(NL):
        hu = rx(h) @ W[f"U{l}"].T
        pre = hu[gr.cols] + gr.ehat[:, None] * W[f"w{l}"] + W[f"c{l}"]
        msg = relu(pre) * gr.offdiag[:, None]
        s = np.zeros_like(h)
        np.add.at(s, gr.rows, msg)
        z = rx(np.concatenate([h, s], axis=1)) @ W[f"V{l}"].T + W[f"d{l}"]
        a = relu(z)
        c[f"Hu{l}"], c[f"pre{l}"], c[f"S{l}"], c[f"Z{l}"] = hu, pre, s, z
        h = h + a
        Hs.append(h)
    c["Hs"] = Hs
    hp = rx(h) @ W["P"].T
    hq = rx(h) @ W["Q"].T
    pre_o = hp[gr.Lrow] + hq[gr.Lcol] + gr.Le[:, None] * W["r"] + W["t"]
    z_d = h @ W["w_d"] + W["b_d"][0]
    g = np.where(gr.isdiag, softplus(z_d[gr.Lrow]), relu(pre_o) @ W["w_o"] + W["b_o"][0])
    c.update(hp=hp, hq=hq, pre_o=pre_o, z_d=z_d)
    return g, c


def loss_and_dg(g, gr: Graph, probes=(), lam=0.0):
    n = gr.n
    tr = 0.0
    logsum = 0.0
    dg = np.zeros_like(g)
    Bg = []
    for i in range(n):
        k0, k1 = gr.Lrp[i], gr.Lrp[i + 1]
        gi = g[k0:k1]
        bgi = gr.blocks[i] @ gi
        Bg.append(bgi)
        tr += gi @ bgi
        logsum += np.log(gi[-1])
    for i in range(n):
        k0, k1 = gr.Lrp[i], gr.Lrp[i + 1]
        dg[k0:k1] = 2.0 * Bg[i] / tr
        dg[k1 - 1] -= 2.0 / (n * g[k1 - 1])
    L = np.log(tr / n) - 2.0 * logsum / n
    if probes is not None and len(probes) and lam > 0:
        G = gr.G_hat(g)
        K = len(probes)
        for r in probes:
            rr = r @ r
            w = gr.Ahat @ r
            u = G @ w
            v = G.T @ u
            d = v - r
            L += lam * (d @ d) / (K * rr)
            dv = 2.0 * lam * d / (K * rr)
            du = G @ dv
            dg += dv[gr.Lcol] * u[gr.Lrow] + du[gr.Lrow] * w[gr.Lcol]
    return L, dg


def backward(p, gr: Graph, c, dg):
    W = unpack(p)
    grad = {k: np.zeros_like(v) for k, v in W.items()}
    h = c["Hs"][NL]
    dh = np.zeros_like(h)
    # output layer
    dz_d = np.zeros(gr.n)
    np.add.at(dz_d, gr.Lrow[gr.isdiag], dg[gr.isdiag] * sigmoid(c["z_d"][gr.Lrow[gr.isdiag]]))
    grad["w_d"] += h.T @ dz_d
    grad["b_d"] += dz_d.sum()
    dh += np.outer(dz_d, W["w_d"])
    off = ~gr.isdiag
    a_o = relu(c["pre_o"])
    grad["w_o"] += (dg[off, None] * a_o[off]).sum(0)
    grad["b_o"] += dg[off].sum()
    dpre = (dg[:, None] * W["w_o"]) * (c["pre_o"] > 0) * off[:, None]
    grad["r"] += (dpre * gr.Le[:, None]).sum(0)
    grad["t"] += dpre.sum(0)
    dhp = np.zeros((gr.n, HO))
    dhq = np.zeros((gr.n, HO))
    np.add.at(dhp, gr.Lrow, dpre)
    np.add.at(dhq, gr.Lcol, dpre)
    grad["P"] += dhp.T @ h
    grad["Q"] += dhq.T @ h
    dh += dhp @ W["P"] + dhq @ W["Q"]
    for l in reversed(range(NL)):
        hl = c["Hs"][l]
        dz = dh * (c[f"Z{l}"] > 0)
        x = np.concatenate([hl, c[f"S{l}"]], axis=1)
        grad[f"V{l}"] += dz.T @ x
        grad[f"d{l}"] += dz.sum(0)
        dx = dz @ W[f"V{l}"]
        dh_l = dh + dx[:, :H]
        ds = dx[:, H:]
        dmsg = ds[gr.rows] * (c[f"pre{l}"] > 0) * gr.offdiag[:, None]
        grad[f"w{l}"] += (dmsg * gr.ehat[:, None]).sum(0)
        grad[f"c{l}"] += dmsg.sum(0)
        dhu = np.zeros_like(hl)
        np.add.at(dhu, gr.cols, dmsg)
        grad[f"U{l}"] += dhu.T @ hl
        dh_l += dhu @ W[f"U{l}"]
        dh = dh_l
    dz0 = dh * (c["H0"] > 0)
    grad["w_in"] += dz0.T @ gr.F
    grad["b_in"] += dz0.sum(0)
    return pack(grad)


def loss_grad(p, gr: Graph, probes=(), lam=0.0):
    g, c = forward(p, gr)
    L, dg = loss_and_dg(g, gr, probes, lam)
    return L, backward(p, gr, c, dg)
