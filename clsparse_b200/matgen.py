"""Seeded synthetic CSR matrices for the workloads the library is measured on.

The reference benchmarks on downloaded University of Florida matrices
(cmake/ExternalMTX.cmake:61-74) that are not available here; these generators
stand in for them with the shapes and value distributions of the workloads
named for this path. Every generator is deterministic for a given seed and
returns (row_ptr uint32[n+1], col uint32[nnz], val float64[nnz]) with columns
sorted inside each row.
"""
from __future__ import annotations

import numpy as np


def _csr_from_coo(n, rows, cols, vals):
    order = np.lexsort((cols, rows))
    rows, cols, vals = rows[order], cols[order], vals[order]
    rp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(rp, rows.astype(np.int64) + 1, 1)
    rp = np.cumsum(rp)
    return rp.astype(np.uint32), cols.astype(np.uint32), vals.astype(np.float64)


def poisson2d(nx: int, ny: int | None = None):
    """2D 5-point Laplacian, Dirichlet: diagonal 4, neighbours -1.
    512x512 gives n = 262,144 and nnz = 1,308,672."""
    ny = nx if ny is None else ny
    n = nx * ny
    idx = np.arange(n, dtype=np.int64)
    i, j = idx % nx, idx // nx
    rows = [idx]
    cols = [idx]
    vals = [np.full(n, 4.0)]
    for di, dj in ((-1, 0), (1, 0), (0, -1), (0, 1)):
        ok = (i + di >= 0) & (i + di < nx) & (j + dj >= 0) & (j + dj < ny)
        rows.append(idx[ok])
        cols.append(idx[ok] + di + dj * nx)
        vals.append(np.full(int(ok.sum()), -1.0))
    return _csr_from_coo(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def _harmonic(a, b):
    return 2.0 * a * b / (a + b)


def diffusion(shape, k):
    """Cell-centred variable-coefficient diffusion on a 2D or 3D grid with
    Dirichlet walls: face coefficient = harmonic mean of the two cells, a wall
    face uses the cell's own coefficient. SPD with a 5- or 7-point pattern."""
    shape = tuple(int(s) for s in shape)
    n = int(np.prod(shape))
    k = np.asarray(k, dtype=np.float64).ravel()
    idx = np.arange(n, dtype=np.int64)
    coords = []
    rem = idx.copy()
    for s in shape:
        coords.append(rem % s)
        rem //= s
    strides = np.cumprod((1,) + shape[:-1])
    diag = np.zeros(n)
    rows, cols, vals = [], [], []
    for ax, s in enumerate(shape):
        for d in (-1, 1):
            ok = (coords[ax] + d >= 0) & (coords[ax] + d < s)
            nb = idx[ok] + d * strides[ax]
            kf = _harmonic(k[idx[ok]], k[nb])
            rows.append(idx[ok])
            cols.append(nb)
            vals.append(-kf)
            diag[idx[ok]] += kf
            diag[idx[~ok]] += k[idx[~ok]]
    rows.append(idx)
    cols.append(idx)
    vals.append(diag)
    return _csr_from_coo(n, np.concatenate(rows), np.concatenate(cols), np.concatenate(vals))


def diffusion3d_lognormal(m: int, sigma: float = 1.5, seed: int = 3):
    """3D 7-point diffusion on an m^3 grid, cell conductivity exp(N(0, sigma^2)).
    m = 128 gives n = 2,097,152 and nnz = 14,581,760."""
    rng = np.random.default_rng(seed)
    k = np.exp(rng.normal(0.0, sigma, size=m ** 3))
    return diffusion((m, m, m), k)


def grf2d(m: int, corr_len: float = 0.05, sigma: float = 2.0, seed: int = 5):
    """Gaussian random field on an m x m grid over [0,1]^2 with squared-
    exponential covariance, by FFT spectral synthesis; scaled to std sigma."""
    rng = np.random.default_rng(seed)
    f = np.fft.fftfreq(m, d=1.0 / m)
    kx, ky = np.meshgrid(f, f, indexing="ij")
    k2 = (2 * np.pi) ** 2 * (kx ** 2 + ky ** 2)
    spec = np.exp(-k2 * corr_len ** 2 / 4.0)
    noise = rng.normal(size=(m, m)) + 1j * rng.normal(size=(m, m))
    g = np.real(np.fft.ifft2(np.sqrt(spec) * noise))
    g = (g - g.mean()) / (g.std() + 1e-300) * sigma
    return g


def diffusion2d_grf(m: int, corr_len: float = 0.05, sigma: float = 2.0, seed: int = 5):
    """2D 5-point diffusion on m x m with coefficients exp(GRF)."""
    return diffusion((m, m), np.exp(grf2d(m, corr_len, sigma, seed)).ravel())


def irregular(n: int, mu: float = 2.5, sigma: float = 1.2, n_dense: int = 50,
              dense_len: int = 200_000, seed: int = 7, ncols: int | None = None):
    """Square matrix with log-normal row lengths max(1, round(exp(N(mu, sigma))))
    plus n_dense rows (seeded positions) of dense_len nonzeros; columns uniform
    without replacement inside each row, sorted; values U[-1, 1]."""
    ncols = n if ncols is None else ncols
    rng = np.random.default_rng(seed)
    lens = np.maximum(1, np.rint(np.exp(rng.normal(mu, sigma, size=n)))).astype(np.int64)
    lens = np.minimum(lens, ncols)
    if n_dense:
        pos = rng.choice(n, size=min(n_dense, n), replace=False)
        lens[pos] = min(dense_len, ncols)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rp[1:])
    nnz = int(rp[-1])
    if nnz >= 2 ** 32:
        raise ValueError("nnz exceeds 32-bit indices")
    if int(lens.max(initial=0)) * 2 > ncols:
        raise ValueError("rows longer than half the columns: use random_lengths")
    row_of = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = rng.integers(0, ncols, size=nnz, dtype=np.int64)
    # draw again wherever a row repeats a column, until every row is distinct
    for _ in range(64):
        key = row_of * ncols + cols
        order = np.argsort(key, kind="stable")
        ks = key[order]
        dup = np.zeros(nnz, dtype=bool)
        dup[1:] = ks[1:] == ks[:-1]
        if not dup.any():
            cols = ks % ncols
            break
        redo = order[dup]
        cols[redo] = rng.integers(0, ncols, size=redo.size, dtype=np.int64)
    else:
        raise RuntimeError("could not draw distinct columns")
    vals = rng.uniform(-1.0, 1.0, size=nnz)
    return rp.astype(np.uint32), cols.astype(np.uint32), vals


def random_lengths(lens, ncols: int, seed: int = 0, spd_shift: float | None = None):
    """CSR with the given row lengths, distinct sorted random columns and U[-1,1]
    values (edge-case matrices for the parity tests)."""
    rng = np.random.default_rng(seed)
    lens = np.minimum(np.asarray(lens, dtype=np.int64), ncols)
    n = len(lens)
    rp = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(lens, out=rp[1:])
    cols = np.empty(int(rp[-1]), dtype=np.int64)
    for r in range(n):
        L = int(lens[r])
        if L:
            cols[rp[r]:rp[r + 1]] = np.sort(rng.choice(ncols, size=L, replace=False))
    vals = rng.uniform(-1.0, 1.0, size=int(rp[-1]))
    return rp.astype(np.uint32), cols.astype(np.uint32), vals


def random_spd(n: int, per_row: int = 6, seed: int = 0):
    """Symmetric, strictly diagonally dominant (hence SPD) random sparse matrix."""
    rng = np.random.default_rng(seed)
    r = rng.integers(0, n, size=n * per_row)
    c = rng.integers(0, n, size=n * per_row)
    keep = r != c
    r, c = r[keep], c[keep]
    v = -rng.uniform(0.1, 1.0, size=r.size)
    rows = np.concatenate([r, c])
    cols = np.concatenate([c, r])
    vals = np.concatenate([v, v])
    key = rows * n + cols
    uk, inv = np.unique(key, return_inverse=True)
    sv = np.zeros(uk.size)
    np.add.at(sv, inv, vals)
    rows, cols, vals = uk // n, uk % n, sv
    diag = np.zeros(n)
    np.add.at(diag, rows, np.abs(vals))
    diag += rng.uniform(0.5, 1.5, size=n)
    rows = np.concatenate([rows, np.arange(n)])
    cols = np.concatenate([cols, np.arange(n)])
    vals = np.concatenate([vals, diag])
    return _csr_from_coo(n, rows, cols, vals)


def spmv_bytes(n_rows: int, n_cols: int, nnz: int, val_bytes: int, vec_bytes: int,
               beta_nonzero: bool = False) -> int:
    """Algorithmic bytes of one SpMV: the reference's formula
    (src/benchmarks/clsparse-bench/functions/clfunc_xSpMdV.hpp:91)
    4*(nnz + nrows) + sizeof(T)*(nnz + ncols + nrows), with value and vector
    sizes kept apart, plus one more read of y when beta != 0."""
    b = 4 * (nnz + n_rows) + val_bytes * nnz + vec_bytes * (n_cols + n_rows)
    if beta_nonzero:
        b += vec_bytes * n_rows
    return b


def stencil_prefix(n: int, dim: int, k):
    """The first n cells (natural order) of a dim-D cell grid just big enough
    to hold them, as a variable-coefficient diffusion operator: the principal
    n x n block of the full grid's operator, so still SPD."""
    side = int(np.ceil(n ** (1.0 / dim) - 1e-9))
    while side ** dim < n:
        side += 1
    rp, col, val = diffusion((side,) * dim, k[: side ** dim] if len(k) >= side ** dim else
                             np.resize(k, side ** dim))
    # keep rows < n and columns < n
    nnz_keep = int(rp[n])
    c = col[:nnz_keep]
    v = val[:nnz_keep]
    keep = c < n
    rows = np.repeat(np.arange(n), np.diff(rp[: n + 1]).astype(np.int64))[keep]
    out_rp = np.zeros(n + 1, dtype=np.int64)
    np.add.at(out_rp, rows + 1, 1)
    return np.cumsum(out_rp).astype(np.uint32), c[keep].astype(np.uint32), v[keep]


def batched_systems(num: int, n_min: int = 500, n_max: int = 50_000, sigma: float = 1.0, seed: int = 11):
    """`num` SPD systems, n log-uniform in [n_min, n_max], each a 2D 5-point or
    3D 7-point variable-coefficient diffusion (coin flip) with coefficients
    exp(N(0, sigma^2)), stacked block-diagonally. Returns (row_ptr, col, val,
    offsets, dims) with offsets the first row of each system (num + 1 entries)."""
    rng = np.random.default_rng(seed)
    ns = np.rint(np.exp(rng.uniform(np.log(n_min), np.log(n_max), size=num))).astype(np.int64)
    dims = rng.integers(2, 4, size=num)
    rps, cols, vals = [], [], []
    offsets = np.zeros(num + 1, dtype=np.int64)
    nnz_base = 0
    for s in range(num):
        n = int(ns[s])
        side = int(np.ceil(n ** (1.0 / dims[s]) - 1e-9)) + 1
        k = np.exp(rng.normal(0.0, sigma, size=side ** int(dims[s])))
        rp, c, v = stencil_prefix(n, int(dims[s]), k)
        offsets[s + 1] = offsets[s] + n
        rps.append(rp[:-1].astype(np.int64) + nnz_base)
        cols.append(c.astype(np.int64) + offsets[s])
        vals.append(v)
        nnz_base += int(rp[-1])
    rp_all = np.concatenate(rps + [np.array([nnz_base])]).astype(np.uint32)
    return rp_all, np.concatenate(cols).astype(np.uint32), np.concatenate(vals), offsets.astype(np.uint32), dims
