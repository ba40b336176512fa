"""Autotuner for the CSR-Adaptive row-block shape and the batched solver's
lanes per row, and the tuning table it writes.

SpMV. The reference fixes the row-block shape at compile time (BLKSIZE 1024,
BLOCK_MULTIPLIER 3, ROWS_FOR_VECTOR 1; src/library/include/clSPARSE-private.hpp:46-50,
used by ComputeRowBlocks, src/library/internal/data-types/csr-meta.hpp:52-269).
`tune_spmv` sweeps those knobs and the adaptive kernel's CTA width for one
matrix: every candidate meta is built with clsparseB200CsrMetaCreateTuned, its
SpMV result is checked against the reference-shape result (parity at every
point: a candidate that disagrees raises), and it is timed with CUDA events
(median of `reps` launches). The fastest shape is returned with the whole
sweep.

Matrices whose rows are all at most 16 long (stencils) take the library's
thread-per-row path whatever the meta's shape, so for them every candidate
times the same kernel and the sweep only confirms parity; the table's entries
for such matrices (poisson512, diffusion3d_64) were measured with the
row-block kernel (CLSPARSE_B200_SHORT_ROWS=0) and apply only under that
setting.

Batched CG. `tune_batched_lanes` times clsparseScsrcgBatched on batches of one
size class at a time with every lanes-per-row width and keeps the fastest per
class.

Table. `TuningTable` holds SpMV entries keyed by matrix features (rows, mean
and maximum row length, coefficient of variation of row lengths) and the
batched size classes; `lookup_shape` returns the shape of the nearest entry
(distance in log-feature space), `lanes_for` the lanes of each system.

    python -m clsparse_b200.autotune --out tuning.json   # sweep the standard set on this GPU
"""
from __future__ import annotations

import argparse
import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

SHAPES_DEFAULT = (1024, 3, 1, 128)

# Candidate shapes: (blk_size, blk_multiplier, rows_for_vector, cta_threads).
CANDIDATES = tuple(
    (blk, mult, rfv, nt)
    for blk in (512, 1024, 2048)
    for mult in (1, 3, 8)
    for rfv in (1, 4)
    for nt in (128, 256)
    if not (blk == 512 and nt == 256)
)

LANES = (1, 2, 4, 8, 16)


def features(rp) -> dict:
    """Row-length statistics of a CSR row pointer."""
    rp = np.asarray(rp, dtype=np.int64)
    n = len(rp) - 1
    lens = np.diff(rp).astype(np.float64)
    mean = float(lens.mean()) if n else 0.0
    std = float(lens.std()) if n else 0.0
    return {"rows": int(n), "mean_row": mean, "max_row": float(lens.max()) if n else 0.0,
            "cv_row": std / mean if mean > 0 else 0.0}


def _fvec(f: dict) -> np.ndarray:
    return np.array([math.log1p(f["rows"]), math.log1p(f["mean_row"]), math.log1p(f["max_row"]),
                     math.log1p(f["cv_row"])])


@dataclass
class TuningTable:
    spmv: list = field(default_factory=list)      # {"features", "shape", "us", "default_us"}
    batched: list = field(default_factory=list)   # {"n_min", "n_max", "lanes"}
    device: str = ""

    def add_spmv(self, feats: dict, shape, us: float, default_us: float, name: str = ""):
        self.spmv.append({"name": name, "features": feats, "shape": list(shape), "us": us,
                          "default_us": default_us})

    def lookup_shape(self, feats: dict):
        """Shape of the nearest tuned matrix; the reference shape when empty."""
        if not self.spmv:
            return SHAPES_DEFAULT
        q = _fvec(feats)
        best = min(self.spmv, key=lambda e: float(np.sum((_fvec(e["features"]) - q) ** 2)))
        return tuple(best["shape"])

    def lanes_for(self, sizes) -> np.ndarray:
        """Lanes per row for systems of the given row counts (0: the library's default)."""
        out = np.zeros(len(sizes), dtype=np.int32)
        for i, n in enumerate(sizes):
            for c in self.batched:
                if c["n_min"] <= n < c["n_max"]:
                    out[i] = c["lanes"]
                    break
        return out

    def save(self, path):
        Path(path).write_text(json.dumps({"device": self.device, "spmv": self.spmv, "batched": self.batched},
                                         indent=1))

    @classmethod
    def load(cls, path):
        d = json.loads(Path(path).read_text())
        return cls(spmv=d.get("spmv", []), batched=d.get("batched", []), device=d.get("device", ""))


def _time_spmv(api, ctrl, A, x, y, one, zero, reps):
    """Median per-launch time (us) with the control in async mode (no host
    synchronisation between launches). The control must run on torch's
    current stream."""
    import torch
    ctrl.enable_async(True)
    try:
        for _ in range(3):
            api.csrmv(one, A, x, zero, y, ctrl)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        stream = torch.cuda.current_stream()
        for s, e in ev:
            s.record(stream)
            api.csrmv(one, A, x, zero, y, ctrl)
            e.record(stream)
        torch.cuda.synchronize()
    finally:
        ctrl.enable_async(False)
    return float(np.median([s.elapsed_time(e) * 1000.0 for s, e in ev]))


def tune_spmv(ctrl, rp, col, val, dtype=None, candidates=CANDIDATES, reps=20, rtol=None):
    """Sweeps row-block shapes for one matrix. Returns (best_shape, best_us,
    default_us, sweep) where sweep is a list of (shape, us). Raises
    AssertionError when a candidate's SpMV result departs from the
    reference-shape result by more than rtol relative to the row scale
    sum_j |a_ij x_j|."""
    import torch

    from . import api
    dtype = dtype or torch.float64
    if rtol is None:
        rtol = 1e-12 if dtype == torch.float64 else 1e-5
    A = api.CsrMatrix.from_numpy(rp, col, val, dtype=dtype)
    n = A.num_rows
    x = torch.tensor(np.random.default_rng(11).uniform(-1, 1, A.num_cols), dtype=dtype, device="cuda")
    y = torch.zeros(n, dtype=dtype, device="cuda")
    one = torch.ones(1, dtype=dtype, device="cuda")
    zero = torch.zeros(1, dtype=dtype, device="cuda")
    # scale of every row for the parity check: |A| |x|
    Aabs = api.CsrMatrix(A.row_ptr, A.col, A.val.abs(), A.num_cols)
    scale = torch.zeros(n, dtype=dtype, device="cuda")
    api.csrmv(one, Aabs, x.abs(), zero, scale, ctrl)
    A.create_meta(ctrl)
    api.csrmv(one, A, x, zero, y, ctrl)
    y_ref = y.clone()
    default_us = _time_spmv(api, ctrl, A, x, y, one, zero, reps)
    sweep = []
    for shape in candidates:
        A.create_meta(ctrl, shape=shape)
        y.fill_(float("nan"))
        api.csrmv(one, A, x, zero, y, ctrl)
        err = (y - y_ref).abs()
        bad = err > rtol * scale + 1e-300
        assert not bool(bad.any()), f"shape {shape}: SpMV differs from the reference shape"
        sweep.append((tuple(shape), _time_spmv(api, ctrl, A, x, y, one, zero, reps)))
    A.delete_meta()
    best_shape, best_us = min(sweep, key=lambda t: t[1])
    if default_us <= best_us:
        best_shape, best_us = SHAPES_DEFAULT, default_us
    return best_shape, best_us, default_us, sweep


def tune_batched_lanes(ctrl, classes=((500, 2000), (2000, 8000), (8000, 50001)), per_class=64, seed=21,
                       lanes=LANES):
    """Fastest lanes-per-row width for the batched solver, per size class of
    system row counts. Returns [{"n_min", "n_max", "lanes", "times_s"}]."""
    import time

    import torch

    from . import _lib as L
    from . import api, matgen
    out = []
    for lo, hi in classes:
        rp, col, val, off, _ = matgen.batched_systems(per_class, lo, hi - 1, sigma=1.0, seed=seed)
        A = api.CsrMatrix.from_numpy(rp, col, val, dtype=torch.float32)
        n = A.num_rows
        b = torch.tensor(np.random.default_rng(seed).uniform(-1, 1, n), dtype=torch.float32, device="cuda")
        times, conv = {}, {}
        for w in lanes:
            x = torch.zeros(n, dtype=torch.float32, device="cuda")
            sc = api.SolverControl(L.DIAGONAL, 20000, 1e-6, 0.0)
            ln = np.full(per_class, w, dtype=np.int32)
            api.cg_batched(x, A, b, off, sc, ctrl, lanes=ln)  # captures the graph
            x.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = api.cg_batched(x, A, b, off, sc, ctrl, lanes=ln)
            torch.cuda.synchronize()
            times[w] = time.perf_counter() - t0
            conv[w] = int(res["converged"])
            sc.release()
        # fastest among the widths that converged the most systems
        top = max(conv.values())
        best = min((w for w in lanes if conv[w] == top), key=times.get)
        out.append({"n_min": lo, "n_max": hi, "lanes": int(best), "times_s": times, "converged": conv,
                    "systems": per_class})
    return out


def standard_set():
    """Synthetic matrices the shipped table is tuned on (name, (rp, col, val))."""
    from . import matgen
    return [
        ("poisson512", matgen.poisson2d(512)),
        ("diffusion3d_64", matgen.diffusion3d_lognormal(64, sigma=1.5, seed=3)),
        ("irregular_500k", matgen.irregular(500_000, mu=2.5, sigma=1.2, n_dense=12, dense_len=200_000, seed=7)),
        ("irregular_2M", matgen.irregular(2_000_000, mu=2.5, sigma=1.2, n_dense=50, dense_len=200_000, seed=7)),
        ("irregular_short_1M", matgen.irregular(1_000_000, mu=1.5, sigma=0.6, n_dense=1, dense_len=5000, seed=9)),
    ]


def main():
    import torch

    from . import api
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--reps", type=int, default=20)
    args = ap.parse_args()
    api.setup()
    ctrl = api.Control()
    table = TuningTable(device=torch.cuda.get_device_name(0))
    for name, (rp, col, val) in standard_set():
        shape, us, dus, sweep = tune_spmv(ctrl, rp, col, val, reps=args.reps)
        table.add_spmv(features(rp), shape, us, dus, name)
        print(json.dumps({"matrix": name, "best": shape, "us": round(us, 2), "default_us": round(dus, 2),
                          "sweep": [(list(s), round(t, 2)) for s, t in sweep]}), flush=True)
    table.batched = tune_batched_lanes(ctrl)
    print(json.dumps({"batched": table.batched}), flush=True)
    table.save(args.out)
    ctrl.release()


if __name__ == "__main__":
    main()
