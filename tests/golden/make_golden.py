"""Generates tests/golden/rowblocks.npz: row-pointer arrays and the row-block
words the reference's own ComputeRowBlocks (src/library/internal/data-types/
csr-meta.hpp:93-269, compiled from the reference sources into oracle/_ref by
oracle/Makefile) produces for them.

Run where the reference tree exists:  python tests/golden/make_golden.py
The fixture pins both the oracle restatement and the library's host binning.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402


# (BLKSIZE, BLOCK_MULTIPLIER, ROWS_FOR_VECTOR) shapes pinned besides the default
SHAPES = [(512, 1, 1), (512, 8, 4), (2048, 3, 1), (2048, 1, 4), (1024, 8, 2)]


def cases():
    """Row-length patterns covering every branch of the binning."""
    rng = np.random.default_rng(20251203)
    out = {
        "empty": [],
        "one_empty_row": [0],
        "single_short": [5],
        "single_1024": [1024],
        "single_1025": [1025],
        "single_3072": [3072],
        "single_3073": [3073],
        "single_200k": [200_000],
        "all_empty_300": [0] * 300,
        "probe_3_3_2000_4": [3, 3, 2000, 4],
        "blk_exact": [512, 512, 1, 1023, 1],
        "long_run_cut": [10, 10, 200, 300, 5, 5, 40, 150, 20],
        "threshold_edges": [0, 1, 31, 32, 33, 127, 128, 129, 1023, 1024, 1025, 3072, 3073, 6145],
        "short_many": list(rng.integers(0, 4, 5000)),
        "uniform_0_40": list(rng.integers(0, 40, 3000)),
        "lognormal": list(np.maximum(1, np.rint(np.exp(rng.normal(2.5, 1.2, 4000)))).astype(int)),
        "mixed_dense": list(np.where(rng.random(3000) < 0.01, rng.integers(1000, 30000, 3000),
                                     rng.integers(0, 12, 3000))),
        "stencil_5pt_rows": [3, 4] * 5 + [5] * 500 + [4, 3],
        "runs_100_300": list(rng.integers(100, 300, 2000)),
    }
    for k in range(6):
        n = int(rng.integers(1, 2500))
        out[f"random_{k}"] = list(rng.choice([0, 1, 2, 7, 31, 32, 33, 100, 129, 700, 1024, 1500, 4000], n))
    return out


def main():
    arrays = {}
    for name, lens in cases().items():
        lens = np.asarray(lens, dtype=np.int64)
        rp = np.zeros(len(lens) + 1, dtype=np.uint32)
        rp[1:] = np.cumsum(lens)
        words, size, dry = oracle.ref_row_blocks(rp)
        arrays[f"{name}__rp"] = rp
        arrays[f"{name}__words"] = words
        arrays[f"{name}__size"] = np.array([size, dry], dtype=np.uint32)
    dst = Path(__file__).resolve().parent / "rowblocks.npz"
    np.savez_compressed(dst, **arrays)
    print(f"wrote {dst} ({len(arrays) // 3} cases)")
    # the same cases under the non-default row-block shapes the tuner sweeps
    shaped = {}
    for shape in SHAPES:
        tag = "x".join(str(v) for v in shape)
        for name, lens in cases().items():
            lens = np.asarray(lens, dtype=np.int64)
            rp = np.zeros(len(lens) + 1, dtype=np.uint32)
            rp[1:] = np.cumsum(lens)
            words, size, dry = oracle.ref_row_blocks(rp, shape)
            shaped[f"{tag}__{name}__words"] = words
            shaped[f"{tag}__{name}__size"] = np.array([size, dry], dtype=np.uint32)
    dst = Path(__file__).resolve().parent / "rowblocks_shapes.npz"
    np.savez_compressed(dst, **shaped)
    print(f"wrote {dst} ({len(shaped) // 2} cases)")


if __name__ == "__main__":
    main()
