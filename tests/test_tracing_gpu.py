"""Opt-in NVTX ranges (CLSPARSE_B200_NVTX=1): the traced calls give the same
results as untraced ones. The switch is read once per process, so the traced
run is a child process."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CHILD = r"""
import sys, json, numpy as np, torch
sys.path.insert(0, sys.argv[1])
from clsparse_b200 import api, matgen
rp, col, val = matgen.poisson2d(64)
ctrl = api.Control()
A = api.CsrMatrix.from_numpy(rp, col, val); A.create_meta(ctrl)
n = A.num_rows
x = torch.tensor(np.random.default_rng(1).uniform(-1, 1, n), device="cuda")
y = torch.zeros(n, dtype=torch.float64, device="cuda")
one = torch.ones(1, dtype=torch.float64, device="cuda"); zero = torch.zeros(1, dtype=torch.float64, device="cuda")
api.csrmv(one, A, x, zero, y, ctrl)
xs = torch.zeros(n, dtype=torch.float64, device="cuda")
sc = api.SolverControl(1, 1000, 1e-10, 0.0)
info = api.solve("cg", xs, A, x, sc, ctrl)
print(json.dumps({"y": float(y.sum()), "it": info["nIters"], "x": float(xs.sum())}))
"""


def run(nvtx: str):
    env = dict(os.environ, CLSPARSE_B200_NVTX=nvtx)
    out = subprocess.run([sys.executable, "-c", CHILD, str(ROOT)], env=env, capture_output=True, text=True,
                         timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    return out.stdout.strip().splitlines()[-1]


def test_traced_calls_match_untraced():
    assert run("1") == run("0")
