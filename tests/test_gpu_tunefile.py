"""Autotuning file (AMG_TUNE_FILE): a first process times the layouts of a PCG solve's
fused CSR ops and records one decision per line; a second process with the same file
reuses them without timing and appends nothing, and its solution is identical (the
layouts are the same, and every layout gives bit-identical outputs per row anyway)."""

import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, numpy as np
sys.path.insert(0, {root!r})
from amjax_b200 import MultilevelSolver, amg_setup, gallery
A = gallery.poisson((48, 48))
W = ("jacobi", {{"iterations": 1, "omega": 2.0 / 3.0}})
ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W, postsmoother=W)
B = np.random.default_rng(5).standard_normal((A.shape[0], 8))
x = ml.pcg(B, tol=1e-8, maxiter=200, precision="mixed")
np.save({out!r}, np.asarray(x.cpu().numpy() if hasattr(x, "cpu") else x))
"""


def _run(tmp_path, tag, tune_file):
    out = str(tmp_path / f"x_{tag}.npy")
    env = dict(os.environ, AMG_TUNE_FILE=str(tune_file))
    env.pop("AMG_TUNE", None)
    env.pop("AMG_KB_G", None)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT, out=out)], env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(out)


def test_tuning_file_written_then_reused(tmp_path):
    tf = tmp_path / "tune.txt"
    x1 = _run(tmp_path, "first", tf)
    lines = tf.read_text().splitlines()
    assert lines, "no tuning decisions recorded"
    for ln in lines:
        name, nnz, k, es, kv, g = ln.split()
        assert int(nnz) >= 0 and int(k) == 8 and int(es) in (4, 8) and int(kv) in (1, 2, 4)
        gl = int(g) % 64  # lane count; 64 + G = lean kernel, 128 + G = wide lean kernel
        assert gl in ((1, 2, 4, 8, 16, 32) if int(g) >= 64 else (4, 8, 16, 32))
    keys = [tuple(ln.split()[:5]) for ln in lines]
    assert len(keys) == len(set(keys)), "a decision was recorded twice"
    x2 = _run(tmp_path, "second", tf)
    assert tf.read_text().splitlines() == lines, "the second process re-tuned"
    np.testing.assert_array_equal(x1, x2)
