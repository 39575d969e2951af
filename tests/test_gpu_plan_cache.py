"""GPU test of the per-hierarchy plan cache limit (AMG_MAX_PLANS).

A plan holds the buffers and graphs of one (precision, k, stream); a hierarchy keeps at most
AMG_MAX_PLANS of them (and as many column-padding stages) and frees the least recently
requested one when a new one is needed.  With the limit at 2, solves that cycle through five
(precision, k) combinations and back give the same solutions and iteration counts as with
the default limit.  Each configuration runs in a child process because the switch is read
once per process.
"""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, json, hashlib, numpy as np
sys.path.insert(0, {root!r})
from amjax_b200 import MultilevelSolver, amg_setup, gallery
W = ("jacobi", {{"iterations": 1, "omega": 2.0 / 3.0}})
A = gallery.poisson((40, 40))
ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W, postsmoother=W)
out = []
for rnd in range(2):
    for prec, k in (("f64", 1), ("mixed", 3), ("f64", 5), ("mixed", 8), ("f32", 2)):
        B = np.random.default_rng(k).standard_normal((A.shape[0], k))
        b = B[:, 0] if k == 1 else B
        x, info = ml.pcg(b, tol=1e-9, maxiter=60, precision=prec, return_info=True)
        x = np.ascontiguousarray(np.asarray(x))
        out.append([prec, k, hashlib.sha256(x.tobytes()).hexdigest(), list(map(int, info["iterations"]))])
print(json.dumps(out))
"""


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_plan_limit_gives_the_same_results(tmp_path):
    tune = str(tmp_path / "tune.txt")
    _run({"AMG_TUNE_FILE": tune})  # records the layouts, so both runs below launch the same ones
    capped = _run({"AMG_TUNE_FILE": tune, "AMG_MAX_PLANS": "2"})
    free = _run({"AMG_TUNE_FILE": tune})
    assert capped == free
    assert capped[:5] == capped[5:]  # a re-created plan gives the same solution as the first
