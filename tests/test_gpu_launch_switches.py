"""GPU test: the launch-level switches change timing, never results.

With one tuning file (so every run launches the same lane layouts), standalone solves and
PCG in FP64, FP32 and mixed precision at k = 1 and k = 8 give bit-identical solutions and
identical iteration counts with the defaults, with the driver's own shared-memory / L1
split (AMG_CARVEOUT=0) and without programmatic dependent launch (AMG_PDL=0).  Each
configuration runs in a child process because the switches are read once per process.
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
A = gallery.poisson((56, 56))
host = amg_setup.smoothed_aggregation_solver(A)
out = {{}}
for dt, precs in ((np.float64, ("f64", "mixed")), (np.float32, ("f32",))):
    ml = MultilevelSolver.from_pyamg(host, presmoother=W, postsmoother=W, dtype=dt)
    for k in (1, 8):
        B = np.random.default_rng(k).standard_normal((A.shape[0], k)).astype(dt)
        b = B[:, 0] if k == 1 else B
        for prec in precs:
            for meth in ("solve", "pcg"):
                x, info = getattr(ml, meth)(b, tol=1e-9, maxiter=80, precision=prec, return_info=True)
                x = np.ascontiguousarray(np.asarray(x))
                out[f"{{dt.__name__}}/{{k}}/{{prec}}/{{meth}}"] = [hashlib.sha256(x.tobytes()).hexdigest(),
                                                               list(map(int, info["iterations"]))]
print(json.dumps(out))
"""


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_launch_switches_do_not_change_results(tmp_path):
    tune = str(tmp_path / "tune.txt")
    _run({"AMG_TUNE_FILE": tune})  # records the layouts
    base = _run({"AMG_TUNE_FILE": tune})
    for switch in ({"AMG_CARVEOUT": "0"}, {"AMG_PDL": "0"}):
        other = _run(dict(switch, AMG_TUNE_FILE=tune))
        assert other == base, (switch, [k for k in base if base[k] != other.get(k)])
