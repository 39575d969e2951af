"""GPU tests of the two-pass levels (one right-hand side, small levels, iterate zero, one
pre- and one post-sweep): the restriction reads the residual of the one-sweep iterate
computed per gathered row, and the post-sweep reads the prolonged and corrected iterate
computed per gathered row, so such a level runs two CSR passes instead of four.

* With two-pass levels on (the default) and off (AMG_FUSE2=0) the standalone solve and PCG
  (V / W / F cycles, FP64, FP32 and mixed precision) take the same iteration counts, and
  their solutions agree to rounding (the on-the-fly residual sums a row's products in
  order, the separate residual pass by lanes): relative difference below 1e-9 in FP64,
  below 1e-4 in FP32.
* The two-pass form launches fewer kernels.
* AMG_FUSE2_ROWS=0 (no level qualifies) launches as many kernels as AMG_FUSE2=0.
* The gather bounds: on a 16³ variable-diffusion SA hierarchy (levels of 4,096 / 514 / 18
  rows; the 514-row level's restriction walks ~2,700 two-hop gathers per coarse row) the
  default gate fuses levels 0 and 2 but not 1, so it launches more kernels than with the
  bounds lifted (AMG_FUSE2_CHAIN, AMG_FUSE2_WORK) and fewer than with AMG_FUSE2=0; the
  three give the same iteration counts and solutions agreeing to rounding.

Each configuration runs in a child process because the switches are read once per process.
"""

import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, json, numpy as np, torch
sys.path.insert(0, {root!r})
from amjax_b200 import MultilevelSolver, amg_setup, gallery
from amjax_b200 import _native as N
W = ("jacobi", {{"iterations": 1, "omega": 2.0 / 3.0}})
out = {{}}
n0 = N.kernel_launch_count()
for kind, n in (("poisson", 64), ("diff", 48)):
    A = gallery.poisson((n, n)) if kind == "poisson" else gallery.variable_diffusion_2d(n, sigma=1.0, seed=5)
    host = amg_setup.smoothed_aggregation_solver(A)
    for dt in (np.float64, np.float32):
        ml = MultilevelSolver.from_pyamg(host, presmoother=W, postsmoother=W, dtype=dt)
        precs = ["f64", "mixed"] if dt == np.float64 else ["f32"]
        b = np.random.default_rng(n).standard_normal(A.shape[0]).astype(dt)
        for prec in precs:
            for meth, cyc in (("solve", "V"), ("solve", "W"), ("solve", "F"), ("pcg", "V"), ("pcg", "F")):
                x, info = getattr(ml, meth)(b, tol=1e-8, maxiter=80, cycle=cyc, precision=prec, return_info=True)
                key = f"{{kind}}/{{dt.__name__}}/{{prec}}/{{meth}}/{{cyc}}"
                out[key] = [np.asarray(x, dtype=np.float64).tolist(), int(info["iterations"][0])]
out["launches"] = N.kernel_launch_count() - n0
print(json.dumps(out))
"""


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT)], env=env, capture_output=True,
                       text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def runs():
    return {"on": _run({}), "off": _run({"AMG_FUSE2": "0"}), "none": _run({"AMG_FUSE2_ROWS": "0"})}


def test_two_pass_levels_match_four_pass(runs):
    on, off = dict(runs["on"]), dict(runs["off"])
    on.pop("launches"), off.pop("launches")
    assert set(on) == set(off)
    for key in on:
        x_on, it_on = on[key]
        x_off, it_off = off[key]
        assert it_on == it_off, (key, it_on, it_off)
        x_on, x_off = np.asarray(x_on), np.asarray(x_off)
        rel = np.linalg.norm(x_on - x_off) / np.linalg.norm(x_off)
        tol = 1e-4 if "float32" in key else 1e-9
        assert rel < tol, (key, rel)


def test_two_pass_levels_launch_fewer_kernels(runs):
    assert runs["on"]["launches"] < runs["off"]["launches"]
    assert runs["none"]["launches"] == runs["off"]["launches"]


DENSE = r"""
import sys, json, numpy as np
sys.path.insert(0, {root!r})
from amjax_b200 import MultilevelSolver, amg_setup, gallery
from amjax_b200 import _native as N
W = ("jacobi", {{"iterations": 1, "omega": 2.0 / 3.0}})
A = gallery.variable_diffusion_3d(16, sigma=1.0, seed=2)
ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W, postsmoother=W)
b = np.random.default_rng(4).standard_normal(A.shape[0])
ml.pcg(b, tol=1e-9, maxiter=100)  # tuning and capture outside the count
n0 = N.kernel_launch_count()
x, info = ml.pcg(b, tol=1e-9, maxiter=100, return_info=True)
print(json.dumps({{"x": np.asarray(x).tolist(), "it": int(info["iterations"][0]),
                  "launches": N.kernel_launch_count() - n0, "levels": [l.A.shape[0] for l in ml.levels]}}))
"""


def _run_dense(env_extra):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", DENSE.format(root=ROOT)], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_gather_bounds_exclude_dense_levels():
    gated = _run_dense({})
    lifted = _run_dense({"AMG_FUSE2_CHAIN": "1e12", "AMG_FUSE2_WORK": "1e12"})
    off = _run_dense({"AMG_FUSE2": "0"})
    assert gated["levels"][:3] == [4096, 514, 18]
    assert lifted["launches"] < gated["launches"] < off["launches"]
    assert gated["it"] == lifted["it"] == off["it"]
    xo = np.asarray(off["x"])
    for run in (gated, lifted):
        assert np.linalg.norm(np.asarray(run["x"]) - xo) / np.linalg.norm(xo) < 1e-9
