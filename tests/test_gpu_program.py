"""GPU tests of the persistent coarse-level program (one cooperative launch that runs a
cycle's coarse levels with grid barriers between dependent steps).

* The program path (AMG_PROGRAM=1) gives bit-identical solutions and identical iteration
  counts to the launch-per-step path for the standalone solve and PCG, V / W / F cycles
  (W and F record more steps than one launch holds, so several programs run in a row),
  k = 1 and k > 1, FP64, FP32 and mixed precision: its row loops keep the launched
  kernels' multiply-add order.
* A barrier wait that runs out (a budget of a few clock cycles, AMG_SPIN_LIMIT) makes the
  kernel give up and return; the solve reports AMG_ERR_TIMEOUT, and the process's GPU
  context stays usable (a plain FP64 SpMV runs afterwards).

Each configuration runs in a child process because the switches are read once per
process; the two runs of a comparison read one tuning file that a first run has completed,
so both launch the same lane layouts (with k = 1 the lanes that split a row's nonzeros set
its summation order, and a process that tunes as it goes can meet an op before its
reducing variant is tuned).  All three runs keep the four-pass form of every level
(AMG_FUSE2=0): the program records that form, while a two-pass level (launches only) sums
each on-the-fly residual in its own order.
"""

import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys, json, hashlib, numpy as np, torch
sys.path.insert(0, {root!r})
from amjax_b200 import MultilevelSolver, amg_setup, gallery
from amjax_b200 import _native as N
W = ("jacobi", {{"iterations": 1, "omega": 2.0 / 3.0}})
out = {{}}
for kind, n in (("poisson", 48), ("diff", 40)):
    A = gallery.poisson((n, n)) if kind == "poisson" else gallery.variable_diffusion_2d(n, sigma=1.0, seed=3)
    host = amg_setup.smoothed_aggregation_solver(A)
    for dt in (np.float64, np.float32):
        ml = MultilevelSolver.from_pyamg(host, presmoother=W, postsmoother=W, dtype=dt)
        precs = ["f64", "mixed", "mixed-f64cg"] if dt == np.float64 else ["f32"]
        for k in (1, 4, 16, 64):
            B = np.random.default_rng(k).standard_normal((A.shape[0], k)).astype(dt)
            b = B[:, 0] if k == 1 else B
            for prec in precs:
                for meth, cyc in (("solve", "V"), ("solve", "W"), ("solve", "F"), ("pcg", "V"), ("pcg", "W")):
                    if k == 64 and cyc != "V":
                        continue
                    x, info = getattr(ml, meth)(b, tol=1e-9, maxiter=60, cycle=cyc, precision=prec, return_info=True)
                    x = np.ascontiguousarray(np.asarray(x))
                    key = f"{{kind}}/{{dt.__name__}}/{{k}}/{{prec}}/{{meth}}/{{cyc}}"
                    out[key] = [hashlib.sha256(x.tobytes()).hexdigest(), list(map(int, info["iterations"]))]
out["launches"] = N.kernel_launch_count()
print(json.dumps(out))
"""


def _run(env_extra, script):
    env = dict(os.environ, **env_extra)
    r = subprocess.run([sys.executable, "-c", script], env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_program_path_is_bit_identical_to_launches(tmp_path):
    script = SCRIPT.format(root=ROOT)
    tune = str(tmp_path / "tune.txt")
    base = {"AMG_TUNE_FILE": tune, "AMG_FUSE2": "0"}
    _run(dict(base, AMG_PROGRAM="0"), script)  # records every layout decision
    with_prog = _run(dict(base, AMG_PROGRAM="1"), script)
    without = _run(dict(base, AMG_PROGRAM="0"), script)
    fewer = with_prog.pop("launches")
    more = without.pop("launches")
    assert set(with_prog) == set(without)
    differ = [key for key in with_prog if with_prog[key] != without[key]]
    assert not differ, differ
    assert fewer < more  # the program replaced launches


TIMEOUT_SCRIPT = r"""
import sys, json, numpy as np, torch
sys.path.insert(0, {root!r})
from amjax_b200 import MultilevelSolver, amg_setup, gallery, CSRMatrix
from amjax_b200 import _native as N
import ctypes as C
W = ("jacobi", {{"iterations": 1, "omega": 2.0 / 3.0}})
A = gallery.poisson((64, 64))
ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W, postsmoother=W)
assert len(ml.levels) >= 3
res = {{}}
for meth in ("solve", "pcg"):
    try:
        getattr(ml, meth)(np.ones(A.shape[0]), tol=1e-8, maxiter=20)
        res[meth] = 0
    except N.NativeError as e:
        res[meth] = e.status
        res[meth + "_msg"] = str(e)
# the context is still usable: a plain SpMV
M = CSRMatrix.from_scipy(A)
x = torch.ones(A.shape[0], dtype=torch.float64, device="cuda")
y = torch.empty_like(x)
N.call("amg_spmv", C.byref(M.desc()), 0, N.ptr(x), N.ptr(y), 1, N.stream_ptr())
torch.cuda.synchronize()
res["spmv_ok"] = bool(np.allclose(y.cpu().numpy(), A @ np.ones(A.shape[0])))
print(json.dumps(res))
"""


def test_barrier_timeout_is_reported_not_hung():
    res = _run({"AMG_PROGRAM": "1", "AMG_SPIN_LIMIT": "16"}, TIMEOUT_SCRIPT.format(root=ROOT))
    assert res["solve"] == 4 and res["pcg"] == 4, res
    assert "ran out of time" in res["pcg_msg"]
    assert res["spmv_ok"]
