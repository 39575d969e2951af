"""Every CSR kernel family the autotuner can pick, forced one at a time (AMG_KB_G: G lanes
per row for csr_kb, 64 + G for the lean csr_kr, 128 + G for the wide 32-byte-vector csr_kr,
192 + G for its software-pipelined form csr_kp and 256 + G for csr_kp sized for 2 CTAs
per SM, including the 1- and 2-lane groups), so
that a layout the tuner picks on some other
matrix or machine is covered by a parity test here.

* Jacobi sweeps through the C ABI: all families accumulate each row in nonzero order with
  fused multiply-adds, so their outputs are bit-identical; each also matches a float64
  torch reference of the same sweep within float32 / float64 rounding.
* Mixed-precision PCG (FP32 cycle, FP64 CG) in a subprocess per family (graphs are cached
  per process, so a family is fixed for the process): FP64-checked residual <= tol and the
  same iteration counts for every family.
"""

import json
import os
import subprocess
import sys

import numpy as np
import pytest
import torch

from amjax_b200 import CSRMatrix, gallery, inverse_diagonal
from amjax_b200 import _native as N

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FAMILIES = ["16", "8", "80", "136", "65", "66", "129", "130", "200", "196", "264", "260"]  # kb 16/8,
# lean 16/1/2, wide 8/1/2, pipelined wide 8/4, pipelined wide at 2 CTAs per SM 8/4


def _sweep(A, dt, x, b, dinv, omega):
    y = torch.empty_like(x)
    N.call("amg_jacobi", A.desc(), 0 if dt == torch.float64 else 1, N.ptr(x), N.ptr(b), N.ptr(dinv), N.ptr(y),
           x.shape[1], 1, float(omega), N.stream_ptr())
    torch.cuda.synchronize()
    return y


@pytest.mark.parametrize("dt,k", [(torch.float32, 64), (torch.float32, 8), (torch.float32, 4),
                                  (torch.float64, 32), (torch.float64, 4), (torch.float32, 16)])
def test_jacobi_families_bit_identical(monkeypatch, dt, k):
    Asp = gallery.poisson((37, 41))
    A = CSRMatrix.from_scipy(Asp)
    dinv = inverse_diagonal(A).to(dt)
    g = torch.Generator(device="cuda").manual_seed(7)
    x = torch.randn(Asp.shape[0], k, dtype=dt, device="cuda", generator=g)
    b = torch.randn(Asp.shape[0], k, dtype=dt, device="cuda", generator=g)
    omega = 2.0 / 3.0
    # float64 reference of the same update, relaxation.py:94-96
    A64 = torch.sparse_csr_tensor(torch.as_tensor(Asp.indptr), torch.as_tensor(Asp.indices),
                                  torch.as_tensor(Asp.data), size=Asp.shape, dtype=torch.float64).cuda()
    x64, b64, d64 = x.double(), b.double(), dinv.double()[:, None]
    ref = (1 - omega) * x64 + omega * (d64 * (b64 - A64 @ x64) + x64)
    tol = 1e-5 if dt == torch.float32 else 1e-12
    outs = {}
    for fam in FAMILIES:
        monkeypatch.setenv("AMG_KB_G", fam)
        outs[fam] = _sweep(A, dt, x, b, dinv, omega)
        err = (outs[fam].double() - ref).abs().max().item() / ref.abs().max().item()
        assert err <= tol, (fam, err)
    base = outs[FAMILIES[0]]
    for fam, y in outs.items():
        assert torch.equal(y, base), f"family {fam} differs from csr_kb"


SCRIPT = r"""
import sys, json, numpy as np
sys.path.insert(0, {root!r})
from amjax_b200 import MultilevelSolver, amg_setup, gallery
A = gallery.poisson((40, 40))
W = ("jacobi", {{"iterations": 1, "omega": 2.0 / 3.0}})
ml = MultilevelSolver.from_pyamg(amg_setup.smoothed_aggregation_solver(A), presmoother=W, postsmoother=W)
out = {{}}
for k in (1, 8, 16):
    B = np.random.default_rng(11).standard_normal((A.shape[0], k))
    x, info = ml.pcg(B if k > 1 else B[:, 0], tol=1e-8, maxiter=200, precision="mixed", return_info=True)
    x = np.asarray(x.cpu().numpy() if hasattr(x, "cpu") else x).reshape(A.shape[0], k)
    rel = np.linalg.norm(B - A @ x, axis=0) / np.linalg.norm(B, axis=0)
    out[k] = {{"iters": [int(i) for i in np.atleast_1d(info["iterations"])], "rel": float(rel.max())}}
print(json.dumps(out))
"""


def test_pcg_families_converge_identically():
    results = {}
    for fam in ["16", "80", "136", "65", "130", "200", "264"]:
        env = dict(os.environ, AMG_KB_G=fam, AMG_TUNE="0")
        r = subprocess.run([sys.executable, "-c", SCRIPT.format(root=ROOT)], env=env, capture_output=True,
                           text=True, timeout=600)
        assert r.returncode == 0, (fam, r.stderr[-2000:])
        results[fam] = json.loads(r.stdout.strip().splitlines()[-1])
    for fam, res in results.items():
        for k, v in res.items():
            assert v["rel"] <= 1e-8, (fam, k, v)
            assert v["iters"] == results["16"][k]["iters"], (fam, k, v["iters"], results["16"][k]["iters"])
