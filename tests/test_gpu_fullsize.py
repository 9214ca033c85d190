"""Full-size parity checks (the sizes of the benchmark workloads) against the
oracle's iteration counts in tests/golden/oracle_iterations.json (written by
oracle/iterations.py from serial oracle runs, plus runs with 2, 4 and 8
OpenMP threads for the BiCGSTAB systems).

CG iteration counts do not depend on the summation order of the dot
products at these sizes (the 128^3 elasticity system takes 1555 iterations
with 1, 2, 4 and 8 oracle threads), so CG is held to +-2. BiCGSTAB counts do:
the oracle itself varies by up to 17 iterations (3.4 %) between its serial
and 8-thread sums at Peclet 0.5, so BiCGSTAB is held to the larger of 2,
three times the oracle's own spread, and 2 % of its count. At these sizes
the size-independent checks are the FP64 residual of the returned solution
(computed with the device FP64 SpMV, bit-identical to the oracle's) and its
agreement with the FP32-refined solution."""
import json
import os

import numpy as np
import pytest

from monolis_b200 import api
from helpers import build, solve

pytestmark = pytest.mark.gpu

with open(os.path.join(os.path.dirname(__file__), "golden", "oracle_iterations.json")) as f:
    FIX = json.load(f)


def bicgstab_bound(key):
    it = FIX[key]
    spread = FIX.get(key + ":by_threads", {})
    sp = max([abs(v - it) for v in spread.values()] + [0])
    return max(2, 3 * sp, int(0.02 * it))


@pytest.mark.parametrize("peclet", [0.5, 5.0, 50.0])
def test_fullsize_convection_diffusion_bicgstab(gpu, peclet):
    key = f"convection_diffusion_n256_pe{peclet:g}_bicgstab_diag_tol1e-08"
    mp, b = build(gpu, "convection_diffusion", n=256, peclet=peclet)
    x, it, res, st = solve(mp, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-8)
    assert st == 0 and res < 1e-8
    bound = bicgstab_bound(key)
    assert abs(it - FIX[key]) <= bound, (it, FIX[key], bound)
    r = b - mp.matvec(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.01e-8
    # the FP32-refined solve reaches the same tolerance on the FP64 residual
    xm, _, resm, stm = solve(mp, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-8, precision=1)
    assert stm == 0 and resm < 1e-8
    assert np.linalg.norm(b - mp.matvec(xm)) / np.linalg.norm(b) < 1.01e-8
    assert np.linalg.norm(xm - x) / np.linalg.norm(x) < 1e-6


def test_fullsize_diffusion_kappa_cg(gpu):
    """The adjoint workload's forward system (128^3 Q1 diffusion, log-normal
    conductivity) to 1e-10: CG iteration count +-2 of the oracle's."""
    key = "diffusion_kappa_n128_cg_diag_tol1e-10"
    mp, b = build(gpu, "diffusion_kappa", n=128)
    x, it, res, st = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=1e-10)
    assert st == 0 and res < 1e-10
    assert abs(it - FIX[key]) <= 2, (it, FIX[key])
    r = b - mp.matvec(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.01e-10
