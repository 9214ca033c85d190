"""Full-size parity checks (the sizes of the benchmark workloads) against the
oracle's results in tests/golden/oracle_iterations.json (written by
oracle/iterations.py).

The FP64 kernels sum every dot product in double-double, the arithmetic of
the reference's pseudo-quadruple inner product (src/linalg/
inner_product.f90:219-258), which makes each dot product the correctly
rounded sum of the rounded products whatever the summation order. The
oracle run with the same dot products ("...:n128" entries) is therefore
the count these solves are held to, +-2: at 256^3 it takes 469 / 445 / 440
BiCGSTAB iterations at Peclet 0.5 / 5 / 50 with 8 threads, and the same with
2 and 4 threads (":n128:by_threads"). The reference's plain serial sums
give 492 / 446 / 440, and the same plain sums over 2, 4 and 8 threads move
by up to 16 iterations at Peclet 0.5 (":by_threads"): that spread is the
summation order, which the double-double sums remove. CG counts do not
depend on the summation order at these sizes (1555 for the elasticity
system in both arithmetics and every thread count). The solution is
compared with a strided sample of the oracle's (":x_sample") to 1e-10.
"""
import json
import os

import numpy as np
import pytest

from monolis_b200 import api
from helpers import build, solve

pytestmark = pytest.mark.gpu

with open(os.path.join(os.path.dirname(__file__), "golden", "oracle_iterations.json")) as f:
    FIX = json.load(f)


def sample_rel_err(x, key):
    stride = FIX[key + ":x_stride"]
    ref = np.asarray(FIX[key + ":x_sample"])
    got = x[::stride]
    assert got.shape == ref.shape
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


@pytest.mark.parametrize("peclet", [0.5, 5.0, 50.0])
def test_fullsize_convection_diffusion_bicgstab(gpu, peclet):
    key = f"convection_diffusion_n256_pe{peclet:g}_bicgstab_diag_tol1e-08"
    mp, b = build(gpu, "convection_diffusion", n=256, peclet=peclet)
    x, it, res, st = solve(mp, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-8)
    assert st == 0 and res < 1e-8
    assert abs(it - FIX[key + ":n128"]) <= 2, (it, FIX[key + ":n128"])
    assert sample_rel_err(x, key + ":n128") < 1e-10
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
    assert abs(it - FIX[key + ":n128"]) <= 2, (it, FIX[key + ":n128"])
    r = b - mp.matvec(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.01e-10


def test_fullsize_elasticity_fp64_solution(gpu):
    """128^3-node elasticity, FP64 CG to 1e-8: iterations +-2 of the oracle's
    (1555, serial plain sums and double-double sums alike) and the solution
    within 1e-10 of the oracle's on a strided sample of 1535 entries."""
    key = "elasticity_n128_cg_diag_tol1e-08"
    mp, b = build(gpu, "elasticity", n=128)
    x, it, res, st = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=1e-8)
    assert st == 0 and res < 1e-8
    assert abs(it - FIX[key]) <= 2 and abs(it - FIX[key + ":n128"]) <= 2, it
    assert sample_rel_err(x, key + ":n128") < 1e-10
    # size-independent check: the FP64 device SpMV of the solution reproduces b
    r = b - mp.matvec(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.01e-8
