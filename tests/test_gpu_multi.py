"""Many right-hand sides on one matrix (monolis_b200_solve_multi_R): every
right-hand side against the CPU oracle's FP64 solve of the same system.

Tolerances: each right-hand side reaches its FP64 relative residual tol
(checked with the oracle's SpMV) and agrees with the oracle's tighter solve to
1e-7 relative; FP64 iteration counts within +-3 of the oracle's (same
recurrence, dot products summed in another order)."""
import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import problems as P
from helpers import build, rel_err, solve

pytestmark = pytest.mark.gpu


def oracle_fv(oracle, side, seed):
    ix, it, v, _ = P.fv_diffusion_csr(side, seed)
    m = api.Monolis(oracle)
    m.set_matrix_BCSR(len(ix) - 1, len(ix) - 1, 1, len(it), v, ix, it)
    m.quiet()
    m.set_error_abort(False)
    return m, (ix, it, v)


def product_fv(gpu, side, seed, precision, tol=1e-8, maxiter=10000):
    ix, it, v, _ = P.fv_diffusion_csr(side, seed)
    m = api.Monolis(gpu)
    m.set_matrix_BCSR(len(ix) - 1, len(ix) - 1, 1, len(it), v, ix, it)
    m.quiet()
    m.set_error_abort(False)
    m.set_method(api.ITER_CG)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(tol)
    m.set_maxiter(maxiter)
    m.set_precision(precision)
    return m


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("n_rhs", [1, 5, 32, 40])
def test_multi_rhs_fv(gpu, oracle, precision, n_rhs):
    side = 12
    mp = product_fv(gpu, side, 77, precision)
    mo, _ = oracle_fv(oracle, side, 77)
    B = np.stack([P.uniform(300 + k, side ** 3) for k in range(n_rhs)])
    X, its, res, st = mp.solve_multi(B)
    assert np.all(st == 0), st
    assert np.all(res < 1e-8), res
    for k in range(n_rhs):
        r = B[k] - mo.matvec(X[k])
        assert np.linalg.norm(r) / np.linalg.norm(B[k]) < 1.01e-8, k
        if k % 7 == 0:
            xo, it_o, _, _ = solve(mo, B[k], api.ITER_CG, api.PREC_DIAG, tol=1e-12)
            assert rel_err(X[k], xo) < 1e-7, k
            if precision == 0:
                _, it8, _, _ = solve(mo, B[k], api.ITER_CG, api.PREC_DIAG, tol=1e-8)
                assert abs(int(its[k]) - it8) <= 3, (k, its[k], it8)


@pytest.mark.parametrize("precision", [0, 1])
def test_multi_rhs_elasticity_blocks(gpu, oracle, precision):
    """ndof 3 blocks, 7 right-hand sides, against single solves of the oracle."""
    mp, b = build(gpu, "elasticity", n=7)
    mo, _ = build(oracle, "elasticity", n=7)
    mp.set_method(api.ITER_CG)
    mp.set_precond(api.PREC_DIAG)
    mp.set_tolerance(1e-9)
    mp.set_maxiter(5000)
    mp.set_precision(precision)
    rng = np.random.default_rng(5)
    B = np.stack([b * (1 + k) + 0.01 * rng.standard_normal(len(b)) for k in range(7)])
    X, its, res, st = mp.solve_multi(B)
    assert np.all(st == 0)
    for k in range(7):
        xo, _, _, _ = solve(mo, B[k], api.ITER_CG, api.PREC_DIAG, tol=1e-12)
        assert rel_err(X[k], xo) < 1e-7, k


def test_multi_rhs_zero_and_maxiter(gpu, oracle):
    mp = product_fv(gpu, 10, 3, 1, tol=1e-8)
    B = np.stack([P.uniform(1, 1000), np.zeros(1000), P.uniform(2, 1000)])
    X, its, res, st = mp.solve_multi(B)
    assert list(st) == [0, 0, 0] and its[1] == 0 and np.all(X[1] == 0.0)
    mp.set_maxiter(4)
    mp.set_tolerance(1e-14)
    X, its, res, st = mp.solve_multi(B)
    assert st[0] == 1 and st[2] == 1 and st[1] == 0 and its[0] == 4


def test_multi_barrier_wait_runs_out(gpu):
    """Every grid-barrier wait of the persistent kernel is bounded. With the
    bound at 2,000 polls and block 0 reaching the first barrier 20 ms late
    (MONOLIS_B200_PRM_I_WAIT_DELAY_US, a bounded sleep), the other blocks'
    waits run out: the solve returns MONOLIS_B200_TIMEOUT (4) after every
    block has left the kernel, and the next solve on the same device and
    buffers (default bound, no delay) succeeds."""
    m = product_fv(gpu, 12, 77, precision=1)
    B = np.stack([P.uniform(900 + k, 12 ** 3) for k in range(3)])
    m.Iarray[api.B200_PRM_I_WAIT_LIMIT] = 2000
    m.Iarray[api.B200_PRM_I_WAIT_DELAY_US] = 20000
    with pytest.raises(RuntimeError, match="timeout"):
        m.solve_multi(B)
    assert m.Iarray[api.PRM_I_IERR] == 4
    m.Iarray[api.B200_PRM_I_WAIT_LIMIT] = 0
    m.Iarray[api.B200_PRM_I_WAIT_DELAY_US] = 0
    X, its, res, st = m.solve_multi(B)
    assert np.all(st == 0) and np.all(res < 1e-8)
    ix, it, v, _ = P.fv_diffusion_csr(12, 77)
    for k in range(3):
        assert np.linalg.norm(B[k] - P.csr_matvec(ix, it, v, X[k])) / np.linalg.norm(B[k]) < 1.01e-8


def test_multi_repeated_solve_reuses_its_graph(gpu):
    """The chunk's launch sequence is a captured CUDA graph; solving again
    with the same device buffers relaunches it and gives the same bits."""
    import torch
    m = product_fv(gpu, 14, 78, precision=0)
    m.set_matrix_cache(True)
    m.device_prepare()
    K, n = 5, 14 ** 3
    d_B = torch.from_numpy(np.stack([P.uniform(950 + k, n) for k in range(K)])).cuda()
    outs = []
    d_X = torch.zeros_like(d_B)
    for _ in range(2):
        d_X.zero_()
        its = np.zeros(K, dtype=np.int32)
        res = np.zeros(K)
        st = np.zeros(K, dtype=np.int32)
        rc = gpu.monolis_b200_device_solve_multi_R(m.p, K, d_B.data_ptr(), d_X.data_ptr(), its.ctypes.data_as(api._ip),
                                                   res.ctypes.data_as(api._dp), st.ctypes.data_as(api._ip))
        assert rc == 0 and np.all(st == 0)
        outs.append((d_X.cpu().numpy(), its.copy()))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])
