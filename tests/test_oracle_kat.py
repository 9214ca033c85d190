"""Pins the CPU oracle against the reference's own known-answer tests, restated.

Each test names the reference test it follows. The reference's values come
from unseeded Fortran `random_number`; the restatements draw from a seeded
generator with the same structure (sizes, diagonal shifts, symmetry), since
the tests assert x = 1 for any such draw.
"""
import ctypes as C

import numpy as np
import pytest

from monolis_b200 import api
from helpers import bits_equal, solve

TOL_EQ = 1e-8  # monolis_test_check_eq_R compares to a small relative tolerance


def chain(lib, n_dof, rng, diag_shift=2.0):
    """src_test/iterative/CG_test.f90:21-72: 10-node chain, random values,
    diagonal + 2, symmetric off-diagonal blocks (j2,i2 transposed)."""
    m = api.Monolis(lib)
    elem = np.array([[i, i + 1] for i in range(9)], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(10, 2, n_dof, elem)
    for i1 in range(10):
        for i2 in range(n_dof):
            m.add_scalar(i1, i1, i2, i2, rng.random() + diag_shift)
    for e in elem:
        for i2 in range(n_dof):
            for j2 in range(n_dof):
                v = rng.random()
                m.add_scalar(int(e[0]), int(e[1]), i2, j2, v)
                m.add_scalar(int(e[1]), int(e[0]), j2, i2, v)
    return m


@pytest.mark.parametrize("n_dof", [1, 2, 3])
@pytest.mark.parametrize("prec", [api.PREC_NONE, api.PREC_DIAG])
@pytest.mark.parametrize("method,tol", [(api.ITER_CG, 1e-10), (api.ITER_BICGSTAB, 1e-12), (api.ITER_PIPECG, 1e-10),
                                        (api.ITER_GROPCG, 1e-10), (api.ITER_BICGSTAB_N128, 1e-12)])
def test_chain_solve_x_equals_one(oracle, n_dof, prec, method, tol):
    # src_test/iterative/CG_test.f90:74-89, BiCGSTAB_test.f90 (tol 1e-12), PipeCG_test.f90:74-89,
    # GropCG_test.f90, BiCGSTAB_N128_test.f90 (tol 1e-12)
    m = chain(oracle, n_dof, np.random.default_rng(10 * n_dof + prec))
    m.quiet()
    b = m.matvec(np.ones(10 * n_dof))
    x, it, res, st = solve(m, b, method, prec, tol=tol)
    assert st == 0 and it >= 1 and res < tol
    np.testing.assert_allclose(x, 1.0, rtol=TOL_EQ)


def test_matvec_11_dense(oracle):
    # src_test/linalg/matvec_test.f90:110-174 (exact)
    m = api.Monolis(oracle)
    elem = np.array([[0, 1], [1, 2], [2, 3], [3, 4]], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(5, 2, 1, elem)
    entries = {(0, 0): 2, (0, 1): 1, (1, 0): 1, (1, 1): 2, (1, 2): 3, (2, 1): 1, (2, 2): 2, (2, 3): 4,
               (3, 2): 1, (3, 3): 2, (3, 4): 5, (4, 3): 1, (4, 4): 2}
    dense = np.zeros((5, 5))
    for (i, j), v in entries.items():
        m.add_scalar(i, j, 0, 0, float(v))
        dense[i, j] = v
    a = np.ones(5)
    assert bits_equal(m.matvec(a), dense @ a)


def test_matvec_33_dense(oracle):
    # src_test/linalg/matvec_test.f90:243-301
    rng = np.random.default_rng(33)
    m = api.Monolis(oracle)
    elem = np.array([[0, 1], [1, 2], [2, 3]], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(4, 2, 3, elem)
    for e in elem:
        for i2 in range(3):
            for j2 in range(3):
                v = rng.random() + 1.0
                m.add_scalar(int(e[0]), int(e[1]), i2, j2, v)
                m.add_scalar(int(e[1]), int(e[0]), j2, i2, v)
    dense = np.zeros((12, 12))
    for i1 in range(4):
        for j1 in range(4):
            for i2 in range(3):
                for j2 in range(3):
                    v, _ = m.get_scalar(i1, j1, i2, j2)
                    dense[3 * i1 + i2, 3 * j1 + j2] = v
    a = np.ones(12)
    np.testing.assert_allclose(m.matvec(a), dense @ a, rtol=1e-15)


def test_check_converge(oracle):
    # src_test/linalg/mat_converge_test.f90:36-55: R = 2*1_4, B2 = 4 -> resid 2.0,
    # not converged, CUR_ITER = 10
    m = api.Monolis(oracle)
    m.quiet()
    R = np.full(4, 2.0)
    conv = oracle.oracle_check_converge(m.p, 4, R.ctypes.data_as(C.POINTER(C.c_double)), 4.0, 10)
    assert conv == 0
    assert m.Iarray[api.PRM_I_CUR_ITER] == 10
    assert m.Rarray[api.PRM_R_CUR_RESID] == 2.0


def test_c_wrapper_solver_test(oracle):
    """wrapper_test/solver/monolis_solver_c_test.c:8-81: ndof 2 chain, diagonal
    rand()%1001 + 5000, off-diagonal rand()%1001 (glibc rand, default seed),
    default method (CG + DIAG), tol 1e-10, x = 1."""
    libc = C.CDLL("libc.so.6")
    libc.srand(1)  # the C test calls rand() unseeded: the default seed is 1
    m = api.Monolis(oracle)
    elem = np.array([[i, i + 1] for i in range(9)], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(10, 2, 2, elem)
    for i in range(10):
        for j in range(2):
            m.set_scalar(i, i, j, j, libc.rand() % 1001 + 5000.0)
    for e in elem:
        for j in range(2):
            for k in range(2):
                v = float(libc.rand() % 1001)
                m.set_scalar(int(e[0]), int(e[1]), j, k, v)
                m.set_scalar(int(e[1]), int(e[0]), j, k, v)
    m.quiet()
    b = m.matvec(np.ones(20))
    m.set_tolerance(1e-10)
    x = np.zeros(20)
    m.solve(b, x)
    np.testing.assert_allclose(x, 1.0, rtol=TOL_EQ)
    assert m.Iarray[api.PRM_I_METHOD] == api.ITER_CG and m.Iarray[api.PRM_I_PRECOND] == api.PREC_DIAG


def mtx_dat(lib):
    """src_test/input.f/mtx.dat (10x10: diagonal 4, super/sub-diagonal 1) as
    2-node elements, assembled as main.f90:176-186 does (self-loops for the
    diagonal, both directions for the others)."""
    m = api.Monolis(lib)
    edges = [(i, i) for i in range(10)] + [(i, i + 1) for i in range(9)]
    elem = np.array(edges, dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(10, 2, 1, elem)
    for (a, b) in edges:
        v = 4.0 if a == b else 1.0
        m.add_scalar(a, b, 0, 0, v)
        if a != b:
            m.add_scalar(b, a, 0, 0, v)
    return m


@pytest.mark.parametrize("method", [api.ITER_CG, api.ITER_BICGSTAB])
@pytest.mark.parametrize("prec", [api.PREC_NONE, api.PREC_DIAG])
def test_mtx_dat_sweep(oracle, method, prec):
    # src_test/input.f/main.f90:193-231: x = 1, iter >= 1, resid <= 1e-10
    m = mtx_dat(oracle)
    m.quiet()
    c = m.matvec(np.ones(10))
    x, it, res, st = solve(m, c, method, prec, tol=1e-10, maxiter=1000)
    np.testing.assert_allclose(x, 1.0, rtol=TOL_EQ)
    assert it >= 1 and res <= 1e-10


@pytest.mark.parametrize("n_dof", [1, 3])
def test_sample_cg_diag_3d(oracle, n_dof):
    # sample/cg_diag_3d/main.f90:52-131: N^3 grid, 5.95 on the diagonal, -1 per edge
    from monolis_b200 import problems
    n = 6
    edges, _ = problems.grid_edges(n)
    m = api.Monolis(oracle)
    m.get_nonzero_pattern_by_simple_mesh(n ** 3, 2, n_dof, edges)
    for i in range(n ** 3):
        for k in range(n_dof):
            m.add_scalar(i, i, k, k, 5.95)
    for e in edges:
        for k in range(n_dof):
            m.add_scalar(int(e[0]), int(e[1]), k, k, -1.0)
            m.add_scalar(int(e[1]), int(e[0]), k, k, -1.0)
    m.quiet()
    b = m.matvec(np.ones(n ** 3 * n_dof))
    x, it, res, st = solve(m, b, api.ITER_CG, api.PREC_DIAG, tol=1e-10)
    assert st == 0
    assert np.max(np.abs(x - 1.0)) < 1e-8


def test_diag_zero_pivot_replaced_by_one(oracle):
    # src/prec/diag/diag_33.f90:74: a zero pivot becomes 1 (then 1/1)
    m = api.Monolis(oracle)
    elem = np.array([[0, 1]], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(2, 2, 3, elem)
    m.add_scalar(0, 0, 0, 0, 2.0)
    m.add_scalar(0, 0, 1, 1, 0.0)   # zero pivot
    m.add_scalar(0, 0, 2, 2, 4.0)
    m.add_scalar(1, 1, 0, 0, 1.0)
    m.add_scalar(1, 1, 1, 1, 1.0)
    m.add_scalar(1, 1, 2, 2, 1.0)
    alu = np.zeros(18)
    oracle.oracle_diag_setup(m.p, alu.ctypes.data_as(C.POINTER(C.c_double)))
    assert alu[0] == 0.5 and alu[4] == 1.0 and alu[8] == 0.25


def test_sorted_inner_product(oracle):
    # src/linalg/inner_product.f90:262-331: products summed in ascending |x_i y_i|
    x = np.array([1e16, 1.0, -1e16, 1.0])
    y = np.ones(4)
    dp = C.POINTER(C.c_double)
    plain = oracle.oracle_dot(4, x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    srt = oracle.oracle_sorted_dot(4, x.ctypes.data_as(dp), y.ctypes.data_as(dp))
    assert srt == 2.0    # 1 + 1 first, then 1e16 + 2 - 1e16
    assert plain == 1.0  # left to right: the first 1 is absorbed by 1e16


def test_zero_rhs_gives_zero(oracle):
    # src/linalg/mat_converge.f90:40-48
    m = mtx_dat(oracle)
    m.quiet()
    x = np.ones(10)
    m.solve(np.zeros(10), x)
    assert np.all(x == 0.0)


def test_inner_product_n128(oracle):
    # src_test/linalg/inner_product_test.f90:146-158 (case 8): the
    # pseudo-quadruple inner product of (1,1,1,1) and (1,2,3,4) is 10
    dp = C.POINTER(C.c_double)
    x, y = np.ones(4), np.array([1.0, 2.0, 3.0, 4.0])
    assert oracle.oracle_dot_n128(4, x.ctypes.data_as(dp), y.ctypes.data_as(dp)) == 10.0
    # the two-double sum keeps what a double sum absorbs
    x = np.array([1e16, 1.0, -1e16, 1.0])
    assert oracle.oracle_dot_n128(4, x.ctypes.data_as(dp), np.ones(4).ctypes.data_as(dp)) == 2.0


@pytest.mark.parametrize("n", [1, 17, 100_003, 2_000_000])
def test_inner_product_n128_is_the_rounded_exact_sum(oracle, n):
    """The double-double sum of the rounded products equals the correctly
    rounded exact sum of those products (math.fsum) for 1 to 8 threads: its
    value does not depend on the summation order."""
    import math
    dp = C.POINTER(C.c_double)
    rng = np.random.default_rng(n)
    x, y = rng.standard_normal(n), rng.standard_normal(n)
    exact = math.fsum((x * y).tolist())
    try:
        for th in (1, 2, 3, 8):
            oracle.oracle_set_threads(th)
            assert oracle.oracle_dot_n128(n, x.ctypes.data_as(dp), y.ctypes.data_as(dp)) == exact
    finally:
        oracle.oracle_set_threads(1)


def test_dot_mode_n128_makes_bicgstab_order_free(oracle):
    """With every dot product in double-double, BiCGSTAB on a 48^3
    convection-diffusion system gives bit-identical solutions and the same
    iteration count for 1, 2, 4 and 8 threads (the reference's plain sums
    are order-dependent: the same runs give different bits)."""
    from helpers import build
    outs = {}
    try:
        oracle.oracle_set_dot_mode(1)
        for th in (1, 2, 4, 8):
            oracle.oracle_set_threads(th)
            m, b = build(oracle, "convection_diffusion", n=48, peclet=50.0)
            x, it, res, st = solve(m, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-8)
            assert st == 0
            outs[th] = (it, x)
    finally:
        oracle.oracle_set_dot_mode(0)
        oracle.oracle_set_threads(1)
    it1, x1 = outs[1]
    for it, x in outs.values():
        assert it == it1 and bits_equal(x, x1)
