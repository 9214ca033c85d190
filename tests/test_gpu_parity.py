"""GPU parity: the CUDA path (libmonolis_b200.so) against the CPU oracle on
the same seeded inputs, through the monolis C API.

Tolerances: SpMV is bit-identical (same per-row summation order, no FMA
contraction in the FP64 path). The FP64 kernels sum dot products in
double-double (the arithmetic of the reference's pseudo-quadruple inner
product), so a dot product equals the correctly rounded sum of the rounded
products; against the reference's plain serial sums it differs by their
rounding (relative 1e-13). FP64 CG/BiCGSTAB reproduce the oracle's
iteration count within +-2 and its solution within 1e-10 relative (x is
compared at the oracle's own tolerance, so the bound is on the difference
of two converged iterates); against the oracle run with double-double dot
products they reproduce its iteration count exactly and its solution bit
for bit."""
import math

import numpy as np
import pytest

from monolis_b200 import api
from helpers import bits_equal, build, oracle_dot_mode, rel_err, solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("problem,kw", [
    ("laplacian", dict(n=16)),
    ("elasticity", dict(n=9)),
    ("convection_diffusion", dict(n=12, peclet=5.0)),
    ("diffusion_kappa", dict(n=9)),
])
def test_spmv_bit_exact(gpu, oracle, problem, kw):
    mp, b = build(gpu, problem, **kw)
    mo, _ = build(oracle, problem, **kw)
    rng = np.random.default_rng(7)
    for _ in range(3):
        x = rng.standard_normal(len(b))
        yo = mo.matvec(x)
        yp = mp.matvec(x)
        assert bits_equal(yp, yo)


@pytest.mark.parametrize("problem,kw", [
    ("elasticity", dict(n=9)),
    ("convection_diffusion", dict(n=13, peclet=5.0)),
    ("laplacian", dict(n=11)),
])
def test_spmv_fp32_paired_layout(gpu, oracle, problem, kw):
    """FP32 SpMV (paired layout, FMA) against the oracle's FP64 SpMV of the
    same FP32-rounded inputs: per row |y32 - y| <= 1e-6 * (|A| |x|)."""
    import torch
    mp, b = build(gpu, problem, **kw)
    mo, _ = build(oracle, problem, **kw)
    mp.set_precision(1)
    mp.device_prepare()
    rng = np.random.default_rng(5)
    x = rng.standard_normal(len(b)).astype(np.float32)
    vals32 = mo.values().astype(np.float32).astype(np.float64)
    mo_abs, _ = build(oracle, problem, **kw)
    mo_abs.values()[:] = np.abs(vals32)
    bound = mo_abs.matvec(np.abs(x.astype(np.float64)))
    mo.values()[:] = vals32
    y_ref = mo.matvec(x.astype(np.float64))
    d_x = torch.from_numpy(x).cuda()
    d_y = torch.empty_like(d_x)
    mp.device_matvec(d_x.data_ptr(), d_y.data_ptr(), fp32=True)
    torch.cuda.synchronize()
    y32 = d_y.cpu().numpy().astype(np.float64)
    assert np.all(np.abs(y32 - y_ref) <= 1e-6 * bound + 1e-30)


def _long_range_graph(n, n_far, seed):
    """Chain 0-1-...-(n-1) plus n_far random edges between distant nodes:
    slices holding a far edge need 32-bit column ids, the rest compress."""
    rng = np.random.default_rng(seed)
    chain = np.stack([np.arange(n - 1), np.arange(1, n)], axis=1)
    far = np.stack([rng.integers(0, n // 4, n_far), rng.integers(3 * n // 4, n, n_far)], axis=1)
    edges = np.ascontiguousarray(np.concatenate([chain, far]), dtype=np.int32)
    vals = rng.standard_normal((len(edges), 4))
    vals[:, 0] += 4.0
    vals[:, 3] += 4.0
    return edges, vals


@pytest.mark.parametrize("n,n_far", [(200_003, 300), (70_001, 0)])
def test_spmv_mixed_wide_and_compressed_slices(gpu, oracle, n, n_far):
    """Column ids are stored as 16-bit differences per slice where they fit
    and as 32-bit ids elsewhere; FP64 SpMV stays bit-identical to the oracle
    on a matrix with both kinds of slices (and a last, partial slice), and
    the FP32 paired layout stays within its rounding bound."""
    import torch
    edges, vals = _long_range_graph(n, n_far, seed=11)
    ms = []
    for lib in (gpu, oracle):
        m = api.Monolis(lib)
        m.get_nonzero_pattern_flat(n, 2, 1, edges)
        m.add_elements(edges, 2, vals.reshape(-1), 4)
        ms.append(m)
    mp, mo = ms
    mp.set_matrix_cache(True)
    mp.set_precision(1)
    mp.device_prepare()
    wide64, wide32 = mp.Iarray[api.B200_PRM_I_WIDE_SLICES_FP64], mp.Iarray[api.B200_PRM_I_WIDE_SLICES_FP32]
    if n_far:
        assert 0 < wide64 < (n + 31) // 32 and 0 < wide32 < (n + 63) // 64
    else:
        assert wide64 == 0 and wide32 == 0
    # the layout's byte count: 2-byte differences (+ bases) in compressed slices
    nz = int(mo.csr_index()[-1])
    full_bytes = nz * (8 + 4) + (n + 1) * 4 + 2 * n * 8
    assert mp.Rarray[api.B200_PRM_R_SPMV_BYTES_FP64] < full_bytes
    rng = np.random.default_rng(2)
    x = rng.standard_normal(n)
    assert bits_equal(mp.matvec(x), mo.matvec(x))
    x32 = x.astype(np.float32)
    vals32 = mo.values().astype(np.float32).astype(np.float64)
    mo.values()[:] = np.abs(vals32)
    bound = mo.matvec(np.abs(x32.astype(np.float64)))
    mo.values()[:] = vals32
    y_ref = mo.matvec(x32.astype(np.float64))
    d_x = torch.from_numpy(x32).cuda()
    d_y = torch.empty_like(d_x)
    mp.device_matvec(d_x.data_ptr(), d_y.data_ptr(), fp32=True)
    torch.cuda.synchronize()
    assert np.all(np.abs(d_y.cpu().numpy().astype(np.float64) - y_ref) <= 1e-6 * bound + 1e-30)


def test_spmv_structured_grid_compresses(gpu, oracle):
    """192^3 7-point grid: the rows at both ends of a grid line put stencil
    neighbours +-n and +-n^2 into one slot; with the midpoint base every
    slice still compresses. The slices inside a grid line have every block
    at the same offset from its row: they are uniform and read no column
    stream (4 of the 6 32-row slices of a line, 1 of the 3 64-row ones). The
    FP64 SpMV stays bit-identical, the FP32 one within its rounding bound."""
    import torch
    n = 192
    mp, b = build(gpu, "convection_diffusion", n=n, peclet=5.0)
    mo, _ = build(oracle, "convection_diffusion", n=n, peclet=5.0)
    mp.set_matrix_cache(True)
    mp.set_precision(1)
    mp.device_prepare()
    assert mp.Iarray[api.B200_PRM_I_WIDE_SLICES_FP64] == 0
    assert mp.Iarray[api.B200_PRM_I_WIDE_SLICES_FP32] == 0
    assert mp.Iarray[api.B200_PRM_I_UNIFORM_SLICES_FP64] == n * n * 4
    assert mp.Iarray[api.B200_PRM_I_UNIFORM_SLICES_FP32] == n * n * 1
    nz = int(mo.csr_index()[-1])
    # the layout's bytes: no difference stream in the uniform slices
    assert mp.Rarray[api.B200_PRM_R_SPMV_BYTES_FP64] < nz * (8 + 2) + (n ** 3 + 1) * 4 + 2 * n ** 3 * 8
    x = np.random.default_rng(4).standard_normal(len(b))
    assert bits_equal(mp.matvec(x), mo.matvec(x))
    x32 = x.astype(np.float32)
    vals32 = mo.values().astype(np.float32).astype(np.float64)
    mo.values()[:] = np.abs(vals32)
    bound = mo.matvec(np.abs(x32.astype(np.float64)))
    mo.values()[:] = vals32
    y_ref = mo.matvec(x32.astype(np.float64))
    d_x = torch.from_numpy(x32).cuda()
    d_y = torch.empty_like(d_x)
    mp.device_matvec(d_x.data_ptr(), d_y.data_ptr(), fp32=True)
    torch.cuda.synchronize()
    assert np.all(np.abs(d_y.cpu().numpy().astype(np.float64) - y_ref) <= 1e-6 * bound + 1e-30)


def test_spmv_ndof2_random_blocks(gpu, oracle):
    # 10-node chain, ndof 2, like wrapper_test/solver/monolis_solver_c_test.c
    elem = np.array([[i, i + 1] for i in range(9)], dtype=np.int32)
    rng = np.random.default_rng(3)
    vals = rng.standard_normal((9, 16))
    out = []
    for lib in (gpu, oracle):
        m = api.Monolis(lib)
        m.get_nonzero_pattern_by_simple_mesh(10, 2, 2, elem)
        m.add_elements(elem, 2, vals.reshape(-1), 16)
        x = np.linspace(-1, 1, 20)
        out.append(m.matvec(x))
    assert bits_equal(out[0], out[1])


def test_inner_product(gpu, oracle):
    mp, b = build(gpu, "laplacian", n=20)
    mo, _ = build(oracle, "laplacian", n=20)
    rng = np.random.default_rng(1)
    x, y = rng.standard_normal(len(b)), rng.standard_normal(len(b))
    sp = mp.inner_product(1, x, y)
    so = mo.inner_product(1, x, y)
    assert abs(sp - so) <= 1e-13 * np.abs(x * y).sum()
    # double-double: the correctly rounded sum of the rounded products
    assert sp == math.fsum((x * y).tolist())
    with oracle_dot_mode(oracle, 1):
        assert sp == mo.inner_product(1, x, y)


@pytest.mark.parametrize("problem,kw,method", [
    ("laplacian", dict(n=32), api.ITER_CG),          # the CPU-runnable configuration, full size
    ("elasticity", dict(n=12), api.ITER_CG),
    ("diffusion_kappa", dict(n=12), api.ITER_CG),
    ("convection_diffusion", dict(n=24, peclet=0.5), api.ITER_BICGSTAB),
    ("convection_diffusion", dict(n=24, peclet=5.0), api.ITER_BICGSTAB),
    ("convection_diffusion", dict(n=24, peclet=50.0), api.ITER_BICGSTAB),
    ("laplacian", dict(n=16), api.ITER_BICGSTAB),
    ("laplacian", dict(n=32), api.ITER_PIPECG),      # PipeCG: iter_RR 50, crossed
    ("elasticity", dict(n=12), api.ITER_PIPECG),
    ("diffusion_kappa", dict(n=12), api.ITER_PIPECG),
    ("laplacian", dict(n=32), api.ITER_GROPCG),
    ("elasticity", dict(n=12), api.ITER_GROPCG),
    ("diffusion_kappa", dict(n=12), api.ITER_GROPCG),
])
@pytest.mark.parametrize("prec", [api.PREC_DIAG, api.PREC_NONE])
def test_solver_parity_fp64(gpu, oracle, problem, kw, method, prec):
    """Iterations within 2 of the oracle's. GropCG and PipeCG carry their
    residuals by recurrence (GropCG never replaces them), which amplifies
    the summation order of the dots: for them the bound is max(2, 3 x the
    oracle's own spread over 1, 2, 4 and 8 threads)."""
    mp, b = build(gpu, problem, **kw)
    mo, _ = build(oracle, problem, **kw)
    xo, it_o, res_o, st_o = solve(mo, b, method, prec, tol=1e-8)
    xp, it_p, res_p, st_p = solve(mp, b, method, prec, tol=1e-8)
    assert st_o == 0 and st_p == 0, (st_o, st_p)
    bound = 2
    if method in (api.ITER_GROPCG, api.ITER_PIPECG):
        its = [it_o]
        try:
            for th in (2, 4, 8):
                oracle.oracle_set_threads(th)
                mt, _ = build(oracle, problem, **kw)
                its.append(solve(mt, b, method, prec, tol=1e-8)[1])
        finally:
            oracle.oracle_set_threads(1)
        bound = max(2, 3 * (max(its) - min(its)))
    assert abs(it_p - it_o) <= bound, (it_p, it_o, bound)
    assert res_p < 1e-8
    # both iterates satisfy the same tolerance; compare them at a tighter solve
    xo2, _, _, _ = solve(mo, b, method, prec, tol=1e-12)
    xp2, _, _, _ = solve(mp, b, method, prec, tol=1e-12)
    assert rel_err(xp2, xo2) < 1e-10
    assert rel_err(xp, xo) < 1e-6
    # the oracle with the product's dot-product arithmetic: same count, same bits
    with oracle_dot_mode(oracle, 1):
        mn, _ = build(oracle, problem, **kw)
        xn, it_n, _, st_n = solve(mn, b, method, prec, tol=1e-8)
    assert st_n == 0 and it_p == it_n, (it_p, it_n)
    assert bits_equal(xp, xn)


@pytest.mark.parametrize("problem,kw", [
    ("convection_diffusion", dict(n=24, peclet=5.0)),
    ("convection_diffusion", dict(n=32, peclet=50.0)),
    ("laplacian", dict(n=16)),
])
@pytest.mark.parametrize("prec", [api.PREC_DIAG, api.PREC_NONE])
def test_bicgstab_n128_parity(gpu, oracle, problem, kw, prec):
    """MONOLIS_ITER_BICGSTAB_N128 (src/iterative/BiCGSTAB_N128.f90): rho and
    c2 in double-double in the reference, every dot product on the device.
    The reference's other sums ((T,S), (T,T), <R,R>) stay order-dependent:
    on the 16^3 Laplacian its count moves between 47 and 48 with 1, 2, 4 and
    8 oracle threads. So: iterations within 2 of the range the oracle's
    restatement gives over those thread counts, exactly the count of the
    oracle with every dot product in double-double, solution 1e-10 at a tight
    tolerance; FP32 refinement is refused (status 5)."""
    mp, b = build(gpu, problem, **kw)
    its = []
    try:
        for th in (1, 2, 4, 8):
            oracle.oracle_set_threads(th)
            mo, _ = build(oracle, problem, **kw)
            xo, it_o, _, st_o = solve(mo, b, api.ITER_BICGSTAB_N128, prec, tol=1e-8)
            assert st_o == 0
            its.append(it_o)
    finally:
        oracle.oracle_set_threads(1)
    xp, it_p, res_p, st_p = solve(mp, b, api.ITER_BICGSTAB_N128, prec, tol=1e-8)
    assert st_p == 0 and res_p < 1e-8
    assert min(its) - 2 <= it_p <= max(its) + 2, (it_p, its)
    with oracle_dot_mode(oracle, 1):
        mn, _ = build(oracle, problem, **kw)
        assert solve(mn, b, api.ITER_BICGSTAB_N128, prec, tol=1e-8)[1] == it_p
    mo, _ = build(oracle, problem, **kw)
    xo2, _, _, _ = solve(mo, b, api.ITER_BICGSTAB_N128, prec, tol=1e-12)
    xp2, _, _, _ = solve(mp, b, api.ITER_BICGSTAB_N128, prec, tol=1e-12)
    assert rel_err(xp2, xo2) < 1e-10
    _, _, _, st_m = solve(mp, b, api.ITER_BICGSTAB_N128, prec, tol=1e-8, precision=1)
    assert st_m == 5


def test_cg_parity_past_residual_replacement(gpu, oracle):
    # 277 oracle iterations: crosses the true-residual replacement at 200
    mp, b = build(gpu, "elasticity", n=24)
    mo, _ = build(oracle, "elasticity", n=24)
    xo, it_o, _, st_o = solve(mo, b, api.ITER_CG, api.PREC_DIAG)
    xp, it_p, _, st_p = solve(mp, b, api.ITER_CG, api.PREC_DIAG)
    assert it_o > 200 and st_o == 0 and st_p == 0
    assert abs(it_p - it_o) <= 2, (it_p, it_o)
    assert rel_err(xp, xo) < 1e-6


@pytest.mark.parametrize("problem,kw,method,prec,rr", [
    ("convection_diffusion", dict(n=48, peclet=5.0), api.ITER_BICGSTAB, api.PREC_DIAG, 20),
    ("convection_diffusion", dict(n=32, peclet=0.5), api.ITER_BICGSTAB, api.PREC_DIAG, 10),
    ("convection_diffusion", dict(n=40, peclet=50.0), api.ITER_BICGSTAB, api.PREC_DIAG, 15),
    ("diffusion_kappa", dict(n=24), api.ITER_CG, api.PREC_DIAG, 25),
    ("elasticity", dict(n=16), api.ITER_CG, api.PREC_NONE, 30),
    ("elasticity", dict(n=12), api.ITER_PIPECG, api.PREC_DIAG, 20),
    ("laplacian", dict(n=24), api.ITER_PIPECG, api.PREC_NONE, 15),
])
def test_parity_with_frequent_residual_replacement(gpu, oracle, problem, kw, method, prec, rr):
    """The replacement interval (200 in the reference) shortened in both
    libraries, so a well-conditioned solve crosses it several times."""
    mp, b = build(gpu, problem, **kw)
    mo, _ = build(oracle, problem, **kw)
    mp.Iarray[api.B200_PRM_I_ITER_RR] = rr
    oracle.oracle_set_iter_rr(rr)
    try:
        xo, it_o, _, st_o = solve(mo, b, method, prec)
    finally:
        oracle.oracle_set_iter_rr(0)  # back to the reference intervals (200; PipeCG 50)
    xp, it_p, _, st_p = solve(mp, b, method, prec)
    assert it_o > 2 * rr and st_o == 0 and st_p == 0
    assert abs(it_p - it_o) <= 2, (it_p, it_o)
    assert rel_err(xp, xo) < 1e-6


@pytest.mark.parametrize("problem,kw,method,prec,tol", [
    ("diffusion_kappa", dict(n=32), api.ITER_BICGSTAB, api.PREC_NONE, 1e-12),
    ("elasticity", dict(n=20), api.ITER_BICGSTAB, api.PREC_NONE, 1e-10),
])
def test_bicgstab_chaotic_cases_converge(gpu, oracle, problem, kw, method, prec, tol):
    """Unpreconditioned BiCGSTAB driven to 1e-10..1e-12: the iteration count
    depends on summation order (the oracle alone gives 348..381 and 235..240
    across 1..8 OpenMP threads), so only convergence and the solution are
    compared."""
    mp, b = build(gpu, problem, **kw)
    mo, _ = build(oracle, problem, **kw)
    xo, it_o, _, st_o = solve(mo, b, method, prec, tol=tol)
    xp, it_p, res_p, st_p = solve(mp, b, method, prec, tol=tol)
    assert st_o == 0 and st_p == 0 and res_p < tol
    assert abs(it_p - it_o) <= 0.15 * it_o, (it_p, it_o)
    assert rel_err(xp, xo) < 1e-6


@pytest.mark.parametrize("n", [8, 12, 16, 24])
def test_cg_mixed_precision_small(gpu, n):
    """Small elasticity systems converge fast; the FP32 correction must not
    carry the whole solution (true FP64 residual checked independently)."""
    mp, b = build(gpu, "elasticity", n=n)
    x, it, res, st = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=1e-8, precision=1)
    assert st == 0 and res < 1e-8
    r = b - mp.matvec(x)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.01e-8


def test_cg_mixed_precision(gpu, oracle):
    mp, b = build(gpu, "elasticity", n=12)
    mo, _ = build(oracle, "elasticity", n=12)
    xo, it_o, _, _ = solve(mo, b, api.ITER_CG, api.PREC_DIAG, tol=1e-12)
    xm, it_m, res_m, st_m = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=1e-8, precision=1)
    assert st_m == 0 and res_m < 1e-8
    # true FP64 residual of the mixed solution
    r = b - mo.matvec(xm)
    r0 = b
    assert np.linalg.norm(r) / np.linalg.norm(r0) < 1.01e-8
    assert mp.Iarray[api.B200_PRM_I_N_REFINE] >= 1
    assert rel_err(xm, xo) < 1e-5


@pytest.mark.parametrize("n,peclet", [(8, 0.5), (12, 5.0), (16, 50.0), (24, 5.0), (32, 0.5)])
@pytest.mark.parametrize("prec", [api.PREC_DIAG, api.PREC_NONE])
def test_bicgstab_mixed_precision(gpu, oracle, n, peclet, prec):
    """FP32-inner BiCGSTAB with FP64 refreshes on the nonsymmetric
    convection-diffusion systems: converged on the true FP64 residual
    (checked with the oracle's SpMV) and within 1e-5 of the FP64 solution."""
    mp, b = build(gpu, "convection_diffusion", n=n, peclet=peclet)
    mo, _ = build(oracle, "convection_diffusion", n=n, peclet=peclet)
    xo, _, _, st_o = solve(mo, b, api.ITER_BICGSTAB, prec, tol=1e-12)
    xm, it_m, res_m, st_m = solve(mp, b, api.ITER_BICGSTAB, prec, tol=1e-8, precision=1)
    assert st_o == 0 and st_m == 0 and res_m < 1e-8
    r = b - mo.matvec(xm)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1.01e-8
    assert mp.Iarray[api.B200_PRM_I_N_REFINE] >= 1
    assert rel_err(xm, xo) < 1e-5


def test_bicgstab_mixed_tight_tolerance(gpu, oracle):
    """Refinement carries the solution well past FP32 accuracy (1e-11)."""
    mp, b = build(gpu, "convection_diffusion", n=20, peclet=5.0)
    mo, _ = build(oracle, "convection_diffusion", n=20, peclet=5.0)
    xo, _, _, _ = solve(mo, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-13)
    xm, _, res_m, st_m = solve(mp, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-11, precision=1)
    assert st_m == 0 and res_m < 1e-11
    assert rel_err(xm, xo) < 1e-8


def test_zero_rhs(gpu, oracle):
    # src/linalg/mat_converge.f90:40-48: <r0,r0> == 0 -> X = 0, converged
    for lib in (gpu, oracle):
        m, b = build(lib, "laplacian", n=8)
        x = np.ones_like(b)
        m.set_init_x(True)
        m.solve(np.zeros_like(b), x)
        assert np.all(x == 0.0)
        assert m.get_error_tag() == 0


def test_maxiter_status(gpu, oracle):
    mp, b = build(gpu, "laplacian", n=16)
    _, it, _, st = solve(mp, b, maxiter=3)
    assert st == 1 and it == 3


def test_nonfinite_status(gpu):
    mp, b = build(gpu, "laplacian", n=8)
    b[5] = np.nan
    _, _, _, st = solve(mp, b)
    assert st == 3


def test_warm_start(gpu, oracle):
    mp, b = build(gpu, "laplacian", n=16)
    mo, _ = build(oracle, "laplacian", n=16)
    x0 = np.linspace(0, 1, len(b))
    xo, it_o, _, _ = solve(mo, b, x0=x0)
    xp, it_p, _, _ = solve(mp, b, x0=x0)
    assert abs(it_o - it_p) <= 2
    assert rel_err(xp, xo) < 1e-6
