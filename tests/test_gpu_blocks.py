"""Block sizes beyond the workloads' 1 and 3 (the kernels take ndof 1..6):
FP64 CG and BiCGSTAB against the oracle (iterations +-2, solution 1e-10 at a
tight tolerance), the FP32-refined CG and the many-right-hand-side solver on
the same systems (FP64 residual below tol)."""
import numpy as np
import pytest

from monolis_b200 import api
from helpers import rel_err, solve

pytestmark = pytest.mark.gpu


def block_chain(lib, n_node, nd, seed, sym=True):
    """3D-ish chain: node i coupled to i+1 and i+7, random blocks, diagonal
    blocks made dominant (SPD when sym)."""
    rng = np.random.default_rng(seed)
    m = api.Monolis(lib)
    elem = np.array([[i, i + 1] for i in range(n_node - 1)] + [[i, i + 7] for i in range(n_node - 7)], dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(n_node, 2, nd, elem)
    for e in elem:
        blk = rng.uniform(-1.0, 1.0, (nd, nd))
        for a in range(nd):
            for c in range(nd):
                m.add_scalar(int(e[0]), int(e[1]), a, c, blk[a, c])
                m.add_scalar(int(e[1]), int(e[0]), c, a, blk[a, c] if sym else rng.uniform(-1, 1))
    for i in range(n_node):
        g = rng.uniform(-0.5, 0.5, (nd, nd))
        d = g @ g.T + np.eye(nd) * (6.0 * nd)
        for a in range(nd):
            for c in range(nd):
                m.add_scalar(i, i, a, c, d[a, c])
    m.quiet()
    m.set_error_abort(False)
    b = np.random.default_rng(seed + 1).standard_normal(n_node * nd)
    return m, b


@pytest.mark.parametrize("nd", [2, 4, 5, 6])
@pytest.mark.parametrize("method", [api.ITER_CG, api.ITER_BICGSTAB])
def test_fp64_solvers_block_sizes(gpu, oracle, nd, method):
    sym = method == api.ITER_CG
    mp, b = block_chain(gpu, 300, nd, 10 * nd, sym)
    mo, _ = block_chain(oracle, 300, nd, 10 * nd, sym)
    assert np.array_equal(mp.values(), mo.values())
    xo, ito, _, sto = solve(mo, b, method, api.PREC_DIAG, tol=1e-8)
    xp, itp, _, stp = solve(mp, b, method, api.PREC_DIAG, tol=1e-8)
    assert sto == 0 and stp == 0 and abs(itp - ito) <= 2, (itp, ito)
    xo2, _, _, _ = solve(mo, b, method, api.PREC_DIAG, tol=1e-12)
    xp2, _, _, _ = solve(mp, b, method, api.PREC_DIAG, tol=1e-12)
    assert rel_err(xp2, xo2) < 1e-10


@pytest.mark.parametrize("nd", [2, 4, 6])
def test_mixed_and_multi_block_sizes(gpu, oracle, nd):
    mp, b = block_chain(gpu, 400, nd, 7 * nd)
    mo, _ = block_chain(oracle, 400, nd, 7 * nd)
    xm, _, resm, stm = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=1e-9, precision=1)
    assert stm == 0 and resm < 1e-9
    assert np.linalg.norm(b - mo.matvec(xm)) / np.linalg.norm(b) < 1.01e-9
    B = np.stack([b, 2.0 * b + 0.5, np.ones_like(b)])
    for precision in (0, 1):
        mp.set_precision(precision)
        X, its, res, st = mp.solve_multi(B)
        assert np.all(st == 0)
        for k in range(3):
            assert np.linalg.norm(B[k] - mo.matvec(X[k])) / np.linalg.norm(B[k]) < 1.01e-9


def _device_and_oracle_factors(mp, mo):
    import ctypes as C
    n = int(mo.s.mat.N) * int(mo.s.mat.NDOF) ** 2
    ao = np.zeros(n)
    mo.lib.oracle_diag_setup(mo.p, ao.ctypes.data_as(C.POINTER(C.c_double)))
    mp.set_precond(api.PREC_DIAG)
    mp.set_precision(0)
    mp.device_prepare()
    ap = np.zeros(n)
    assert mp.lib.monolis_b200_device_get_diag(mp.p, ap.ctypes.data_as(C.POINTER(C.c_double))) == 0
    return ap, ao


@pytest.mark.parametrize("nd", [1, 2, 3, 4, 5, 6])
def test_diag_factors_bit_exact(gpu, oracle, nd):
    """Device DIAG setup (diagonal block extracted from the CSR row, LU
    without pivoting, reciprocal pivots) against the oracle's restatement of
    src/prec/diag/diag_33.f90:16-99 and diag_nn.f90:16-86, bit for bit,
    nonsymmetric blocks included."""
    from helpers import bits_equal
    mp, _ = block_chain(gpu, 200, nd, 3 * nd, sym=False)
    mo, _ = block_chain(oracle, 200, nd, 3 * nd, sym=False)
    ap, ao = _device_and_oracle_factors(mp, mo)
    assert bits_equal(ap, ao)


@pytest.mark.parametrize("nd", [1, 3, 5])
def test_diag_factors_zero_pivot(gpu, oracle, nd):
    """A zero pivot is replaced by 1 (src/prec/diag/diag_33.f90:74,
    diag_nn.f90): rows whose diagonal block is zero or has a zero leading
    entry give the same factors on the device as in the oracle."""
    from helpers import bits_equal
    elem = np.array([[i, i + 1] for i in range(7)], dtype=np.int32)
    libs = []
    for lib in (gpu, oracle):
        m = api.Monolis(lib)
        m.get_nonzero_pattern_by_simple_mesh(8, 2, nd, elem)
        rng = np.random.default_rng(nd)
        for i in range(8):
            for a in range(nd):
                for c in range(nd):
                    v = rng.uniform(1.0, 2.0) if a == c else rng.uniform(-0.3, 0.3)
                    if i == 2 or (i == 5 and a == 0):
                        v = 0.0  # whole block zero / first pivot zero
                    m.add_scalar(i, i, a, c, v)
        libs.append(m)
    ap, ao = _device_and_oracle_factors(*libs)
    assert bits_equal(ap, ao)
    nd2 = nd * nd
    assert all(ap[2 * nd2 + k * (nd + 1)] == 1.0 for k in range(nd))
