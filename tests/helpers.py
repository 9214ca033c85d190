"""Shared helpers: build a problem in a library, solve it, compare."""
import contextlib

import numpy as np

from monolis_b200 import api
from monolis_b200 import problems as P

BUILDERS = {
    "laplacian": P.laplacian,
    "elasticity": P.elasticity,
    "convection_diffusion": P.convection_diffusion,
    "diffusion_kappa": P.diffusion_kappa,
}


def build(lib, problem, **kw):
    m = api.Monolis(lib)
    b = BUILDERS[problem](m, **kw)
    if isinstance(b, tuple):
        b = b[0]
    m.quiet()
    m.set_error_abort(False)
    return m, np.ascontiguousarray(b)


def solve(m, b, method=api.ITER_CG, prec=api.PREC_DIAG, tol=1e-8, maxiter=10000, precision=0, x0=None):
    m.set_method(method)
    m.set_precond(prec)
    m.set_tolerance(tol)
    m.set_maxiter(maxiter)
    if m.lib.is_product:
        m.set_precision(precision)
    x = np.zeros_like(b) if x0 is None else np.array(x0, dtype=np.float64)
    m.set_init_x(x0 is None)
    m.solve(b, x)
    return x, m.get_converge_iter(), m.get_converge_residual(), m.get_error_tag()


def rel_err(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bits_equal(a, b):
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    return a.shape == b.shape and np.array_equal(a.view(np.uint64), b.view(np.uint64))


@contextlib.contextmanager
def oracle_dot_mode(oracle, mode):
    """Runs the oracle with its dot products in the given arithmetic: 0 the
    reference's plain sums, 1 double-double (the product's FP64 kernels)."""
    old = oracle.oracle_get_dot_mode()
    oracle.oracle_set_dot_mode(mode)
    try:
        yield
    finally:
        oracle.oracle_set_dot_mode(old)
