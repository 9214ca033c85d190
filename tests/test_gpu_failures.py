"""Failure paths that the host or the kernels turn into status codes, with
inputs made on the host (no GPU fault is provoked): CSR validation before the
upload (MONOLIS_B200_PRM_I_CHECK) and a BiCGSTAB breakdown (c2 = <RT,V> = 0).
Status codes: 2 breakdown, 5 bad input (Iarray[MONOLIS_PRM_I_IERR])."""
import numpy as np
import pytest

from monolis_b200 import api
from helpers import build, solve

pytestmark = pytest.mark.gpu


def test_check_mode_rejects_out_of_range_column(gpu):
    """With the check on, a block column outside 1..NP in the host CSR is
    found before anything is uploaded: status 5, x untouched; the repaired
    matrix then solves."""
    m, b = build(gpu, "laplacian", n=8)
    m.Iarray[api.B200_PRM_I_CHECK] = 1
    item = m.csr_item()
    saved = int(item[17])
    item[17] = m.N + 5
    x0 = np.full_like(b, 7.0)
    x, _, _, st = solve(m, b, api.ITER_CG, api.PREC_DIAG, x0=x0)
    assert st == 5 and np.all(x == 7.0)
    item[17] = 0  # 1-based ids: 0 is out of range too
    _, _, _, st = solve(m, b, api.ITER_CG, api.PREC_DIAG)
    assert st == 5
    item[17] = saved
    m.matrix_changed()
    _, _, res, st = solve(m, b, api.ITER_CG, api.PREC_DIAG)
    assert st == 0 and res < 1e-8


def test_check_mode_rejects_decreasing_offsets(gpu):
    m, b = build(gpu, "laplacian", n=6)
    m.Iarray[api.B200_PRM_I_CHECK] = 1
    index = m.csr_index()
    saved = int(index[10])
    index[10] = index[9] - 1
    _, _, _, st = solve(m, b, api.ITER_CG, api.PREC_DIAG)
    assert st == 5
    index[10] = saved
    m.matrix_changed()
    _, _, _, st = solve(m, b, api.ITER_CG, api.PREC_DIAG)
    assert st == 0


def test_bicgstab_breakdown_status(gpu):
    """A = [[0, 1], [-1, 0]] without preconditioner, b = (1, 1): the first
    V = A P is orthogonal to the shadow residual, c2 = <RT,V> = 0, and the
    solve stops with status 2 (breakdown) instead of dividing by zero."""
    m = api.Monolis(gpu)
    index = np.array([0, 1, 2], dtype=np.int32)
    item = np.array([1, 0], dtype=np.int32)
    m.set_matrix_BCSR(2, 2, 1, 2, np.array([1.0, -1.0]), index, item)
    m.quiet()
    m.set_error_abort(False)
    _, _, _, st = solve(m, np.array([1.0, 1.0]), api.ITER_BICGSTAB, api.PREC_NONE)
    assert st == 2
