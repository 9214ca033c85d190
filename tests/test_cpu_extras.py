"""CPU-side checks of the pieces added around the hot path: the product has no
CPU fallback (without a CUDA device every solve reports status 6 and leaves x
alone), and the synthetic problem builders of the batched and adjoint
workloads produce what their docstrings state."""
import ctypes as C

import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import problems as P


def _has_cuda():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_cuda(), reason="checks the behaviour without a CUDA device")
def test_product_has_no_cpu_fallback(product):
    m = api.Monolis(product)
    b = P.laplacian(m, n=4)
    m.quiet()
    m.set_error_abort(False)
    x = np.full_like(b, 7.0)
    m.set_init_x(False)
    m.solve(b, x)
    assert m.get_error_tag() == 6 and np.all(x == 7.0)
    assert m.solve_transpose(b, x) == 6
    B = np.stack([b, b])
    with pytest.raises(RuntimeError):
        m.solve_multi(B)
    batch = api.Batch(product)
    ix, it, v, _ = P.fv_diffusion_csr(4, 1)
    batch.add_csr(64, 1, ix, it, v)
    with pytest.raises(RuntimeError):
        batch.prepare()
    batch.destroy()
    out = C.c_double()
    assert product.monolis_b200_inner_product_noalloc_R(4, None, None, C.byref(out), None) != 0


def test_fv_diffusion_system():
    ix, it, v, kappa = P.fv_diffusion_csr(5, 3)
    n = 125
    A = np.zeros((n, n))
    for r in range(n):
        cols = it[ix[r]:ix[r + 1]]
        assert np.all(np.diff(cols) > 0)  # ascending columns
        A[r, cols] = v[ix[r]:ix[r + 1]]
    assert np.array_equal(A, A.T)
    assert np.linalg.eigvalsh(A).min() > 0
    # interior face transmissibility is the harmonic mean 2 k_i k_j / (k_i + k_j)
    i, j = 62, 63  # neighbours along x inside the cube
    assert np.isclose(-A[i, j], 2 * kappa[i] * kappa[j] / (kappa[i] + kappa[j]))
    # row sums: the Dirichlet boundary faces (2 k_i each) make boundary rows dominant
    assert np.isclose(A[62].sum(), 0.0, atol=1e-12)  # interior cell
    assert A[0].sum() > 0


def test_batch_sides_distribution():
    s = P.batch_sides()
    assert len(s) == 512 and s.min() >= 10 and s.max() <= 60
    total = int((s ** 3).sum())
    assert 1.5e7 < total < 3e7  # about 2e7 unknowns


def test_adjoint_target_and_mask():
    n = 9
    t = P.smooth_target(n)
    assert t.shape == (n ** 3,) and np.all(np.isfinite(t))
    grid = t.reshape(n, n, n)  # [z, y, x]
    assert np.allclose(grid[:, :, 0], 0.0) and np.allclose(grid[0], 0.0)  # zero on the faces
    fixed = P.face_x0_fixed(n, 3).reshape(n ** 3, 3)
    assert fixed.sum() == 3 * n * n and np.all(fixed[0::n] == 1)
