"""Adjoint pieces on the GPU: transpose SpMV and solve, the sampled outer
product, the per-element gradient, and the whole gradient of the adjoint
workload (3D Q1 diffusion, L = 1/2 ||x - x_target||^2, dL/dkappa_e) checked
against central finite differences and against an FP64 reference gradient
computed from the CPU oracle.

Tolerances: transpose SpMV bit-identical to the oracle's SpMV of the explicit
transpose (same row order, no FMA); transpose solves like the forward ones
(iterations +-2, solution 1e-10); the sampled outer product bit-identical to
numpy; element gradients 1e-12 relative to the pattern-level reduction;
gradient vs FD 1e-5 relative, vs the oracle's gradient 1e-8."""
import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import problems as P
from helpers import bits_equal, build, rel_err, solve

pytestmark = pytest.mark.gpu


def explicit_transpose(lib, m):
    """A^T of m as a new struct in lib, from m's CSC arrays
    (monolis_get_CSC_format): row j lists column j's rows in ascending order."""
    nd = m.NDOF
    vals = m.values().reshape(-1, nd, nd)
    perm = m.csc_perm().astype(np.int64) - 1
    vt = np.ascontiguousarray(vals[perm].transpose(0, 2, 1).reshape(-1))
    t = api.Monolis(lib)
    idx = np.ascontiguousarray(m.csc_index(), dtype=np.int32)
    item = np.ascontiguousarray(m.csc_item() - 1, dtype=np.int32)
    t.set_matrix_BCSR(m.N, m.N, nd, len(item), vt, idx, item)
    t.quiet()
    t.set_error_abort(False)
    return t


def random_nonsymmetric(lib, n_node, nd, seed):
    """Chain-plus-skip pattern with random nonsymmetric blocks and a dominant diagonal."""
    rng = np.random.default_rng(seed)
    m = api.Monolis(lib)
    elem = np.array([[i, (i + 1) % n_node] for i in range(n_node)] + [[i, (i + 5) % n_node] for i in range(0, n_node, 3)],
                    dtype=np.int32)
    m.get_nonzero_pattern_by_simple_mesh(n_node, 2, nd, elem)
    vals = m.values()
    vals[:] = rng.uniform(-1.0, 1.0, len(vals))
    idx, item = m.csr_index(), m.csr_item()
    for i in range(n_node):
        for k in range(idx[i], idx[i + 1]):
            if item[k] - 1 == i:
                blk = vals[k * nd * nd:(k + 1) * nd * nd].reshape(nd, nd)
                blk += np.eye(nd) * (8.0 + 4.0 * nd)
    m.quiet()
    m.set_error_abort(False)
    return m


@pytest.mark.parametrize("case", ["convdiff", "random3", "random1"])
def test_transpose_matvec_bit_exact(gpu, oracle, case):
    if case == "convdiff":
        mp, b = build(gpu, "convection_diffusion", n=9, peclet=50.0)
    else:
        mp = random_nonsymmetric(gpu, 40, 3 if case == "random3" else 1, seed=11)
        b = np.zeros(mp.N * mp.NDOF)
    mt = explicit_transpose(oracle, mp)
    rng = np.random.default_rng(3)
    for _ in range(2):
        x = rng.standard_normal(len(b))
        assert bits_equal(mp.matvec_transpose(x), mt.matvec(x))
    # and A^T differs from A for these matrices
    x = rng.standard_normal(len(b))
    assert not bits_equal(mp.matvec_transpose(x), mp.matvec(x))


def transpose_solve(m, b, method, tol, precision=0):
    m.set_method(method)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(tol)
    m.set_maxiter(10000)
    m.set_precision(precision)
    m.set_init_x(True)
    x = np.zeros_like(b)
    rc = m.solve_transpose(b, x)
    return x, m.get_converge_iter(), rc


@pytest.mark.parametrize("problem,kw,method", [
    ("convection_diffusion", dict(n=12, peclet=5.0), api.ITER_BICGSTAB),
    ("convection_diffusion", dict(n=10, peclet=50.0), api.ITER_BICGSTAB),
    ("elasticity", dict(n=7), api.ITER_CG),  # symmetric: A^T = A
])
def test_transpose_solve_matches_oracle(gpu, oracle, problem, kw, method):
    """monolis_b200_solve_transpose_R against the oracle's monolis_solve_R on
    the explicit transpose: iterations +-2 at 1e-8, solutions 1e-10 at 1e-12."""
    mp, b = build(gpu, problem, **kw)
    mt = explicit_transpose(oracle, mp)
    xo, ito, _, sto = solve(mt, b, method, api.PREC_DIAG, tol=1e-8)
    xp, itp, rc = transpose_solve(mp, b, method, 1e-8)
    assert rc == 0 and sto == 0
    assert abs(itp - ito) <= 2, (itp, ito)
    xo2, _, _, _ = solve(mt, b, method, api.PREC_DIAG, tol=1e-12)
    xp2, _, rc = transpose_solve(mp, b, method, 1e-12)
    assert rc == 0
    assert rel_err(xp2, xo2) < 1e-10
    r = b - mt.matvec(xp2)
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-11


def test_transpose_solve_mixed(gpu):
    mp, b = build(gpu, "diffusion_kappa", n=10)
    x, _, rc = transpose_solve(mp, b, api.ITER_CG, 1e-10, precision=1)
    assert rc == 0
    x64, _, rc = transpose_solve(mp, b, api.ITER_CG, 1e-10, precision=0)
    assert rc == 0
    assert rel_err(x, x64) < 1e-8


def test_sampled_outer_product_bit_exact(gpu):
    for mp in (random_nonsymmetric(gpu, 30, 3, seed=5), build(gpu, "diffusion_kappa", n=6)[0]):
        nd = mp.NDOF
        rng = np.random.default_rng(9)
        lam = rng.standard_normal(mp.N * nd)
        x = rng.standard_normal(mp.N * nd)
        G = mp.sampled_outer_product(lam, x, scale=-1.0)
        idx, item = mp.csr_index(), mp.csr_item() - 1
        rows = np.repeat(np.arange(mp.N), np.diff(idx))
        L = (-1.0 * lam.reshape(-1, nd))[rows]  # (nz, nd)
        X = x.reshape(-1, nd)[item]
        ref = (L[:, :, None] * X[:, None, :]).reshape(-1)
        assert bits_equal(G, ref)


def element_reduction_from_pattern(m, elem, kref, fixed, G):
    """dL/dk_e = sum over the element's (a, b) of K(a,b) * G at the stored
    entry (n_a, n_b), rows of fixed dofs excluded (numpy, from G)."""
    idx, item = m.csr_index(), m.csr_item() - 1
    out = np.zeros(len(elem))
    for e, en in enumerate(elem):
        s = 0.0
        for a, na in enumerate(en):
            if fixed[na]:
                continue
            row = item[idx[na]:idx[na + 1]]
            for bb, nb in enumerate(en):
                k = idx[na] + int(np.searchsorted(row, nb))
                s += kref[a, bb] * G[k]
        out[e] = s
    return out


def test_element_gradient_equals_pattern_reduction(gpu):
    n = 6
    mp, _ = build(gpu, "diffusion_kappa", n=n)
    elem, kref, fixed = P.hex_elements(n), P.hex8_diffusion_ke(1.0 / (n - 1)), P.face_x0_fixed(n, 1)
    rng = np.random.default_rng(4)
    lam = rng.standard_normal(n ** 3)
    x = rng.standard_normal(n ** 3)
    g = mp.element_gradient(elem, 8, kref.reshape(-1), 0, lam, x, fixed=fixed, scale=-1.0)
    G = mp.sampled_outer_product(lam, x, scale=-1.0)
    ref = element_reduction_from_pattern(mp, elem, kref, fixed, G)
    assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))
    # per-element matrices (stride) give the same result for copies of kref
    kper = np.tile(kref.reshape(-1), len(elem))
    g2 = mp.element_gradient(elem, 8, kper, 64, lam, x, fixed=fixed, scale=-1.0)
    assert bits_equal(g, g2)


def test_element_gradient_elasticity_blocks(gpu):
    """ndof 3 (24 local dofs, register path) and a generic size (2-node
    elements, ndof 3 -> 6 local dofs) against numpy."""
    rng = np.random.default_rng(8)
    n = 5
    mp, _ = build(gpu, "elasticity", n=n)
    elem = P.hex_elements(n)
    ke = rng.standard_normal((24, 24))
    lam = rng.standard_normal(n ** 3 * 3)
    x = rng.standard_normal(n ** 3 * 3)
    fixed = P.face_x0_fixed(n, 3)
    g = mp.element_gradient(elem, 8, ke.reshape(-1), 0, lam, x, fixed=fixed, scale=-1.0)
    dofs = (elem[:, :, None] * 3 + np.arange(3)).reshape(len(elem), 24)
    le = np.where(fixed[dofs] != 0, 0.0, lam[dofs])
    ref = -np.einsum("ea,ab,eb->e", le, ke, x[dofs])
    assert np.max(np.abs(g - ref)) <= 1e-12 * np.max(np.abs(ref))
    edges = elem[:, :2].copy()
    k2 = rng.standard_normal((6, 6))
    g2 = mp.element_gradient(edges, 2, k2.reshape(-1), 0, lam, x, scale=1.0)
    d2 = (edges[:, :, None] * 3 + np.arange(3)).reshape(len(edges), 6)
    ref2 = np.einsum("ea,ab,eb->e", lam[d2], k2, x[d2])
    assert np.max(np.abs(g2 - ref2)) <= 1e-12 * np.max(np.abs(ref2))


def test_element_gradient_rejects_bad_node(gpu):
    mp, _ = build(gpu, "diffusion_kappa", n=4)
    elem = P.hex_elements(4).copy()
    elem[3, 2] = 4 ** 3  # out of range
    with pytest.raises(RuntimeError):
        mp.element_gradient(elem, 8, np.eye(8).reshape(-1), 0, np.zeros(64), np.zeros(64))


@pytest.mark.parametrize("precision", [0, 1])
def test_adjoint_gradient_fd_and_reference(gpu, oracle, precision):
    """The adjoint workload at 12^3 nodes: gradient from the test-only
    torch.autograd.Function vs central finite differences on 32 seeded
    directions (1e-5 relative) and vs the FP64 gradient of the CPU oracle."""
    from adjoint_torch import DiffusionSystem, loss_and_grad

    n = 12
    tol = 1e-12 if precision == 0 else 1e-11
    sys_p = DiffusionSystem(gpu, n, tol=tol, precision=precision)
    kappa = np.exp(P.normal(5, (n - 1) ** 3, 0.0, 1.0))
    target = P.smooth_target(n)
    L, g = loss_and_grad(sys_p, kappa, target)
    assert np.all(np.isfinite(g)) and np.linalg.norm(g) > 0

    # FP64 reference gradient: oracle forward solve, oracle solve of the
    # explicit transpose, element reduction in numpy
    sys_o = DiffusionSystem(oracle, n, tol=1e-13)
    mo, xo = sys_o.forward(kappa)
    mt = explicit_transpose(oracle, mo)
    lam_o, _, _, st = solve(mt, xo - target, api.ITER_CG, api.PREC_DIAG, tol=1e-13)
    assert st == 0
    le = np.where(sys_o.fixed[sys_o.elem] != 0, 0.0, lam_o[sys_o.elem])
    g_ref = -np.einsum("ea,ab,eb->e", le, sys_o.kref, xo[sys_o.elem])
    assert rel_err(g, g_ref) < (1e-8 if precision == 0 else 1e-7)

    # central differences along 32 seeded directions (relative to kappa)
    rng = np.random.default_rng(2025)
    h = 1e-4
    worst = 0.0
    for _ in range(32):
        d = kappa * rng.standard_normal(len(kappa))
        fd = (sys_p.loss(kappa + h * d, target) - sys_p.loss(kappa - h * d, target)) / (2 * h)
        an = float(np.dot(g, d))
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    assert worst < 1e-5, worst
