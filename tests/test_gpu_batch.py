"""Batched solver (monolis_b200_batch_*): many independent systems solved by CG
+ DIAG in one persistent kernel, against per-system FP64 solves of the CPU
oracle on the same systems.

Tolerances: with refinement every system reaches the FP64 relative residual
tol (checked with an FP64 numpy SpMV) and its solution agrees with the
oracle's tighter solve to 1e-6 relative; without refinement (FP32 recursion)
the true residual of the result is within 10x of the 1e-6 target."""
import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import problems as P
from helpers import rel_err, solve

pytestmark = pytest.mark.gpu


def make_systems(sides, seed0=100):
    return [P.fv_diffusion_csr(int(s), seed0 + i) for i, s in enumerate(sides)]


def rhs(systems, seed0=500):
    return [P.uniform(seed0 + i, len(ix) - 1) for i, (ix, _, _, _) in enumerate(systems)]


def new_batch(lib, systems, config=None):
    b = api.Batch(lib)
    for ix, it, v, _ in systems:
        b.add_csr(len(ix) - 1, 1, ix, it, v)
    b.prepare(precond=api.PREC_DIAG, autotune=config is None)
    if config is not None:
        b.set_config(*config)
    return b


def oracle_solution(oracle, sysm, b, tol=1e-12):
    ix, it, v, _ = sysm
    m = api.Monolis(oracle)
    m.set_matrix_BCSR(len(ix) - 1, len(ix) - 1, 1, len(it), v, ix, it)
    m.quiet()
    m.set_error_abort(False)
    x, _, _, st = solve(m, b, api.ITER_CG, api.PREC_DIAG, tol=tol, maxiter=20000)
    assert st == 0
    return x


def true_resid(sysm, x, b):
    ix, it, v, _ = sysm
    return float(np.linalg.norm(b - P.csr_matvec(ix, it, v, x)) / np.linalg.norm(b))


SIDES = [4, 13, 7, 9, 12, 5, 16, 3, 10, 8, 11, 6, 14, 4, 9, 15, 7, 12]


@pytest.mark.parametrize("config", [None, (1, 256, 0), (2, 256, 0), (4, 512, 0), (8, 256, 0), (4, 256, 1024),
                                    (8, 512, 4096)])
def test_batch_refined_matches_oracle(gpu, oracle, config):
    systems = make_systems(SIDES)
    bs = rhs(systems)
    batch = new_batch(gpu, systems, config)
    xs, its, res, st = batch.solve(bs, tol=1e-8, max_iter=5000, refine=True)
    assert np.all(st == 0), st
    assert np.all(res < 1e-8), res
    for k, (sysm, x, b) in enumerate(zip(systems, xs, bs)):
        assert true_resid(sysm, x, b) < 1.01e-8, k
        xo = oracle_solution(oracle, sysm, b)
        assert rel_err(x, xo) < 1e-6, k
        assert its[k] >= 1
    batch.destroy()


def test_batch_fp32_only(gpu):
    systems = make_systems(SIDES[:10], seed0=300)
    bs = rhs(systems, seed0=900)
    batch = new_batch(gpu, systems, (4, 256, 2048))
    xs, its, res, st = batch.solve(bs, tol=1e-6, max_iter=5000, refine=False)
    assert np.all(st == 0), st
    for k, (sysm, x, b) in enumerate(zip(systems, xs, bs)):
        tr = true_resid(sysm, x, b)
        assert tr < 1e-5, (k, tr)
        assert abs(tr - res[k]) <= 1e-3 * tr + 1e-12  # the reported residual is the FP64 one of x
    batch.destroy()


def test_batch_zero_rhs_and_maxiter(gpu):
    systems = make_systems([6, 12, 9], seed0=40)
    bs = rhs(systems)
    bs[0] = np.zeros_like(bs[0])
    batch = new_batch(gpu, systems, (2, 256, 0))
    xs, its, res, st = batch.solve(bs, tol=1e-8, max_iter=5000, refine=True)
    assert st[0] == 0 and its[0] == 0 and np.all(xs[0] == 0.0)
    assert st[1] == 0 and st[2] == 0
    xs, its, res, st = batch.solve(bs, tol=1e-12, max_iter=3, refine=True)
    assert st[1] == 1 and st[2] == 1 and its[1] == 3  # max_iter reached (status 1)
    batch.destroy()


def test_batch_configs_agree_and_autotune(gpu):
    systems = make_systems([20, 9, 15, 30, 5, 11, 25, 7], seed0=70)
    bs = rhs(systems, seed0=71)
    batch = new_batch(gpu, systems, (1, 256, 0))
    cands = batch.autotune(iters=10)
    assert len(cands) >= 4 and all(c[3] > 0 for c in cands)
    chosen = batch.config()
    assert chosen in [(c[0], c[1], c[2]) for c in cands]
    ref, _, _, _ = batch.solve(bs, tol=1e-10, max_iter=5000, refine=True)
    for cfg in [(1, 512, 0), (2, 256, 512), (8, 256, 0)]:
        batch.set_config(*cfg)
        xs, _, res, st = batch.solve(bs, tol=1e-10, max_iter=5000, refine=True)
        assert np.all(st == 0)
        for a, b in zip(xs, ref):
            assert rel_err(a, b) < 1e-8
    batch.destroy()


def test_batch_device_vectors_layout(gpu):
    """The device-resident form: b written into the stacked device vector at
    the reported offsets, x read back from there."""
    import ctypes
    import torch
    cudart = ctypes.CDLL("libcudart.so.12")  # already loaded by torch
    cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
    d2d = 3  # cudaMemcpyDeviceToDevice
    systems = make_systems([5, 8, 3], seed0=10)
    bs = rhs(systems, seed0=11)
    batch = new_batch(gpu, systems, (2, 256, 0))
    off = batch.offsets()
    assert off[0] == 0 and np.all(off % 64 == 0)
    assert list(np.diff(off)) == [128, 512]  # 125 rows -> 128, 512 rows
    d_b, d_x = batch.device_vectors()
    total = int(off[-1]) + 64  # last system (27 rows) padded to 64
    tb = torch.zeros(total, dtype=torch.float64, device="cuda")
    for o, b in zip(off, bs):
        tb[int(o):int(o) + len(b)] = torch.from_numpy(b)
    torch.cuda.synchronize()
    assert cudart.cudaMemcpy(d_b, tb.data_ptr(), total * 8, d2d) == 0
    its, res, st = batch.device_solve(tol=1e-8, max_iter=5000, refine=True)
    assert np.all(st == 0)
    tx = torch.empty(total, dtype=torch.float64, device="cuda")
    assert cudart.cudaMemcpy(tx.data_ptr(), d_x, total * 8, d2d) == 0
    xh = tx.cpu().numpy()
    for o, sysm, b in zip(off, systems, bs):
        x = xh[int(o):int(o) + len(b)]
        assert true_resid(sysm, x, b) < 1.01e-8
    assert np.all(xh[int(off[0]) + 125:int(off[1])] == 0.0)  # padding rows stay zero
    batch.destroy()
