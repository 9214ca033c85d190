"""The multi-rank device path (halo updates through NCCL, dot products summed
by an NCCL all-reduce, scalar updates in separate one-thread kernels), FP64
CG, GropCG, PipeCG and BiCGSTAB and FP32-refined CG and BiCGSTAB, run with a
one-rank communicator: it must give exactly the
bits and iteration count of the single-rank solve, also past the
true-residual replacement at iteration 200. (Runs here have one GPU; more
ranks cannot share it.)"""
import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import partition
from helpers import bits_equal, build, solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("problem,kw,method,rr", [
    ("elasticity", dict(n=8), api.ITER_CG, 0),
    ("elasticity", dict(n=24), api.ITER_CG, 0),
    ("laplacian", dict(n=20), api.ITER_CG, 0),
    ("convection_diffusion", dict(n=16, peclet=5.0), api.ITER_BICGSTAB, 0),
    ("convection_diffusion", dict(n=16, peclet=0.5), api.ITER_BICGSTAB, 7),
    ("laplacian", dict(n=24), api.ITER_BICGSTAB, 5),
    ("elasticity", dict(n=10), api.ITER_BICGSTAB, 0),
    ("elasticity", dict(n=12), api.ITER_PIPECG, 0),
    ("laplacian", dict(n=20), api.ITER_PIPECG, 9),
    ("elasticity", dict(n=12), api.ITER_GROPCG, 0),
    ("convection_diffusion", dict(n=16, peclet=50.0), api.ITER_BICGSTAB_N128, 0),
])
def test_sharded_path_one_rank_bit_identical(gpu, problem, kw, method, rr):
    """rr > 0: true residual every rr iterations (instead of 200), so the
    replacement step of the multi-rank plan runs several times."""
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    mp.Iarray[api.B200_PRM_I_ITER_RR] = rr
    xp, itp, resp, stp = solve(mp, b, method, api.PREC_DIAG, tol=1e-8)
    assert stp == 0
    p = partition.partition_rows(mp.csr_index(), mp.csr_item() - 1, mp.values(), nd, 1)[0]
    assert p["N"] == p["NP"] == mp.N
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(p["N"], p["NP"], nd, len(p["item"]), p["val"], p["index"], p["item"])
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(p, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    ms.Iarray[api.B200_PRM_I_ITER_RR] = rr
    xs, its, ress, sts = solve(ms, b, method, api.PREC_DIAG, tol=1e-8)
    assert sts == 0
    assert its == itp and ress == resp
    assert bits_equal(xs, xp)
    if problem == "elasticity" and kw.get("n") == 24:
        assert itp > 200  # crosses the true-residual replacement
    if rr:
        assert itp > 2 * rr
    ms.finalize()


def test_sharded_path_rejects_unsupported(gpu):
    mp, b = build(gpu, "laplacian", n=6)
    p = partition.partition_rows(mp.csr_index(), mp.csr_item() - 1, mp.values(), 1, 1)[0]
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(p["N"], p["NP"], 1, len(p["item"]), p["val"], p["index"], p["item"])
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(p, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    _, _, _, st = solve(ms, b, api.ITER_PIPECG, api.PREC_DIAG, precision=1)
    assert st == 5  # the FP32-refined form is CG and BiCGSTAB only
    ms.finalize()


@pytest.mark.parametrize("problem,kw,method", [
    ("laplacian", dict(n=14), api.ITER_CG),
    ("elasticity", dict(n=7), api.ITER_CG),
    ("convection_diffusion", dict(n=14, peclet=5.0), api.ITER_BICGSTAB),
    ("laplacian", dict(n=14), api.ITER_PIPECG),
    ("elasticity", dict(n=7), api.ITER_GROPCG),
])
def test_sharded_boundary_rows_through_self_halo(gpu, problem, kw, method):
    """A one-rank system whose rows read some columns through ghost entries:
    every 7th node gets a ghost copy, filled by a halo list the rank sends to
    itself. The rows that read a ghost form the boundary slices, multiplied
    after the halo update while the interior slices run beside it; the
    solution must match the plain solve (the rows' sums run in a different
    order, so to the solver tolerance, not bit for bit)."""
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    N = mp.N
    x_ref, it_ref, _, st = solve(mp, b, method, api.PREC_DIAG, tol=1e-12)
    assert st == 0
    index = mp.csr_index().astype(np.int64)
    item = (mp.csr_item() - 1).astype(np.int64)
    val = mp.values().reshape(-1, nd * nd)
    mirrored = np.arange(3, N, 7)
    ghost = np.full(N, -1, dtype=np.int64)
    ghost[mirrored] = N + np.arange(len(mirrored))
    NP = N + len(mirrored)
    new_index, new_item, new_val = [0], [], []
    for i in range(N):
        cols = item[index[i]:index[i + 1]]
        cols2 = np.where((ghost[cols] >= 0) & (cols != i), ghost[cols], cols)
        order = np.argsort(cols2, kind="stable")
        new_item.extend(cols2[order].tolist())
        new_val.append(val[index[i]:index[i + 1]][order])
        new_index.append(len(new_item))
    new_index += [new_index[-1]] * (NP - N)  # ghost rows hold no blocks
    new_val = np.concatenate(new_val).reshape(-1)
    assert any(c >= N for c in new_item)
    halo = {"N": N, "recv_pe": [0], "recv_index": [0, len(mirrored)], "recv_item": np.arange(N, NP),
            "send_pe": [0], "send_index": [0, len(mirrored)], "send_item": mirrored}
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(N, NP, nd, len(new_item), new_val, np.array(new_index, dtype=np.int32),
                       np.array(new_item, dtype=np.int32))
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(halo, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    bl = np.zeros(NP * nd)
    bl[:N * nd] = b
    xs, its, _, sts = solve(ms, bl, method, api.PREC_DIAG, tol=1e-12)
    assert sts == 0
    assert abs(its - it_ref) <= 2, (its, it_ref)
    assert np.linalg.norm(xs[:N * nd] - x_ref) / np.linalg.norm(x_ref) < 1e-9
    # the solve ends with the ghost entries of x updated from their owners
    # (src/iterative/CG.f90:105 and the other solvers' last step)
    assert bits_equal(xs[N * nd:].reshape(-1, nd), xs[:N * nd].reshape(-1, nd)[mirrored])
    ms.finalize()


@pytest.mark.parametrize("problem,kw,method", [
    ("elasticity", dict(n=10), api.ITER_CG),
    ("convection_diffusion", dict(n=16, peclet=5.0), api.ITER_BICGSTAB),
])
def test_device_solve_com_one_rank(gpu, problem, kw, method):
    """monolis_b200_device_solve_com_R (device b and x, multi-rank plan through
    a one-rank NCCL communicator) gives the bits of the plain device solve;
    without a communicator it is the plain device solve."""
    import torch
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    mp.set_method(method)
    mp.set_precond(api.PREC_DIAG)
    mp.set_tolerance(1e-8)
    mp.set_matrix_cache(True)
    mp.device_prepare()
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros_like(d_b)
    assert mp.device_solve(d_b.data_ptr(), d_x.data_ptr()) == 0
    x_ref, it_ref = d_x.cpu().numpy(), mp.get_converge_iter()
    d_x.zero_()
    assert mp.device_solve_com(d_b.data_ptr(), d_x.data_ptr()) == 0  # no communicator attached
    assert bits_equal(d_x.cpu().numpy(), x_ref)
    p = partition.partition_rank(mp.csr_index(), mp.csr_item() - 1, mp.values(), nd, 1, 0)
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(p["N"], p["NP"], nd, len(p["item"]), p["val"], p["index"], p["item"])
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_method(method)
    ms.set_precond(api.PREC_DIAG)
    ms.set_tolerance(1e-8)
    ms.set_matrix_cache(True)
    ms.set_halo(p, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    ms.device_prepare()
    d_x2 = torch.zeros_like(d_b)
    assert ms.device_solve_com(d_b.data_ptr(), d_x2.data_ptr()) == 0
    assert ms.get_converge_iter() == it_ref
    assert bits_equal(d_x2.cpu().numpy(), x_ref)
    ms.finalize()


@pytest.mark.parametrize("problem,kw,tol", [
    ("elasticity", dict(n=12), 1e-8),
    ("laplacian", dict(n=20), 1e-10),
    ("diffusion_kappa", dict(n=10), 1e-9),
])
def test_sharded_mixed_cg_one_rank_bit_identical(gpu, problem, kw, tol):
    """The multi-rank FP32-refined CG (FP32 halo update of p, all-reduced dot
    products, the refresh's all-reduce in every iteration, y and x kept on
    the ghost rows) through a one-rank NCCL communicator: the iteration
    count, residual, refresh count and solution bits of the plain refined
    solve."""
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    xp, itp, resp, stp = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=tol, precision=1)
    assert stp == 0 and resp < tol
    nref = mp.Iarray[api.B200_PRM_I_N_REFINE]
    p = partition.partition_rank(mp.csr_index(), mp.csr_item() - 1, mp.values(), nd, 1, 0)
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(p["N"], p["NP"], nd, len(p["item"]), p["val"], p["index"], p["item"])
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(p, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    xs, its, ress, sts = solve(ms, b, api.ITER_CG, api.PREC_DIAG, tol=tol, precision=1)
    assert sts == 0
    assert its == itp and ress == resp and ms.Iarray[api.B200_PRM_I_N_REFINE] == nref
    assert bits_equal(xs, xp)
    ms.finalize()


@pytest.mark.parametrize("problem,kw,tol", [
    ("convection_diffusion", dict(n=16, peclet=5.0), 1e-8),
    ("convection_diffusion", dict(n=20, peclet=50.0), 1e-9),
    ("laplacian", dict(n=18), 1e-10),
    ("elasticity", dict(n=9), 1e-8),
])
def test_sharded_mixed_bicgstab_one_rank_bit_identical(gpu, problem, kw, tol):
    """The multi-rank FP32-refined BiCGSTAB (FP32 halo updates of PT and ST,
    all-reduced dot products, the refresh's all-reduce in every iteration,
    y and x kept on the ghost rows) through a one-rank NCCL communicator:
    the iteration count, residual, refresh count and solution bits of the
    plain refined solve."""
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    xp, itp, resp, stp = solve(mp, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=tol, precision=1)
    assert stp == 0 and resp < tol
    nref = mp.Iarray[api.B200_PRM_I_N_REFINE]
    assert nref >= 1
    p = partition.partition_rank(mp.csr_index(), mp.csr_item() - 1, mp.values(), nd, 1, 0)
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(p["N"], p["NP"], nd, len(p["item"]), p["val"], p["index"], p["item"])
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(p, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    xs, its, ress, sts = solve(ms, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=tol, precision=1)
    assert sts == 0
    assert its == itp and ress == resp and ms.Iarray[api.B200_PRM_I_N_REFINE] == nref
    assert bits_equal(xs, xp)
    ms.finalize()


def _mirrored_system(mp, every=7, first=3):
    """The system of mp with the columns of every `every`-th node (from
    `first`) read through a ghost copy filled by a one-rank self-exchange:
    (N, NP, index, item, val, halo, mirrored)."""
    nd = mp.NDOF
    N = mp.N
    index = mp.csr_index().astype(np.int64)
    item = (mp.csr_item() - 1).astype(np.int64)
    val = mp.values().reshape(-1, nd * nd)
    mirrored = np.arange(first, N, every)
    ghost = np.full(N, -1, dtype=np.int64)
    ghost[mirrored] = N + np.arange(len(mirrored))
    NP = N + len(mirrored)
    new_index, new_item, new_val = [0], [], []
    for i in range(N):
        cols = item[index[i]:index[i + 1]]
        cols2 = np.where((ghost[cols] >= 0) & (cols != i), ghost[cols], cols)
        order = np.argsort(cols2, kind="stable")
        new_item.extend(cols2[order].tolist())
        new_val.append(val[index[i]:index[i + 1]][order])
        new_index.append(len(new_item))
    new_index += [new_index[-1]] * (NP - N)
    new_val = np.concatenate(new_val).reshape(-1)
    halo = {"N": N, "recv_pe": [0], "recv_index": [0, len(mirrored)], "recv_item": np.arange(N, NP),
            "send_pe": [0], "send_index": [0, len(mirrored)], "send_item": mirrored}
    return (N, NP, np.array(new_index, dtype=np.int32), np.array(new_item, dtype=np.int32), new_val, halo,
            mirrored)


@pytest.mark.parametrize("problem,kw", [("convection_diffusion", dict(n=14, peclet=5.0)),
                                        ("laplacian", dict(n=14))])
def test_sharded_mixed_bicgstab_through_self_halo(gpu, problem, kw):
    """FP32-refined BiCGSTAB on a one-rank system whose rows read every 7th
    node through a ghost copy (filled by a self-exchange): PT and ST cross
    the halo in FP32, the FP64 refreshes multiply x + y on the ghost rows,
    which the solver keeps with the owners' arithmetic; the solution reaches
    the tolerance on the FP64 residual of the original system and matches
    the plain refined solve to it."""
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    tol = 1e-9
    x_ref, it_ref, _, st = solve(mp, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=tol, precision=1)
    assert st == 0
    N, NP, index, item, val, halo, mirrored = _mirrored_system(mp)
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(N, NP, nd, len(item), val, index, item)
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(halo, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    bl = np.zeros(NP * nd)
    bl[:N * nd] = b
    xs, its, ress, sts = solve(ms, bl, api.ITER_BICGSTAB, api.PREC_DIAG, tol=tol, precision=1)
    assert sts == 0 and ress < tol
    assert ms.Iarray[api.B200_PRM_I_N_REFINE] >= 1
    x = xs[:N * nd]
    assert np.linalg.norm(b - mp.matvec(x)) / np.linalg.norm(b) < 1.01 * tol
    assert abs(its - it_ref) <= max(5, it_ref // 5), (its, it_ref)
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-6
    assert bits_equal(xs[N * nd:].reshape(-1, nd), xs[:N * nd].reshape(-1, nd)[mirrored])
    ms.finalize()


@pytest.mark.parametrize("problem,kw", [("laplacian", dict(n=14)), ("elasticity", dict(n=7))])
def test_sharded_mixed_cg_through_self_halo(gpu, problem, kw):
    """FP32-refined CG on a one-rank system whose rows read every 7th node
    through a ghost copy (filled by a self-exchange): the FP64 refreshes
    multiply x + y on the ghost rows, which the solver keeps with the owners'
    arithmetic; the solution reaches the tolerance on the FP64 residual of
    the original system and matches the plain refined solve to it."""
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    N = mp.N
    tol = 1e-10
    x_ref, it_ref, _, st = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=tol, precision=1)
    assert st == 0
    index = mp.csr_index().astype(np.int64)
    item = (mp.csr_item() - 1).astype(np.int64)
    val = mp.values().reshape(-1, nd * nd)
    mirrored = np.arange(3, N, 7)
    ghost = np.full(N, -1, dtype=np.int64)
    ghost[mirrored] = N + np.arange(len(mirrored))
    NP = N + len(mirrored)
    new_index, new_item, new_val = [0], [], []
    for i in range(N):
        cols = item[index[i]:index[i + 1]]
        cols2 = np.where((ghost[cols] >= 0) & (cols != i), ghost[cols], cols)
        order = np.argsort(cols2, kind="stable")
        new_item.extend(cols2[order].tolist())
        new_val.append(val[index[i]:index[i + 1]][order])
        new_index.append(len(new_item))
    new_index += [new_index[-1]] * (NP - N)
    new_val = np.concatenate(new_val).reshape(-1)
    halo = {"N": N, "recv_pe": [0], "recv_index": [0, len(mirrored)], "recv_item": np.arange(N, NP),
            "send_pe": [0], "send_index": [0, len(mirrored)], "send_item": mirrored}
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(N, NP, nd, len(new_item), new_val, np.array(new_index, dtype=np.int32),
                       np.array(new_item, dtype=np.int32))
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(halo, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    bl = np.zeros(NP * nd)
    bl[:N * nd] = b
    xs, its, ress, sts = solve(ms, bl, api.ITER_CG, api.PREC_DIAG, tol=tol, precision=1)
    assert sts == 0 and ress < tol
    assert ms.Iarray[api.B200_PRM_I_N_REFINE] >= 1
    x = xs[:N * nd]
    # the FP64 residual of the original (unmirrored) system
    assert np.linalg.norm(b - mp.matvec(x)) / np.linalg.norm(b) < 1.01 * tol
    assert abs(its - it_ref) <= max(3, it_ref // 10), (its, it_ref)
    assert np.linalg.norm(x - x_ref) / np.linalg.norm(x_ref) < 1e-7
    # the solve ends with the ghost entries of x updated from their owners
    assert bits_equal(xs[N * nd:].reshape(-1, nd), xs[:N * nd].reshape(-1, nd)[mirrored])
    ms.finalize()
