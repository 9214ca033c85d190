"""The multi-rank device path (halo updates through NCCL, dot products summed
by an NCCL all-reduce, scalar updates in a separate one-thread kernel) run
with a one-rank communicator: it must give exactly the bits and iteration
count of the single-rank solve, also past the true-residual replacement at
iteration 200. (Runs here have one GPU; more ranks cannot share it.)"""
import numpy as np
import pytest

from monolis_b200 import api
from monolis_b200 import partition
from helpers import bits_equal, build, solve

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("problem,kw", [("elasticity", dict(n=8)), ("elasticity", dict(n=24)),
                                        ("laplacian", dict(n=20))])
def test_sharded_path_one_rank_bit_identical(gpu, problem, kw):
    mp, b = build(gpu, problem, **kw)
    nd = mp.NDOF
    xp, itp, resp, stp = solve(mp, b, api.ITER_CG, api.PREC_DIAG, tol=1e-8)
    assert stp == 0
    p = partition.partition_rows(mp.csr_index(), mp.csr_item() - 1, mp.values(), nd, 1)[0]
    assert p["N"] == p["NP"] == mp.N
    ms = api.Monolis(gpu)
    ms.set_matrix_BCSR(p["N"], p["NP"], nd, len(p["item"]), p["val"], p["index"], p["item"])
    ms.quiet()
    ms.set_error_abort(False)
    ms.set_halo(p, 0, 1)
    ms.com_init_nccl(api.nccl_unique_id(gpu), 0, 1)
    xs, its, ress, sts = solve(ms, b, api.ITER_CG, api.PREC_DIAG, tol=1e-8)
    assert sts == 0
    assert its == itp and ress == resp
    assert bits_equal(xs, xp)
    if kw.get("n") == 24:
        assert itp > 200  # crosses the true-residual replacement
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
    _, _, _, st = solve(ms, b, api.ITER_BICGSTAB, api.PREC_DIAG)
    assert st == 5  # the multi-rank solve is FP64 CG
    ms.finalize()
