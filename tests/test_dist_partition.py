"""The multi-rank solve's host-side contract, checked on CPU with gloo ranks:
monolis_b200.partition builds rank-local systems and MONOLIS_COM halo tables
whose halo exchange (pack send_item -> neighbour -> unpack into recv_item)
and per-rank dot products, followed by the scalar updates the device code
applies (FP64 CG and BiCGSTAB with block-Jacobi: halo updates of the
multiplied vectors P, PT, ST and X, all-reduced sums for every dot),
reproduce the single-rank solve of the oracle: same solution, iteration
count within 2."""
import os
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle", "_build", "libmonolis_oracle.so")


def global_system(problem):
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from monolis_b200 import api
    from monolis_b200 import problems as P
    lib = api.load_library(ORACLE, oracle=True)
    m = api.Monolis(lib)
    if problem == "laplacian":
        b = P.laplacian(m, n=7)
    elif problem == "convection_diffusion":
        b = P.convection_diffusion(m, n=8, peclet=5.0)
    else:
        b = P.elasticity(m, n=5)
    return m, np.ascontiguousarray(b)


def local_matvec(p, nd, x):
    """y (owned rows) = A_local x (owned + ghost entries)."""
    n, ix, it, v = p["N"], p["index"], p["item"], p["val"].reshape(-1, nd, nd)
    y = np.zeros((n, nd))
    xb = x.reshape(-1, nd)
    for i in range(n):
        for k in range(ix[i], ix[i + 1]):
            y[i] += v[k] @ xb[it[k]]
    return y.reshape(-1)


def _worker(rank, world, port, problem, q, method="cg"):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        if ROOT not in sys.path:
            sys.path.insert(0, ROOT)
        from monolis_b200 import partition
        m, b = global_system(problem)
        nd = m.NDOF
        parts = partition.partition_rows(m.csr_index(), m.csr_item() - 1, m.values(), nd, world)
        p = parts[rank]
        n, npr = p["N"], p["NP"]
        bl = np.zeros(npr * nd)
        bl[:n * nd] = b[p["glob"][:n].repeat(nd) * nd + np.tile(np.arange(nd), n)]

        def halo(v):
            reqs, bufs = [], []
            for qd, s in enumerate(p["send_pe"]):
                items = p["send_item"][p["send_index"][qd]:p["send_index"][qd + 1]]
                buf = torch.from_numpy(np.ascontiguousarray(v.reshape(-1, nd)[items].reshape(-1)))
                reqs.append(dist.isend(buf, int(s)))
                bufs.append(buf)
            for qd, s in enumerate(p["recv_pe"]):
                items = p["recv_item"][p["recv_index"][qd]:p["recv_index"][qd + 1]]
                buf = torch.empty(len(items) * nd, dtype=torch.float64)
                dist.recv(buf, int(s))
                v.reshape(-1, nd)[items] = buf.numpy().reshape(-1, nd)
            for r_ in reqs:
                r_.wait()

        def gdot(a, c):
            t = torch.tensor([float(np.dot(a[:n * nd], c[:n * nd]))], dtype=torch.float64)
            dist.all_reduce(t)
            return t.item()

        # block-Jacobi factors of the owned diagonal blocks (inverse blocks)
        vb = p["val"].reshape(-1, nd, nd)
        dinv = np.zeros((n, nd, nd))
        for i in range(n):
            for k in range(p["index"][i], p["index"][i + 1]):
                if p["item"][k] == i:
                    dinv[i] = np.linalg.inv(vb[k])
        prec = lambda r_: np.einsum("iab,ib->ia", dinv, r_[:n * nd].reshape(n, nd)).reshape(-1)
        x = np.zeros(npr * nd)
        halo(x)
        r = bl[:n * nd] - local_matvec(p, nd, x)
        if method == "bicgstab":
            it = _bicgstab(r, x, p, nd, n, npr, halo, gdot, prec)
            q.put((rank, p["glob"][:n].tolist(), x[:n * nd].tolist(), it))
            return
        if method == "gropcg":
            it = _gropcg(r, x, p, nd, n, npr, halo, gdot, prec)
            q.put((rank, p["glob"][:n].tolist(), x[:n * nd].tolist(), it))
            return
        if method == "pipecg":
            it = _pipecg(r, x, bl, p, nd, n, npr, halo, gdot, prec)
            q.put((rank, p["glob"][:n].tolist(), x[:n * nd].tolist(), it))
            return
        z = prec(r)
        B2 = gdot(bl, bl)
        rho = gdot(r, z)
        pvec = np.zeros(npr * nd)
        it = 0
        while it < 5000:
            it += 1
            pvec[:n * nd] = z if it == 1 else z + (rho / rho_old) * pvec[:n * nd]
            halo(pvec)
            qv = local_matvec(p, nd, pvec)
            alpha = rho / gdot(pvec, qv)
            x[:n * nd] += alpha * pvec[:n * nd]
            r -= alpha * qv
            z = prec(r)
            rr = gdot(r, r)
            rho_old, rho = rho, gdot(r, z)
            if np.sqrt(rr / B2) < 1e-8:
                break
        q.put((rank, p["glob"][:n].tolist(), x[:n * nd].tolist(), it))
    finally:
        dist.destroy_process_group()


def _bicgstab(r, x, p, nd, n, npr, halo, gdot, prec):
    """BiCGSTAB of the device code's multi-rank plan (src/iterative/BiCGSTAB.f90:87-170):
    PT and ST get their ghost entries before each product; every dot is a
    local sum followed by an all-reduce. Returns the iteration count."""
    rt = r.copy()
    B2 = gdot(r, r)
    rho = gdot(r, rt)
    pv = np.zeros(n * nd)
    vv = np.zeros(n * nd)
    pt = np.zeros(npr * nd)
    st = np.zeros(npr * nd)
    alpha = omega = 1.0
    for it in range(1, 5000):
        if it == 1:
            pv = r.copy()
        else:
            beta = (rho / rho1) * (alpha / omega)
            pv = r + beta * (pv - omega * vv)
        pt[:n * nd] = prec(pv)
        halo(pt)
        vv = local_matvec(p, nd, pt)
        alpha = rho / gdot(rt, vv)
        s = r - alpha * vv
        st[:n * nd] = prec(s)
        halo(st)
        t = local_matvec(p, nd, st)
        ts, tt = gdot(t, s), gdot(t, t)
        omega = ts / tt if tt != 0.0 else 0.0
        x[:n * nd] += alpha * pt[:n * nd] + omega * st[:n * nd]
        r = s - omega * t
        rr = gdot(r, r)
        if np.sqrt(rr / B2) < 1e-8:
            return it
        rho1, rho = rho, gdot(r, rt)
    return 5000


def _pipecg(r, x, bl, p, nd, n, npr, halo, gdot, prec, iter_rr=50):
    """PipeCG of the device code's multi-rank plan (src/iterative/PipeCG.f90:67-149):
    U and M get their ghost entries before their products; <R,U> and <V,U>
    are all-reduced together (on the device, while L = A M runs), <R,R> for
    the convergence check. Returns the iteration count."""
    B2 = gdot(r, r)
    u = np.zeros(npr * nd)
    u[:n * nd] = prec(r)
    halo(u)
    v = local_matvec(p, nd, u)
    m = np.zeros(npr * nd)
    z, qv, s, pv = (np.zeros(n * nd) for _ in range(4))
    gamma, alpha = 1.0, 1.0
    for it in range(1, 5000):
        g, d = gdot(r, u), gdot(v, u)
        m[:n * nd] = prec(v)
        halo(m)
        l = local_matvec(p, nd, m)
        gamma1, alpha1 = 1.0 / gamma, 1.0 / alpha
        gamma, delta = g, d
        if it > 1:
            beta = gamma * gamma1
            alpha = gamma / (delta - beta * gamma * alpha1)
        else:
            alpha, beta = gamma / delta, 0.0
        z = beta * z + l
        qv = beta * qv + m[:n * nd]
        s = beta * s + v
        pv = beta * pv + u[:n * nd]
        if it % iter_rr == 0:
            x[:n * nd] += alpha * pv
            halo(x)
            r = bl[:n * nd] - local_matvec(p, nd, x)
            u[:n * nd] = prec(r)
            halo(u)
            v = local_matvec(p, nd, u)
        else:
            r = r - alpha * s
            u[:n * nd] = u[:n * nd] - alpha * qv
            v = v - alpha * z
            x[:n * nd] += alpha * pv
        if np.sqrt(gdot(r, r) / B2) < 1e-8:
            return it
    return 5000


def _gropcg(r, x, p, nd, n, npr, halo, gdot, prec):
    """GropCG of the device code's multi-rank plan (src/iterative/GropCG.f90:80-125):
    U gets its ghost entries before V = A U, while <R,U> and <R,R> are
    all-reduced; delta = <P,S> all-reduced before alpha. Returns the
    iteration count."""
    B2 = gdot(r, r)
    u = np.zeros(npr * nd)
    u[:n * nd] = prec(r)
    pv = u[:n * nd].copy()
    halo(u)
    s = local_matvec(p, nd, u)
    gamma = gdot(r, u)
    for it in range(1, 5000):
        delta = gdot(pv, s)
        qv = prec(s)
        alpha = gamma / delta
        x[:n * nd] += alpha * pv
        r = r - alpha * s
        u[:n * nd] = u[:n * nd] - alpha * qv
        gamma1, rr = gdot(r, u), gdot(r, r)
        halo(u)
        v = local_matvec(p, nd, u)
        beta = gamma1 / gamma
        gamma = gamma1
        pv = beta * pv + u[:n * nd]
        s = beta * s + v
        if np.sqrt(rr / B2) < 1e-8:
            return it
    return 5000


@pytest.mark.parametrize("problem,world,method", [("laplacian", 2, "pipecg"), ("elasticity", 3, "pipecg"),
                                                  ("laplacian", 3, "gropcg"), ("elasticity", 2, "gropcg")])
def test_partitioned_pipelined_cg_matches_single_rank(problem, world, method, oracle):
    from monolis_b200 import api
    from helpers import solve
    mth = api.ITER_PIPECG if method == "pipecg" else api.ITER_GROPCG
    m, b = global_system(problem)
    nd = m.NDOF
    x_ref, it_ref, _, st = solve(m, b, mth, api.PREC_DIAG, tol=1e-8)
    assert st == 0
    out = _run_ranks(problem, world, method, 33900 + (os.getpid() % 2000) + 13 * world + (7 if method == "gropcg" else 0))
    x = np.zeros_like(b)
    its = set()
    for rank, glob, xl, it in out:
        glob = np.array(glob)
        x[(glob[:, None] * nd + np.arange(nd)).reshape(-1)] = xl
        its.add(it)
    assert len(its) == 1
    assert abs(its.pop() - it_ref) <= 2
    x_tight, _, _, _ = solve(m, b, mth, api.PREC_DIAG, tol=1e-12)
    assert np.linalg.norm(x - x_tight) / np.linalg.norm(x_tight) < 1e-6


def _run_ranks(problem, world, method, port):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_worker, args=(r, world, port, problem, q, method)) for r in range(world)]
    for p_ in procs:
        p_.start()
    out = [q.get(timeout=180) for _ in range(world)]
    for p_ in procs:
        p_.join(timeout=60)
        assert p_.exitcode == 0
    return out


@pytest.mark.parametrize("world", [2, 3])
def test_partitioned_bicgstab_matches_single_rank(world, oracle):
    from monolis_b200 import api
    from helpers import solve
    m, b = global_system("convection_diffusion")
    x_ref, it_ref, _, st = solve(m, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-8)
    assert st == 0
    out = _run_ranks("convection_diffusion", world, "bicgstab", 32700 + (os.getpid() % 2000) + 11 * world)
    x = np.zeros_like(b)
    its = set()
    for rank, glob, xl, it in out:
        x[np.array(glob)] = xl
        its.add(it)
    assert len(its) == 1  # every rank stops at the same iteration
    assert abs(its.pop() - it_ref) <= 2
    x_tight, _, _, _ = solve(m, b, api.ITER_BICGSTAB, api.PREC_DIAG, tol=1e-12)
    assert np.linalg.norm(x - x_tight) / np.linalg.norm(x_tight) < 1e-6


@pytest.mark.parametrize("problem,world", [("laplacian", 2), ("laplacian", 3), ("elasticity", 2)])
def test_partitioned_cg_matches_single_rank(problem, world, oracle):
    from monolis_b200 import api
    from helpers import solve
    m, b = global_system(problem)
    nd = m.NDOF
    x_ref, it_ref, _, st = solve(m, b, api.ITER_CG, api.PREC_DIAG, tol=1e-8)
    assert st == 0
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + (os.getpid() % 2000) + 7 * world
    procs = [ctx.Process(target=_worker, args=(r, world, port, problem, q)) for r in range(world)]
    for p_ in procs:
        p_.start()
    out = [q.get(timeout=180) for _ in range(world)]
    for p_ in procs:
        p_.join(timeout=60)
        assert p_.exitcode == 0
    x = np.zeros_like(b)
    its = set()
    for rank, glob, xl, it in out:
        glob = np.array(glob)
        x[(glob[:, None] * nd + np.arange(nd)).reshape(-1)] = xl
        its.add(it)
    assert len(its) == 1  # every rank stops at the same iteration
    assert abs(its.pop() - it_ref) <= 2
    x_tight, _, _, _ = solve(m, b, api.ITER_CG, api.PREC_DIAG, tol=1e-12)
    assert np.linalg.norm(x - x_tight) / np.linalg.norm(x_tight) < 1e-6


def test_partition_tables_are_consistent():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from monolis_b200 import partition
    m, b = global_system("laplacian")
    parts = partition.partition_rows(m.csr_index(), m.csr_item() - 1, m.values(), 1, 4)
    assert sum(p["N"] for p in parts) == m.N
    for r, p in enumerate(parts):
        # what r receives from s is exactly what s sends to r, in the same order
        for qd, s in enumerate(p["recv_pe"]):
            recv_glob = p["glob"][p["recv_item"][p["recv_index"][qd]:p["recv_index"][qd + 1]]]
            ps = parts[s]
            k = list(ps["send_pe"]).index(r)
            send_glob = ps["glob"][ps["send_item"][ps["send_index"][k]:ps["send_index"][k + 1]]]
            assert np.array_equal(recv_glob, send_glob)
        assert np.all(p["item"] < p["NP"])


@pytest.mark.parametrize("problem,nd,world", [("laplacian", 1, 4), ("laplacian", 1, 3), ("elasticity", 3, 2),
                                              ("elasticity", 3, 5)])
def test_partition_rank_matches_partition_rows(problem, nd, world):
    """The vectorised one-rank partitioner (used for the 56 M-block headline
    system) gives exactly the arrays of the row-by-row one for every rank."""
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from monolis_b200 import partition
    m, b = global_system(problem)
    args = (m.csr_index(), m.csr_item() - 1, m.values(), nd, world)
    parts = partition.partition_rows(*args)
    for r in range(world):
        q = partition.partition_rank(*args, r)
        p = parts[r]
        for k in ("N", "NP", "lo", "hi"):
            assert p[k] == q[k], k
        for k in ("glob", "index", "item", "val", "recv_pe", "recv_index", "recv_item", "send_pe", "send_index",
                  "send_item"):
            assert np.array_equal(np.asarray(p[k]), np.asarray(q[k])), k
            if k != "val" and k != "glob":
                assert np.asarray(q[k]).dtype == np.int32, k
