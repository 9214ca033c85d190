"""CPU baselines of the benchmark configurations: the oracle (the C++
restatement of the reference's FP64 solvers, built -O2 like the reference's
Makefile) timed on this host, wall clock around monolis_solve_R, for given
OpenMP thread counts (1 = the reference's default build, which has no OpenMP).

    python oracle/cpu_baselines.py --threads 1 8 [--only c1 c2 ...] [--out FILE]

Configurations (seeded synthetic inputs of monolis_b200.problems):
  c1  3D 7-point Laplacian 32^3, CG + DIAG, 1e-8
  c2  3D elasticity 128^3 nodes (ndof 3), CG + DIAG, 1e-8
  c3  convection-diffusion 256^3 at Peclet 0.5, 5, 50, BiCGSTAB + DIAG, 1e-8
  c4  the 512 batched FV diffusion systems one after another, CG + DIAG,
      1e-8 (the CPU has no batched form), and the 96^3 system with 32
      right-hand sides one after another
  c5  the adjoint workload: forward CG to 1e-10 and the adjoint solve (A is
      symmetric: the same solver) of 3D Q1 diffusion on 128^3 nodes
Prints one JSON object per configuration and thread count (seconds,
iterations) and appends it to --out when given. Long at full size: the
1-thread c2 solve takes about 17 minutes on an 8-core Xeon at 2.7 GHz.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from monolis_b200 import api, problems  # noqa: E402

SO = os.path.join(ROOT, "oracle", "_build", "libmonolis_oracle.so")


def solve(m, b, method, tol, maxiter=100000):
    m.quiet()
    m.set_error_abort(False)
    m.set_method(method)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(tol)
    m.set_maxiter(maxiter)
    x = np.zeros_like(b)
    t0 = time.perf_counter()
    m.solve(b, x)
    return time.perf_counter() - t0, m.get_converge_iter(), m.get_error_tag(), x


def run(lib, name):
    if name == "c1":
        m = api.Monolis(lib)
        b = problems.laplacian(m, n=32)
        t, it, st, _ = solve(m, b, api.ITER_CG, 1e-8)
        return {"s": t, "iterations": it, "status": st}
    if name == "c2":
        m = api.Monolis(lib)
        b = problems.elasticity(m, n=128)
        t, it, st, _ = solve(m, b, api.ITER_CG, 1e-8)
        return {"s": t, "iterations": it, "status": st}
    if name == "c3":
        out = {}
        for pe in (0.5, 5.0, 50.0):
            m = api.Monolis(lib)
            b = problems.convection_diffusion(m, n=256, peclet=pe)
            t, it, st, _ = solve(m, b, api.ITER_BICGSTAB, 1e-8)
            out[f"pe{pe:g}"] = {"s": t, "iterations": it, "status": st}
            m.finalize()
        return out
    if name == "c4":
        sides = problems.batch_sides(512)
        total, its, bad = 0.0, [], 0
        for i, s in enumerate(sides):
            ix, it_, v, _ = problems.fv_diffusion_csr(int(s), 4000 + i)
            b = problems.uniform(5000 + i, int(s) ** 3)
            m = api.Monolis(lib)
            n = len(ix) - 1
            m.set_matrix_BCSR(n, n, 1, len(it_), v, ix, it_)
            t, it, st, _ = solve(m, b, api.ITER_CG, 1e-8)
            total += t
            its.append(it)
            bad += st != 0
            m.finalize()
        ix, it_, v, _ = problems.fv_diffusion_csr(96, 4999)
        n = len(ix) - 1
        m = api.Monolis(lib)
        m.set_matrix_BCSR(n, n, 1, len(it_), v, ix, it_)
        t_rhs, its_rhs = 0.0, []
        for k in range(32):
            t, it, st, _ = solve(m, problems.uniform(6000 + k, n), api.ITER_CG, 1e-8)
            t_rhs += t
            its_rhs.append(it)
            bad += st != 0
        return {"many_systems_s": total, "many_systems_iterations_max": int(max(its)),
                "many_rhs_s": t_rhs, "many_rhs_iterations_max": int(max(its_rhs)), "failures": int(bad)}
    if name == "c5":
        m = api.Monolis(lib)
        b, _, _, _ = problems.diffusion_kappa(m, n=128)
        t1, it1, st1, x = solve(m, b, api.ITER_CG, 1e-10)
        target = problems.smooth_target(128)
        t2, it2, st2, _ = solve(m, np.ascontiguousarray(x - target), api.ITER_CG, 1e-10)
        return {"forward_s": t1, "forward_iterations": it1, "adjoint_s": t2, "adjoint_iterations": it2,
                "s": t1 + t2, "status": max(st1, st2)}
    raise ValueError(name)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, nargs="+", default=[1, os.cpu_count()])
    ap.add_argument("--only", nargs="*", default=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--out")
    args = ap.parse_args()
    lib = api.load_library(SO, oracle=True)
    for th in args.threads:
        lib.oracle_set_threads(th)
        for name in args.only:
            r = {"config": name, "threads": th, "host_cores": os.cpu_count(), **run(lib, name)}
            line = json.dumps(r)
            print(line, flush=True)
            if args.out:
                with open(args.out, "a") as f:
                    f.write(line + "\n")


if __name__ == "__main__":
    main()
