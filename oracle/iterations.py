"""Records the oracle's iteration counts and final residuals at full benchmark
sizes into tests/golden/oracle_iterations.json (test fixture and the
extrapolation count of the CPU baseline).

    python oracle/iterations.py [--threads T] [--only KEY ...]

Runs the CPU oracle (oracle/_build/libmonolis_oracle.so); long at full size
(minutes per system on a few cores). Keys: <problem>_n<size>[_pe<P>]_<method>_<prec>_tol<tol>.

--spread runs each case with 2, 4 and 8 OpenMP threads instead (three more
summation orders of every dot product) and stores the counts under
"<key>:by_threads": how far the iteration count moves when only the
summation order changes.

--dot-mode n128 runs the oracle with every dot product summed in
double-double (the arithmetic of the reference's pseudo-quadruple inner
product, src/linalg/inner_product.f90:219-258, which the product library's
FP64 kernels use) and stores the results under "<key>:n128...": the
iteration count, the thread counts it was reproduced with (--spread), and
a strided sample of the solution ("<key>:n128:x_sample", every
--sample-stride-th entry, first entry at 0).
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

OUT = os.path.join(ROOT, "tests", "golden", "oracle_iterations.json")
SO = os.path.join(ROOT, "oracle", "_build", "libmonolis_oracle.so")

CASES = {
    "laplacian_n32_cg_diag_tol1e-08": (problems.laplacian, dict(n=32), api.ITER_CG, 1e-8),
    "elasticity_n128_cg_diag_tol1e-08": (problems.elasticity, dict(n=128), api.ITER_CG, 1e-8),
    "diffusion_kappa_n128_cg_diag_tol1e-10": (problems.diffusion_kappa, dict(n=128), api.ITER_CG, 1e-10),
    "convection_diffusion_n256_pe0.5_bicgstab_diag_tol1e-08":
        (problems.convection_diffusion, dict(n=256, peclet=0.5), api.ITER_BICGSTAB, 1e-8),
    "convection_diffusion_n256_pe5_bicgstab_diag_tol1e-08":
        (problems.convection_diffusion, dict(n=256, peclet=5.0), api.ITER_BICGSTAB, 1e-8),
    "convection_diffusion_n256_pe50_bicgstab_diag_tol1e-08":
        (problems.convection_diffusion, dict(n=256, peclet=50.0), api.ITER_BICGSTAB, 1e-8),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--only", nargs="*")
    ap.add_argument("--spread", action="store_true")
    ap.add_argument("--dot-mode", choices=("reference", "n128"), default="reference")
    ap.add_argument("--sample-stride", type=int, default=0)
    args = ap.parse_args()
    lib = api.load_library(SO, oracle=True)
    lib.oracle_set_threads(args.threads)
    n128 = args.dot_mode == "n128"
    lib.oracle_set_dot_mode(1 if n128 else 0)
    sfx = ":n128" if n128 else ""
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    for key, (fn, kw, method, tol) in CASES.items():
        if args.only and key not in args.only:
            continue
        if args.spread:
            counts = {}
            for th in (2, 4, 8):
                lib.oracle_set_threads(th)
                m = api.Monolis(lib)
                b = fn(m, **kw)
                if isinstance(b, tuple):
                    b = b[0]
                m.quiet()
                m.set_error_abort(False)
                m.set_method(method)
                m.set_precond(api.PREC_DIAG)
                m.set_tolerance(tol)
                m.set_maxiter(100000)
                x = np.zeros_like(b)
                m.solve(b, x)
                counts[str(th)] = m.get_converge_iter()
                m.finalize()
                print(key, th, counts[str(th)], flush=True)
            data[key + sfx + ":by_threads"] = counts
            with open(OUT, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
            continue
        m = api.Monolis(lib)
        b = fn(m, **kw)
        if isinstance(b, tuple):
            b = b[0]
        m.quiet()
        m.set_error_abort(False)
        m.set_method(method)
        m.set_precond(api.PREC_DIAG)
        m.set_tolerance(tol)
        m.set_maxiter(100000)
        x = np.zeros_like(b)
        t0 = time.time()
        m.solve(b, x)
        dt = time.time() - t0
        k = key + sfx
        data[k] = m.get_converge_iter()
        data[k + ":residual"] = m.get_converge_residual()
        data[k + ":status"] = m.get_error_tag()
        data[k + ":threads"] = args.threads
        data[k + ":seconds"] = round(dt, 1)
        if args.sample_stride > 0:
            data[k + ":x_stride"] = args.sample_stride
            data[k + ":x_sample"] = [float(v) for v in x[::args.sample_stride]]
            data[k + ":x_norm"] = float(np.linalg.norm(x))
        print(k, data[k], data[k + ":residual"], f"{dt:.0f}s", flush=True)
        m.finalize()
        with open(OUT, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
