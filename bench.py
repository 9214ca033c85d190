"""Benchmark: time to relative residual 1e-8 on 3D linear elasticity, 128^3 nodes.

Workload (one step = one full solve): 3D linear elasticity on a 128^3-node
structured hex8 mesh (E = 1, nu = 0.3, face x = 0 clamped, body force with a
seeded perturbation), block CSR with ndof = 3 (2,097,152 block rows,
55,742,968 3x3 blocks), CG + DIAG (3x3 block Jacobi), relative residual
sqrt(<r,r>/<r0,r0>) < 1e-8. Inputs are synthetic (monolis_b200.problems).

Our arm (one GPU): headline `value` = the plain FP64 CG (the reference's
arithmetic) with b and x resident in HBM, mean over the timed solves; `e2e` =
the same FP64 solve through monolis_solve_R with pinned host b/x, which
includes uploading the matrix (the library re-uploads by default), mean over
the calls. Beside them: the FP32-inner / FP64-refined CG (`mixed`,
`speedup_mixed_vs_fp64`), in-solve kernel times and the roofline of the
dominant kernel, standalone SpMV figures, a bounded CPU-baseline sample and
the secondary workloads (C3 BiCGSTAB, C4 batched / many right-hand sides, C5
adjoint).
`--impl reference`: the CPU oracle (restatement of the reference's FP64 CG)
on every host core: one complete solve to 1e-8, measured whole and cut into
`steps` consecutive iteration ranges by its per-iteration clock.
Several GPUs: the system row-partitioned over the ranks (NCCL halo updates
and all-reduced dot products, strong scaling, max over ranks); --replicas
runs independent copies instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

# OpenMP threads of the host assembly and of the CPU baseline sleep between
# parallel regions instead of spinning, so they do not take the cores the
# solver's host loop (graph launches, state reads) runs on. Set before any
# library that links the OpenMP runtime is loaded.
os.environ.setdefault("OMP_WAIT_POLICY", "PASSIVE")

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from monolis_b200 import api, problems  # noqa: E402

ORACLE_SO = os.path.join(ROOT, "oracle", "_build", "libmonolis_oracle.so")
FIXTURE = os.path.join(ROOT, "tests", "golden", "oracle_iterations.json")
def metric_name(n):
    """The headline metric, shared by both arms (the arithmetic is in `dtype`)."""
    return f"time to rel.res 1e-8, block-CSR CG (3D elasticity {n}^3 nodes, ndof=3)"


def workload_name(n, nz):
    return (f"3D linear elasticity {n}^3 nodes, hex8 Q1, E=1 nu=0.3, ndof=3, {nz} 3x3 blocks, "
            f"CG + 3x3 block-Jacobi, rel.res 1e-8")
TOL = 1e-8
# DRAM bytes (read + write) per launch of the FP64 cg_spmv_kernel divided by
# its layout bytes, from the ncu --set full capture at 64^3 nodes
# (527.12 MB / 522.13 MB); traffic scales with the blocks processed.
NCU_SPMV64_TRAFFIC_RATIO = 1.0096
NCU_SPMV64_TRAFFIC_SOURCE = ("ncu --set full capture of cg_spmv_kernel<3,3,double> at 64^3 nodes (dram read+write "
                             "527.12 MB / layout bytes 522.13 MB = 1.0096), scaled by the layout bytes of a 128^3 "
                             "launch")


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": 0}
        busy = [s for s in sm if s > 0.5 * (smax or max(sm))] or sm
        return {"sm_mhz": float(np.median(busy)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def max_over_ranks(v, world, device="cuda"):
    """The slowest rank's value (all ranks take part in the collective)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.item()


def fixture():
    try:
        with open(FIXTURE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def oracle_iterations(n):
    return fixture().get(f"elasticity_n{n}_cg_diag_tol1e-08")


def device_solve_timed(m, stream, d_b, d_x):
    """One device-resident solve timed with CUDA events on the library stream."""
    import torch
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    rc = m.device_solve(d_b.data_ptr(), d_x.data_ptr())
    e1.record(stream)
    e1.synchronize()
    if rc != 0:
        raise RuntimeError(f"solve failed: {api.STATUS_NAMES.get(rc, rc)}")
    return e0.elapsed_time(e1) * 1e-3


def kernel_times(m, stream, d_b, d_x):
    """Per-kernel average seconds of one solve in the library's kernel-timer
    mode (every kernel bracketed by CUDA events on the library stream)."""
    m.Iarray[api.B200_PRM_I_KERNEL_TIMERS] = 1
    try:
        device_solve_timed(m, stream, d_b, d_x)
    finally:
        m.Iarray[api.B200_PRM_I_KERNEL_TIMERS] = 0
    it = max(m.get_converge_iter(), 1)
    return [m.Rarray[api.B200_PRM_R_TIME_KERNEL + k] / it for k in range(8)], it


def workload_c1(lib, args):
    """The reference's CPU-runnable configuration: 3D 7-point Laplacian 32^3,
    CG + DIAG to 1e-8, FP64 and FP32-refined, device-resident b and x (five
    timed solves after one untimed)."""
    import torch
    m = api.Monolis(lib)
    b = problems.laplacian(m, n=32)
    m.quiet()
    m.set_error_abort(False)
    m.set_method(api.ITER_CG)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(TOL)
    m.set_maxiter(10000)
    m.set_matrix_cache(True)
    stream = torch.cuda.ExternalStream(api.stream_handle(lib))
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros_like(d_b)
    out = {"workload": "3D 7-point Laplacian 32^3 (32,768 unknowns), CG + DIAG, rel.res 1e-8",
           "oracle_iterations": fixture().get("laplacian_n32_cg_diag_tol1e-08")}
    for prec, name in ((0, "fp64"), (1, "mixed")):
        m.set_precision(prec)
        m.device_prepare()
        device_solve_timed(m, stream, d_b, d_x)
        ts = [device_solve_timed(m, stream, d_b, d_x) for _ in range(5)]
        out[name] = {"s": float(np.median(ts)), "s_each": ts, "iterations": m.get_converge_iter(),
                     "rel_residual": m.get_converge_residual()}
    m.finalize()
    return out


def workload_c3(lib, args, peak):
    """Nonsymmetric 7-point upwind convection-diffusion, 256^3 unknowns,
    BiCGSTAB + DIAG to 1e-8: FP64 and FP32-refined, three cell Peclet numbers."""
    import torch
    fx = fixture()
    out = {}
    for pe in args.c3_peclet:
        m = api.Monolis(lib)
        t0 = time.perf_counter()
        b = problems.convection_diffusion(m, n=args.c3_n, peclet=pe)
        t_asm = time.perf_counter() - t0
        m.quiet()
        m.set_error_abort(False)
        m.set_method(api.ITER_BICGSTAB)
        m.set_precond(api.PREC_DIAG)
        m.set_tolerance(TOL)
        m.set_maxiter(20000)
        m.set_matrix_cache(True)
        stream = torch.cuda.ExternalStream(api.stream_handle(lib))
        d_b = torch.from_numpy(b).cuda()
        d_x = torch.zeros_like(d_b)
        res = {}
        for prec, name in ((0, "fp64"), (1, "mixed")):
            m.set_precision(prec)
            m.device_prepare()
            device_solve_timed(m, stream, d_b, d_x)  # warm-up
            with ClockSampler(torch.cuda.current_device()) as clk:
                ts = [device_solve_timed(m, stream, d_b, d_x) for _ in range(3)]
            t = float(np.mean(ts))
            d_r = torch.empty_like(d_x)
            m.device_matvec(d_x.data_ptr(), d_r.data_ptr())
            stream.synchronize()
            res[name] = {"s": t, "s_each": ts, "clocks": clk.summary(), "iterations": m.get_converge_iter(),
                         "true_rel_residual": (torch.linalg.norm(d_b - d_r) / torch.linalg.norm(d_b)).item(),
                         "fp64_refreshes": int(m.Iarray[api.B200_PRM_I_N_REFINE])}
            if prec == 0:
                x64 = d_x.clone()
                kt, _ = kernel_times(m, stream, d_b, d_x)
                res[name]["kernel_us_per_iteration"] = {"p": kt[0] * 1e6, "v=A*pt": kt[1] * 1e6, "s": kt[2] * 1e6,
                                                        "t=A*st": kt[3] * 1e6, "x,r": kt[4] * 1e6}
                byts = float(m.Rarray[api.B200_PRM_R_SPMV_BYTES_FP64])
                res[name]["spmv_layout_bytes"] = byts
                res[name]["wide_slices"] = int(m.Iarray[api.B200_PRM_I_WIDE_SLICES_FP64])
                res[name]["spmv_in_solve_gbs"] = byts / kt[1] / 1e9
                res[name]["spmv_in_solve_frac_of_measured"] = byts / kt[1] / 1e9 / peak
        res["mixed"]["rel_error_vs_fp64_solution"] = float(torch.linalg.norm(d_x - x64) / torch.linalg.norm(x64))
        key = f"convection_diffusion_n{args.c3_n}_pe{pe:g}_bicgstab_diag_tol1e-08"
        out[f"pe{pe:g}"] = {"assembly_s": t_asm, **res, "speedup_mixed_vs_fp64": res["fp64"]["s"] / res["mixed"]["s"],
                            "oracle_iterations": fx.get(key), "oracle_iterations_by_threads": fx.get(key + ":by_threads")}
        m.finalize()
        del d_b, d_x, x64
    return {"workload": f"3D upwind convection-diffusion {args.c3_n}^3 unknowns, ndof=1, BiCGSTAB + DIAG, "
                        f"rel.res 1e-8, FP64 vs FP32-inner/FP64-refined", "by_peclet": out}


def device_assembly_c2(lib, n, b_host):
    """Elasticity assembled on the device (monolis_b200_device_add_elements_R +
    monolis_b200_device_set_Dirichlet_bc_R) against the host assembly."""
    import ctypes as C
    import torch
    host = api.Monolis(lib)
    problems.elasticity(host, n=n)
    m = api.Monolis(lib)
    elem = problems.hex_elements(n)
    m.get_nonzero_pattern_flat(n ** 3, 8, 3, elem)
    ke = problems.hex8_elasticity_ke(1.0 / (n - 1)).reshape(-1)
    d_elem = torch.from_numpy(elem).cuda()
    d_ke = torch.from_numpy(np.ascontiguousarray(ke)).cuda()
    h = 1.0 / (n - 1)
    cnt = np.bincount(elem.reshape(-1), minlength=n ** 3).astype(np.float64) * (h ** 3 / 8.0)
    f = np.zeros((n ** 3, 3))
    f[:, 2] = -1.0
    f += problems.normal(2, n ** 3 * 3, 0.0, 0.01).reshape(n ** 3, 3)
    b0 = np.ascontiguousarray((f * cnt[:, None]).reshape(-1))
    nodes = np.repeat(np.arange(0, n ** 3, n, dtype=np.int32), 3)
    dofs = np.tile(np.arange(3, dtype=np.int32), n * n)
    vals = np.zeros(len(nodes))
    d_b = torch.from_numpy(b0).cuda()
    dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = lib.monolis_b200_device_clear_matrix(m.p)
    rc = rc or lib.monolis_b200_device_add_elements_R(m.p, len(elem), 8, d_elem.data_ptr(), d_ke.data_ptr(), 0, None)
    rc = rc or lib.monolis_b200_device_set_Dirichlet_bc_R(m.p, d_b.data_ptr(), len(nodes), nodes.ctypes.data_as(ip),
                                                          dofs.ctypes.data_as(ip), vals.ctypes.data_as(dp))
    torch.cuda.synchronize()
    t_dev = time.perf_counter() - t0
    if rc:
        return {"failed": int(rc)}
    vals_dev = np.empty(m.NZ * 9)
    lib.monolis_b200_device_get_values(m.p, vals_dev.ctypes.data_as(dp))
    same = bool(np.array_equal(vals_dev.view(np.uint64), host.values().view(np.uint64)) and
                np.array_equal(d_b.cpu().numpy().view(np.uint64), b_host.view(np.uint64)))
    m.finalize()
    host.finalize()
    return {"device_s": t_dev, "bit_identical_to_host": same,
            "includes": "clear + 2,048,383 hex8 element matrices (24x24) + 49,152 Dirichlet conditions + layout rebuild"}


def fp64_one_by_one(lib, systems, bs, tol):
    """The plain FP64 GPU CG (monolis_b200_device_solve_R) on each system in
    turn, device-resident b and x; returns summed device seconds, iterations."""
    import torch
    stream = torch.cuda.ExternalStream(api.stream_handle(lib))
    total, iters = 0.0, []
    for (ix, it, v, _), b in zip(systems, bs):
        m = api.Monolis(lib)
        n = len(ix) - 1
        m.set_matrix_BCSR(n, n, 1, len(it), v, ix, it)
        m.quiet()
        m.set_error_abort(False)
        m.set_method(api.ITER_CG)
        m.set_precond(api.PREC_DIAG)
        m.set_tolerance(tol)
        m.set_maxiter(20000)
        m.set_matrix_cache(True)
        m.device_prepare()
        d_b = torch.from_numpy(b).cuda()
        d_x = torch.zeros_like(d_b)
        total += device_solve_timed(m, stream, d_b, d_x)
        iters.append(m.get_converge_iter())
        m.finalize()
    return total, iters


def batch_run(lib, systems, bs, label):
    """Stack the systems into one batch, autotune, solve FP32-refined to 1e-8
    and FP32-only to 1e-6; check every system's FP64 residual in numpy."""
    import torch
    batch = api.Batch(lib)
    for ix, it, v, _ in systems:
        batch.add_csr(len(ix) - 1, 1, ix, it, v)
    t0 = time.perf_counter()
    batch.prepare(precond=api.PREC_DIAG, autotune=True)
    t_prep = time.perf_counter() - t0
    cands = batch.autotune(iters=30)
    cfg = batch.config()
    out = {"systems": len(systems), "unknowns": int(sum(len(b) for b in bs)), "prepare_s": t_prep,
           "config": {"cluster": cfg[0], "threads": cfg[1], "split_rows": cfg[2], "unroll": batch.unroll()},
           "autotune": [{"cluster": c[0], "threads": c[1], "split_rows": c[2], "s": c[3]} for c in cands]}
    for name, tol, refine in (("refined_1e-8", 1e-8, True), ("fp32_1e-6", 1e-6, False)):
        xs, its, res, st = batch.solve(bs, tol=tol, max_iter=20000, refine=refine)  # warm-up; uploads b
        t_e2e0 = time.perf_counter()
        xs, its, res, st = batch.solve(bs, tol=tol, max_iter=20000, refine=refine)
        t_e2e = time.perf_counter() - t_e2e0
        torch.cuda.nvtx.range_push(f"c4_batch_{name}")  # ncu --nvtx-include "c4_batch_refined_1e-8/"
        its2, res2, st2 = batch.device_solve(tol=tol, max_iter=20000, refine=refine)
        torch.cuda.nvtx.range_pop()
        t_dev = batch.last_seconds()
        true = [float(np.linalg.norm(b - problems.csr_matvec(ix, it, v, x)) / np.linalg.norm(b))
                for (ix, it, v, _), x, b in zip(systems, xs, bs)]
        # roofline: every system's iterations x the minimum fused FP32 CG schedule of its size (SpMV:
        # values and 32-bit column ids, offsets, x and y; 12 vector passes; DIAG factors), FP64 refreshes
        # not counted (a lower bound on the bytes of the refined solve)
        peak, _ = measured_peak()
        byts = sum(int(k) * (len(it) * 8 + (len(ix) + 1) * 4 + 2 * (len(ix) - 1) * 4 + 13 * (len(ix) - 1) * 4)
                   for k, (ix, it, v, _) in zip(its2, systems))
        out[name] = {"s": t_dev, "e2e_s": t_e2e, "all_converged": bool(np.all(st2 == 0)),
                     "max_true_rel_residual": max(true), "iterations_max": int(its2.max()),
                     "iterations_mean": float(its2.mean()),
                     "roofline": {"bound": "hbm", "fp32_loop_bytes": float(byts),
                                  "achieved_gbs": byts / t_dev / 1e9, "frac_of_measured": byts / t_dev / 1e9 / peak}}
    batch.destroy()
    log(f"[rank 0] batch {label}: {json.dumps({k: out[k] for k in out if k != 'autotune'})[:300]}")
    return out


def workload_c4(lib, args):
    """512 independent FV diffusion systems (side log-uniform in [10, 60]) in
    one batch, and one 96^3 system with 32 right-hand sides; each against the
    plain FP64 GPU CG solving the systems one by one."""
    sides = problems.batch_sides(args.c4_count)
    systems = [problems.fv_diffusion_csr(int(s), 4000 + i) for i, s in enumerate(sides)]
    bs = [problems.uniform(5000 + i, int(s) ** 3) for i, s in enumerate(sides)]
    res = {"workload": f"{len(sides)} cell-centred FV diffusion systems, side round(exp(U(ln10, ln60))), "
                       f"log-normal kappa, CG + DIAG; FP32 batched (1e-6) and FP32-refined (1e-8) vs FP64 GPU "
                       f"CG one system at a time (1e-8)"}
    res["many_systems"] = batch_run(lib, systems, bs, "many systems")
    t64, it64 = fp64_one_by_one(lib, systems, bs, 1e-8)
    res["many_systems"]["fp64_one_by_one_s"] = t64
    res["many_systems"]["speedup_refined_vs_fp64"] = t64 / res["many_systems"]["refined_1e-8"]["s"]
    # one 96^3 system with 32 right-hand sides (monolis_b200_device_solve_multi_R)
    one = problems.fv_diffusion_csr(args.c4_rhs_side, 4999)
    rhs = [problems.uniform(6000 + k, args.c4_rhs_side ** 3) for k in range(args.c4_rhs)]
    res["many_rhs"] = multi_rhs_run(lib, one, rhs)
    t64r, it64r = fp64_one_by_one(lib, [one] * args.c4_rhs, rhs, 1e-8)
    res["many_rhs"]["fp64_one_by_one_s"] = t64r
    res["many_rhs"]["fp64_one_by_one_iterations_max"] = int(max(it64r))
    res["many_rhs"]["speedup_refined_vs_fp64"] = t64r / res["many_rhs"]["refined_1e-8"]["s"]
    return res


def workload_c4_sharded(lib, args, rank, world):
    """C4's independent systems over the ranks: replicas with no data-path
    collective (monolis_b200.partition.split_systems, greedy by stored
    blocks); every rank solves its share in one batch, FP32-refined to 1e-8;
    the job time is the max over ranks. Every rank reaches the same barrier
    and reduction whatever happens locally (a rank without systems, or one
    whose solve fails, reports 0 s or inf)."""
    from monolis_b200 import partition
    sides = problems.batch_sides(args.c4_count)
    share = partition.split_systems([7 * int(s) ** 3 for s in sides], world)[rank]
    t, err, converged, unknowns, batch = 0.0, None, True, 0, None
    try:
        if share:
            systems = [problems.fv_diffusion_csr(int(sides[i]), 4000 + i) for i in share]
            bs = [problems.uniform(5000 + i, int(sides[i]) ** 3) for i in share]
            unknowns = int(sum(len(b) for b in bs))
            batch = api.Batch(lib)
            for ix, it, v, _ in systems:
                batch.add_csr(len(ix) - 1, 1, ix, it, v)
            batch.prepare(precond=api.PREC_DIAG, autotune=True)
            batch.solve(bs, tol=1e-8, max_iter=20000, refine=True)  # warm-up; uploads b
    except Exception as e:  # reported below, after the collectives every rank takes
        err = repr(e)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    try:
        if batch is not None and err is None:
            _, _, st = batch.device_solve(tol=1e-8, max_iter=20000, refine=True)
            t = batch.last_seconds()
            converged = bool(np.all(st == 0))
    except Exception as e:
        err = repr(e)
    finally:
        if batch is not None:
            batch.destroy()
    t_max = max_over_ranks(t if err is None else float("inf"), world)
    out = {"workload": f"{len(sides)} C4 systems over {world} ranks (greedy by stored blocks), FP32-refined 1e-8",
           "systems_this_rank": len(share), "unknowns_this_rank": unknowns,
           "all_converged_this_rank": converged and err is None,
           "s": t_max, "scaling": f"strong (the {len(sides)} systems are split)"}
    if err is not None:
        out["failed_this_rank"] = err
    return out


def multi_rhs_run(lib, sysm, rhs):
    """All right-hand sides in one persistent kernel (matrix read once per
    iteration for all of them): FP32-refined to 1e-8 and FP64 to 1e-8."""
    import torch
    ix, it, v, _ = sysm
    n = len(ix) - 1
    m = api.Monolis(lib)
    m.set_matrix_BCSR(n, n, 1, len(it), v, ix, it)
    m.quiet()
    m.set_error_abort(False)
    m.set_method(api.ITER_CG)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(1e-8)
    m.set_maxiter(20000)
    m.set_matrix_cache(True)
    stream = torch.cuda.ExternalStream(api.stream_handle(lib))
    K = len(rhs)
    d_B = torch.from_numpy(np.ascontiguousarray(np.stack(rhs))).cuda()
    d_X = torch.zeros_like(d_B)
    out = {"unknowns": n, "rhs": K, "nz": len(it)}
    for name, prec in (("refined_1e-8", 1), ("fp64_1e-8", 0)):
        m.set_precision(prec)
        m.device_prepare()
        its = np.zeros(K, dtype=np.int32)
        res = np.zeros(K)
        st = np.zeros(K, dtype=np.int32)
        times = []
        for rep in range(2):  # warm-up, timed
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            torch.cuda.nvtx.range_push(f"c4_multi_{name}_{rep}")  # ncu --nvtx-include "c4_multi_refined_1e-8_1/"
            rc = lib.monolis_b200_device_solve_multi_R(m.p, K, d_B.data_ptr(), d_X.data_ptr(),
                                                       its.ctypes.data_as(api._ip), res.ctypes.data_as(api._dp),
                                                       st.ctypes.data_as(api._ip))
            torch.cuda.nvtx.range_pop()
            e1.record(stream)
            e1.synchronize()
            if rc:
                raise RuntimeError(f"multi-RHS solve failed: {rc}")
            times.append(e0.elapsed_time(e1) * 1e-3)
        X = d_X.cpu().numpy()
        true = [float(np.linalg.norm(b - problems.csr_matvec(ix, it, v, X[k])) / np.linalg.norm(b))
                for k, b in enumerate(rhs)]
        # roofline: per iteration the matrix and the DIAG factors once (values + 32-bit column ids +
        # offsets, in the loop precision) while any right-hand side is active, and 11 vector passes per
        # active right-hand side (product: z, p read, p, q written; update: p, q, r, y read, y, r, z
        # written); FP64 refreshes not counted
        peak, _ = measured_peak()
        sv = 4 if prec == 1 else 8
        byts = int(its.max()) * (len(it) * (sv + 4) + (n + 1) * 4 + n * sv) + float(its.sum()) * 11 * n * sv
        out[name] = {"s": times[-1], "all_converged": bool(np.all(st == 0)), "max_true_rel_residual": max(true),
                     "iterations_max": int(its.max()), "iterations_mean": float(its.mean()),
                     "roofline": {"bound": "hbm", "loop_bytes": float(byts), "achieved_gbs": byts / times[-1] / 1e9,
                                  "frac_of_measured": byts / times[-1] / 1e9 / peak}}
    m.finalize()
    log(f"[rank 0] many rhs: {json.dumps(out)[:300]}")
    return out


def workload_c5(lib, args):
    """Adjoint gradient of L = 1/2 ||x - x_target||^2 for 3D Q1 diffusion with
    per-element log-normal conductivity (128^3 nodes): forward CG to 1e-10,
    transpose solve, per-element gradient; FP64 and FP32-refined, plus
    central differences on a few seeded directions."""
    import torch
    n = args.c5_n
    m = api.Monolis(lib)
    t0 = time.perf_counter()
    b, kappa, kref, elem = problems.diffusion_kappa(m, n=n)
    t_asm = time.perf_counter() - t0
    target = problems.smooth_target(n)
    fixed = problems.face_x0_fixed(n, 1)
    m.quiet()
    m.set_error_abort(False)
    m.set_method(api.ITER_CG)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(1e-10)
    m.set_maxiter(20000)
    m.set_matrix_cache(True)
    stream = torch.cuda.ExternalStream(api.stream_handle(lib))
    d_b = torch.from_numpy(b).cuda()
    d_t = torch.from_numpy(target).cuda()
    d_elem = torch.from_numpy(np.ascontiguousarray(elem)).cuda()
    d_k = torch.from_numpy(np.ascontiguousarray(kref.reshape(-1))).cuda()
    d_fix = torch.from_numpy(fixed).cuda()
    n_elem = len(elem)
    res = {}
    grads = {}
    for prec, name in ((0, "fp64"), (1, "mixed")):
        m.set_precision(prec)
        m.device_prepare()
        d_x = torch.zeros_like(d_b)
        d_lam = torch.zeros_like(d_b)
        d_g = torch.empty(n_elem, dtype=torch.float64, device="cuda")
        for rep in range(2):  # warm-up, then timed
            t_fwd = device_solve_timed(m, stream, d_b, d_x)
            it_f = m.get_converge_iter()
            d_rhs = d_x - d_t
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            rc = lib.monolis_b200_device_solve_transpose_R(m.p, d_rhs.data_ptr(), d_lam.data_ptr())
            e1.record(stream)
            e1.synchronize()
            if rc:
                raise RuntimeError(f"adjoint solve failed: {rc}")
            t_adj = e0.elapsed_time(e1) * 1e-3
            it_a = m.get_converge_iter()
            e0.record(stream)
            for _ in range(10):
                rc = lib.monolis_b200_device_element_gradient_R(m.p, n_elem, 8, d_elem.data_ptr(), d_k.data_ptr(), 0,
                                                               d_lam.data_ptr(), d_x.data_ptr(), d_fix.data_ptr(),
                                                               -1.0, d_g.data_ptr())
            e1.record(stream)
            e1.synchronize()
            if rc:
                raise RuntimeError(f"element gradient failed: {rc}")
            t_grad = e0.elapsed_time(e1) * 1e-3 / 10
        grads[name] = d_g.cpu().numpy()
        gbytes = n_elem * (8 * 4 + 8) + 3 * (n ** 3) * 8  # connectivity, gradient, lambda + x + mask once
        res[name] = {"forward_s": t_fwd, "forward_iterations": it_f, "adjoint_s": t_adj, "adjoint_iterations": it_a,
                     "gradient_kernel_us": t_grad * 1e6, "gradient_kernel_gbs": gbytes / t_grad / 1e9,
                     "total_s": t_fwd + t_adj + t_grad}
        if prec == 0:
            x_ref = d_x.cpu().numpy()
            # roofline: the minimum fused CG schedule per iteration (SpMV + 12 vector passes + the
            # DIAG factors, ndof 1) x iterations / solve time; the gradient kernel's bytes / its time
            peak, peak_kind = measured_peak()
            nn = n ** 3
            it_bytes = float(m.Rarray[api.B200_PRM_R_SPMV_BYTES_FP64]) + 12 * nn * 8 + nn * 8
            c5_roofline = {"bound": "hbm", "peak_gbs": peak, "peak_kind": peak_kind,
                           "cg_bytes_per_iteration": it_bytes,
                           "fp64_forward_frac": it_f * it_bytes / t_fwd / 1e9 / peak,
                           "fp64_adjoint_frac": it_a * it_bytes / t_adj / 1e9 / peak,
                           "gradient_kernel_bytes": gbytes,
                           "gradient_kernel_frac": gbytes / t_grad / 1e9 / peak}
    g64 = grads["fp64"]
    res["mixed"]["gradient_rel_diff_vs_fp64"] = float(np.linalg.norm(grads["mixed"] - g64) / np.linalg.norm(g64))
    fd = []
    t_fd = 0.0
    if args.c5_fd_dirs > 0:
        # central differences: A(kappa +- h d) assembled on the device (element matrices scaled per element,
        # Dirichlet face), solved to 1e-11 on the device, loss summed on the device
        import ctypes as C
        rng = np.random.default_rng(2025)
        h = 1e-4
        fm = api.Monolis(lib)
        fm.get_nonzero_pattern_flat(n ** 3, 8, 1, elem)
        fm.quiet()
        fm.set_error_abort(False)
        fm.set_method(api.ITER_CG)
        fm.set_precond(api.PREC_DIAG)
        fm.set_tolerance(1e-11)
        fm.set_maxiter(20000)
        nodes = np.arange(0, n ** 3, n, dtype=np.int32)
        zeros = np.zeros(len(nodes), dtype=np.int32)
        vals = np.zeros(len(nodes))
        ones = torch.ones(n ** 3, dtype=torch.float64, device="cuda")
        d_fb = torch.empty_like(ones)
        d_fx = torch.empty_like(ones)
        dp, ip = C.POINTER(C.c_double), C.POINTER(C.c_int)

        def loss(d_kap):
            d_fb.copy_(ones)
            rc = lib.monolis_b200_device_clear_matrix(fm.p)
            rc = rc or lib.monolis_b200_device_add_elements_R(fm.p, n_elem, 8, d_elem.data_ptr(), d_k.data_ptr(), 0,
                                                              d_kap.data_ptr())
            rc = rc or lib.monolis_b200_device_set_Dirichlet_bc_R(fm.p, d_fb.data_ptr(), len(nodes),
                                                                  nodes.ctypes.data_as(ip), zeros.ctypes.data_as(ip),
                                                                  vals.ctypes.data_as(dp))
            if rc:
                raise RuntimeError(f"FD assembly failed: {rc}")
            d_fx.zero_()
            rc = fm.device_solve(d_fb.data_ptr(), d_fx.data_ptr())
            fd_solves.append((int(rc), fm.get_converge_iter(), fm.get_converge_residual()))
            return 0.5 * float(torch.dot(d_fx - d_t, d_fx - d_t))
        fd_solves = []
        d_kap0 = torch.from_numpy(kappa).cuda()
        g64_d = torch.from_numpy(g64).cuda()
        t0 = time.perf_counter()
        for _ in range(args.c5_fd_dirs):
            d = torch.from_numpy(kappa * rng.standard_normal(n_elem)).cuda()
            fdv = (loss(d_kap0 + h * d) - loss(d_kap0 - h * d)) / (2 * h)
            an = float(torch.dot(g64_d, d))
            fd.append(abs(fdv - an) / abs(an))
        t_fd = time.perf_counter() - t0
        fm.finalize()
    m.finalize()
    return {"workload": f"adjoint of L=1/2||x-x_target||^2, 3D Q1 diffusion {n}^3 nodes, log-normal kappa per element "
                        f"({n_elem} elements), forward/adjoint CG+DIAG to 1e-10",
            "assembly_s": t_asm, "loss": 0.5 * float(np.dot(x_ref - target, x_ref - target)), **res,
            "fd_directions": len(fd), "fd_max_rel_err_fp64": max(fd) if fd else None,
            "fd_median_rel_err_fp64": float(np.median(fd)) if fd else None, "fd_s": t_fd,
            "fd_solves": ({"count": len(fd_solves), "status_nonzero": sum(1 for q in fd_solves if q[0]),
                           "iterations_max": max(q[1] for q in fd_solves),
                           "rel_residual_max": max(q[2] for q in fd_solves)} if fd else None),
            "fd_method": "central differences, h = 1e-4 along kappa * N(0,1) directions; each side assembled on "
                         "the device (scaled element matrices + Dirichlet face) and solved to 1e-11 in FP64",
            "roofline": c5_roofline}


def shared_config(n, nz, unknowns):
    """The workload, identical in both arms' lines."""
    mat_gb = nz * 9 * 8 / 1e9
    l2 = (f"inputs larger than L2 (FP64 matrix {mat_gb:.1f} GB)" if mat_gb > 0.126
          else f"matrix {mat_gb * 1e3:.0f} MB fits in L2")
    return {"workload": workload_name(n, nz), "unknowns": int(unknowns), "nz_blocks": int(nz),
            "arithmetic": "f64 (CG recurrences, SpMV, DIAG)", "l2": l2}


def run_reference(args, rank):
    """The reference arm: the CPU oracle (the restatement of the reference's
    FP64 CG, DIAG and SpMV) on every host core. One step is a contiguous
    range of iterations of ONE complete solve to 1e-8: the solve is timed
    whole, and the oracle's wall-clock log (end of every iteration) cuts it
    into `steps` consecutive ranges, so `value` is a measured solve time and
    steps x ms_per_step is the measured timed region. The warm-up is one
    solve capped at `warmup` steps' worth of iterations. A single-threaded
    sample (the reference's default build has no OpenMP) is reported beside
    it, extrapolated by the iteration count, together with the fixture's
    measured complete serial solve."""
    if rank != 0:
        return  # other ranks of a multi-rank launch exit without work
    orc = api.load_library(ORACLE_SO, oracle=True)
    threads = os.cpu_count() or 1
    orc.oracle_set_threads(threads)
    m = api.Monolis(orc)
    t0 = time.perf_counter()
    b = problems.elasticity(m, n=args.n)
    t_asm = time.perf_counter() - t0
    nz = int(m.csr_index()[-1])
    m.quiet()
    m.set_error_abort(False)
    m.set_method(api.ITER_CG)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(TOL)
    fx = fixture()
    key = f"elasticity_n{args.n}_cg_diag_tol1e-08"
    it_hint = fx.get(key) or 200
    K = max(1, args.steps)
    seg = max(1, -(-it_hint // K))
    # warm-up: `warmup` steps of the timed steps' size
    m.set_maxiter(max(1, args.warmup * seg))
    x = np.zeros_like(b)
    m.solve(b, x)
    # timed: one complete solve with the iteration clock
    max_iter = 20000
    clock = np.zeros(max_iter + 2)
    orc.oracle_set_iter_clock(api._dptr(clock), len(clock))
    m.set_maxiter(max_iter)
    x = np.zeros_like(b)
    t1 = time.perf_counter()
    m.solve(b, x)
    t_solve = time.perf_counter() - t1
    orc.oracle_set_iter_clock(None, 0)
    it = m.get_converge_iter()
    status = m.get_error_tag()
    bounds = [round(k * it / K) for k in range(K + 1)]
    step_s = [float(clock[bounds[k + 1]] - clock[bounds[k]]) for k in range(K)]
    # single thread: a bounded sample of the same solve
    orc.oracle_set_threads(1)
    m.set_maxiter(args.cpu_sample_iters)
    x1 = np.zeros_like(b)
    t1 = time.perf_counter()
    m.solve(b, x1)
    t_1 = time.perf_counter() - t1
    value = t_solve
    line = {
        "impl": "reference", "metric": metric_name(args.n), "value": value,
        "unit": "s", "n_gpus": args.gpus, "steps": K, "warmup": args.warmup,
        "ms_per_step": value / K * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": shared_config(args.n, nz, len(b)),
        "parallelism": f"cpu, {threads} threads (oracle, FP64)",
        "cpu_baseline": {"value": value, "unit": "s", "cores": threads, "kind": "port",
                         "sample": f"one complete FP64 CG + DIAG solve to rel.res 1e-8 ({it} iterations, "
                                   f"status {status}) on {threads} threads, measured whole; steps are "
                                   f"{K} consecutive iteration ranges of it"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "iterations": it, "step_s": step_s, "assembly_s": t_asm,
        "single_thread": {
            "value_extrapolated": t_1 / args.cpu_sample_iters * it, "unit": "s", "cores": 1,
            "sample": f"{args.cpu_sample_iters} iterations on 1 thread ({t_1:.2f} s), x {it} iterations",
            "measured_full_solve_other_host": fx.get(key + ":seconds"),
            "measured_full_solve_other_host_note": "complete serial oracle solve recorded by oracle/iterations.py "
                                                   "on an 8-core Xeon @ 2.7 GHz (tests/golden)"},
    }
    print(json.dumps(line), flush=True)


def timed_device_solves(m, stream, d_b, d_x, precision, warmup, steps, clock_index=None):
    """warmup + steps device-resident solves (CUDA events on the library
    stream); returns per-step seconds, iterations, launches, clocks."""
    import torch
    m.set_precision(precision)

    def one():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = m.device_solve(d_b.data_ptr(), d_x.data_ptr())
        e1.record(stream)
        e1.synchronize()
        if rc != 0:
            raise RuntimeError(f"solve failed: {api.STATUS_NAMES.get(rc, rc)}")
        return e0.elapsed_time(e1) * 1e-3

    for _ in range(warmup):
        one()
    torch.cuda.synchronize()
    times, iters, launches = [], [], 0
    sampler = ClockSampler(clock_index) if clock_index is not None else None
    torch.cuda.nvtx.range_push("timed")  # ncu --nvtx-include "timed/" selects these launches
    if sampler:
        sampler.__enter__()
    try:
        for _ in range(steps):
            times.append(one())
            iters.append(m.get_converge_iter())
            launches += int(m.Iarray[api.B200_PRM_I_LAUNCHES])
    finally:
        if sampler:
            sampler.__exit__(None, None, None)
        torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    return times, iters, launches, (sampler.summary() if sampler else None)


def e2e_calls(m, b, n_unk, precision, calls, parts=None):
    """monolis_solve_R with pinned host b and x, matrix uploaded by every
    call (the library's default, like the reference's GPU build); one
    untimed call first. Returns the per-call wall seconds; `parts` (a list)
    receives each timed call's split as the library reports it: host->device
    copies (matrix and b), the device loop, the device->host copy of x."""
    import torch
    hb = torch.from_numpy(b).pin_memory()
    hx = torch.zeros(n_unk, dtype=torch.float64).pin_memory()
    m.set_matrix_cache(False)
    m.set_precision(precision)
    out = []
    for k in range(1 + calls):
        hx.zero_()
        t1 = time.perf_counter()
        m.solve(hb.numpy(), hx.numpy())
        dt = time.perf_counter() - t1
        if m.get_error_tag() != 0:
            raise RuntimeError(f"monolis_solve_R failed: status {m.get_error_tag()}")
        if k >= 1:
            out.append(dt)
            if parts is not None:
                R = m.Rarray
                parts.append({"wall_s": round(dt, 4), "h2d_s": round(R[api.B200_PRM_R_TIME_H2D], 4),
                              "loop_s": round(R[api.B200_PRM_R_TIME_LOOP], 4),
                              "d2h_s": round(R[api.B200_PRM_R_TIME_D2H], 4)})
    return out


def stats(v):
    return {"mean_s": float(np.mean(v)), "median_s": float(np.median(v)), "max_s": float(np.max(v)),
            "min_s": float(np.min(v)), "n": len(v)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--cpu-sample-iters", type=int, default=10)
    ap.add_argument("--cpu-baseline-iters", type=int, default=200,
                    help="iterations of the CPU-baseline sample in our arm (about 10-30 s on the host)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workloads", default="c1,c3,c4,c5",
                    help="secondary workloads to run after the headline (any of c1,c3,c4,c5, or none)")
    ap.add_argument("--replicas", action="store_true",
                    help="with N > 1: N independent copies of the headline system (weak scaling) instead of "
                         "the row-partitioned solve of one system")
    ap.add_argument("--sharded", action="store_true",
                    help="force the row-partitioned multi-rank code path (NCCL halo + all-reduce), also at N = 1")
    ap.add_argument("--c4-count", type=int, default=512)
    ap.add_argument("--c4-sharded", action="store_true",
                    help="the C4 systems split over the N ranks (greedy by stored blocks), each rank "
                         "solving its share in one batch, max over ranks (N = 1: the whole batch)")
    ap.add_argument("--c4-rhs-side", type=int, default=96)
    ap.add_argument("--c4-rhs", type=int, default=32)
    ap.add_argument("--c3-n", type=int, default=256)
    ap.add_argument("--c3-peclet", type=float, nargs="+", default=[0.5, 5.0, 50.0])
    ap.add_argument("--c5-n", type=int, default=128)
    ap.add_argument("--c5-fd-dirs", type=int, default=32)
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if (world > 1 and not args.replicas) or args.sharded:
        main_sharded(args, world, rank, local)
    else:
        main_ours(args, world, rank, local)


def main_sharded(args, world, rank, local):
    """The headline system row-partitioned over the ranks, the reference's
    multi-rank model (src/linalg/matvec.f90:144: halo update before each
    product; src/linalg/inner_product.f90:185: every dot product summed over
    the ranks; src/solver/solver.f90:44: N = n_internal_vertex): contiguous
    row ranges of about equal stored blocks (z-slabs of the structured mesh),
    an NCCL communicator on the MONOLIS_COM of every rank, FP64 CG + DIAG
    device-resident (monolis_b200_device_solve_com_R). Strong scaling: one
    system, time = max over ranks. Every rank takes the same collective steps
    in the same order, whatever happens locally."""
    import datetime

    # NCCL's own log of every communicator (ranks, devices, transports),
    # before the process group or the library creates one. NCCL writes it to
    # the process's stdout; that descriptor is pointed at stderr, and the one
    # JSON line goes to the original stdout.
    os.environ["NCCL_DEBUG"] = "INFO"
    sys.stdout.flush()
    json_out = os.fdopen(os.dup(1), "w")
    os.dup2(2, 1)
    import torch
    import torch.distributed as dist

    from monolis_b200 import partition
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    lib = api.load_product()
    g = api.Monolis(lib)
    t0 = time.perf_counter()
    b = problems.elasticity(g, n=args.n)
    nd, n_glob, nz_glob = g.NDOF, g.N, g.NZ
    t1 = time.perf_counter()
    p = partition.partition_rank(g.csr_index(), g.csr_item() - 1, g.values(), nd, world, rank)
    t_part = time.perf_counter() - t1
    rows = (p["glob"][:, None] * nd + np.arange(nd)[None, :]).reshape(-1)
    b_loc = np.ascontiguousarray(b[rows])
    g.finalize()
    del g
    m = api.Monolis(lib)
    m.set_matrix_BCSR(p["N"], p["NP"], nd, len(p["item"]), p["val"], p["index"], p["item"])
    m.quiet()
    m.set_error_abort(False)
    m.set_method(api.ITER_CG)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(TOL)
    m.set_maxiter(20000)
    m.set_matrix_cache(True)
    m.set_precision(0)
    m.set_halo(p, rank, world)
    # one NCCL unique id from rank 0 (through the process group's store)
    uid = [api.nccl_unique_id(lib) if rank == 0 else None]
    if world > 1:
        dist.broadcast_object_list(uid, src=0)
    m.com_init_nccl(uid[0], rank, world)
    t_setup = time.perf_counter() - t0
    log(f"[rank {rank}] rows {p['lo']}..{p['hi']} of {n_glob}, ghosts {p['NP'] - p['N']}, "
        f"neighbours {list(p['recv_pe'])}, setup {t_setup:.1f}s (partition {t_part:.1f}s)")
    stream = torch.cuda.ExternalStream(api.stream_handle(lib))
    d_b = torch.from_numpy(b_loc).cuda()
    d_x = torch.zeros_like(d_b)
    m.device_prepare()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def one():
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        rc = m.device_solve_com(d_b.data_ptr(), d_x.data_ptr())
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) * 1e-3, rc

    failed = None
    for _ in range(args.warmup):
        _, rc = one()
        failed = failed or (rc or None)
    barrier()
    times, iters = [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            t, rc = one()
            failed = failed or (rc or None)
            times.append(t)
            iters.append(m.get_converge_iter())
    barrier()
    t_mean = float(np.mean(times)) if failed is None else float("inf")
    t_max = max_over_ranks(t_mean, world)
    it = int(np.median(iters))
    res = m.get_converge_residual()
    launches = int(m.Iarray[api.B200_PRM_I_LAUNCHES]) * args.steps
    # the FP32-refined CG on the same partition (FP32 halo of p, all-reduced dots)
    m.set_precision(1)
    m.device_prepare()
    barrier()
    t32, it32, failed32 = [], [], None
    for k in range(1 + args.steps):
        t, rc = one()
        failed32 = failed32 or (rc or None)
        if k >= 1:
            t32.append(t)
            it32.append(m.get_converge_iter())
    barrier()
    t32_max = max_over_ranks(float(np.mean(t32)) if failed32 is None else float("inf"), world)
    nref32 = int(m.Iarray[api.B200_PRM_I_N_REFINE])
    m.set_precision(0)
    # e2e: monolis_solve_R with this rank's host b and x (pinned), device matrix kept
    hb = torch.from_numpy(b_loc).pin_memory()
    hx = torch.zeros(len(b_loc), dtype=torch.float64).pin_memory()
    e2e = []
    for k in range(1 + args.steps):
        hx.zero_()
        barrier()
        t1 = time.perf_counter()
        m.solve(hb.numpy(), hx.numpy())
        if k >= 1:
            e2e.append(time.perf_counter() - t1)
    e2e_max = max_over_ranks(float(np.mean(e2e)), world)
    if rank == 0:
        peak, peak_kind = measured_peak()
        line = {
            "metric": metric_name(args.n), "value": t_max, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max * 1e3, "higher_is_better": False, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": shared_config(args.n, nz_glob, n_glob * nd),
            "parallelism": f"row partition over {world} ranks (z-slabs; NCCL halo updates + all-reduced dots)",
            "statistic": f"mean of {len(times)} solves, max over ranks", "iterations": it, "rel_residual": res,
            "failed_status": failed,
            "mixed": {"value": t32_max, "unit": "s", "dtype": "f32 inner / f64 refinement",
                      "iterations": int(np.median(it32)), "fp64_refreshes": nref32, "failed_status": failed32,
                      "statistic": f"mean of {len(t32)} solves after one untimed, max over ranks"},
            "speedup_mixed_vs_fp64": t_max / t32_max,
            "rank0": {"rows": int(p["N"]), "ghost_rows": int(p["NP"] - p["N"]),
                      "neighbours": [int(v) for v in p["recv_pe"]], "step_s": times},
            "e2e": {"value": e2e_max, "unit": "s",
                    "h2d_bytes_per_step": int(len(b_loc) * 8), "d2h_bytes_per_step": int(len(b_loc) * 8),
                    "path": "monolis_solve_R with the MONOLIS_COM (NCCL), pinned host b/x of rank 0's rows, "
                            "device matrix kept (cache); bytes per step are rank 0's",
                    "statistic": f"mean of {len(e2e)} calls, max over ranks", **stats(e2e)},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "roofline": None, "roofline_note": "see the one-GPU line (the same kernels on 1/N of the rows)",
            "cpu_baseline": None, "peak_gbs": peak, "peak_kind": peak_kind,
        }
        print(json.dumps(line), file=json_out, flush=True)
    m.finalize()
    if world > 1:
        dist.destroy_process_group()


def main_ours(args, world, rank, local):
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    lib = api.load_product()
    m = api.Monolis(lib)
    t0 = time.perf_counter()
    b = problems.elasticity(m, n=args.n)
    t_asm = time.perf_counter() - t0
    m.quiet()
    m.set_error_abort(False)
    m.set_method(api.ITER_CG)
    m.set_precond(api.PREC_DIAG)
    m.set_tolerance(TOL)
    m.set_maxiter(20000)
    N, nd, nz = m.N, m.NDOF, m.NZ
    n_unk = N * nd
    log(f"[rank {rank}] assembled n={args.n}: N={N} nz={nz} in {t_asm:.1f}s")

    stream = torch.cuda.ExternalStream(api.stream_handle(lib))
    d_b = torch.from_numpy(b).cuda()
    d_x = torch.zeros(n_unk, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # headline: the plain FP64 CG (the reference's arithmetic), device-resident
    # b and x; the device matrix is kept between these solves
    m.set_matrix_cache(True)
    m.set_precision(0)
    m.device_prepare()
    barrier()
    t64s, it64s, launches, clocks = timed_device_solves(m, stream, d_b, d_x, 0, args.warmup, args.steps, local)
    barrier()
    t64 = float(np.mean(t64s))
    it64 = int(np.median(it64s))
    res64 = m.get_converge_residual()
    x64 = d_x.clone()
    # the FP32-inner / FP64-refined CG on the same system
    m.set_precision(1)
    m.device_prepare()
    barrier()
    t32s, it32s, _, clocks32 = timed_device_solves(m, stream, d_b, d_x, 1, max(2, args.warmup), args.steps, local)
    barrier()
    t_mixed = float(np.mean(t32s))
    nref = int(m.Iarray[api.B200_PRM_I_N_REFINE])  # FP64 refreshes of the last timed solve
    err_vs_fp64 = float(torch.linalg.norm(d_x - x64) / torch.linalg.norm(x64))
    d_r = torch.empty_like(d_x)
    m.device_matvec(d_x.data_ptr(), d_r.data_ptr())
    stream.synchronize()
    true_res = torch.linalg.norm(d_b - d_r).item() / torch.linalg.norm(d_b).item()  # x0 = 0: r0 = b
    # per-kernel durations inside a solve (kernel-timer mode, one extra solve of each precision)
    kt32, _ = kernel_times(m, stream, d_b, d_x)
    m.set_precision(0)
    kt64, _ = kernel_times(m, stream, d_b, d_x)

    # SpMV roofline (standalone kernels, FP64 and FP32), CUDA events on the library stream
    nzb, padded, nslices = m.device_info()
    u64, u32 = int(m.Iarray[api.B200_PRM_I_UNROLL_FP64]), int(m.Iarray[api.B200_PRM_I_UNROLL_FP32])
    layout_bytes = {"fp64": float(m.Rarray[api.B200_PRM_R_SPMV_BYTES_FP64]),
                    "fp32": float(m.Rarray[api.B200_PRM_R_SPMV_BYTES_FP32])}
    layout = {"bytes_fp64": layout_bytes["fp64"], "bytes_fp32": layout_bytes["fp32"],
              "bytes_fp64_32bit_columns": problems.spmv_bytes(nz, N, nd, 8),
              "bytes_fp32_32bit_columns": problems.spmv_bytes(nz, N, nd, 4),
              "wide_slices_fp64": int(m.Iarray[api.B200_PRM_I_WIDE_SLICES_FP64]),
              "wide_slices_fp32": int(m.Iarray[api.B200_PRM_I_WIDE_SLICES_FP32])}
    xs64 = torch.randn(n_unk, dtype=torch.float64, device="cuda")
    ys64 = torch.empty_like(xs64)
    xs32 = xs64.float()
    ys32 = torch.empty_like(xs32)
    torch.cuda.synchronize()
    spmv = {}
    reps = 20
    for name, fp32, xs, ys in (("fp64", False, xs64, ys64), ("fp32", True, xs32, ys32)):
        for _ in range(3):
            m.device_matvec(xs.data_ptr(), ys.data_ptr(), fp32=fp32)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            m.device_matvec(xs.data_ptr(), ys.data_ptr(), fp32=fp32)
        e1.record(stream)
        e1.synchronize()
        dt = e0.elapsed_time(e1) * 1e-3 / reps
        spmv[name] = {"seconds": dt, "bytes": layout_bytes[name], "gbs": layout_bytes[name] / dt / 1e9}
    del xs64, ys64, xs32, ys32
    peak, peak_kind = measured_peak()

    # device assembly of the same system, checked bit for bit against the host assembly
    asm = device_assembly_c2(lib, args.n, b)

    # e2e through monolis_solve_R with pinned host buffers (matrix upload included)
    e2e64_parts = []
    e2e64 = e2e_calls(m, b, n_unk, 0, args.steps, e2e64_parts)
    e2e32 = e2e_calls(m, b, n_unk, 1, min(args.steps, 5))
    h2d = nz * nd * nd * 8 + nz * 4 + (N + 1) * 4 + n_unk * 8  # values, items, offsets, b
    d2h = n_unk * 8

    t64_max = max_over_ranks(t64, world)
    t_mixed_max = max_over_ranks(t_mixed, world)
    e2e64_max = max_over_ranks(float(np.mean(e2e64)), world)

    workloads = {}
    if args.c4_sharded:
        try:
            workloads["c4_sharded"] = workload_c4_sharded(lib, args, rank, world)
        except Exception as e:  # report, do not hide
            workloads["c4_sharded"] = {"failed": repr(e)}
    if rank == 0 and world == 1:
        for w in [w for w in args.workloads.split(",") if w and w != "none"]:
            try:
                if w == "c1":
                    workloads["c1"] = workload_c1(lib, args)
                elif w == "c3":
                    workloads["c3"] = workload_c3(lib, args, peak)
                elif w == "c5":
                    workloads["c5"] = workload_c5(lib, args)
                elif w == "c4":
                    workloads["c4"] = workload_c4(lib, args)
            except Exception as e:  # report, do not hide
                workloads[w] = {"failed": repr(e)}
            log(f"[rank 0] workload {w}: {json.dumps(workloads[w])[:400]}")

    # the CPU baseline last: its OpenMP threads would otherwise share the
    # host cores with the graph-launching threads of the GPU workloads
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            orc = api.load_library(ORACLE_SO, oracle=True)
            threads = os.cpu_count() or 1
            orc.oracle_set_threads(threads)
            mo = api.Monolis(orc)
            ind = m.csr_index().copy()
            item0 = (m.csr_item() - 1).astype(np.int32)
            mo.set_matrix_BCSR(N, N, nd, nz, m.values(), ind, item0)
            mo.quiet()
            mo.set_error_abort(False)
            mo.set_method(api.ITER_CG)
            mo.set_precond(api.PREC_DIAG)
            mo.set_maxiter(args.cpu_baseline_iters)
            xo = np.zeros_like(b)
            t1 = time.perf_counter()
            mo.solve(b, xo)
            t_s = time.perf_counter() - t1
            t_it = t_s / args.cpu_baseline_iters
            cpu = {"value": t_it * it64, "unit": "s", "cores": threads, "kind": "port",
                   "sample": f"{args.cpu_baseline_iters} oracle FP64 CG iterations on the same system "
                             f"({t_s:.2f} s on {threads} threads), x {it64} iterations"}
            mo.finalize()
        except Exception as e:  # report, do not hide
            cpu = {"value": None, "unit": "s", "cores": None, "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        spmv32_bytes = layout_bytes["fp32"]
        spmv64_bytes = layout_bytes["fp64"]
        in_solve = {
            "fp64_us_per_iteration": {"p": kt64[0] * 1e6, "q=A*p (+<p,q>)": kt64[1] * 1e6,
                                      "update (+M^-1, dots)": kt64[2] * 1e6, "residual (gated)": kt64[3] * 1e6},
            "mixed_us_per_iteration": {"p+fold": kt32[0] * 1e6, "q=A*p (fp32, +<p,q>)": kt32[1] * 1e6,
                                       "update (+M^-1, dots)": kt32[2] * 1e6, "refresh (gated)": kt32[3] * 1e6},
            "spmv_fp64_in_solve_gbs": spmv64_bytes / kt64[1] / 1e9,
            "spmv_fp32_in_solve_gbs": spmv32_bytes / kt32[1] / 1e9,
        }
        # solver roofline: the minimum fused CG schedule per iteration, {SpMV + <p,q>},
        # {x (y), r update, z = M^-1 r, <r,z>, <r,r>}, {p = z + beta p}: the SpMV bytes +
        # 12 vector passes + the block-Jacobi factors (9 per block row); the refined
        # solver adds its FP64 refreshes (FP64 SpMV + x, y, b, r, z and the factors)
        it_mixed = int(np.median(it32s))
        bytes_it64 = spmv64_bytes + 12 * n_unk * 8 + 9 * N * 8
        bytes_it32 = spmv32_bytes + 12 * n_unk * 4 + 9 * N * 4
        bytes_refresh = spmv64_bytes + n_unk * (8 + 4 + 8 + 4 + 4) + 9 * N * 4
        total32 = it_mixed * bytes_it32 + nref * bytes_refresh
        solver_roofline = {
            "fp64": {"bytes_per_iteration": bytes_it64, "iterations": it64,
                     "achieved_gbs": it64 * bytes_it64 / t64_max / 1e9,
                     "frac_of_measured": it64 * bytes_it64 / t64_max / 1e9 / peak},
            "mixed": {"bytes_per_iteration": bytes_it32, "bytes_per_refresh": bytes_refresh, "refreshes": nref,
                      "iterations": it_mixed, "achieved_gbs": total32 / t_mixed_max / 1e9,
                      "frac_of_measured": total32 / t_mixed_max / 1e9 / peak},
        }
        achieved = in_solve["spmv_fp64_in_solve_gbs"]
        line = {
            "metric": metric_name(args.n), "value": t64_max, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t64_max * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": shared_config(args.n, nz, n_unk),
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "statistic": f"mean of {len(t64s)} solves", "step_s": t64s,
            "iterations": it64, "rel_residual": res64,
            "mixed": {"value": t_mixed_max, "unit": "s", "dtype": "f32 inner / f64 refinement",
                      "iterations": it_mixed, "fp64_refreshes": nref, "true_rel_residual": true_res,
                      "rel_error_vs_fp64_solution": err_vs_fp64, "statistic": f"mean of {len(t32s)} solves",
                      "step_s": t32s, "clocks": clocks32,
                      "e2e": {"value": float(np.mean(e2e32)), "unit": "s", **stats(e2e32)}},
            "speedup_mixed_vs_fp64": t64_max / t_mixed_max,
            "spmv": {k: {"gbs": v["gbs"], "us": v["seconds"] * 1e6, "bytes": v["bytes"],
                         "frac_of_measured": v["gbs"] / peak, "frac_of_8tbs": v["gbs"] / 8000.0}
                     for k, v in spmv.items()},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "traffic": (NCU_SPMV64_TRAFFIC_RATIO * spmv64_bytes
                                     if NCU_SPMV64_TRAFFIC_RATIO else None),
                         "traffic_source": NCU_SPMV64_TRAFFIC_SOURCE,
                         "kernel": "cg_spmv_kernel (FP64 sliced-ELL SpMV q=A*p with the fused double-double "
                                   "<p,q>), average launch inside an FP64 solve, kernel-timer mode",
                         "algorithmic_bytes_per_launch": spmv64_bytes, "peak_kind": peak_kind},
            "in_solve_kernels": in_solve,
            "solver_roofline": solver_roofline,
            "spmv_layout": layout,
            "e2e": {"value": e2e64_max, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": "monolis_solve_R (FP64), pinned host b/x, matrix uploaded every call",
                    "statistic": f"mean of {len(e2e64)} calls", **stats(e2e64), "calls": e2e64_parts},
            "gpu_launches": launches,
            "autotuned_unroll": {"fp64": u64, "fp32": u32},
            "clocks": clocks,
            "cpu_baseline": cpu,
            "assembly_s": t_asm,
            "device_assembly": asm,
            "workloads": workloads,
        }
        print(json.dumps(line), flush=True)
    m.finalize()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
