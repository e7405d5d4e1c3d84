#!/usr/bin/env python
"""Benchmark: Helmholtz combined-field dense assembly on B200.

Workload (default): regular_sphere(6) (32768 triangles), DP0 spaces, k = 10,
the indirect combined-field operator  A = DLP - 1/2 I - i k SLP  as a dense
32768 x 32768 complex128 matrix.  One step = one full assembly of A (regular
pairs + Sauter-Schwab singular pairs + identity), matrix resident in HBM.

* ``value``: entries/s of the mixed-precision assembly (FP32 regular pairs,
  FP64 singular pairs, FP64 per-entry sums), inputs already on the device.
* ``fp64``: the same for the FP64 path, plus the mixed/FP64 ratio and the
  relative Frobenius error of the mixed matrix against the FP64 matrix.
* ``e2e``: entries/s through the public operator API (``dlp - 0.5*ident -
  1j*k*slp`` then ``weak_form()``), with every step re-uploading the grid
  from pinned host memory and copying the whole matrix back into pinned host
  memory.
* ``roofline``: the regular-pair kernel (the dominant launch), algorithmic
  flops / CUDA-event time against the FP32 (or FP64) FMA peak measured in the
  same run by ``bemppcuda_fma_probe``.
* ``cpu_baseline``: the reference's own Numba path (bempp_cl installed under
  baseline/_ref, through its public API) on a seeded random row sample of the
  same operator, all host cores; the oracle port when the reference is not
  importable.  ``parity`` compares the GPU matrices with it on those rows, and
  the breadth operators with the oracle on 48 rows at their own sizes.
* ``shape_gradient``: gradients/s of the far-field objective of a perturbed
  L5 sphere (k = 6) with respect to all vertex coordinates and k, with the
  adjoint-kernel cost relative to one forward assembly and a central
  difference check on 20 coordinates.
* ``breadth``: FP64 throughput of the other operator families on their
  configurations (Laplace DP0 L4 with its matvec; Helmholtz P1 SLP / DLP /
  ADLP / hypersingular L5, k = 5; Maxwell EFIE / MFIE RWG-SNC L4, k = 2;
  Helmholtz potential at 10 000 points), each beside the oracle on the host.
* ``batch``: 64 DP0 Helmholtz single-layer problems on seeded ellipsoids
  (regular_sphere(3..5) scaled per axis, k ~ U[1, 16]) assembled in one
  persistent launch per precision after autotuning, then replayed as a CUDA
  graph together with the 8-right-hand-side product of every problem; the
  same problems assembled one launch pair at a time give the unbatched time.
  ``batch.many_small`` repeats this for 256 problems of 128 / 512 elements,
  where separate launches cannot fill the GPU.

Multi-GPU (torchrun): symmetric stripes -- rank r sweeps the element pairs
(i, j), i <= j, of its rows [lo_r, hi_r) (equal pair counts over the ranks),
keeping A_ij and the transposed A_ji in two local buffers, with no collective
(strong scaling, total work fixed, each pair's kernel work done once as on
one GPU); the distributed solve runs on the stripes.  ``--impl reference`` times the reference's CPU
path (as ``cpu_baseline``) on rank 0 only.
"""

import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "bempp-cl_b200"))
sys.path.insert(0, ROOT)
os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))

import numpy as np  # noqa: E402

# algorithmic flops per quadrature-point pair (add/sub/mul = 1, FMA = 2, sqrt,
# div, sin, cos, exp = 1 each; software expansions not counted)
FLOPS_PER_QPE = {
    "helmholtz_combined_field": 35,  # shared r, exp(ikr) of DLP and SLP
    "helmholtz_single_layer": 20,
    "helmholtz_double_layer": 30,
    "laplace_single_layer": 13,
}


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--level", type=int, default=6)
    ap.add_argument("--k", type=float, default=10.0)
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-solve", action="store_true")
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--skip-shape", action="store_true")
    ap.add_argument("--skip-fd", action="store_true")
    ap.add_argument("--skip-breadth", action="store_true")
    ap.add_argument("--shape-level", type=int, default=5)
    ap.add_argument("--shape-solver", choices=["lu32", "gmres", "gmres32"], default="lu32")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU time per baseline sample")
    ap.add_argument("--profile-case", choices=sorted(PROFILE_CASES), default=None,
                    help="run one kernel on a few-GB case (for ncu captures; prints its CUDA-event time) and exit")
    return ap.parse_args(argv)


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def row_block(n, world, rank):
    from bempp_cuda.distributed import row_block as rb

    return rb(n, world, rank)


def build_problem(level, world, rank):
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(level)
    domain = function_space(grid, "DP", 0)
    lo, hi = row_block(grid.number_of_elements, world, rank)
    dual = domain if (lo, hi) == (0, grid.number_of_elements) else function_space(
        grid, "DP", 0, support_elements=np.arange(lo, hi)
    )
    return grid, domain, dual


def combined_descriptor(k):
    from bempp_cuda.operators import OperatorDescriptor

    eta = -1j * k
    return OperatorDescriptor("helmholtz_combined_field_boundary", [k, 0.0, eta.real, eta.imag],
                              "helmholtz_combined_field", "default_scalar", "double", True, None, 1)


# ----------------------------------------------------------------------------- clocks
class ClockSampler(object):
    """nvidia-smi samples every 200 ms while the timed region runs."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.device_index = device_index
        self.proc = None
        self.path = os.path.join("/tmp", "bempp_cuda_clocks_%d.csv" % os.getpid())

    def start(self):
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device_index), "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() in ("active", "1"):
                    reasons.add(name)
        os.unlink(self.path)
        return {
            "sm_mhz": float(np.median(sm)) if sm else None,
            "sm_max_mhz": float(max(smax)) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


# ----------------------------------------------------------------------------- GPU arm
def measure_fma_peaks(torch):
    """FP32 and FP64 FMA throughput (TFLOP/s) from the library's probe kernel."""
    import ctypes

    from bempp_cuda import _lib
    from bempp_cuda.device import current_stream

    lib = _lib.load()
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    blocks = props.multi_processor_count * 8
    out = {}
    for name, prec, dtype, iters in (("fp32", _lib.MIXED, torch.float32, 20000), ("fp64", _lib.FP64, torch.float64, 10000)):
        sink = torch.zeros(blocks, dtype=dtype, device="cuda")
        flops = ctypes.c_double(0.0)
        best = 0.0
        for rep in range(4):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            _lib.check(lib.bemppcuda_fma_probe(prec, iters, blocks, ctypes.c_void_p(sink.data_ptr()),
                                               ctypes.byref(flops), current_stream()))
            e1.record()
            torch.cuda.synchronize()
            if rep:
                best = max(best, flops.value / (e0.elapsed_time(e1) * 1e-3) / 1e12)
        out[name] = best
    return out


def traffic_estimate(rows, cols):
    """DRAM bytes per regular launch: 1.054e9 B measured at 8192^2 (ncu), scaled by the entries."""
    return 1.054e9 * (rows * cols) / 8192.0**2


def gpu_arm(args, world, rank, local):
    import torch

    from bempp_cuda import _lib
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.device import clear_cache, device_grid, device_singular_rule, device_space
    from bempp_cuda.operators import Parameters

    torch.cuda.set_device(local)
    grid, domain, dual = build_problem(args.level, world, rank)
    params = Parameters()
    desc = combined_descriptor(args.k)
    rows, cols = dual.global_dof_count, domain.global_dof_count
    entries = rows * cols
    dist = None
    if world > 1:
        import torch.distributed as dist

    # device-resident inputs (uploaded once, outside the timed region)
    device_grid(grid)
    device_space(domain)
    device_space(dual)
    n_el = int(grid.number_of_elements)
    stripe = None
    if world == 1:
        rule = device_singular_rule(grid, params.quadrature.singular, dual.support, domain.support)
        npairs_singular = rule.npairs
        out = torch.empty((rows, cols), dtype=torch.complex128, device="cuda")
        rank_entries = rows * cols
    else:
        # symmetric stripes: this rank sweeps the pairs (i, j), i <= j, of rows [lo, hi) (equal pair counts
        # over the ranks) into U (A_ij) and L (A_ji), both (hi - lo) x (n - lo)
        from bempp_cuda.distributed import singular_into_stripe, stripe_bounds, stripe_entries, stripe_singular_pairs

        lo, hi = stripe_bounds(n_el, world)[rank]
        stripe = (lo, hi)
        out = torch.zeros((hi - lo, n_el - lo), dtype=torch.complex128, device="cuda")
        out_t = torch.zeros_like(out)
        rank_entries = stripe_entries(n_el, lo, hi)
        npairs_singular = stripe_singular_pairs(domain, params, lo, hi)  # builds the stripe's pair list

    def one_step(precision, events=None):
        if events is not None:
            events[0].record()
        if stripe is None:
            regular_into(out, desc, domain, dual, params, precision=precision, overwrite=True)
        else:
            regular_into(out, desc, domain, domain, params, precision=precision, overwrite=True, rows=stripe,
                         tresult=out_t, col_begin=stripe[0])
        if events is not None:
            events[1].record()
        if stripe is None:
            singular_into_dense(out, desc, domain, dual, params, diag_shift=-0.5)
        else:
            singular_into_stripe(out, out_t, stripe[0], stripe[1], desc, domain, params, diag_shift=-0.5)
        if events is not None:
            events[2].record()

    def barrier():
        if dist is not None:
            dist.barrier()

    def timed(precision, steps, warmup, sample_clocks):
        for _ in range(warmup):
            one_step(precision)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        ev = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(steps)]
        start = torch.cuda.Event(enable_timing=True)
        stop = torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(local) if sample_clocks else None
        if sampler:
            sampler.start()
            time.sleep(0.3)
        start.record()
        for s in range(steps):
            one_step(precision, ev[s])
        stop.record()
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        total_ms = start.elapsed_time(stop)
        reg_ms = [ev[s][0].elapsed_time(ev[s][1]) for s in range(steps)]
        sing_ms = [ev[s][1].elapsed_time(ev[s][2]) for s in range(steps)]
        if dist is not None:
            t = torch.tensor([total_ms], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
        return total_ms, float(np.mean(reg_ms)), float(np.mean(sing_ms)), clocks

    peaks = measure_fma_peaks(torch)

    result = {}
    # FP64 path first, keep its matrix for the operator error of the mixed path
    fp64 = None
    ref64 = None
    total_entries = int(grid.number_of_elements) ** 2
    if not args.skip_fp64:
        t64, reg64, sing64, _ = timed(_lib.FP64, args.steps, args.warmup, False)
        fp64 = {"value": total_entries * args.steps / (t64 * 1e-3), "unit": "entries/s",
                "ms_per_step": t64 / args.steps, "regular_ms": reg64, "singular_ms": sing64}
        fits = rank_entries * 16 * 3 < torch.cuda.get_device_properties(local).total_memory * 0.85
        ref64 = (out.clone() if stripe is None else (out.clone(), out_t.clone())) if fits else None
    tmx, regmx, singmx, clocks = timed(_lib.MIXED, args.steps, args.warmup, True)
    value = total_entries * args.steps / (tmx * 1e-3)
    # seeded rows of both matrices for the parity check against the CPU reference (after timing)
    gpu_rows = None
    if world == 1:
        idx = torch.as_tensor(parity_rows(rows), device="cuda")
        gpu_rows = {"mixed": out.index_select(0, idx).cpu().numpy()}
        if ref64 is not None:
            gpu_rows["fp64"] = ref64.index_select(0, idx).cpu().numpy()
    solve = None
    if fp64 is not None:
        fp64["mixed_over_fp64"] = value / fp64["value"]
        if ref64 is not None:
            if stripe is None:
                err = torch.linalg.norm(out - ref64) / torch.linalg.norm(ref64)
            else:
                err = torch.sqrt((torch.linalg.norm(out - ref64[0]) ** 2 + torch.linalg.norm(out_t - ref64[1]) ** 2)
                                 / (torch.linalg.norm(ref64[0]) ** 2 + torch.linalg.norm(ref64[1]) ** 2))
            fp64["mixed_rel_fro_err"] = float(err.item())
            if not args.skip_solve:
                if world == 1:
                    solve = solve_measure(args, torch, grid, domain, ref64, out, desc, params)
                else:
                    solve = solve_measure_distributed(args, torch, grid, domain, ref64, world, rank, dist)
            del ref64
        torch.cuda.empty_cache()

    # roofline of the regular-pair kernel (mixed precision); entries of this rank's block or stripe
    regular_pairs = rank_entries - npairs_singular
    qpe = 36 * regular_pairs
    flops = qpe * FLOPS_PER_QPE["helmholtz_combined_field"]
    achieved = flops / (regmx * 1e-3) / 1e12
    roof = {"bound": "fp32", "achieved": achieved, "peak": peaks["fp32"], "unit": "TFLOP/s",
            "frac": achieved / peaks["fp32"], "traffic": traffic_estimate(rank_entries, 1),
            "kernel": "regular_dp0_mixed_sym<HELMHOLTZ_COMBINED>", "kernel_ms": regmx,
            "flops_per_qpe": FLOPS_PER_QPE["helmholtz_combined_field"], "qpe_per_launch": qpe,
            "flops_convention": "algorithmic flops of evaluating every entry on its own (the reference's "
                                "work); the symmetric sweep evaluates each point pair once for A_ij and A_ji, "
                                "so the hardware evaluates qpe_per_launch / 2 point pairs",
            "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the same kernel at "
                              "regular_sphere(5), scaled by the entry count; the output write is the whole "
                              "traffic",
            "peak_source": "bemppcuda_fma_probe, measured in this run"}
    if fp64 is not None:
        a64 = flops / (fp64["regular_ms"] * 1e-3) / 1e12
        fp64["roofline"] = {"bound": "fp64", "achieved": a64, "peak": peaks["fp64"], "unit": "TFLOP/s",
                            "frac": a64 / peaks["fp64"], "kernel_ms": fp64["regular_ms"]}

    # end to end through the public API (host in, host out)
    e2e = None
    if not args.skip_e2e:
        e2e = e2e_measure(args, torch, grid, domain, dual, world, dist, clear_cache, total_entries)

    batch = None
    if not args.skip_batch:
        del out
        torch.cuda.empty_cache()
        batch = batch_measure(args, torch, world, rank, dist)
        torch.cuda.empty_cache()
        batch["many_small"] = batch_measure(args, torch, world, rank, dist, count=256, levels=(2, 3))
        del batch["many_small"]["elements"]
    breadth = None
    if not args.skip_breadth and world == 1:
        torch.cuda.empty_cache()
        breadth = breadth_measure(args, torch, peaks["fp64"], peaks["fp32"])
    shape = None
    if not args.skip_shape and world == 1:
        torch.cuda.empty_cache()
        shape = shape_measure(args, torch)

    line = {
        "metric": METRIC,
        "value": value,
        "unit": "entries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": tmx / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f32+f64",
        "data": "synthetic: regular_sphere(%d) unit sphere, generated by octahedron subdivision" % args.level,
        "config": bench_config(args),
        "precision": "mixed: FP32 regular pairs, FP64 singular pairs and per-entry sums",
        "parallelism": ("symmetric stripes x%d (equal pair counts; U and L per rank)" % world) if world > 1
                       else "one GPU",
        "gpu_launches": 2 * args.steps,
        "clocks": clocks,
        "roofline": roof,
        "fp64": fp64,
        "fma_peaks_tflops": peaks,
        "regular_ms": regmx,
        "singular_ms": singmx,
    }
    if e2e is not None:
        line["e2e"] = e2e
    if solve is not None:
        line["solve"] = solve
    if batch is not None:
        line["batch"] = batch
    if shape is not None:
        line["shape_gradient"] = shape
    if breadth is not None:
        line["breadth"] = breadth
        checks = {e["operator"]: e["parity_rel_fro_vs_oracle"] for e in breadth if "parity_rel_fro_vs_oracle" in e}
        if checks:
            line["parity"] = {"breadth_fp64_vs_oracle": checks, "bound": 1e-12,
                              "sample": "48 seeded rows per operator at its configured level; 500 of the 10 000 "
                                        "potential points"}
    return line, gpu_rows


def hbm_peak():
    """(GB/s, source): the driver's measured copy bandwidth, else the fallback figure of this pool."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured copy)"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback 6.65 TB/s"


def matvec_measure(torch, a64):
    """GEMV on the resident matrix (the GMRES matvec): HBM-bound, one read of the matrix per product.
    The library's kernel (bemppcuda_gemv, used by the solves) beside cuBLAS through torch.mv."""
    from bempp_cuda.matmat import gemv

    peak, source = hbm_peak()
    n = a64.shape[0]
    out = {"peak_gbs": peak, "peak_source": source}
    a32 = a64.to(torch.complex64)
    for name, mat in (("complex128", a64), ("complex64", a32)):
        x = torch.ones(n, dtype=mat.dtype, device="cuda")
        nbytes = mat.numel() * mat.element_size()
        entry = {"bytes": nbytes}
        for impl, fn in (("library", lambda: gemv(mat, x)), ("cublas", lambda: torch.mv(mat, x))):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(10):
                fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / 10
            gbs = nbytes / (ms * 1e-3) / 1e9
            entry[impl] = {"ms": ms, "gbs": gbs, "frac": gbs / peak}
        ref = torch.mv(mat, x)
        entry["library_rel_diff_vs_cublas"] = float((torch.linalg.norm(gemv(mat, x) - ref) / torch.linalg.norm(ref)).item())
        out[name] = entry
    del a32
    torch.cuda.empty_cache()
    return out


def solve_measure(args, torch, grid, domain, a64, amx, desc, params):
    """C3 solve: plane wave exp(i k z).  FP64 GMRES on the FP64 matrix against the mixed matrix with
    iterative refinement whose residuals use the FP64 operator, evaluated matrix-free (the mixed
    matrix only preconditions the corrections), both to relative residual 1e-8; then both again to
    1e-11, where the two solutions must agree to 1e-8."""
    from bempp_cuda.grid_function import GridFunction
    from bempp_cuda.linalg import gmres_tensor, solve_refined
    from bempp_cuda.matmat import matvec_of
    from bempp_cuda.operators import fp64_matvec_of

    k = args.k

    def minus_incident(x, n, domain_index, result):
        result[0] = -np.exp(1j * k * x[2])

    b = torch.as_tensor(GridFunction(domain, fun=minus_incident).projections(domain), device="cuda")
    fp64_apply = fp64_matvec_of(desc, 1.0, domain, params, amx)
    # warm-up (first-call costs of the solver's kernels and host loop), so both solves are timed warm
    gemv64 = matvec_of(a64)
    gmres_tensor(gemv64, b, tol=1e-8, restart=200, maxiter=5)
    fp64_apply(b)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(3):
        fp64_apply(b)
    e1.record()
    torch.cuda.synchronize()
    apply_ms = e0.elapsed_time(e1) / 3
    out = {"rhs": "projection of -exp(i k z) onto DP0", "fp64_residual_apply_ms": apply_ms,
           "fp64_residual_apply_note": "FP64 operator product without the FP64 matrix: regular pairs evaluated "
                                       "on the fly (bemppcuda_apply_regular) + adjacent entries of the mixed matrix"}
    solutions = {}
    for tol in (1e-8, 1e-11):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        x64, info, res, its = gmres_tensor(gemv64, b, tol=tol, restart=200, maxiter=2000)
        torch.cuda.synchronize()
        t64 = time.perf_counter() - t0
        xmx, rinfo = solve_refined(amx, b, tol=tol, inner_tol=1e-4, restart=200, residual=fp64_apply)
        res_true = float((torch.linalg.norm(b - torch.mv(a64, xmx)) / torch.linalg.norm(b)).item())
        out["tol_%g" % tol] = {
            "fp64": {"iterations": its, "info": info, "seconds": t64, "final_residual": res[-1]},
            "mixed_refined": {"refinements": rinfo["refinements"], "inner_iterations": rinfo["inner_iterations"],
                              "residuals": rinfo["relative_residuals"], "seconds": rinfo["seconds"],
                              "inner_dtype": "complex64", "residual_operator": "FP64, matrix-free"},
            "mixed_solution_residual_in_fp64_matrix": res_true,
        }
        solutions[tol] = (x64, xmx)
    x64, xmx = solutions[1e-11]
    out["solution_rel_diff_vs_fp64"] = float((torch.linalg.norm(xmx - x64) / torch.linalg.norm(x64)).item())
    x64, xmx = solutions[1e-8]
    out["solution_rel_diff_vs_fp64_at_tol_1e-8"] = float(
        (torch.linalg.norm(xmx - x64) / torch.linalg.norm(x64)).item())
    out["note"] = ("solution_rel_diff_vs_fp64 compares both solves run to relative residual 1e-11 (bound 1e-8); "
                   "at 1e-8 each solution carries its own GMRES error of about cond x 1e-8")
    out["matvec"] = matvec_measure(torch, a64)
    return out


def batch_measure(args, torch, world, rank, dist, count=64, levels=(3, 4, 5)):
    """``count`` DP0 Helmholtz SLP problems (ellipsoids L in ``levels``, k ~ U[1,16]) in one persistent launch.

    Each precision is autotuned, then one CUDA graph holding the batched
    assembly and the 8-right-hand-side products of every problem is replayed.
    The same problems assembled one after another through the single-problem
    kernels give the unbatched time.
    """
    from bempp_cuda import _lib, operators
    from bempp_cuda.assembly import regular_into, singular_into_dense
    from bempp_cuda.batch import BatchAssembler, c4_problems
    from bempp_cuda.operators import Parameters

    probs = c4_problems(count, seed=0, levels=levels)
    from bempp_cuda.distributed import shard_problems

    mine = shard_problems([g.number_of_elements for g, _ in probs], world, rank)
    grids = [probs[i][0] for i in mine]
    ks = [probs[i][1] for i in mine]
    rhs = []
    for i in mine:
        rng = np.random.default_rng(1000 + i)
        n = probs[i][0].number_of_elements
        rhs.append(torch.as_tensor(rng.standard_normal((n, 8)) + 1j * rng.standard_normal((n, 8)), device="cuda"))
    entries_all = sum(g.number_of_elements ** 2 for g, _ in probs)

    def max_ms(ms):
        if dist is None:
            return ms
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def events_ms(fn, steps):
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return max_ms(e0.elapsed_time(e1) / steps)

    res = {"problems": len(probs), "elements": sorted(g.number_of_elements for g, _ in probs),
           "entries": entries_all, "rhs_per_problem": 8, "shards": "largest-first onto least-loaded rank"}
    outputs64 = None
    for prec in ("fp64", "mixed"):
        ba = BatchAssembler(grids, ks, precision=prec)
        t0 = time.perf_counter()
        shape, timings = ba.autotune()
        tune_s = time.perf_counter() - t0
        prods = [torch.empty_like(x) for x in rhs]
        ba.capture(rhs, prods)
        for _ in range(args.warmup):
            ba.replay()
        launch_ms = events_ms(ba.launch, args.steps)
        # assembly + 8-RHS products: issued eagerly, then replayed from the graph
        eager_ms = events_ms(lambda: ba.step(rhs, prods), args.steps)
        graph_ms = events_ms(ba.replay, args.steps)
        entry = {"rows_per_item": shape[0], "ctas_per_sm": shape[1], "autotune_s": tune_s,
                 "shapes_timed": len(timings), "launch_ms": launch_ms,
                 "entries_per_s": entries_all / (launch_ms * 1e-3),
                 "step_with_products": {"eager_ms": eager_ms, "graph_ms": graph_ms,
                                        "graph_speedup": eager_ms / graph_ms,
                                        "products_ms": graph_ms - launch_ms,
                                        "entries_per_s": entries_all / (graph_ms * 1e-3)}}
        if prec == "fp64":
            # the batched 8-RHS product kernel alone against one library GEMM per problem
            prod_ms = events_ms(ba._product.launch, args.steps)
            torch_ms = events_ms(lambda: [torch.matmul(a, x, out=y) for a, x, y in zip(ba.outputs, rhs, prods)],
                                 args.steps)
            nbytes = sum(16 * (o.shape[0] * o.shape[1] + (o.shape[0] + o.shape[1]) * x.shape[1])
                         for o, x in zip(ba.outputs, rhs))
            peak, source = hbm_peak()
            entry["products"] = {"kernel": "matmat_c128_tc<8> (FP64 tensor cores, one launch, all problems)", "kernel_ms": prod_ms,
                                 "torch_matmul_ms": torch_ms, "bytes": nbytes,
                                 "gbs": nbytes / (prod_ms * 1e-3) / 1e9,
                                 "frac": nbytes / (prod_ms * 1e-3) / 1e9 / peak, "peak_gbs": peak,
                                 "peak_source": source}
            outputs64 = [o.clone() for o in ba.outputs]
        else:
            errs = [(torch.linalg.norm(a - b) / torch.linalg.norm(b)).item() for a, b in zip(ba.outputs, outputs64)]
            entry["max_rel_fro_err_vs_fp64"] = max(errs) if errs else 0.0
        res[prec] = entry
        del ba, prods
        torch.cuda.empty_cache()
    del outputs64

    # unbatched: the same problems one by one (two launches each), device inputs resident
    params = Parameters()
    singles = []
    for g, k in zip(grids, ks):
        from bempp_cuda.space import function_space

        sp = function_space(g, "DP", 0)
        desc = operators.boundary.helmholtz.single_layer(sp, sp, sp, k).descriptor
        singles.append((sp, desc, torch.empty((g.number_of_elements,) * 2, dtype=torch.complex128, device="cuda")))

    def sequential(precision):
        def run():
            for sp, desc, out in singles:
                regular_into(out, desc, sp, sp, params, precision=precision, overwrite=True)
                singular_into_dense(out, desc, sp, sp, params)
        return run

    for prec, code in (("fp64", _lib.FP64), ("mixed", _lib.MIXED)):
        run = sequential(code)
        for _ in range(args.warmup):
            run()
        ms = events_ms(run, args.steps)
        res[prec]["unbatched_ms"] = ms
        res[prec]["batched_speedup"] = ms / res[prec]["launch_ms"]
    res["mixed_over_fp64"] = res["mixed"]["entries_per_s"] / res["fp64"]["entries_per_s"]
    del singles
    torch.cuda.empty_cache()
    return res


def shape_measure(args, torch):
    """Shape gradient of J = sum_j |u_inf(d_j)|^2 (32 Fibonacci directions) on a perturbed L5 sphere, k = 6.

    One step = forward (device geometry, combined-field assembly, LU, solve,
    far field, J) + backward (adjoint solve, adjoint kernels).  The adjoint
    kernels are compared with one forward assembly (regular + singular pass).
    Central differences (h = 1e-6) on 20 seeded coordinates and on k check
    the gradient at this size.
    """
    from bempp_cuda.matmat import matvec_of
    from bempp_cuda.shape_gradient import FarFieldObjective
    from bempp_cuda.shapes import perturbed_sphere

    grid, _ = perturbed_sphere(args.shape_level, seed=0)
    solver = args.shape_solver
    obj = FarFieldObjective(grid, solver=solver, tol=1e-12)
    k = 6.0
    x0 = obj.vertices.clone()
    names = ("geometry", "assembly", "solve", "farfield", "adjoint_solve", "adjoint_kernels")
    from bempp_cuda.shape_gradient import ScatteringState

    iters = {}

    def step(ev=None):
        def mark(i):
            if ev is not None:
                ev[i].record()
        mark(0)
        geo = obj.geometry(x0)
        mark(1)
        a = obj.assemble(geo, k)
        mark(2)
        b = obj.rhs(geo, k)
        if solver == "lu32":
            lu, piv = torch.linalg.lu_factor(a.to(torch.complex64))
            phi, its = obj._refine(lu, piv, matvec_of(a), b)
            low = None
            iters["forward_refinements"] = its
        elif solver == "gmres32":
            lu = piv = None
            low = a.to(torch.complex64)
            phi, its = obj._gmres32(matvec_of(a), matvec_of(low), b)
            iters["forward_inner_iterations"] = its
        else:  # gmres
            lu = piv = low = None
            phi, its = obj._gmres(matvec_of(a), b)
            iters["forward_iterations"] = its
        mark(3)
        ff = obj.farfield_matrix(geo, k)
        u = ff @ phi
        value = (u.real ** 2 + u.imag ** 2).sum()
        mark(4)
        state = ScatteringState(geo, lu, piv, phi, u, ff, a, its, low)
        lam = obj.adjoint(state)
        mark(5)
        vgrad, kgrad = obj.gradient(state, k, lam=lam)
        mark(6)
        return value, vgrad, kgrad

    for _ in range(max(args.warmup, 1)):
        step()
    torch.cuda.synchronize()
    steps = max(args.steps, 1)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(7)] for _ in range(steps)]
    t0 = time.perf_counter()
    for s in range(steps):
        value, vgrad, kgrad = step(evs[s])
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) / steps
    parts = {n: float(np.mean([evs[s][i].elapsed_time(evs[s][i + 1]) for s in range(steps)]))
             for i, n in enumerate(names)}
    device_ms = evs[0][0].elapsed_time(evs[-1][6]) / steps
    res = {"workload": "perturbed regular_sphere(%d) (%d elements, %d vertices), k=6, DP0 combined field, "
                       "32 Fibonacci far-field directions, incident exp(i k z)"
                       % (args.shape_level, grid.number_of_elements, obj.base.nvertices),
           "shape_grads_per_s": 1e3 / max(device_ms, wall * 1e3),
           "ms_per_gradient": max(device_ms, wall * 1e3), "parts_ms": parts,
           "adjoint_kernels_over_forward_assembly": parts["adjoint_kernels"] / parts["assembly"],
           "backward_over_forward": (parts["adjoint_solve"] + parts["adjoint_kernels"])
           / (parts["geometry"] + parts["assembly"] + parts["solve"] + parts["farfield"]),
           "solver": ("complex64 LU (cuSOLVER via torch) refined with complex128 residuals of the FP64 matrix to "
                      "relative residual 1e-12; the adjoint reuses the factors") if solver == "lu32" else
                     ("GMRES on a complex64 copy of the matrix (inner tolerance 1e-5) refined with complex128 "
                      "residuals of the FP64 matrix to relative residual 1e-12, forward and adjoint (transposed "
                      "view)") if solver == "gmres32" else
                     ("GMRES on the complex128 matrix to relative residual 1e-12, forward and adjoint (transposed "
                      "view); each Arnoldi step one CUDA-graph replay, convergence checked every 16 steps"),
           "refinements": dict(iters),
           "J": float(value.item())}
    if not args.skip_fd:
        h = 1e-6
        rng = np.random.default_rng(7)
        flat = rng.choice(obj.base.nvertices * 3, size=20, replace=False)
        fd, ad = [], []
        for f in flat:
            v, c = int(f) // 3, int(f) % 3
            xp = x0.clone()
            xm = x0.clone()
            xp[v, c] += h
            xm[v, c] -= h
            fd.append((obj.evaluate(xp, k, solver="lu").item() - obj.evaluate(xm, k, solver="lu").item()) / (2 * h))
            ad.append(vgrad[v, c].item())
        fd = np.array(fd)
        ad = np.array(ad)
        fdk = (obj.evaluate(x0, k + h, solver="lu").item() - obj.evaluate(x0, k - h, solver="lu").item()) / (2 * h)
        # the same coordinates with the fourth-order stencil (f(-2H) - 8 f(-H) + 8 f(H) - f(2H)) / (12 H),
        # H = 1e-4: truncation O(H^4) and roundoff eps_J |J| / H both far below the h = 1e-6 central
        # difference's roundoff, which dominates on the small gradient components
        H = 1e-4
        fd4 = []
        for f in flat:
            v, c = int(f) // 3, int(f) % 3
            vals = []
            for step in (-2, -1, 1, 2):
                xs = x0.clone()
                xs[v, c] += step * H
                vals.append(obj.evaluate(xs, k, solver="lu").item())
            fd4.append((vals[0] - 8 * vals[1] + 8 * vals[2] - vals[3]) / (12 * H))
        fd4 = np.array(fd4)
        res["fd_check"] = {"h": h, "coordinates": 20,
                           "fd_solver": "complex128 dense LU (independent of the refined complex64 solve above)",
                           "rel_err_norm": float(np.linalg.norm(ad - fd) / np.linalg.norm(fd)),
                           "max_rel_err": float(np.max(np.abs(ad - fd) / np.abs(fd))),
                           "max_err_over_max_grad": float(np.max(np.abs(ad - fd)) / np.max(np.abs(fd))),
                           "fourth_order_H": H,
                           "fourth_order_rel_err_norm": float(np.linalg.norm(ad - fd4) / np.linalg.norm(fd4)),
                           "fourth_order_max_rel_err": float(np.max(np.abs(ad - fd4) / np.abs(fd4))),
                           "central_vs_fourth_order_max_rel": float(np.max(np.abs(fd - fd4) / np.abs(fd4))),
                           "smallest_component_over_max": float(np.min(np.abs(fd4)) / np.max(np.abs(fd4))),
                           "k_rel_err": float(abs(kgrad.item() - fdk) / abs(fdk)),
                           "criterion": "per coordinate relative error <= 1e-6 against the fourth-order stencil; "
                                        "the h = 1e-6 central difference is reported as configured, its "
                                        "per-coordinate error is its own roundoff (central_vs_fourth_order)"}
    return res


# (name, factory path, domain space, dual space, level, wavenumber, algorithmic flops per point pair)
# Flops per point pair (same convention as FLOPS_PER_QPE): kernels 13 (Laplace SLP), 20
# (Helmholtz SLP), 30 (Helmholtz DLP / ADLP); a 3 x 3 shape product block adds 2 * 9 (P1);
# the hypersingular form adds 2 * 9 more for the k^2 n.n term; Maxwell EFIE adds 9 x (5 for
# the RWG dot product + 4 for the complex accumulation), MFIE 9 x (9 cross product + 5 dot
# + 4 accumulation) on top of the Helmholtz DLP factor.
BREADTH = [
    ("laplace.single_layer dp0", "laplace.single_layer", ("DP", 0), ("DP", 0), 4, None, 13),
    ("helmholtz.single_layer p1", "helmholtz.single_layer", ("P", 1), ("P", 1), 5, 5.0, 38),
    ("helmholtz.double_layer p1", "helmholtz.double_layer", ("P", 1), ("P", 1), 5, 5.0, 48),
    ("helmholtz.adjoint_double_layer p1", "helmholtz.adjoint_double_layer", ("P", 1), ("P", 1), 5, 5.0, 48),
    ("helmholtz.hypersingular p1", "helmholtz.hypersingular", ("P", 1), ("P", 1), 5, 5.0, 56),
    ("maxwell.electric_field rwg/snc", "maxwell.electric_field", ("RWG", 0), ("SNC", 0), 4, 2.0, 101),
    ("maxwell.magnetic_field rwg/snc", "maxwell.magnetic_field", ("RWG", 0), ("SNC", 0), 4, 2.0, 192),
]


def breadth_measure(args, torch, fp64_peak=None, fp32_peak=None):
    """FP64 throughput of the other operator families (dense weak form through the operator API).

    GPU: CUDA events around the full assembly (regular + singular passes) of
    each operator on its configuration, inputs resident.  CPU: the oracle
    (port) on 48 seeded rows of the same operator at the same level, with all
    host cores; the same rows of the GPU matrix are its FP64 parity check
    (``parity_rel_fro_vs_oracle``, bound 1e-12).  Potential: 10 000 points in
    the shell 1.5 < r < 3 from complex N(0,1) P1 coefficients on the level-5
    sphere; the oracle evaluates 500 seeded points of them.
    """
    from bempp_cuda import operators
    from bempp_cuda.quadrature import SingularPairs, triangle_rule
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    from oracle import oracle as orc

    grids = {}

    def grid_of(level):
        if level not in grids:
            grids[level] = regular_sphere(level)
        return grids[level]

    def factory(path):
        obj = operators.boundary
        for part in path.split("."):
            obj = getattr(obj, part)
        return obj

    def build(path, dsp, tsp, level, k):
        g = grid_of(level)
        dom = function_space(g, *dsp)
        dual = function_space(g, *tsp)
        f = factory(path)
        return (f(dom, dom, dual) if k is None else f(dom, dom, dual, k)), dom, dual

    out = []
    for name, path, dsp, tsp, level, k, flops_pp in BREADTH:
        op, dom, dual = build(path, dsp, tsp, level, k)
        op._assemble()  # uploads and warms
        torch.cuda.synchronize()
        ms = []
        for _ in range(max(args.steps, 1)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            mat = op._assemble()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
            del mat
        rows, cols = dual.global_dof_count, dom.global_dof_count
        entry = {"operator": name, "level": level, "k": k, "shape": [rows, cols],
                 "gpu_ms": float(np.median(ms)), "gpu_entries_per_s": rows * cols / (np.median(ms) * 1e-3)}
        ne = dom.grid.number_of_elements
        qpe = 36.0 * ne * ne  # regular point pairs of every element pair, counted per pair as the reference does
        achieved = qpe * flops_pp / (np.median(ms) * 1e-3) / 1e12
        entry["roofline"] = {"bound": "fp64", "flops_per_qpe": flops_pp, "qpe": qpe, "achieved": achieved,
                             "unit": "TFLOP/s", "peak": fp64_peak,
                             "frac": achieved / fp64_peak if fp64_peak else None}
        if not args.skip_cpu:
            # oracle (port) on a seeded sample of rows of the same operator: CPU rate and FP64 parity
            d = op.descriptor
            qp, qw = triangle_rule(4)
            sample = np.sort(np.random.default_rng(48).choice(rows, min(48, rows), replace=False))
            t0 = time.perf_counter()
            ref_rows = orc.assemble_rows(d.kernel_type, d.assembly_type, d.options, d.is_complex, dom, dual, sample,
                                         qp, qw, 4)
            tc = time.perf_counter() - t0
            got = op._assemble().tensor.index_select(0, torch.as_tensor(sample, device="cuda")).cpu().numpy()
            entry["cpu_rows"] = int(len(sample))
            entry["cpu_entries_per_s"] = len(sample) * cols / tc
            entry["gpu_over_cpu"] = entry["gpu_entries_per_s"] / entry["cpu_entries_per_s"]
            entry["parity_rel_fro_vs_oracle"] = float(np.linalg.norm(got - ref_rows) / np.linalg.norm(ref_rows))
        if name.startswith("laplace"):
            # C1 matvec: HBM-bound GEMV on the resident matrix
            mat = op._assemble()
            x = torch.as_tensor(np.random.default_rng(0).standard_normal(cols), device="cuda")
            for _ in range(3):
                mat @ x
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(20):
                mat @ x
            e1.record()
            torch.cuda.synchronize()
            entry["matvec_us"] = e0.elapsed_time(e1) * 1e3 / 20
            entry["matvec_note"] = "2048^2 f64 = 33.5 MB, resident in the 126 MB L2 between calls"
            del mat
        out.append(entry)
        torch.cuda.empty_cache()

    # mixed precision on P1 (device_interface "cuda_mixed"): FP32 regular pairs, against the FP64 weak form
    for name, path, level, k, flops_pp in (("helmholtz.single_layer p1 mixed", "helmholtz.single_layer", 5, 5.0, 38),
                                           ("helmholtz.double_layer p1 mixed", "helmholtz.double_layer", 5, 5.0, 48),
                                           ("helmholtz.adjoint_double_layer p1 mixed",
                                            "helmholtz.adjoint_double_layer", 5, 5.0, 48),
                                           ("helmholtz.hypersingular p1 mixed", "helmholtz.hypersingular", 5, 5.0, 56),
                                           ("maxwell.electric_field rwg/snc mixed", "maxwell.electric_field", 4, 2.0,
                                            101),
                                           ("maxwell.magnetic_field rwg/snc mixed", "maxwell.magnetic_field", 4, 2.0,
                                            192)):
        g = grid_of(level)
        if path.startswith("maxwell"):
            sp, dual = function_space(g, "RWG", 0), function_space(g, "SNC", 0)
        else:
            sp = dual = function_space(g, "P", 1)
        f = factory(path)
        op64, opmx = f(sp, sp, dual, k), f(sp, sp, dual, k, device_interface="cuda_mixed")
        ref = op64._assemble()
        opmx._assemble()
        torch.cuda.synchronize()
        ms = []
        for _ in range(max(args.steps, 1)):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            mat = opmx._assemble()
            e1.record()
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        err = float((torch.linalg.norm(mat.tensor - ref.tensor) / torch.linalg.norm(ref.tensor)).item())
        rows, cols = dual.global_dof_count, sp.global_dof_count
        ne = g.number_of_elements
        qpe = 36.0 * ne * ne
        gms = float(np.median(ms))
        achieved = qpe * flops_pp / (gms * 1e-3) / 1e12
        from bempp_cuda.assembly import FP64_FALLBACKS

        fallback = any(key[1] == opmx.descriptor.kernel_type and key[2] == opmx.descriptor.assembly_type
                       for key in FP64_FALLBACKS)
        out.append({"operator": name, "level": level, "k": k, "shape": [rows, cols], "gpu_ms": gms,
                    "gpu_entries_per_s": rows * cols / (gms * 1e-3), "rel_fro_err_vs_fp64": err,
                    "roofline": {"bound": "fp64" if fallback else "fp32", "flops_per_qpe": flops_pp, "qpe": qpe,
                                 "achieved": achieved, "unit": "TFLOP/s",
                                 "peak": fp64_peak if fallback else fp32_peak,
                                 "frac": achieved / (fp64_peak if fallback else fp32_peak)
                                 if (fp64_peak if fallback else fp32_peak) else None},
                    "note": ("no mixed-precision kernel: FP64 under cuda_mixed" if fallback else
                             "FP32 regular pairs, FP64 singular pairs and per-pair blocks")})
        del ref, mat
        torch.cuda.empty_cache()

    # potential: 10 000 shell points, P1 coefficients, k = 5
    g = grid_of(5)
    sp = function_space(g, "P", 1)
    rng = np.random.default_rng(1)
    dirs = rng.standard_normal((3, 10000))
    dirs /= np.linalg.norm(dirs, axis=0)
    pts = dirs * (1.5**3 + rng.random(10000) * (3.0**3 - 1.5**3)) ** (1.0 / 3.0)
    coeffs = rng.standard_normal(sp.global_dof_count) + 1j * rng.standard_normal(sp.global_dof_count)
    pot = operators.potential.helmholtz.single_layer(sp, pts, 5.0)
    pot.evaluate_device(coeffs)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(max(args.steps, 1)):
        pot.evaluate_device(coeffs)
    e1.record()
    torch.cuda.synchronize()
    pms = e0.elapsed_time(e1) / max(args.steps, 1)
    # the same evaluation with points and element coefficients already on the device
    from bempp_cuda.assembly import evaluate_potential_device

    pts_dev = torch.as_tensor(np.ascontiguousarray(pts.T), device="cuda")
    local_dev = torch.as_tensor(sp.map_to_full_grid @ coeffs, device="cuda")
    for _ in range(3):
        evaluate_potential_device(sp, pot.descriptor, pts_dev, local_dev, pot.parameters)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(max(args.steps, 1) * 5):
        evaluate_potential_device(sp, pot.descriptor, pts_dev, local_dev, pot.parameters)
    e1.record()
    torch.cuda.synchronize()
    kms = e0.elapsed_time(e1) / (max(args.steps, 1) * 5)
    qpe = 10000 * g.number_of_elements * 6
    pach = qpe * 28 / (kms * 1e-3) / 1e12  # 20 (kernel) + 8 (complex multiply-accumulate) per point pair
    pentry = {"operator": "potential.helmholtz.single_layer p1", "level": 5, "k": 5.0, "points": 10000,
              "gpu_ms": pms, "kernel_ms": kms, "gpu_qpe_per_s": qpe / (kms * 1e-3),
              "roofline": {"bound": "fp64", "flops_per_qpe": 28, "qpe": qpe, "achieved": pach, "unit": "TFLOP/s",
                           "peak": fp64_peak, "frac": pach / fp64_peak if fp64_peak else None},
              "note": "gpu_ms: public API call with the coefficient upload and the device gather to element slots; "
                      "kernel_ms: device-resident points and element coefficients (source table + evaluation)"}
    if not args.skip_cpu:
        # oracle (port) at 500 seeded points of the 10 000: CPU rate (scaled to 10 000) and FP64 parity
        qp, qw = triangle_rule(4)
        d = pot.descriptor
        pick = np.sort(np.random.default_rng(500).choice(10000, 500, replace=False))
        t0 = time.perf_counter()
        ref_pts = orc.evaluate_potential(d.kernel_type, d.assembly_type, d.options, sp, pts[:, pick], coeffs, qp, qw)
        tc = (time.perf_counter() - t0) * 20.0
        got = pot.evaluate(coeffs)[:, pick]
        pentry["cpu_s_scaled"] = tc
        pentry["gpu_over_cpu"] = tc / (pms * 1e-3)
        pentry["parity_points"] = 500
        pentry["parity_rel_fro_vs_oracle"] = float(np.linalg.norm(got - ref_pts) / np.linalg.norm(ref_pts))
    out.append(pentry)
    # the same potential with FP32 point-source pairs (device_interface="cuda_mixed")
    from bempp_cuda import _lib

    ref = evaluate_potential_device(sp, pot.descriptor, pts_dev, local_dev, pot.parameters)
    for _ in range(3):
        evaluate_potential_device(sp, pot.descriptor, pts_dev, local_dev, pot.parameters, precision=_lib.MIXED)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(max(args.steps, 1) * 5):
        mix = evaluate_potential_device(sp, pot.descriptor, pts_dev, local_dev, pot.parameters, precision=_lib.MIXED)
    e1.record()
    torch.cuda.synchronize()
    mms = e0.elapsed_time(e1) / (max(args.steps, 1) * 5)
    mach = qpe * 28 / (mms * 1e-3) / 1e12
    out.append({"operator": "potential.helmholtz.single_layer p1 mixed", "level": 5, "k": 5.0, "points": 10000,
                "gpu_ms": mms, "kernel_ms": mms, "gpu_qpe_per_s": qpe / (mms * 1e-3),
                "rel_fro_err_vs_fp64": float((torch.linalg.norm(mix - ref) / torch.linalg.norm(ref)).item()),
                "over_fp64_kernel": kms / mms,
                "roofline": {"bound": "fp32", "flops_per_qpe": 28, "qpe": qpe, "achieved": mach, "unit": "TFLOP/s",
                             "peak": fp32_peak, "frac": mach / fp32_peak if fp32_peak else None},
                "note": "device-resident points and element coefficients; FP32 point-source pairs, FP64 "
                        "per-element phase and sums"})
    return out


def solve_measure_distributed(args, torch, grid, domain, stripes, world, rank, dist):
    """C3 solve on symmetric stripes: FP64 GMRES, per matvec one all-gather of the iterate and one
    all-reduce of the product (NCCL)."""
    from bempp_cuda.distributed import StripeOperator, gmres_distributed
    from bempp_cuda.grid_function import GridFunction

    k = args.k

    def minus_incident(x, n, domain_index, result):
        result[0] = -np.exp(1j * k * x[2])

    n = grid.number_of_elements
    op = StripeOperator(stripes[0], stripes[1], n, world, rank)
    lo, hi = op.local_range
    b = GridFunction(domain, fun=minus_incident).projections(domain)
    b_local = torch.as_tensor(b[lo:hi], device="cuda")
    torch.cuda.synchronize()
    dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    x_local, info, res, its = gmres_distributed(op, b_local, tol=1e-8, restart=200, maxiter=2000)
    e1.record()
    torch.cuda.synchronize()
    t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    r_local = b_local - op.matvec(x_local)
    rr = torch.stack([torch.linalg.vector_norm(r_local) ** 2, torch.linalg.vector_norm(b_local) ** 2])
    dist.all_reduce(rr)
    return {"rhs": "projection of -exp(i k z) onto DP0", "tol": 1e-8, "ranks": world,
            "fp64_distributed": {"iterations": its, "info": info, "seconds": float(t.item()) / 1e3,
                                 "final_residual": res[-1],
                                 "true_residual": float(torch.sqrt(rr[0] / rr[1]).item()),
                                 "collectives": "per iteration: all-gather of the iterate and all-reduce of the "
                                                "stripe products (NCCL), all-reduce of the orthogonalisation "
                                                "coefficients and norms"}}


def e2e_measure(args, torch, grid, domain, dual, world, dist, clear_cache, total_entries):
    """Public-API steps: pinned host grid in, pinned host matrix out."""
    from bempp_cuda import operators
    from bempp_cuda.grid import Grid
    from bempp_cuda.space import function_space

    rows, cols = dual.global_dof_count, domain.global_dof_count
    host_out = torch.empty((rows, cols), dtype=torch.complex128, pin_memory=True)
    # the user's host objects: grid and spaces are built once, as in a bempp script
    g = Grid(np.asarray(grid.vertices), np.asarray(grid.elements))
    d = function_space(g, "DP", 0)
    lo = int(dual.support_elements[0])
    t = d if rows == cols else function_space(g, "DP", 0, support_elements=np.arange(lo, lo + rows))

    def step():
        # device copies are dropped, so every step uploads vertices, elements, dof maps and singular tables
        for obj in (g, d, t):
            clear_cache(obj, device_only=True)
        slp = operators.boundary.helmholtz.single_layer(d, d, t, args.k, device_interface="cuda_mixed")
        dlp = operators.boundary.helmholtz.double_layer(d, d, t, args.k, device_interface="cuda_mixed")
        ident = operators.boundary.sparse.identity(d, d, t, device_interface="cuda_mixed")
        lhs = dlp - 0.5 * ident - 1j * args.k * slp
        # the weak form as a host matrix (what the reference returns); the copy overlaps the assembly
        operators.weak_form_to_host(lhs, out=host_out)

    for _ in range(max(1, args.warmup)):
        step()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(args.steps):
        step()
    stop.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = max(start.elapsed_time(stop), wall * 1e3)
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    from bempp_cuda.device import device_grid, device_singular_rule, device_space

    h2d = (device_grid(g).h2d_bytes + device_space(d).h2d_bytes + (device_space(t).h2d_bytes if t is not d else 0)
           + device_singular_rule(g, 4, t.support, d.support).h2d_bytes)
    return {"value": total_entries * args.steps / (ms * 1e-3), "unit": "entries/s", "ms_per_step": ms / args.steps,
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(rows * cols * 16),
            "note": "each step re-uploads the grid, spaces and singular tables from host memory (device copies "
                    "dropped), assembles the fused operator in 16 row blocks of the symmetric sweep and streams "
                    "each finished block to pinned host memory while the next is assembled "
                    "(operators.weak_form_to_host)"}


# ----------------------------------------------------------------------------- CPU arm
METRIC = "entries/s Helmholtz assembly, mixed vs FP64 GPU at rel err <=1e-6; shape-grads/s"
PARITY_ROWS = 512  # seeded rows of the benchmark operator kept from the GPU matrices for the CPU comparison


def bench_config(args):
    """The workload description both arms print (identical dicts)."""
    n = 8 * 4**args.level
    return {
        "workload": "Helmholtz combined-field DLP - 1/2 I - i k SLP, DP0, regular_sphere(%d), %d x %d complex128, "
                    "k=%g, regular order 4, singular order 4" % (args.level, n, n, args.k),
        "elements": n,
        "k": args.k,
        "l2": "output %.1f GB per step > 126 MB L2; compute-bound kernel" % (n * n * 16 / 1e9),
    }


def parity_rows(n):
    """The seeded random rows (test elements) used for CPU timing samples and parity checks."""
    return np.random.default_rng(20240).permutation(n)[: min(PARITY_ROWS, n)]


class CpuReference(object):
    """The reference's CPU path on a row sample of the benchmark operator.

    With the unmodified bempp_cl importable (installed under baseline/_ref,
    oracle/reference.py): its own public API with device_interface="numba"
    -- ``(dlp - 0.5 * identity - 1j * k * slp).weak_form()`` with the dual space
    restricted to the sampled elements (``support_elements``), so every step
    runs the reference's regular, singular and sparse assemblers on those rows
    (kind "reference").  Otherwise the oracle, the C/OpenMP restatement of the
    reference Numba kernels (kind "port").  Rows are a seeded random sample of
    the test elements, sized so one step takes about ``target_seconds``.
    """

    def __init__(self, args):
        self.args = args
        self.n = 8 * 4**args.level
        from oracle import reference

        self.bempp_cl = reference.load()
        self.kind = "reference" if self.bempp_cl is not None else "port"
        self.why_port = None if self.bempp_cl is not None else reference.reason()
        var = "NUMBA_NUM_THREADS" if self.bempp_cl is not None else "OMP_NUM_THREADS"
        self.cores = int(os.environ.get(var, os.cpu_count() or 1))
        from bempp_cuda.shapes import regular_sphere

        self.grid = regular_sphere(args.level)
        self._ref_grid = None

    def rows(self, rows):
        """(matrix rows of ``sorted(rows)``, seconds of the timed call)."""
        rows = np.sort(np.asarray(rows))
        k = self.args.k
        if self.bempp_cl is not None:
            from oracle import reference

            api = self.bempp_cl.api
            if self._ref_grid is None:
                self._ref_grid = reference.grid_from(self.grid)
            g = self._ref_grid
            d = api.function_space(g, "DP", 0)
            t = api.function_space(g, "DP", 0, support_elements=rows)
            H = api.operators.boundary.helmholtz
            t0 = time.perf_counter()
            slp = H.single_layer(d, d, t, k, assembler="dense", device_interface="numba")
            dlp = H.double_layer(d, d, t, k, assembler="dense", device_interface="numba")
            ident = api.operators.boundary.sparse.identity(d, d, t)
            mat = (dlp - 0.5 * ident - 1j * k * slp).weak_form().to_dense()
            return np.asarray(mat), time.perf_counter() - t0
        from oracle import oracle as orc

        from bempp_cuda.quadrature import triangle_rule
        from bempp_cuda.space import function_space

        domain = function_space(self.grid, "DP", 0)
        qp, qw = triangle_rule(4)
        eta = -1j * k
        t0 = time.perf_counter()
        mat = orc.assemble_rows("helmholtz_combined_field", "default_scalar", [k, 0.0, eta.real, eta.imag], True,
                                domain, domain, rows, qp, qw, 4)
        mat[np.arange(len(rows)), rows] += -0.5 * self.grid.volumes[rows]
        return mat, time.perf_counter() - t0

    def calibrate(self, target_seconds):
        """Warm the path (Numba compiles on its first call) and pick the sample size."""
        sample = parity_rows(self.n)
        self.rows(sample[:8])
        _, t = self.rows(sample[:32])
        self.count = int(min(len(sample), max(32, 32 * target_seconds / max(t, 1e-3))))
        self.sample = sample[: self.count]
        return self.count

    def describe(self):
        if self.bempp_cl is not None:
            what = ("bempp_cl %s Numba path through its public API (weak_form of the combined field with the "
                    "dual space on the sampled elements)" % getattr(self.bempp_cl, "__version__", ""))
        else:
            what = "oracle port (C/OpenMP restatement of the reference Numba kernels; %s)" % self.why_port
        return ("%d seeded random rows x %d columns of the %d x %d operator per step, regular + singular + "
                "identity: %s" % (self.count, self.n, self.n, self.n, what))


def reference_arm(args, world, rank):
    if rank != 0:
        return None
    cpu = CpuReference(args)
    cpu.calibrate(args.cpu_seconds)
    for _ in range(max(0, args.warmup - 1)):
        cpu.rows(cpu.sample[: max(8, cpu.count // 8)])
    times = [cpu.rows(cpu.sample)[1] for _ in range(args.steps)]
    total = sum(times)
    value = cpu.count * cpu.n * args.steps / total
    return {
        "metric": METRIC,
        "value": value,
        "unit": "entries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True,
        "scaling": "strong",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: regular_sphere(%d) unit sphere, generated by octahedron subdivision" % args.level,
        "config": bench_config(args),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "entries/s", "cores": cpu.cores, "kind": cpu.kind,
                         "sample": cpu.describe()},
        "e2e": {"value": value, "unit": "entries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def cpu_leg(args, line, gpu_rows):
    """cpu_baseline of the GPU arm, and the parity of the GPU matrices on the same rows."""
    cpu = CpuReference(args)
    cpu.calibrate(args.cpu_seconds)
    mat, t = cpu.rows(cpu.sample)
    line["cpu_baseline"] = {"value": cpu.count * cpu.n / t, "unit": "entries/s", "cores": cpu.cores,
                            "kind": cpu.kind, "sample": cpu.describe()}
    if gpu_rows is None:
        return
    order = np.argsort(cpu.sample)
    parity = {"rows": int(cpu.count), "against": cpu.kind, "bound_fp64": 1e-12, "bound_mixed": 1e-6}
    for name, rows in gpu_rows.items():
        got = rows[: cpu.count][order]
        parity[name + "_rel_fro"] = float(np.linalg.norm(got - mat) / np.linalg.norm(mat))
    line.setdefault("parity", {})["benchmark_operator"] = parity


# ----------------------------------------------------------------------------- single-kernel cases
def _case_matmat(torch):
    """The FP64 tensor-core product: 3 x (8192 x 8192) complex128 times 8 right-hand sides (3.2 GB)."""
    from bempp_cuda.matmat import BatchedProduct

    gen = torch.Generator(device="cuda").manual_seed(0)
    mats = [torch.randn((8192, 8192), dtype=torch.complex128, device="cuda", generator=gen) for _ in range(3)]
    xs = [torch.randn((8192, 8), dtype=torch.complex128, device="cuda", generator=gen) for _ in range(3)]
    ys = [torch.empty_like(x) for x in xs]
    bp = BatchedProduct(mats, xs, ys)
    return bp.launch, 3 * 16 * (8192 * 8192 + 2 * 8192 * 8)


def _case_gemv(torch):
    """The solves' one-right-hand-side product on a 16384 x 16384 complex128 matrix (4.3 GB)."""
    from bempp_cuda.matmat import gemv

    gen = torch.Generator(device="cuda").manual_seed(0)
    a = torch.randn((16384, 16384), dtype=torch.complex128, device="cuda", generator=gen)
    x = torch.randn(16384, dtype=torch.complex128, device="cuda", generator=gen)
    return (lambda: gemv(a, x)), a.numel() * 16


def _combined_l5(torch, args):
    from bempp_cuda.operators import Parameters
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    grid = regular_sphere(5)
    sp = function_space(grid, "DP", 0)
    return sp, Parameters(), combined_descriptor(5.0)


def _case_mixed_sym(torch, args=None):
    """The mixed symmetric combined-field sweep on regular_sphere(5), k = 5 (1.07 GB output)."""
    from bempp_cuda import _lib
    from bempp_cuda.assembly import regular_into

    sp, prm, desc = _combined_l5(torch, args)
    out = torch.empty((8192, 8192), dtype=torch.complex128, device="cuda")
    return (lambda: regular_into(out, desc, sp, sp, prm, precision=_lib.MIXED, overwrite=True)), out.numel() * 16


def _case_apply(torch, args=None):
    """The FP64 matrix-free apply of the combined field's regular part on regular_sphere(5), k = 5."""
    from bempp_cuda.assembly import apply_regular

    sp, prm, desc = _combined_l5(torch, args)
    x = torch.ones(8192, dtype=torch.complex128, device="cuda")
    y = torch.zeros(8192, dtype=torch.complex128, device="cuda")
    return (lambda: apply_regular(y, x, desc, sp, sp, prm)), 0


def _p1_case(torch, name, precision):
    """The regular pass of a Helmholtz operator on P1 of regular_sphere(5), k = 5, added into a 4098 x 4098
    complex128 matrix (269 MB)."""
    from bempp_cuda import operators
    from bempp_cuda.assembly import regular_into
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    sp = function_space(regular_sphere(5), "P", 1)
    op = getattr(operators.boundary.helmholtz, name)(sp, sp, sp, 5.0)
    n = sp.global_dof_count
    out = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    return (lambda: regular_into(out, op.descriptor, sp, sp, op.parameters, precision=precision)), out.numel() * 16


def _case_p1_mixed_dlp(torch, args=None):
    """The mixed Helmholtz double layer on P1 of regular_sphere(5), k = 5 (the skew sweep)."""
    from bempp_cuda import _lib

    return _p1_case(torch, "double_layer", _lib.MIXED)


def _case_p1_fp64_dlp(torch, args=None):
    """The FP64 Helmholtz double layer on P1 of regular_sphere(5), k = 5 (the skew sweep)."""
    from bempp_cuda import _lib

    return _p1_case(torch, "double_layer", _lib.FP64)


def _case_p1_fp64_slp(torch, args=None):
    """The FP64 Helmholtz single layer on P1 of regular_sphere(5), k = 5 (the symmetric sweep)."""
    from bempp_cuda import _lib

    return _p1_case(torch, "single_layer", _lib.FP64)


def _points_case(torch, path, k, directions):
    """A mixed-precision potential or far field of P1 coefficients on regular_sphere(5) at 10 000 seeded points
    (the shell 1.5 < r < 3) or directions, inputs on the device."""
    from bempp_cuda import _lib, operators
    from bempp_cuda.assembly import evaluate_potential_device
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    sp = function_space(regular_sphere(5), "P", 1)
    rng = np.random.default_rng(1)
    dirs = rng.standard_normal((3, 10000))
    dirs /= np.linalg.norm(dirs, axis=0)
    pts = dirs if directions else dirs * (1.5**3 + rng.random(10000) * (3.0**3 - 1.5**3)) ** (1.0 / 3.0)
    f = operators
    for part in path.split("."):
        f = getattr(f, part)
    op = f(sp, pts, k)
    coeffs = rng.standard_normal(sp.global_dof_count) + 1j * rng.standard_normal(sp.global_dof_count)
    local = torch.as_tensor(sp.map_to_full_grid @ coeffs, device="cuda")
    pdev = torch.as_tensor(np.ascontiguousarray(pts.T), device="cuda")
    return (lambda: evaluate_potential_device(sp, op.descriptor, pdev, local, op.parameters,
                                              precision=_lib.MIXED)), 0


def _singular_p1_case(torch, name):
    """The singular pass of a Helmholtz operator on P1 of regular_sphere(5), k = 5 (Sauter-Schwab pairs of
    one space), added into a 4098 x 4098 complex128 matrix."""
    from bempp_cuda import operators
    from bempp_cuda.assembly import singular_into_dense
    from bempp_cuda.shapes import regular_sphere
    from bempp_cuda.space import function_space

    sp = function_space(regular_sphere(5), "P", 1)
    op = getattr(operators.boundary.helmholtz, name)(sp, sp, sp, 5.0)
    n = sp.global_dof_count
    out = torch.zeros((n, n), dtype=torch.complex128, device="cuda")
    return (lambda: singular_into_dense(out, op.descriptor, sp, sp, op.parameters)), 0


def _case_singular_p1_dlp(torch, args=None):
    """The FP64 singular pass of the Helmholtz double layer on P1 of regular_sphere(5), k = 5."""
    return _singular_p1_case(torch, "double_layer")


def _case_singular_p1_slp(torch, args=None):
    """The FP64 singular pass of the Helmholtz single layer on P1 of regular_sphere(5), k = 5."""
    return _singular_p1_case(torch, "single_layer")


def _case_potential_mixed(torch, args=None):
    """The mixed Helmholtz single-layer potential, 10 000 points, P1 on regular_sphere(5), k = 5."""
    return _points_case(torch, "potential.helmholtz.single_layer", 5.0, False)


def _case_farfield_mixed(torch, args=None):
    """The mixed Helmholtz single-layer far field, 10 000 directions, P1 on regular_sphere(5), k = 5."""
    return _points_case(torch, "far_field.helmholtz.single_layer", 5.0, True)


PROFILE_CASES = {"matmat_3x8192": _case_matmat, "gemv_16384": _case_gemv, "mixed_sym_l5": _case_mixed_sym,
                 "apply_l5": _case_apply, "p1_mixed_dlp_l5": _case_p1_mixed_dlp, "p1_fp64_dlp_l5": _case_p1_fp64_dlp,
                 "p1_fp64_slp_l5": _case_p1_fp64_slp, "singular_p1_dlp_l5": _case_singular_p1_dlp,
                 "singular_p1_slp_l5": _case_singular_p1_slp,
                 "potential_mixed_l5": _case_potential_mixed, "farfield_mixed_l5": _case_farfield_mixed}


def profile_case(args):
    import torch

    from bempp_cuda import _lib

    _lib.load()
    fn, nbytes = PROFILE_CASES[args.profile_case](torch)
    for _ in range(max(1, args.warmup)):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    print(json.dumps({"profile_case": args.profile_case, "ms": ms, "bytes": nbytes,
                      "gbs": nbytes / (ms * 1e-3) / 1e9 if nbytes else None}))


def main():
    args = parse()
    if args.profile_case:
        profile_case(args)
        return
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        line = reference_arm(args, world, rank)
        if line is not None:
            print(json.dumps(line))
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    line, gpu_rows = gpu_arm(args, world, rank, local)
    if rank == 0 and world == 1 and not args.skip_cpu:
        cpu_leg(args, line, gpu_rows)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
