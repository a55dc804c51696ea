"""Benchmark of the electrostatic BEM hot path on B200 (one JSON line on rank 0).

Workload (default): coaxial electrodes -- inner cylinder r = 0.5 m at -1000 V, outer r = 1.0 m
at 0 V, length 4 m, 40,000 rectangles + 4,000 annular cap triangles -- charge densities from a
GMRES solve to 1e-10, then the field and potential at 1,000,000 seeded points uniform in the
gap. A step is one evaluation of all 1,000,000 points.

  value     points/s of the MIXED form on device-resident points (all ranks, weak scaling)
  e2e       the same through the C ABI with pinned host buffers (H2D + D2H inside the step)
  extra     the plain FP64 form on the same points, the mixed-vs-FP64 error, GMRES solve
            times (plain FP64 matrix-free vs mixed assembled), a tracking and an adjoint
            sample, Robin Hood on the 1,280-triangle sphere, the 100,000-triangle 8-RHS
            stacked-ring solve, the FP64 roofline of the field kernel and the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl native|reference]

Multi-GPU runs are launched with torch.distributed.run; points are independent, so every
rank evaluates its own 1,000,000 points against the same (replicated) geometry with no
data-path collective ("weak" scaling); timings are reduced with max over ranks.
"""

from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_POINTS = 1_000_000
TOL = 1e-10
# DRAM bytes (read + write) of one MIXED direct-sum launch over the default 1,000,000-point
# workload, from a one-pass ncu capture (profiles/field_kernel_coax1m_dram.md); bench.py
# cannot run ncu itself, so the figure is reported only for that workload
FIELD_TRAFFIC_BYTES_1M = 69.49e6 + 83.10e6
# algorithmic flops per element-point interaction (field + potential) by band:
# cubature / Gauss with n nodes: 20 n + 30 (node sums, ratio test); analytic near field:
# fixed counts of one pass through the non-degenerate branch (frozen here)
RWG_FLOPS = {0: 420, 1: 520, 2: 160}  # triangle, rectangle, analytic wire
NODES = {0: {1: 33, 2: 12, 3: 7}, 1: {1: 33, 2: 12, 3: 7}, 2: {1: 16, 2: 4}}


def flops_per_band(counts):
    c = np.asarray(counts, dtype=np.float64).reshape(3, 4)
    total = 0.0
    for shape in range(3):
        total += c[shape, 0] * RWG_FLOPS[shape]
        for band, n in NODES[shape].items():
            total += c[shape, band] * (20 * n + 30)
    return total


# ----------------------------------------------------------------------------- CPU reference
def _ref_worker(args):
    """Reference field solver (oracle/_ref, the reference's own FP64 CPU code) on a slice."""
    mesh_arrays, sigma, pts = args
    sys.path.insert(0, ROOT)
    from kassiopeia_b200.geometry import Mesh
    from oracle import ref

    m = Mesh(*mesh_arrays)
    p = ref.RefProblem(m)
    p.set_sigma(sigma)
    t0 = time.perf_counter()
    p.field(pts)
    return time.perf_counter() - t0, len(pts)


def cpu_reference_rate(mesh, sigma, pts, workers, seconds_target=12.0):
    """points/s of the reference CPU direct sum on `workers` processes (spawned), each taking a
    disjoint slice of a bounded point sample; returns (points/s, sample description)."""
    from oracle import ref as R

    if not R.available():
        return None, "oracle/_ref not built"
    # calibrate: one point on one process
    ctx = mp.get_context("spawn")
    arrays = (mesh.shape, mesh.boundary, mesh.geom, mesh.value)
    with ctx.Pool(1) as pool:
        dt, _ = pool.map(_ref_worker, [(arrays, sigma, pts[:2])])[0]
    per_point = dt / 2
    per_worker = max(1, int(seconds_target / max(per_point, 1e-6)))
    n = min(len(pts), per_worker * workers)
    sample = pts[:n]
    chunks = [sample[i::workers] for i in range(workers)]
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        res = pool.map(_ref_worker, [(arrays, sigma, c) for c in chunks if len(c)])
    wall = time.perf_counter() - t0
    busy = max(r[0] for r in res)
    return n / busy, f"{n} of the {len(pts)} gap points on {workers} processes ({wall:.1f} s wall incl. setup)"


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index=0):
        self.index, self.samples, self._stop = index, [], threading.Event()
        self._t = threading.Thread(target=self._run, daemon=True)

    def _run(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                f = [x.strip() for x in out.stdout.strip().split(",")]
                if len(f) >= 8:
                    self.samples.append(f)
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no nvidia-smi samples"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if "Active" in s[4 + k]
                          and "Not" not in s[4 + k]})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ----------------------------------------------------------------------------- native arm
def run_native(args, rank, world, dist):
    import torch

    import kassiopeia_b200 as K
    from kassiopeia_b200 import _native as NN
    from kassiopeia_b200 import geometry as G
    from kassiopeia_b200 import ranks as RK

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    mesh = G.coax()
    P = RK.rank_points(N_POINTS, rank)
    ctx = K.CUDAElectrostaticContext(dev)
    ctx.SetGeometry(mesh)

    # charge densities: plain FP64 matrix-free GMRES (the reference algorithm) vs the
    # assembled mixed-precision solve with FP64 refinement
    if args.profile:
        x_asm = np.where(mesh.value < -1.0, -1e-8, 1e-8)
        st_plain = st_asm = {"seconds": float("nan"), "iterations": 0, "rel_residual": float("nan")}
        sigma_diff = float("nan")
    else:
        x_plain, st_plain = ctx.Solve(tol=TOL, max_iter=300, mode=K.SOLVE_PLAIN)
        x_asm, st_asm = ctx.Solve(tol=TOL, max_iter=300, mode=K.SOLVE_ASSEMBLED)  # includes the assembly
        st_asm["repeat_seconds"] = ctx.Solve(tol=TOL, max_iter=300, mode=K.SOLVE_ASSEMBLED)[1]["seconds"]
        sigma_diff = float(np.max(np.abs(x_asm - x_plain)) / np.max(np.abs(x_plain)))
    ctx.SetSigma(x_asm)

    def barrier():
        RK.barrier(dist, device=torch.device("cuda", dev))

    def max_over_ranks(v):
        return RK.max_over_ranks(v, dist, device=torch.device("cuda", dev))

    dP = torch.from_numpy(P).cuda()
    dOut = torch.empty((N_POINTS, 4), dtype=torch.float64, device="cuda")

    def device_steps(precision, k):
        ms = 0.0
        for _ in range(k):
            ctx.FieldDevice(dP.data_ptr(), N_POINTS, dOut.data_ptr(), precision=precision)
            ms += ctx.last_kernel_ms
        return ms

    # warm-up, then K timed steps per form; inputs (24 MB points, 44k x 256 B elements) are
    # resident and every step re-reads them: the working set is compute-bound, not cache-bound
    device_steps(K.MIXED, args.warmup)
    device_steps(K.FP64, max(1, args.warmup // 2))
    launches0 = NN.lib().kemcu_launch_count(ctx._h)
    with ClockSampler(dev) as clk:
        barrier()
        t0 = time.perf_counter()
        ms_mixed = device_steps(K.MIXED, args.steps)
        barrier()
        wall_mixed = time.perf_counter() - t0
    launches = NN.lib().kemcu_launch_count(ctx._h) - launches0
    ms_mixed = max_over_ranks(ms_mixed)
    barrier()
    ms_fp64 = max_over_ranks(device_steps(K.FP64, args.steps))

    # end-to-end through the C ABI with pinned host buffers
    hP = torch.from_numpy(P).pin_memory()
    hOut = torch.empty((N_POINTS, 4), dtype=torch.float64).pin_memory()
    import ctypes as C
    pP = C.cast(hP.data_ptr(), C.POINTER(C.c_double))
    pO = C.cast(hOut.data_ptr(), C.POINTER(C.c_double))
    NN.lib().kemcu_field(ctx._h, pP, N_POINTS, pO, K.MIXED, K.FIELD_AND_POTENTIAL)
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rc = NN.lib().kemcu_field(ctx._h, pP, N_POINTS, pO, K.MIXED, K.FIELD_AND_POTENTIAL)
        assert rc == 0, NN.lib().kemcu_last_error(ctx._h)
    barrier()
    e2e_s = max_over_ranks((time.perf_counter() - t0) / args.steps)

    # accuracy of the mixed form against the plain FP64 form (the metric bound is 1e-9)
    sub = P[:20000]
    o64 = ctx.ElectricFieldAndPotential(sub, precision=K.FP64)
    o32 = ctx.ElectricFieldAndPotential(sub, precision=K.MIXED)
    err_E = float(np.max(np.linalg.norm(o32[:, :3] - o64[:, :3], axis=1) / np.linalg.norm(o64[:, :3], axis=1)))
    err_phi = float(np.max(np.abs(o32[:, 3] - o64[:, 3])) / np.max(np.abs(o64[:, 3])))

    # algorithmic work (band histogram on a 2% sample, scaled) and the FP64 roofline
    hs = P[::50]
    counts = np.zeros(12, dtype=np.int64)
    NN.lib().kemcu_band_histogram(ctx._h, np.ascontiguousarray(hs).ctypes.data_as(C.POINTER(C.c_double)), len(hs),
                                  counts.ctypes.data_as(C.POINTER(C.c_longlong)))
    flops_per_step = flops_per_band(counts) * (N_POINTS / len(hs))
    f64 = C.c_double()
    f32 = C.c_double()
    NN.lib().kemcu_fma_peak(ctx._h, C.byref(f64), C.byref(f32))

    # tracking sample (configuration 3: 65,536 electrons in the 1,280-triangle sphere field)
    extra = {}
    axisym_case = None
    if not args.quick:
        sph = G.icosphere(3)
        tctx = K.CUDAElectrostaticContext(dev)
        tctx.SetGeometry(sph)
        tctx.Solve(tol=TOL, mode=K.SOLVE_ASSEMBLED)
        E = G.electrons(65536, seed=99 + rank)
        for prec, name in ((K.FP64, "fp64"), (K.MIXED, "mixed")):
            _, _, _, ts = tctx.TrackRK8(E, 1e-11, 10000, step_budget=2, sphere_radius=1.0, precision=prec)
            extra[f"tracking_track_steps_per_s_{name}"] = ts["steps"] / ts["seconds"]
        # adjoint sample (configuration 4: 20,480 triangles, 4,096 probes)
        s5 = G.icosphere(5)
        tctx.SetGeometry(s5)
        xs, _ = tctx.Solve(tol=TOL, mode=K.SOLVE_ASSEMBLED)
        rng = np.random.default_rng(4)
        tctx.SetSigma(xs * (1 + 0.1 * rng.normal(size=s5.n)))
        probes = G.shell_points(4096, seed=44)
        w = np.zeros((4096, 4))
        w[:, 2] = 1.0
        w[:, 3] = 1.0
        tctx.FieldVJP(probes, w)
        extra["adjoint_vjp_ms_fp64"] = tctx.last_kernel_ms
        # Robin Hood (configuration 1: 1,280-triangle sphere, tolerance 1e-8, the reference's
        # KRobinHood defaults), matrix-free columns and assembled columns
        tctx.SetGeometry(G.icosphere(3))
        for assembled, name in ((False, "matrix_free"), (True, "assembled")):
            tctx.SolveRobinHood(tol=1e-8, assembled=assembled)
            _, rs = tctx.SolveRobinHood(tol=1e-8, assembled=assembled)
            extra[f"robinhood_c1_{name}"] = {"seconds": rs["seconds"], "corrections": rs["subiterations"],
                                             "checks": rs["iterations"], "rel_residual_inf": rs["rel_residual"]}
        # axisymmetric model (conic sections and rings, KElectrostaticAnalyticConicSectionIntegrator
        # / ...RingIntegrator): coax of 2 x 2,000 cylinder sections, 2 x 200 cap sections and 16
        # rings; assembled solve, then the FP64 field at 100,000 gap points
        ax = G.conic_coax(n_z=2000, n_cap=200, n_rings=16)
        tctx.SetGeometry(ax)
        xa, sa = tctx.Solve(tol=TOL, mode=K.SOLVE_ASSEMBLED)
        Pa = G.gap_points(100_000, seed=77)
        tctx.ElectricFieldAndPotential(Pa[:4096])
        tctx.ElectricFieldAndPotential(Pa)
        ms_ax = tctx.last_kernel_ms
        extra["axisym_conic_coax"] = {
            "elements": ax.n, "points": len(Pa), "field_ms": ms_ax, "points_per_s": len(Pa) / (ms_ax * 1e-3),
            "epi_per_s": len(Pa) * ax.n / (ms_ax * 1e-3), "assembled_solve_s": sa["seconds"],
            "krylov_iterations": sa["iterations"], "rel_residual": sa["rel_residual"]}
        axisym_case = (ax, xa, Pa)
        tctx.close()
        # configuration 5: 100,000 jittered triangles on 8 stacked rings, 8 right-hand sides:
        # one matrix-free FP64 matvec for 8 RHS, and the assembled solve (120 GB operator; the
        # coax context is re-used so that its 23 GB operator is released first)
        c5 = ctx
        rings = G.stacked_rings()
        c5.SetGeometry(rings)
        B = G.ring_potentials(rings, n_rhs=8)
        for _ in range(2):  # the second of each pair is kept
            c5.Multiply(B[0] * 1e-12, precision=K.FP64)
        t1 = c5.last_kernel_ms
        for _ in range(2):
            c5.Multiply(B * 1e-12, precision=K.FP64)
        t8 = c5.last_kernel_ms
        _, s5 = c5.Solve(B, tol=TOL, mode=K.SOLVE_ASSEMBLED)  # allocates and assembles the operator
        _, s5r = c5.Solve(B, tol=TOL, mode=K.SOLVE_ASSEMBLED)
        extra["c5_stacked_rings_100k_8rhs"] = {
            "matrix_free_fp64_matvec_ms_1rhs": t1, "matrix_free_fp64_matvec_ms_8rhs": t8,
            "assembled_solve_s": s5["seconds"], "assembled_solve_repeat_s": s5r["seconds"],
            "krylov_iterations": s5["iterations"], "rel_residual": s5["rel_residual"]}

    res = dict(
        ms_mixed=ms_mixed, ms_fp64=ms_fp64, wall_mixed=wall_mixed, e2e_s=e2e_s, launches=int(launches),
        err_E=err_E, err_phi=err_phi, flops_per_step=flops_per_step, fp64_peak=f64.value, fp32_peak=f32.value,
        counts=counts.tolist(), st_plain=st_plain, st_asm=st_asm, sigma_diff=sigma_diff, clocks=clk.summary(),
        extra=extra, mesh=mesh, sigma=x_asm, P=P, axisym=axisym_case)
    ctx.close()
    return res


def profile_operator():
    import kassiopeia_b200 as K
    from kassiopeia_b200 import geometry as G

    ctx = K.CUDAElectrostaticContext(int(os.environ.get("LOCAL_RANK", 0)))
    mesh = G.coax(n_phi=60, n_z=120, n_cap_rings=8)
    ctx.SetGeometry(mesh)
    x = np.ones(mesh.n)
    X = np.stack([x * (r + 1) for r in range(8)])
    # one right-hand side (dense_matvec_kernel): 3 FP32 then 2 FP64 launches; then 8 right-hand
    # sides (dense_mma_kernel): 2 FP32 then 2 FP64 launches
    for prec, xx in ((K.MIXED, x),) * 3 + ((K.FP64, x),) * 2 + ((K.MIXED, X),) * 2 + ((K.FP64, X),) * 2:
        ctx.Multiply(xx, precision=prec, assembled=True)  # the first call assembles the operator
        entry = 4 if prec == K.MIXED else 8
        ms = ctx.last_kernel_ms
        print(json.dumps({"operator": "dense " + ("FP32" if prec == K.MIXED else "FP64"), "n": mesh.n,
                          "rhs": 1 if xx.ndim == 1 else xx.shape[0], "ms": ms,
                          "GB/s": mesh.n * mesh.n * entry / (ms * 1e-3) / 1e9}), flush=True)


def profile_tracker():
    import kassiopeia_b200 as K
    from kassiopeia_b200 import geometry as G

    ctx = K.CUDAElectrostaticContext(int(os.environ.get("LOCAL_RANK", 0)))
    ctx.SetGeometry(G.icosphere(3))
    ctx.Solve(tol=TOL, mode=K.SOLVE_ASSEMBLED)
    E = G.electrons(65536, seed=99)
    for prec, name in ((K.FP64, "FP64"), (K.MIXED, "MIXED")):
        _, _, _, ts = ctx.TrackRK8(E, 1e-11, 10000, step_budget=8, sphere_radius=1.0, precision=prec)
        print(json.dumps({"tracker": name, "tracks": len(E), "steps": ts["steps"], "seconds": ts["seconds"],
                          "track_steps_per_s": ts["steps"] / ts["seconds"]}), flush=True)


def profile_axisym():
    import kassiopeia_b200 as K
    from kassiopeia_b200 import geometry as G

    ctx = K.CUDAElectrostaticContext(int(os.environ.get("LOCAL_RANK", 0)))
    ax = G.conic_coax(n_z=2000, n_cap=200, n_rings=16)
    ctx.SetGeometry(ax)
    ctx.Solve(tol=TOL, mode=K.SOLVE_ASSEMBLED)
    P = G.gap_points(10_000, seed=77)
    for _ in range(2):  # the first launch warms up, the second is the one to capture
        ctx.ElectricFieldAndPotential(P)
        print(json.dumps({"axisym_field": "FP64", "elements": ax.n, "points": len(P), "ms": ctx.last_kernel_ms,
                          "points_per_s": len(P) / (ctx.last_kernel_ms * 1e-3)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--quick", action="store_true", help="skip the tracking/adjoint/CPU samples")
    ap.add_argument("--profile", action="store_true",
                    help="profiling case for ncu: no solves (fixed charge density, no assembled operator) and "
                         "--points points; prints the same JSON line")
    ap.add_argument("--points", type=int, default=N_POINTS, help="gap points per GPU (default 1,000,000)")
    ap.add_argument("--profile-operator", action="store_true",
                    help="profiling case for ncu: assembled operator of a 16,320-element coax (2.1 GB FP64 + "
                         "1.1 GB FP32), three FP32 and two FP64 dense matvecs with one right-hand side, then two "
                         "FP32 and two FP64 with eight; prints one JSON line per matvec")
    ap.add_argument("--profile-tracker", action="store_true",
                    help="profiling case for ncu: 65,536 electrons in the field of the 1,280-triangle sphere, "
                         "one persistent RK8 launch of 8 steps per track, FP64 then MIXED; prints track steps/s")
    ap.add_argument("--profile-axisym", action="store_true",
                    help="profiling case for ncu: axisymmetric coax (4,416 conic sections and rings), field and "
                         "potential at 10,000 gap points, two launches; prints points/s")
    args = ap.parse_args()
    if args.profile_axisym:
        profile_axisym()
        return
    if args.profile_operator:
        profile_operator()
        return
    if args.profile_tracker:
        profile_tracker()
        return
    globals()["N_POINTS"] = args.points
    if args.profile:
        args.quick = True

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None

    if args.impl == "reference":
        if rank != 0:
            return
        run_reference(args)
        return

    if world > 1:
        import datetime

        import torch
        import torch.distributed as D

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        D.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = D
    r = run_native(args, rank, world, dist)

    cpu = None
    if rank == 0 and world == 1 and not args.quick:
        workers = os.cpu_count() or 1
        rate, sample = cpu_reference_rate(r["mesh"], r["sigma"], r["P"], workers)
        if rate is not None:
            cpu = {"value": rate, "unit": "points/s", "cores": workers, "kind": "reference", "sample": sample}
            # the single-core figure beside it (one process, a ~5 s sample)
            rate1, sample1 = cpu_reference_rate(r["mesh"], r["sigma"], r["P"], 1, seconds_target=5.0)
            cpu["one_core"] = {"value": rate1, "sample": sample1}
            if r["axisym"] is not None:
                # the axisymmetric model's field on the reference CPU code, one core
                am, ax_sigma, ax_pts = r["axisym"]
                rate_ax, sample_ax = cpu_reference_rate(am, ax_sigma, ax_pts, 1, seconds_target=4.0)
                cpu["axisym_conic_coax_one_core"] = {"value": rate_ax, "unit": "points/s",
                                                     "sample": sample_ax.replace("gap points", "axisymmetric gap points")}
        else:
            cpu = {"value": None, "unit": "points/s", "cores": 0, "kind": "reference", "sample": sample}

    if rank == 0:
        steps = args.steps
        pts = N_POINTS * world
        ms_step = r["ms_mixed"] / steps
        value = pts / (ms_step * 1e-3)
        fp64_value = pts / (r["ms_fp64"] / steps * 1e-3)
        achieved = r["flops_per_step"] / (ms_step * 1e-3) / 1e12
        line = {
            "metric": "field evals/s (points/s; EPI/s = points/s x 44,000 elements) at <=1e-9 rel. error vs FP64",
            "value": value,
            "unit": "points/s",
            "n_gpus": world,
            "steps": steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64 (mixed form: FP32-class hardware rsqrt estimate + FP64 Newton step per cubature node; FP64 elsewhere)",
            "data": "synthetic (seeded coax mesh and gap points)",
            "config": {"workload": "coax: 40,000 rectangles + 4,000 cap triangles, 1,000,000 gap points per GPU, "
                                   "GMRES to 1e-10", "elements": 44000, "points_per_gpu": N_POINTS,
                       "parallelism": f"replicated geometry, points sharded over {world} GPU(s)",
                       "l2": "inputs re-read every step; 24 MB points + 11 MB elements, compute-bound kernel"},
            "e2e": {"value": pts / r["e2e_s"], "unit": "points/s",
                    "h2d_bytes_per_step": N_POINTS * 24, "d2h_bytes_per_step": N_POINTS * 32},
            "gpu_launches": r["launches"],
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": r["fp64_peak"], "unit": "TFLOP/s",
                         "frac": achieved / r["fp64_peak"] if r["fp64_peak"] else None,
                         "traffic": FIELD_TRAFFIC_BYTES_1M if N_POINTS == 1_000_000 else None,
                         "traffic_unit": "bytes per launch (ncu dram read + write)",
                         "algorithmic_bytes": N_POINTS * (24 + 32) + 44000 * (256 + 8),
                         "peak_source": "measured FP64 FMA throughput of this GPU (kemcu_fma_peak); "
                                        "MEASURED_PEAKS.json has no FP64 CUDA-core figure",
                         "flops_per_step": r["flops_per_step"], "band_counts": r["counts"]},
            "plain_fp64": {"value": fp64_value, "unit": "points/s", "ms_per_step": r["ms_fp64"] / steps,
                           "speedup_mixed_over_plain": value / fp64_value},
            "accuracy_mixed_vs_fp64": {"max_rel_err_E_per_point": r["err_E"],
                                       "max_abs_err_phi_over_max_phi": r["err_phi"]},
            "gmres": {"plain_fp64_matrix_free_s": r["st_plain"]["seconds"],
                      "plain_iterations": r["st_plain"]["iterations"],
                      "mixed_assembled_s": r["st_asm"]["seconds"],
                      "mixed_assembled_repeat_s": r["st_asm"].get("repeat_seconds"),
                      "mixed_assembled_iterations": r["st_asm"]["iterations"],
                      "mixed_assembled_rel_residual": r["st_asm"]["rel_residual"],
                      "speedup": r["st_plain"]["seconds"] / r["st_asm"]["seconds"],
                      "sigma_rel_diff": r["sigma_diff"]},
            "fp32_fma_peak_tflops": r["fp32_peak"],
            "clocks": r["clocks"],
            "cpu_baseline": cpu,
        }
        line.update(r["extra"])
        print(json.dumps(line))


def run_reference(args):
    """Reference arm: the reference's own CPU direct sum (oracle/_ref) on all host cores, same
    workload and metric, each step a bounded sample of the 1,000,000 gap points."""
    from kassiopeia_b200 import geometry as G
    from oracle import ref as R

    if not R.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libkemref.so not built here"}))
        return
    mesh = G.coax()
    P = G.gap_points(N_POINTS, seed=2024)  # rank 0's block (kassiopeia_b200.ranks.rank_points)
    # charge densities from the reference's own solver would take hours at 44,000 elements
    # (N^2 matrix entries per GMRES iteration on the CPU); the reference field sum is timed
    # with a fixed smooth density instead -- the direct sum's cost does not depend on sigma
    sigma = np.where(mesh.value < -1.0, -1e-8, 1e-8)
    workers = os.cpu_count() or 1
    rates = []
    for _ in range(max(1, args.warmup // 3)):
        cpu_reference_rate(mesh, sigma, P, workers, seconds_target=2.0)
    for _ in range(args.steps):
        rate, sample = cpu_reference_rate(mesh, sigma, P, workers, seconds_target=8.0)
        rates.append(rate)
    v = float(np.median(rates))
    print(json.dumps({
        "impl": "reference", "metric": "field evals/s (points/s; EPI/s = points/s x 44,000 elements) at <=1e-9 rel. "
                                       "error vs FP64",
        "value": v, "unit": "points/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": N_POINTS / v * 1e3,  # one step = the 1,000,000 points at the sampled rate
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded coax mesh and gap points)",
        "config": {"workload": "coax: 40,000 rectangles + 4,000 cap triangles, 1,000,000 gap points per GPU, "
                               "GMRES to 1e-10", "elements": 44000, "points_per_gpu": N_POINTS},
        "cpu_baseline": {"value": v, "unit": "points/s", "cores": workers, "kind": "reference", "sample": sample},
        "e2e": {"value": v, "unit": "points/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


if __name__ == "__main__":
    main()
