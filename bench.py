"""Benchmark: time to relative residual 1e-8 and DoF-updates/s of the P1 geometric-
multigrid solve on one B200, FP32-inner/FP64-refinement (mixed) against plain FP64.

Workload (the reference configuration the metric is quoted on): Poisson -lap(u) = f
on the unit cube split into a 2x2x2 macro-cube mesh (48 macro-tets), refinement
level 7 (16.97M micro-vertices), Dirichlet u = 0, f ~ U[-1,1] per micro-vertex
(seed 0), zero initial guess, V(3,3) cycles with SOR (omega = 1) and an FP64 CG
coarse solve on level 0, each solve run to ||f - Au|| / ||f|| <= 1e-8.

A step is one full solve from the zero initial guess with f resident in HBM. Each
FP64 vector of the finest level is 140 MB, larger than the 126 MB L2, so no L2 flush
is needed between steps. Under torchrun every rank solves its own replica of the
problem (the path has no exchange step on one mesh: replicas only); the time is the
maximum over ranks.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "hyteg-vara_b200")
sys.path.insert(0, os.path.join(PKG, "python"))
sys.path.insert(0, PKG)

METRIC = "MG time-to-1e-8 & DoF-updates/s, mixed vs FP64 on 1 B200; p50/p99 solve latency"
UNIT = "DoF-updates/s"
TOL = 1e-8


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait()

    def summary(self):
        sm, smax, reasons = [], None, set()
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                sm.append(float(f[1]))
                smax = float(f[2])
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for n, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except Exception:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def profile_figure(name, key):
    """A figure recorded as `key = value` in an ncu summary under profiles/ (None if absent)."""
    import re

    try:
        text = open(os.path.join(ROOT, "profiles", name)).read()
    except OSError:
        return None
    m = re.search(r"\b" + re.escape(key) + r"\s*=\s*([0-9.eE+]+)", text)
    return float(m.group(1)) if m else None


def rank_reduce(vals, op, world, device):
    """All-reduce floats over the ranks of the default process group ("max" for times,
    "sum" for throughputs); identity on a single rank. Every rank calls it in the same
    order."""
    if world == 1:
        return [float(v) for v in vals]
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.tolist()]


def replica_value(world, unknowns, cycles, max_ms):
    """Whole-job DoF-updates/s of N replicas: every rank solves its own copy, the time is the
    slowest rank's."""
    return world * unknowns * cycles / (max_ms / 1e3)


def ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist

    import build as B
    import hyb_inputs as I
    import hyteg_b200 as H

    B.build()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream
    L, nc = args.level, args.cubes

    st = H.PrimitiveStorage.cuboid(nc, nc, nc, L)
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0, coarse_tol=1e-12)
    xyz = st.dof_coords(L)
    f = I.uniform_rhs(xyz, 0, nc << L)
    ndof = st.num_dofs(L)
    u, b = H.P1Function("u", st, 0, L), H.P1Function("f", st, 0, L)
    b.set(f, L, stream=sh)
    m_col, _ = st.colouring()
    # interior (non-Dirichlet) DoFs: the unknowns each V-cycle updates
    mask = H.P1Function("mask", st, 0, L)
    mask.interpolate(1.0, L, flag=H.INNER | H.NEUMANN)
    n_unknowns = int(round(mask.dot_global(mask, L, H.INNER | H.NEUMANN)))
    del mask

    def solve(precision):
        u.interpolate(0.0, L, flag=H.ALL, stream=sh)
        return gmg.solve_to_tolerance(u, b, L, TOL, max_cycles=60, precision=precision, stream=sh)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        return rank_reduce([v], "max", world, dev)[0]

    def timed(fn, steps):
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = [fn() for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1)), out

    for _ in range(args.warmup):
        solve(32)
        solve(64)
    # headline: mixed precision solves, inputs resident
    with Clocks(local_rank) as clk:
        k0 = H.kernel_launch_count()
        t_mixed, hist_mixed = timed(lambda: solve(32), args.steps)
        launches = H.kernel_launch_count() - k0
    clocks = clk.summary()
    t_fp64, hist_fp64 = timed(lambda: solve(64), args.steps)
    cyc_mixed = [len(h) - 1 for h in hist_mixed]
    cyc_fp64 = [len(h) - 1 for h in hist_fp64]
    ms_mixed = t_mixed / args.steps
    ms_fp64 = t_fp64 / args.steps
    value = replica_value(world, n_unknowns, sum(cyc_mixed), t_mixed)

    # error of the mixed solution against a tightly converged FP64 solve of the same system
    solve(32)
    u_mixed = u.get(L, stream=sh)
    u.interpolate(0.0, L, flag=H.ALL, stream=sh)
    gmg.solve_to_tolerance(u, b, L, 1e-13, max_cycles=80, precision=64, stream=sh)
    u_ref = u.get(L, stream=sh)
    err_mixed = float(np.abs(u_mixed - u_ref).max() / np.abs(u_ref).max())

    # End to end through the C ABI with host buffers: every step copies its f from pinned host
    # memory to the device, solves, and copies u back to pinned host memory, all inside the
    # timed region. The copies run on a second stream and overlap the neighbouring steps'
    # solves (step k+1's f is uploaded and step k-1's u downloaded while step k solves), as a
    # serving pipeline would: two device staging buffers each way, events order them, and
    # the canonical-order conversions (set_device / get_device) run on the solve's stream.
    f_host = [torch.from_numpy(f.copy()).pin_memory() for _ in range(2)]
    u_host = [torch.empty(ndof, dtype=torch.float64).pin_memory() for _ in range(2)]
    d_f = [torch.empty(ndof, dtype=torch.float64, device=dev) for _ in range(2)]
    d_u = [torch.empty(ndof, dtype=torch.float64, device=dev) for _ in range(2)]
    copy = torch.cuda.Stream(device=dev)

    def e2e_run(steps):
        ev_h2d = [torch.cuda.Event() for _ in range(steps)]
        ev_read = [torch.cuda.Event() for _ in range(steps)]
        ev_d2h = [torch.cuda.Event() for _ in range(steps)]
        copy.wait_stream(stream)  # the first upload starts inside the timed region
        with torch.cuda.stream(copy):
            d_f[0].copy_(f_host[0], non_blocking=True)
            ev_h2d[0].record(copy)
        for k in range(steps):
            if k + 1 < steps:
                with torch.cuda.stream(copy):
                    if k >= 1:
                        copy.wait_event(ev_read[k - 1])  # step k-1 has read d_f[(k + 1) % 2]
                    d_f[(k + 1) % 2].copy_(f_host[(k + 1) % 2], non_blocking=True)
                    ev_h2d[k + 1].record(copy)
            stream.wait_event(ev_h2d[k])
            b.set_device(d_f[k % 2].data_ptr(), L, stream=sh)
            ev_read[k].record(stream)
            solve(32)
            if k >= 2:
                stream.wait_event(ev_d2h[k - 2])  # step k-2's download has read d_u[k % 2]
            u.get_device(d_u[k % 2].data_ptr(), L, stream=sh)
            done = torch.cuda.Event()
            done.record(stream)
            with torch.cuda.stream(copy):
                copy.wait_event(done)
                u_host[k % 2].copy_(d_u[k % 2], non_blocking=True)
                ev_d2h[k].record(copy)
        stream.wait_stream(copy)  # the last download ends the timed region

    e2e_run(2)
    t_e2e, _ = timed(lambda: e2e_run(args.steps), 1)
    assert np.array_equal(u_host[(args.steps - 1) % 2].numpy(), u_mixed), "end-to-end result differs"
    e2e = {"value": world * n_unknowns * sum(cyc_mixed) / (t_e2e / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": ndof * 8, "d2h_bytes_per_step": ndof * 8, "ms_per_step": t_e2e / args.steps,
           "copies": "pinned host <-> device every step, on a second stream overlapping the neighbouring solves"}

    # kernel rooflines (CUDA events on the launching stream, 20 launches each)
    peak, peak_kind = peaks()

    def kernel_time(fn, reps=20):
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps / 1e3

    y = H.P1Function("y", st, L, L)
    t_apply = kernel_time(lambda: A.apply(b, y, L, H.INNER | H.NEUMANN, stream=sh))
    t_sor = kernel_time(lambda: A.smooth_sor(u, b, 1.0, L, H.INNER | H.NEUMANN, stream=sh))
    u32, b32 = H.P1Function("u32", st, L, L, H.F32), H.P1Function("b32", st, L, L, H.F32)
    b32.copy_from(b, L, stream=sh)
    t_sor32 = kernel_time(lambda: A.smooth_sor(u32, b32, 1.0, L, H.INNER | H.NEUMANN, stream=sh))
    # algorithmic bytes: apply reads src and writes dst (16 B/DoF); an SOR sweep reads rhs,
    # reads and writes u (24 B/DoF FP64, 12 B/DoF FP32)
    apply_gbs = ndof * 16 / t_apply / 1e9
    sor_gbs = ndof * 24 / t_sor / 1e9
    sor32_gbs = ndof * 12 / t_sor32 / 1e9

    def roof(a, t_bytes=None, t_src=None):
        return {"bound": "hbm", "achieved": round(a, 1), "peak": peak, "unit": "GB/s", "frac": round(a / peak, 3),
                "peak_source": peak_kind, "traffic": t_bytes, "traffic_source": t_src}

    # DRAM bytes (read + write) per launch from the warm-cache ncu captures of the same kernels
    # and workload that profiles/ summarises (one sweep = the sum over its ten launches)
    sweep_prof, apply_prof = "k_sor_fp64_fp32_level7_cube48.md", "k_apply_fp64_level7_cube48.md"
    sweep64_traffic = profile_figure(sweep_prof, "fp64_sweep_bytes")
    sweep32_traffic = profile_figure(sweep_prof, "fp32_sweep_bytes")
    apply_traffic = profile_figure(apply_prof, "fp64_apply_bytes")
    if (L, nc) != (7, 2):
        sweep64_traffic = sweep32_traffic = apply_traffic = None

    # The reference's own SOR order on the GPU (hyb_operator_smooth_sor_reference_order): the
    # same FP64 algorithm, with the same iterates up to rounding, as the reference arm times
    # on the host; one solve from zero to 1e-8 and one level-7 sweep.
    ref_order = None
    if not args.no_reference_order:
        g_ref = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0, smoother=H.SMOOTHER_SOR_REFERENCE_ORDER,
                                           coarse_tol=1e-12)

        def solve_ref():
            u.interpolate(0.0, L, flag=H.ALL, stream=sh)
            return g_ref.solve_to_tolerance(u, b, L, TOL, max_cycles=60, precision=64, stream=sh)

        solve_ref()
        t_ref, h_ref = timed(solve_ref, 1)
        cyc_ref = len(h_ref[0]) - 1

        def solve_ref32():
            u.interpolate(0.0, L, flag=H.ALL, stream=sh)
            return g_ref.solve_to_tolerance(u, b, L, TOL, max_cycles=60, precision=32, stream=sh)

        solve_ref32()
        t_ref32, h_ref32 = timed(solve_ref32, 1)
        t_sweep_ref = kernel_time(lambda: A.smooth_sor_reference_order(u, b, 1.0, L, H.INNER | H.NEUMANN, stream=sh),
                                  reps=5)
        ref_order = {"smoother": "SOR in the reference's staged lexicographic order (V, E, F, C), FP64",
                     "time_to_tol_ms": t_ref, "cycles": cyc_ref, "final_rel_residual": float(h_ref[0][-1]),
                     "mixed": {"time_to_tol_ms": t_ref32, "cycles": len(h_ref32[0]) - 1,
                               "final_rel_residual": float(h_ref32[0][-1])},
                     "dof_updates_per_s": world * n_unknowns * cyc_ref / (t_ref / 1e3),
                     "sweep_ms": t_sweep_ref * 1e3, "sweep_level": L,
                     "multicolour_sweep_ms": t_sor * 1e3}
        del g_ref

    varcoef = None
    if not args.no_varcoef:
        del y, u32, b32
        torch.cuda.synchronize()
        varcoef = variable_coefficient(args, H, I, stream)

    shell = None
    if not args.no_shell:
        torch.cuda.synchronize()
        shell = spherical_shell(args, H, I, stream)

    blend = None
    if not args.no_blend:
        torch.cuda.synchronize()
        blend = blended_shell(args, H, stream)

    serve = None
    if not args.no_serve:
        torch.cuda.synchronize()
        serve = serving(args, H)
        if world > 1:
            serve["solves_per_s"] = rank_reduce([serve["solves_per_s"]], "sum", world, dev)[0]
            serve["p99_ms_max_over_ranks"] = rank_reduce([serve["p99_ms"]], "max", world, dev)[0]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_mixed, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 V-cycles in f64 refinement", "data": "synthetic",
            "config": {"workload": f"Poisson, {nc}x{nc}x{nc} cuboid ({6 * nc ** 3} macro-tets), level {L}, "
                                   f"V(3,3) multicolour SOR w=1, FP64 CG coarse on level 0, to rel. residual 1e-8",
                       "dofs": ndof, "unknowns": n_unknowns, "colours": {"interface": m_col, "interior": 4},
                       "l2": "inputs larger than L2 (FP64 finest vector 140 MB > 126 MB)",
                       "parallelism": "replicas" if world > 1 else "single GPU"},
            "time_to_tol_ms": {"mixed": ms_mixed, "fp64": ms_fp64},
            "speedup_mixed_vs_fp64": ms_fp64 / ms_mixed,
            "cycles": {"mixed": cyc_mixed[-1], "fp64": cyc_fp64[-1]},
            "final_rel_residual": {"mixed": float(hist_mixed[-1][-1]), "fp64": float(hist_fp64[-1][-1])},
            "error_mixed_vs_fp64_solution": err_mixed,
            "dof_updates_per_s_fp64": world * n_unknowns * sum(cyc_fp64) / (t_fp64 / 1e3),
            "roofline": dict(roof(sor_gbs, sweep64_traffic, "ncu (warm caches), profiles/" + sweep_prof),
                             kernel="k_sor_iface + k_sor_interior (one FP64 multicolour SOR sweep, 10 launches, level 7)",
                             ms=t_sor * 1e3),
            "roofline_apply": dict(roof(apply_gbs, apply_traffic, "ncu (warm caches), profiles/" + apply_prof),
                                   kernel="k_apply (FP64 stencil apply, level 7)", ms=t_apply * 1e3),
            "roofline_sor_fp32": dict(roof(sor32_gbs, sweep32_traffic, "ncu (warm caches), profiles/" + sweep_prof),
                                      kernel="k_sor_iface + k_sor_interior (FP32 sweep, level 7)", ms=t_sor32 * 1e3),
            "reference_order_fp64": ref_order,
            "e2e": e2e, "gpu_launches": launches, "clocks": clocks, "cpu_baseline": cpu,
            "variable_coefficient": varcoef, "spherical_shell": shell, "blended_shell": blend, "serving": serve,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def variable_coefficient(args, H, I, stream, nc=4, L=6, steps=2):
    """-div(k grad u) = f with the P1 elementwise operator on the 4x4x4 cuboid (384
    macro-tets) at level 6; k = exp(g), g a Gaussian random field (correlation length 0.2,
    sigma 1, seed 1; 64 random Fourier features, evaluated on the device); f ~ U[-1,1]
    seeded; V(3,3) multicolour SOR, FP64 and FP32-inner/FP64-refinement, each to 1e-8."""
    import numpy as np
    import torch

    sh = stream.cuda_stream
    st = H.PrimitiveStorage.cuboid(nc, nc, nc, L)
    w, ph = I.grf_features(0.2, 1, 64)
    A = H.P1ElementwiseDivKGradOperator.random_features(st, 0, L, w, ph, 1.0)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0, coarse_tol=1e-12)
    u, b = H.P1Function("u", st, 0, L), H.P1Function("f", st, 0, L)
    b.fill_uniform_random(L, 0, float(nc << L), stream=sh)
    n_unknowns = (nc * (1 << L) - 1) ** 3

    def solve(precision, tol=TOL):
        u.interpolate(0.0, L, flag=H.ALL, stream=sh)
        return gmg.solve_to_tolerance(u, b, L, tol, max_cycles=200, precision=precision, stream=sh)

    out = {}
    for prec in (32, 64):
        solve(prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hist = [solve(prec) for _ in range(steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        out[prec] = (ms, len(hist[-1]) - 1, float(hist[-1][-1]))
    solve(32)
    u_mixed = u.get(L, stream=sh)
    solve(64, 1e-13)
    u_ref = u.get(L, stream=sh)
    # the same problem with the coefficient at every micro-tet's quadrature points on every
    # level (the reference form's callback semantics) instead of the levels' nodal values
    Aq = H.P1ElementwiseDivKGradOperator.quadrature(st, 0, L, 2, w, ph, sigma=1.0)
    gq = H.GeometricMultigridSolver(st, Aq, 0, L, 3, 3, 1.0, coarse_tol=1e-12)
    quad = {}
    for prec in (32, 64):
        u.interpolate(0.0, L, flag=H.ALL, stream=sh)
        gq.solve_to_tolerance(u, b, L, TOL, max_cycles=200, precision=prec, stream=sh)
        u.interpolate(0.0, L, flag=H.ALL, stream=sh)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hq = gq.solve_to_tolerance(u, b, L, TOL, max_cycles=200, precision=prec, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        quad[prec] = (e0.elapsed_time(e1), len(hq) - 1)
    u.interpolate(0.0, L, flag=H.ALL, stream=sh)
    gq.solve_to_tolerance(u, b, L, 1e-13, max_cycles=200, precision=64, stream=sh)
    u_q = u.get(L, stream=sh)
    return {"workload": f"-div(k grad u)=f, {nc}x{nc}x{nc} cuboid ({6 * nc ** 3} macro-tets), level {L}, k=exp(GRF "
                        f"corr 0.2 sigma 1 seed 1), V(3,3) multicolour SOR, to rel. residual 1e-8",
            "dofs": st.num_dofs(L), "time_to_tol_ms": {"mixed": out[32][0], "fp64": out[64][0]},
            "speedup_mixed_vs_fp64": out[64][0] / out[32][0], "cycles": {"mixed": out[32][1], "fp64": out[64][1]},
            "final_rel_residual": {"mixed": out[32][2], "fp64": out[64][2]},
            "dof_updates_per_s": {"mixed": n_unknowns * out[32][1] / (out[32][0] / 1e3),
                                  "fp64": n_unknowns * out[64][1] / (out[64][0] / 1e3)},
            "error_mixed_vs_fp64_solution": float(np.abs(u_mixed - u_ref).max() / np.abs(u_ref).max()),
            "quadrature_coefficient": {
                "time_to_tol_ms": {"mixed": quad[32][0], "fp64": quad[64][0]},
                "cycles": {"mixed": quad[32][1], "fp64": quad[64][1]},
                "solution_vs_nodal_coefficient": float(np.abs(u_q - u_ref).max() / np.abs(u_ref).max()),
                "note": "coefficient at every micro-tet's quadrature points on every level (the reference "
                        "form's callback semantics); one timed solve each"}}


def spherical_shell(args, H, I, stream, ntan=5, nrad=4, L=6):
    """Thick spherical shell, radii 0.55..1.0, icosahedral tangential resolution ntan = 5,
    nrad = 4 radii (3 radial layers), affine macro-tets, level 6; -div(k grad u) = f with
    k = exp(5 (1 - r)) times lognormal noise exp(0.5 g), g a Gaussian random field
    (correlation length 0.2, seed 2); f ~ U[-1,1] seeded; V(2,2) cycles, mixed precision
    and FP64, each to 1e-8."""
    import numpy as np
    import torch

    sh = stream.cuda_stream
    t0 = time.perf_counter()
    st = H.PrimitiveStorage.spherical_shell(ntan, nrad, 0.55, 1.0, L)
    setup_s = time.perf_counter() - t0
    w, ph = I.grf_features(0.2, 2, 64)
    A = H.P1ElementwiseDivKGradOperator.random_features(st, 0, L, w, ph, 0.5, radial=5.0)
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 2, 2, 1.0, coarse_tol=1e-12)
    u, b = H.P1Function("u", st, 0, L), H.P1Function("f", st, 0, L)
    b.fill_uniform_random(L, 0, float(1 << 20), stream=sh)  # points are not on a lattice: a fine one
    mask = H.P1Function("mask", st, L, L)
    mask.interpolate(1.0, L, flag=H.INNER | H.NEUMANN)
    n_unknowns = int(round(mask.dot_global(mask, L, H.INNER | H.NEUMANN)))
    del mask

    def solve(precision, tol=TOL):
        u.interpolate(0.0, L, flag=H.ALL, stream=sh)
        return gmg.solve_to_tolerance(u, b, L, tol, max_cycles=300, precision=precision, stream=sh)

    out = {}
    for prec in (32, 64):
        solve(prec)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hist = solve(prec)
        e1.record(stream)
        torch.cuda.synchronize()
        out[prec] = (e0.elapsed_time(e1), len(hist) - 1, float(hist[-1]))
    solve(32)
    u_mixed = u.get(L, stream=sh)
    solve(64, 1e-12)
    u_ref = u.get(L, stream=sh)
    m_col, _ = st.colouring()
    err = float(np.abs(u_mixed - u_ref).max() / np.abs(u_ref).max())
    ndofs = st.num_dofs(L)
    del gmg, A, u, b, st
    torch.cuda.synchronize()
    # the same shape as serving requests: four solves, 0.1 s apart, after a warm-up round
    # that leaves four resident hierarchies
    sv = H.Server(int(args.serve_budget_gb * (1 << 30)), max_active=4, max_level=L)
    for i in range(4):
        sv.submit(H.Server.request(ntan, nrad, 1, L, H.COEFF_RADIAL, 32, 500 + i, mesh=H.MESH_SHELL))
    sv.run(600)
    ids = [sv.submit(H.Server.request(ntan, nrad, 1, L, H.COEFF_RADIAL, 32, 600 + i, mesh=H.MESH_SHELL),
                     arrival_s=0.1 * i) for i in range(4)]
    sv.run(600)
    res = [sv.result(i) for i in ids]
    lat = [(r.done_s - r.arrival_s) * 1e3 for r in res]
    served = {"requests": 4, "arrivals_s": [0.0, 0.1, 0.2, 0.3], "statuses": sorted({r.status for r in res}),
              "latency_ms": lat, "cycles": [r.cycles for r in res],
              "solves_per_s": 4 / (max(r.done_s for r in res) - min(r.arrival_s for r in res))}
    sv.close()
    return {"workload": f"spherical shell ntan={ntan} nrad={nrad} (3 radial layers) r in [0.55, 1], "
                        f"{60 * (ntan - 1) ** 2 * (nrad - 1)} macro-tets, level {L}, "
                        f"k=exp(5(1-r))*exp(0.5 GRF corr 0.2 seed 2), V(2,2) multicolour SOR, to rel. residual 1e-8",
            "dofs": ndofs, "unknowns": n_unknowns, "interface_colours": m_col, "setup_s": setup_s,
            "time_to_tol_ms": {"mixed": out[32][0], "fp64": out[64][0]},
            "speedup_mixed_vs_fp64": out[64][0] / out[32][0], "cycles": {"mixed": out[32][1], "fp64": out[64][1]},
            "final_rel_residual": {"mixed": out[32][2], "fp64": out[64][2]},
            "dof_updates_per_s": {"mixed": n_unknowns * out[32][1] / (out[32][0] / 1e3),
                                  "fp64": n_unknowns * out[64][1] / (out[64][0] / 1e3)},
            "error_mixed_vs_fp64_solution": err, "as_serving_requests": served}


# flops of one blended micro-tet row evaluation as the kernel formulates it (edges 54,
# inverse Jacobian 42, coefficient products 25, five quadrature points 111 each, row sums
# and accumulation 10): the map Jacobian's rank-one inverse and the 5-point rule
BLEND_FLOPS_PER_TET_ROW = 690
FP64_NOMINAL_TFLOPS = 37.0  # B200 FP64 (CUDA cores), nominal; no measured FP64 peak on this pool


def blended_shell(args, H, stream, ntan=5, nrad=4, L=5):
    """The curved shell: the mesh of the spherical-shell leg with every macro-cell carrying
    its IcosahedralShellMap, -div(k grad u) = f with p1_div_k_grad_blending_q3 element
    matrices integrated on the device per row, k = exp(5 (1 - |x|)) at the mapped points,
    f ~ U[-1,1] seeded; V(2,2) cycles, mixed precision and FP64 to 1e-8, and the FP64
    apply's arithmetic rate (4 N^3 micro-tet rows per cell and apply)."""
    import torch

    sh = stream.cuda_stream
    t0 = time.perf_counter()
    st = H.PrimitiveStorage.spherical_shell(ntan, nrad, 0.55, 1.0, L)
    A = H.P1ElementwiseBlendingDivKGradOperator(st, 0, L, 5.0)
    setup_s = time.perf_counter() - t0
    gmg = H.GeometricMultigridSolver(st, A, 0, L, 2, 2, 1.0, coarse_tol=1e-12)
    u, b = H.P1Function("u", st, 0, L), H.P1Function("f", st, 0, L)
    b.fill_uniform_random(L, 0, float(1 << 20), stream=sh)
    out = {}
    for prec in (32, 64):
        u.interpolate(0.0, L, flag=H.ALL, stream=sh)
        gmg.solve_to_tolerance(u, b, L, TOL, max_cycles=2, precision=prec, stream=sh)
        torch.cuda.synchronize()
        u.interpolate(0.0, L, flag=H.ALL, stream=sh)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        hist = gmg.solve_to_tolerance(u, b, L, TOL, max_cycles=100, precision=prec, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        out[prec] = (e0.elapsed_time(e1), len(hist) - 1, float(hist[-1]))
    y = H.P1Function("y", st, L, L)
    for _ in range(2):
        A.apply(b, y, L, H.ALL, stream=sh)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    e0.record(stream)
    for _ in range(reps):
        A.apply(b, y, L, H.ALL, stream=sh)
    e1.record(stream)
    torch.cuda.synchronize()
    t_apply = e0.elapsed_time(e1) / reps / 1e3
    n_cells = 60 * (ntan - 1) ** 2 * (nrad - 1)
    flops = 4 * (1 << L) ** 3 * n_cells * BLEND_FLOPS_PER_TET_ROW
    ndofs = st.num_dofs(L)
    del gmg, A, u, b, y, st
    torch.cuda.synchronize()
    return {"workload": f"curved spherical shell ntan={ntan} nrad={nrad} r in [0.55, 1], {n_cells} macro-tets with "
                        f"IcosahedralShellMap, level {L}, p1_div_k_grad_blending_q3 with k=exp(5(1-|x|)), "
                        f"V(2,2) multicolour SOR, to rel. residual 1e-8",
            "dofs": ndofs, "setup_s": setup_s,
            "time_to_tol_ms": {"mixed": out[32][0], "fp64": out[64][0]},
            "cycles": {"mixed": out[32][1], "fp64": out[64][1]},
            "final_rel_residual": {"mixed": out[32][2], "fp64": out[64][2]},
            "apply": {"kernel": "k_row_pass_blend<double, kRowApply> (FP64 apply, all rows)", "ms": t_apply * 1e3,
                      "bound": "fp64", "achieved_tflops": flops / t_apply / 1e12,
                      "peak_tflops": FP64_NOMINAL_TFLOPS, "peak_source": "nominal",
                      "frac": flops / t_apply / 1e12 / FP64_NOMINAL_TFLOPS,
                      "flops_per_apply": flops, "flops_per_tet_row": BLEND_FLOPS_PER_TET_ROW}}


def serve_stream(n, rate, seed, levels=(3, 7), cubes=(1, 4)):
    """Open-loop request stream: Poisson arrivals at `rate` per second; per request a
    cuboid mesh of c x c x c macro-cubes (c uniform in `cubes`), a level uniform in
    `levels`, a constant or lognormal coefficient with equal odds, its own seed for f and
    k; mixed precision to 1e-8."""
    import numpy as np

    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n))
    t -= t[0]
    out = []
    for i in range(n):
        c = int(rng.integers(cubes[0], cubes[1] + 1))
        out.append((float(t[i]), (c, c, c, int(rng.integers(levels[0], levels[1] + 1)), int(rng.integers(0, 2)), 32,
                                  int(rng.integers(1, 1 << 62)))))
    return out


def serving(args, H):
    """Serving stream at --rate requests/s through the continuous-batching loop. Warm-up:
    one request of every shape the stream holds, so that hierarchies are resident and
    their graphs captured before the timed stream (as in a long-running server). Then the
    same requests one at a time (the mix's throughput without overlap) and a second stream
    at 0.7x the measured capacity (latency without a backlog)."""
    import numpy as np

    stream = serve_stream(args.serve_requests, args.rate, 1234)
    sv = H.Server(int(args.serve_budget_gb * (1 << 30)), max_active=args.serve_slots, max_level=7)
    t0 = time.perf_counter()
    shapes = sorted({q[:6] for _, q in stream})
    for i, sh in enumerate(shapes):
        sv.submit(H.Server.request(*sh, seed=10_000 + i), arrival_s=0.0)
    sv.run(600)
    warm_s = time.perf_counter() - t0
    ids = [sv.submit(H.Server.request(*q), arrival_s=a) for a, q in stream]
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        sv.run(900)
    res = [sv.result(i) for i in ids]
    ok = [r for r in res if r.status == 0]
    lat = np.array([(r.done_s - r.arrival_s) * 1e3 for r in ok])
    wait = np.array([(r.admit_s - r.arrival_s) * 1e3 for r in ok])
    makespan = max(r.done_s for r in res) - min(r.arrival_s for r in res)

    # unknowns (interior micro-vertices) x cycles of the completed solves
    def work_of(strm, results):
        return sum((q[0] * (1 << q[3]) - 1) ** 3 * r.cycles for (a, q), r in zip(strm, results) if r.status == 0)

    work = work_of(stream, res)
    stats = sv.stats()
    # the same requests one at a time (one slot, all present at the start): the throughput of
    # this mix without overlap, what the concurrent loop is compared with
    sq = H.Server(int(args.serve_budget_gb * (1 << 30)), max_active=1, max_level=7)
    for i, sh in enumerate(shapes):
        sq.submit(H.Server.request(*sh, seed=10_000 + i), arrival_s=0.0)
    sq.run(600)
    sids = [sq.submit(H.Server.request(*q), arrival_s=0.0) for a, q in stream]
    sq.run(900)
    sres = [sq.result(i) for i in sids]
    s_span = max(r.done_s for r in sres) - min(r.arrival_s for r in sres)
    sq.close()
    # a stream at a rate the loop sustains (0.7 x the measured capacity): latency without a backlog
    rate2 = max(1.0, round(0.7 * len(ok) / makespan, 1))
    stream2 = serve_stream(args.serve_requests, rate2, 4321)
    ids2 = [sv.submit(H.Server.request(*q), arrival_s=a) for a, q in stream2]
    sv.run(900)
    res2 = [sv.result(i) for i in ids2]
    ok2 = [r for r in res2 if r.status == 0]
    lat2 = np.array([(r.done_s - r.arrival_s) * 1e3 for r in ok2])
    sv.close()
    return {"rate_req_per_s": args.rate, "requests": len(res), "completed": len(ok),
            "statuses": sorted({r.status for r in res}),
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "p50_queue_ms": float(np.percentile(wait, 50)),
            "solves_per_s": len(ok) / makespan, "makespan_s": makespan,
            "dof_updates_per_s": work / makespan,
            "one_at_a_time": {"dof_updates_per_s": work_of(stream, sres) / s_span, "solves_per_s": len(sres) / s_span,
                              "makespan_s": s_span},
            "concurrent_over_one_at_a_time": (work / makespan) / (work_of(stream, sres) / s_span),
            "sustained": {"rate_req_per_s": rate2, "completed": len(ok2), "p50_ms": float(np.percentile(lat2, 50)),
                          "p99_ms": float(np.percentile(lat2, 99)), "mean_ms": float(lat2.mean())},
            "max_rel_residual": max(r.rel_residual for r in ok),
            "slots": args.serve_slots, "budget_gb": args.serve_budget_gb, "warmup_s": warm_s,
            "peak_gb": stats["peak_bytes"] / 2 ** 30, "hierarchies_built": stats["hierarchies_built"],
            "graphs_captured": stats["graphs_captured"], "batched_solves": stats["batched_solves"],
            "batch_launches": stats["batches"], "clocks": clk.summary(),
            "workload": "Poisson arrivals; c x c x c cubes c~U{1..4}, level~U{3..7}, k constant or lognormal "
                        "(exp of GRF, corr. 0.2, sigma 1), seeded f, mixed V(3,3) to 1e-8; latency = arrival "
                        "to result on the host"}


def cpu_baseline(args, steps=1):
    """The CPU oracle (a restatement of the reference's algorithm) on the host cores:
    FP64 V(3,3) cycles with the reference's SOR ordering on the same problem."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O

    cores = os.cpu_count() or 1
    threads = O.set_threads(cores)
    c, t = O.mesh_cuboid(args.cubes, args.cubes, args.cubes)
    orc = O.Oracle(c, t, args.level)
    L = args.level
    b = O.uniform_rhs(orc.coords_of(L), 0, args.cubes << L)
    kind, bc = orc.info(L)
    n_unknowns = int(np.sum((bc & (O.INNER | O.NEUMANN)) != 0))
    x = np.zeros(orc.n(L))
    t0 = time.perf_counter()
    orc.gmg(x, b, 0, L, smoother=0, max_cycles=steps)
    dt = time.perf_counter() - t0
    return {"value": n_unknowns * steps / dt, "unit": UNIT, "cores": threads, "host_cores": cores, "threads": threads,
            "kind": "port",
            "sample": f"{steps} FP64 V(3,3) cycle(s) at level {L} on the {6 * args.cubes ** 3}-tet mesh, "
                      f"reference SOR ordering, {threads} OpenMP threads, {dt:.2f} s"}


def reference(args, rank, world):
    """The reference's algorithm on the host CPU: the oracle port (the reference itself cannot
    be built here: its waLBerla and Eigen submodules and MPI are absent), FP64 with the
    reference's staged lexicographic SOR, OpenMP over all host threads (the count is stated).
    Each timed step is one V(3,3) cycle of the workload (a bounded sample; the unit is the
    same DoF-updates/s per V-cycle as ours). Besides the K timed cycles, the line reports one
    whole FP64 solve from zero to relative residual 1e-8 (its cycles and seconds: the
    time-to-tolerance form of the metric) and one cycle on a single thread (the reference's
    default build has no OpenMP)."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle as O

    cores = os.cpu_count() or 1
    threads = O.set_threads(cores)
    c, t = O.mesh_cuboid(args.cubes, args.cubes, args.cubes)
    L = args.level
    orc = O.Oracle(c, t, L)
    b = O.uniform_rhs(orc.coords_of(L), 0, args.cubes << L)
    kind, bc = orc.info(L)
    n_unknowns = int(np.sum((bc & (O.INNER | O.NEUMANN)) != 0))
    x = np.zeros(orc.n(L))
    for _ in range(args.warmup):
        orc.gmg(x, b, 0, L, smoother=0, max_cycles=1)
    x[:] = 0
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.gmg(x, b, 0, L, smoother=0, max_cycles=1)
    dt = time.perf_counter() - t0
    value = n_unknowns * args.steps / dt
    # one whole solve to tolerance from the zero guess
    x[:] = 0
    t0 = time.perf_counter()
    _, hist = orc.gmg(x, b, 0, L, smoother=0, max_cycles=60, rel_tol=TOL)
    t_tol = time.perf_counter() - t0
    # one cycle on one thread
    O.set_threads(1)
    x[:] = 0
    t0 = time.perf_counter()
    orc.gmg(x, b, 0, L, smoother=0, max_cycles=1)
    t_one = time.perf_counter() - t0
    O.set_threads(threads)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"Poisson, {args.cubes}x{args.cubes}x{args.cubes} cuboid "
                                   f"({6 * args.cubes ** 3} macro-tets), level {L}, FP64 V(3,3) cycles, "
                                   f"reference SOR ordering (one cycle per timed step)",
                       "unknowns": n_unknowns, "threads": threads, "host_cores": cores},
            "time_to_tol_s": {"fp64": t_tol, "cycles": len(hist) - 1, "final_rel_residual": float(hist[-1]),
                              "dof_updates_per_s": n_unknowns * (len(hist) - 1) / t_tol},
            "single_thread": {"dof_updates_per_s": n_unknowns / t_one, "s_per_cycle": t_one},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "host_cores": cores, "threads": threads,
                             "kind": "port",
                             "sample": f"{args.steps} FP64 V(3,3) cycles at level {L}, reference SOR ordering, "
                                       f"{threads} OpenMP threads"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def single_op(args):
    """Run one level operation repeatedly (for ncu captures of a single kernel):
    --op apply|residual|sor|sor32|restrict|prolong at --level on the bench mesh, or
    --op vcycle: FP64 V(3,3) cycles from --level down to level 0 (program kernel, row
    passes of the middle levels, CG); --op blend_apply: the blending operator's FP64 apply
    on the curved shell (ntan 5, nrad 4) at --level (blend_apply32: FP32 rows)."""
    import torch

    import build as B
    import hyb_inputs as I
    import hyteg_b200 as H

    B.build()
    L, nc = args.level, args.cubes
    if args.op in ("blend_apply", "blend_apply32"):
        # the curved shell (ntan 5, nrad 4) with the blending operator, FP64 (FP32) apply
        st = H.PrimitiveStorage.spherical_shell(5, 4, 0.55, 1.0, L)
        A = H.P1ElementwiseBlendingDivKGradOperator(st, L, L, 5.0)
        bt = H.F32 if args.op == "blend_apply32" else H.F64
        b, y = H.P1Function("b", st, L, L, bt), H.P1Function("y", st, L, L, bt)
        b.interpolate(1.0, L, flag=H.ALL)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            A.apply(b, y, L, H.ALL)
        torch.cuda.synchronize()
        print(json.dumps({"op": args.op, "level": L, "dofs": st.num_dofs(L), "reps": args.steps,
                          "us_per_call_wall": (time.perf_counter() - t0) / args.steps * 1e6}))
        return
    st = H.PrimitiveStorage.cuboid(nc, nc, nc, L)
    A = H.P1ConstantLaplaceOperator(st, 0, L)
    dt = H.F32 if args.op == "sor32" else H.F64
    u, b, y = (H.P1Function(n, st, 0, L, dt) for n in "uby")
    for lv in range(L + 1):
        f = I.uniform_rhs(st.dof_coords(lv), 0, nc << lv)
        if dt == H.F64:
            b.set(f, lv)
            u.set(0.1 * f, lv)
        else:
            b.set(f.astype("float32"), lv)
            u.set((0.1 * f).astype("float32"), lv)
    F = H.INNER | H.NEUMANN
    # a solver's first cycle builds the levels' row tables, as in every solve
    x64, b64 = H.P1Function("x64", st, 0, L), H.P1Function("b64", st, 0, L)
    H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0).solve(x64, b64, L)
    del x64, b64
    P, R = H.P1toP1LinearProlongation(), H.P1toP1LinearRestriction()
    ops = {"apply": lambda: A.apply(b, y, L, F), "residual": lambda: A.residual(u, b, y, L, F),
           "sor": lambda: A.smooth_sor(u, b, 1.0, L, F), "sor32": lambda: A.smooth_sor(u, b, 1.0, L, F),
           "restrict": lambda: R.restrict(y, L, F), "prolong": lambda: P.prolongate_and_add(u, L - 1, F)}
    if args.op == "vcycle":
        gmg = H.GeometricMultigridSolver(st, A, 0, L, 3, 3, 1.0)
        ops["vcycle"] = lambda: gmg.solve(u, b, L)
    fn = ops[args.op]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        fn()
    torch.cuda.synchronize()
    print(json.dumps({"op": args.op, "level": L, "dofs": st.num_dofs(L), "reps": args.steps,
                      "us_per_call_wall": (time.perf_counter() - t0) / args.steps * 1e6}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--level", type=int, default=7)
    ap.add_argument("--cubes", type=int, default=2)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-stream leg")
    ap.add_argument("--no-varcoef", action="store_true", help="skip the variable-coefficient leg")
    ap.add_argument("--no-shell", action="store_true", help="skip the spherical-shell leg")
    ap.add_argument("--no-blend", action="store_true", help="skip the curved-shell (blending operator) leg")
    ap.add_argument("--no-reference-order", action="store_true",
                    help="skip the FP64 solve with SOR in the reference's own order")
    ap.add_argument("--serve-only", action="store_true", help="run only the serving-stream leg")
    ap.add_argument("--rate", type=float, default=200.0, help="serving arrival rate, requests/s")
    ap.add_argument("--serve-requests", type=int, default=100)
    ap.add_argument("--serve-slots", type=int, default=16)
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--op", default=None, choices=["apply", "residual", "sor", "sor32", "restrict", "prolong", "vcycle",
                                                       "blend_apply", "blend_apply32"],
                    help="profiling mode: repeat one level operation --steps times")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.op:
        single_op(args)
    elif args.serve_only:
        import torch

        import build as B
        import hyteg_b200 as H

        B.build()
        torch.cuda.set_device(local_rank)
        print(json.dumps(serving(args, H)), flush=True)
    elif args.impl == "reference":
        reference(args, rank, world)
    else:
        ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
