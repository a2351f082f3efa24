"""Benchmark: PPE time to 1e-8 relative residual on one B200 (plus CCD bandwidth).

Workload (the configuration the headline metric is quoted on): variable-density
PPE on a 512^2 unit box, rho_l/rho_g = 1000, 12 seeded droplets, RHS = the
divergence of an 8-mode seeded velocity, Neumann walls with the centre node
pinned, stop at ||r|| < 1e-8 ||b|| of the control-volume-weighted SPD system
(the reference's CG route).  A "step" is one full PPE solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

value  = ms per solve of the B200 method (device-resident inputs, L2 flushed
         between steps), max over ranks.
e2e    = the same through the public Python API with host NumPy inputs:
         rhs and rho copied host->device and p copied back inside the timed region.
The reference arm (--impl reference) times the CPU restatement of the
reference's CG + Jacobi solve on the host cores: full solves, as many as fit
in about 150 s (``steps`` says how many), beside the quick-start step's
CPU time.

Output: one detail line (``"bench_detail": true``: the CCD table, the 257^3
operator blocks, held-out learned fields, batching, the 192^3 step), then the
headline line last: plain / mixed / learned PPE ms and speed-ups, the
quick-start step ms (``c1_ms_per_step``), ``roofline``, ``cpu_baseline``,
``e2e`` and ``clocks``.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

N_PPE = (512, 512)
TOL = 1e-8
METRIC = "PPE ms to 1e-8 relative residual (512^2, rho ratio 1000, 12 droplets)"
WORKLOAD = "ppe_512x512_rho1000_12drops"


class _Cfg:
    def __init__(self, **kw):
        self.__dict__.update(kw)


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region (clocks + throttle reasons)."""

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def _max_over_ranks(x, ws):
    """Max of a per-rank device time over the replicas (NCCL on GPUs, gloo on CPU)."""
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def make_inputs():
    from twophaseflow_b200.workloads import divergence_rhs, droplet_density
    rho = droplet_density(N_PPE, seed=0)
    rhs = divergence_rhs(N_PPE, seed=1)
    return rho, rhs


def _solver(precision):
    """'fp64' / 'mixed': Jacobi PCG; 'learned': the learned solver's defaults."""
    from twophaseflow_b200 import PPESolverFVMMatrixFree, UniformGrid
    if precision == "learned":
        from twophaseflow_b200.learned import PPESolverLearned
        return PPESolverLearned(None, _Cfg(pseudo_tol=TOL, pseudo_maxiter=1_000_000, ppe_learned_maxiter=20000),
                                UniformGrid(N_PPE))
    cfg = _Cfg(pseudo_tol=TOL, pseudo_maxiter=1_000_000, ppe_iteration_method="cg", ppe_preconditioner="jacobi",
               ppe_precision=precision, ppe_inner_tol=1e-3)
    return PPESolverFVMMatrixFree(None, cfg, UniformGrid(N_PPE))


def time_ppe(precision, rho_d, rhs_d, steps, warmup, flush, cg_kernel=0):
    """Device-resident solves; L2 flushed before every step (untimed).
    ``cg_kernel``: 0 the default choice, 1 the all-global persistent kernel."""
    import ctypes
    import torch
    from twophaseflow_b200 import _lib
    s = _solver(precision)
    if cg_kernel:
        _lib.check(s.lib.tpf_ppe_set_cg_kernel(s._handle, ctypes.c_int(cg_kernel)))
    for _ in range(warmup):
        s.solve(rhs_d, rho_d)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        p = s.solve(rhs_d, rho_d)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return s, p, times


def time_learned(rho_d, rhs_d, steps, warmup, flush, **opts):
    """Network-preconditioned solve (shipped weights, two-level mode; the
    solver's defaults -- flexible GMRES(60), 16 sweeps -- unless ``opts`` give
    ``ppe_learned_*`` settings), device-resident inputs."""
    import torch
    from twophaseflow_b200 import UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned
    cfg = _Cfg(pseudo_tol=TOL, pseudo_maxiter=1_000_000, ppe_learned_maxiter=20000, **opts)
    s = PPESolverLearned(None, cfg, UniformGrid(N_PPE))
    for _ in range(warmup):
        s.solve(rhs_d, rho_d)
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        p = s.solve(rhs_d, rho_d)
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return s, p, times


def learned_heldout(sizes=((512, 512), (1024, 1024)), seeds=(11, 12, 13), **opts):
    """Learned preconditioner against plain FP64 PCG on density fields that were
    used neither in training nor in choosing its settings (12 droplets, seeded
    as the benchmark field): one warm-up and one timed solve of each, CUDA
    events, to 1e-8 relative residual; ``opts``: ``ppe_learned_*`` settings
    (default: the solver's)."""
    import torch
    from twophaseflow_b200 import PPESolverFVMMatrixFree, UniformGrid
    from twophaseflow_b200.learned import PPESolverLearned
    from twophaseflow_b200.workloads import divergence_rhs, droplet_density

    def timed(solver, rhs, rho):
        solver.solve(rhs, rho)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        p = solver.solve(rhs, rho)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), p

    out = {}
    for N in sizes:
        pc = PPESolverFVMMatrixFree(None, _Cfg(pseudo_tol=TOL, pseudo_maxiter=1_000_000, ppe_iteration_method="cg",
                                               ppe_preconditioner="jacobi"), UniformGrid(N))
        lr = PPESolverLearned(None, _Cfg(pseudo_tol=TOL, pseudo_maxiter=1_000_000, ppe_learned_maxiter=20000,
                                         **opts), UniformGrid(N))
        rows = []
        for seed in seeds:
            rho = torch.from_numpy(droplet_density(N, seed=seed)).cuda()
            rhs = torch.from_numpy(divergence_rhs(N, seed=seed + 100)).cuda()
            tp, pp = timed(pc, rhs, rho)
            tl, pl = timed(lr, rhs, rho)
            d = lr.last_diagnostics
            diff = float(torch.max(torch.abs((pl - pl.mean()) - (pp - pp.mean()))) / torch.max(torch.abs(pp - pp.mean())))
            rows.append({"seed": seed, "pcg_ms": round(tp, 2), "pcg_iterations": pc.last_diagnostics["ppe_low_order_cg_iterations"],
                         "learned_ms": round(tl, 2), "learned_iterations": d["ppe_learned_iterations"],
                         "fallback_iterations": d["ppe_learned_fallback_iterations"], "max_rel_diff": diff})
        geo = float(np.exp(np.mean([np.log(r["pcg_ms"] / r["learned_ms"]) for r in rows])))
        out[f"{N[0]}x{N[1]}"] = {"coarsen": lr.coarsen, "fields": rows, "speedup_geomean": round(geo, 3)}
    return out


def time_ppe_e2e(precision, rho_h, rhs_h, steps, warmup):
    """Public API with host NumPy inputs; H2D + solve + D2H inside the timed region."""
    import torch
    s = _solver(precision)
    for _ in range(warmup):
        s.solve(rhs_h, rho_h)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        p = s.solve(rhs_h, rho_h)
    e1.record()
    torch.cuda.synchronize()
    wall = (time.perf_counter() - t0) * 1e3 / steps
    return e0.elapsed_time(e1) / steps, wall, p


def time_ccd(N, bc, axis, dtype="f64", reps=10):
    """CCD line-kernel device time per call: `reps` calls captured in one CUDA
    graph and replayed (inputs 136 MB / 8 MB; a 3-D field exceeds L2)."""
    from twophaseflow_b200.kernel_cases import ccd_case
    r = ccd_case(tuple(N), axis, bc, dtype, reps)
    return {"N": list(N), "bc": bc, "axis": axis, "dtype": dtype, "us": r["us_per_call"], "GBps": r["GBps"]}


# DRAM bytes read + written by one cg1_band_kernel solve at 513^2 (ncu,
# dram__bytes_read.sum + dram__bytes_write.sum of the launch)
PCG_BAND_DRAM_BYTES_PER_SOLVE = 11.5e6
# DRAM bytes of one smooth_block_kernel launch (4 sweeps) at 513^2 (ncu,
# cold caches: the five inputs read once; the output stays in L2)
SMOOTH_DRAM_BYTES_PER_LAUNCH = 10.5e6


def time_c1(steps, warmup):
    """The quick-start step on the GPU (64^2 rising bubble, density and
    viscosity ratio 0.1, Re 100, Fr 1, We 10; UCCD6 convection, mass-corrected
    transport, Neumann reinitialization, GMRES(80) with the line
    preconditioner, no-slip walls): ms per step over ``steps`` steps after
    ``warmup`` steps, each at the CFL time step read back from the device, with
    the pre- and post-PPE work replayed from CUDA graphs."""
    import torch
    from twophaseflow_b200 import TwoPhaseStep, UniformGrid
    from twophaseflow_b200.workloads import quickstart_psi
    s = TwoPhaseStep(UniformGrid((64, 64)), quickstart_psi(), rho_ratio=0.1, mu_ratio=0.1, convection="uccd6",
                     transport_mass_correction=True, reinit_bc="neumann", ppe_method="gmres", ppe_maxiter=500,
                     no_slip=True, zero_velocity_shortcut=True)
    dt = 0.3 * float(np.sqrt(1.1 * 10.0 * (1.0 / 64) ** 3 / (2.0 * np.pi)))
    s.step(dt)
    for _ in range(warmup):
        s.step(s.cfl_dt())
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    its = []
    e0.record()
    for _ in range(steps):
        s.step(s.cfl_dt())
        its.append(s.last_ppe_iterations)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    return {"ms_per_step": round(ms, 3), "steps": steps, "gmres_iterations_mean": round(float(np.mean(its)), 1),
            "dt": s.cfl_dt(), "u_max": round(float(max(v.abs().max().item() for v in s.vel)), 6)}


def cpu_baseline_sample(rho, rhs, iters_full, max_iters=300):
    """Oracle (CPU restatement of the reference CG + Jacobi) timed on a bounded
    sample of iterations, extrapolated to the full iteration count."""
    from oracle import ppe as oppe
    coords = oppe.uniform_coords(N_PPE, (1.0, 1.0))
    o = oppe.FVMMatrixFree(coords, method="cg", preconditioner="jacobi", tol=1e-300, maxiter=max_iters)
    t0 = time.perf_counter()
    try:
        o.solve(rhs, rho)
    except RuntimeError:
        pass  # budget exhausted by design: this is a timing sample
    dt = time.perf_counter() - t0
    per_iter = dt / max_iters
    try:
        from threadpoolctl import threadpool_info
        cores = max([d.get("num_threads", 1) for d in threadpool_info()] + [1])
    except Exception:
        cores = 1
    return {"value": round(per_iter * iters_full * 1e3, 1), "unit": "ms", "cores": int(cores), "kind": "port",
            "sample": f"{max_iters} CG+Jacobi iterations of the 512^2 solve ({dt:.1f} s), "
                      f"extrapolated to {iters_full} iterations"}


def c1_reference_sample(n_steps=3):
    """The oracle's restatement of the reference quick-start step (64^2,
    density ratio 0.1, GMRES(80) + line preconditioner) on the host cores:
    ms per step over ``n_steps`` steps at the capillary-limited dt."""
    from oracle.ns_step import QuickStartStep
    from twophaseflow_b200.workloads import quickstart_psi
    s = QuickStartStep((64, 64), (1.0, 1.0), quickstart_psi())
    dt = 0.3 * np.sqrt(1.1 * 10.0 * (1.0 / 64) ** 3 / (2.0 * np.pi))
    s.step(dt)   # first step: zero velocity, setup
    t0 = time.perf_counter()
    for _ in range(n_steps):
        s.step(dt)
    return (time.perf_counter() - t0) * 1e3 / n_steps


def run_reference(args):
    """The reference's CPU path on the host cores: the oracle's restatement of
    PPESolverFVMMatrixFree's CG + Jacobi route (fvm_matrixfree.py:150-260 over
    SciPy cg), one FULL solve of the 512^2 system per timed step.  A full
    solve takes ~20 s, so the timed steps are capped to about 150 s of work;
    ``steps`` reports the solves actually timed and ``steps_requested`` the
    request.  Warm-up steps are bounded 200-iteration samples (untimed)."""
    ws, rank, _ = _dist()
    if rank != 0:
        return 0
    rho, rhs = make_inputs()
    from oracle import ppe as oppe
    coords = oppe.uniform_coords(N_PPE, (1.0, 1.0))
    for _ in range(args.warmup):
        cpu_baseline_sample(rho, rhs, 1, max_iters=200)
    times, iters = [], 0
    budget_s = 150.0
    t_all = time.perf_counter()
    while len(times) < args.steps:
        o = oppe.FVMMatrixFree(coords, method="cg", preconditioner="jacobi", tol=TOL, maxiter=1_000_000)
        t0 = time.perf_counter()
        o.solve(rhs, rho)
        times.append((time.perf_counter() - t0) * 1e3)
        iters = o.last_iterations
        if (time.perf_counter() - t_all) + times[-1] * 1e-3 > budget_s:
            break
    v = float(np.mean(times))
    try:
        from threadpoolctl import threadpool_info
        cores = max([d.get("num_threads", 1) for d in threadpool_info()] + [1])
    except Exception:
        cores = 1
    c1_ms = c1_reference_sample()
    line = {"impl": "reference", "metric": METRIC, "value": round(v, 1), "unit": "ms", "n_gpus": args.gpus,
            "steps": len(times), "steps_requested": args.steps, "warmup": args.warmup,
            "ms_per_step": round(v, 1), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded droplets, seeded velocity divergence)",
            "config": {"workload": WORKLOAD, "grid": list(N_PPE), "tol": TOL,
                       "method": "CG + Jacobi (the reference's CG route), NumPy on the host cores"},
            "cpu_baseline": {"value": round(v, 1), "unit": "ms", "cores": int(cores), "kind": "port",
                             "sample": f"{len(times)} full solves of the 512^2 system ({iters} CG iterations each)"},
            "e2e": {"value": round(v, 1), "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "iterations": iters,
            "c1_ms_per_step": round(c1_ms, 1),
            "c1_note": "quick-start 64^2 step (density ratio 0.1, GMRES(80) + line preconditioner), oracle port, 3 steps"}
    print(json.dumps(line), flush=True)
    return 0


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args(argv)
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    ws, rank, local = _dist()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    dev = torch.device("cuda", torch.cuda.current_device())
    rho, rhs = make_inputs()
    rho_d = torch.from_numpy(rho).to(dev)
    rhs_d = torch.from_numpy(rhs).to(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    # per plain solve: prepare (face couplings), rhs weighting, the persistent
    # CG kernel and the pin/copy-out = 4 kernel launches

    # plain FP64 PCG (the comparator of the headline), mixed precision, learned
    _barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        s64, p64, t64 = time_ppe("fp64", rho_d, rhs_d, args.steps, args.warmup, flush)
        torch.cuda.synchronize()
        _barrier(ws)
        # the learned solve (flexible GMRES(60), U-Net two-level preconditioner),
        # the same steps / warm-up and L2 flush
        slr, plr, tlr = time_learned(rho_d, rhs_d, args.steps, args.warmup, flush)
        torch.cuda.synchronize()
    _barrier(ws)
    it64 = s64.last_diagnostics["ppe_low_order_cg_iterations"]
    smx, pmx, tmx = time_ppe("mixed", rho_d, rhs_d, max(2, args.steps // 2), 1, flush)
    _barrier(ws)
    dmx = smx.last_diagnostics
    # the same mixed solve on the all-global FP32 kernel (kernel-for-kernel context)
    smg, _, tmg = time_ppe("mixed", rho_d, rhs_d, 2, 1, flush, cg_kernel=1)
    _barrier(ws)
    dmg = smg.last_diagnostics
    dlr = slr.last_diagnostics
    # the configuration's flexible GMRES(30), and flexible CG(8) with 3 sweeps
    sgm, pgm, tgm = time_learned(rho_d, rhs_d, 2, 1, flush, ppe_learned_outer="fgmres", ppe_learned_restart=30)
    _barrier(ws)
    dgm = dict(sgm.last_diagnostics)
    sfc, pfc, tfc = time_learned(rho_d, rhs_d, 2, 1, flush, ppe_learned_outer="fcg", ppe_learned_smooth=3)
    _barrier(ws)
    dfc = dict(sfc.last_diagnostics)
    heldout = learned_heldout()
    _barrier(ws)
    heldout30 = learned_heldout(ppe_learned_outer="fgmres", ppe_learned_restart=30)
    _barrier(ws)
    ms_mx = _max_over_ranks(float(np.mean(tmx)), ws)
    ms_64 = _max_over_ranks(float(np.mean(t64)), ws)
    ms_lr = _max_over_ranks(float(np.mean(tlr)), ws)
    err = float(torch.max(torch.abs(pmx - p64)).item() / torch.max(torch.abs(p64)).item())
    err_lr = float(torch.max(torch.abs(plr - p64)).item() / torch.max(torch.abs(p64)).item())
    best = min((ms_64, "fp64"), (ms_mx, "mixed"), (ms_lr, "learned"))[1]
    ms_best = min(ms_64, ms_mx, ms_lr)

    # e2e through the public API with host buffers (same method as the headline)
    e2e_ms, e2e_wall, _ = time_ppe_e2e(best, rho, rhs, max(2, args.steps // 2), 1)
    e2e_ms = _max_over_ranks(e2e_ms, ws)

    # roofline of the dominant kernel (persistent PCG, one launch per solve):
    # algorithmic bytes per FP64 iteration = 112 B/DOF (survey's fused 3-kernel
    # count); the 512^2 working set (~13 MB) is L2-resident, so this is a
    # latency-bound kernel measured against the HBM copy peak
    ndof = (N_PPE[0] + 1) * (N_PPE[1] + 1)
    peak, peak_kind = _peaks()
    alg64 = it64 * 112 * ndof
    ach64 = alg64 / (np.mean(t64) * 1e-3) / 1e9
    roof_plain = {"kernel": "cg1_band_kernel", "bound": "hbm", "achieved": round(ach64, 1), "peak": peak,
                  "peak_kind": peak_kind, "unit": "GB/s", "frac": round(ach64 / peak, 3),
                  "traffic": PCG_BAND_DRAM_BYTES_PER_SOLVE,
                  "note": "112 B/DOF/iteration algorithmic over the solve; vectors live in shared memory, "
                          "DRAM traffic is the inputs once (ncu); the iteration is bound by the grid reduction"}
    # the learned solve's top kernel by time share: the blocked damped-Jacobi
    # smoother (48 B per node and launch algorithmic, 4 sweeps per launch)
    from twophaseflow_b200.kernel_cases import smoother_case
    smo = smoother_case(N_PPE)
    roof_learned = {"kernel": "smooth_block_kernel", "bound": "hbm", "achieved": smo["GBps"], "peak": peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": round(smo["GBps"] / peak, 3),
                    "us_per_launch": smo["us_per_launch"], "traffic": SMOOTH_DRAM_BYTES_PER_LAUNCH,
                    "note": "48 B/node per launch algorithmic (z, r, D^-1, couplings read, z written; 4 sweeps); "
                            "the 513^2 operator is L2-resident"}
    # launches of the learned solve (flexible GMRES, two-level mode), counted
    # from its launch sequence: per Arnoldi column 27 for the preconditioner
    # (fused restriction, input packing, 14 convolutions, 6 resampling layers,
    # output layer, 4 blocked smoother launches, the first starting from the
    # prolongation), 1 operator and 4 Gram-Schmidt; per restart cycle 6; 12
    # for the set-up
    its_lr = dlr["ppe_learned_iterations"]
    launches_lr = its_lr * 32 + 6 * ((its_lr + 59) // 60) + 12

    # CCD line kernels (2-D 1024^2 and 3-D 256^3, FP64 and FP32), graph-timed
    ccd = []
    for N in ((1024, 1024), (256, 256, 256)):
        for dt in ("f64", "f32"):
            for bc in ("wall", "periodic"):
                for axis in range(len(N)):
                    ccd.append(time_ccd(N, bc, axis, dtype=dt))
    # FP32 line solves under FP64 iterative refinement against the direct FP64
    # solve (257^3 wall, strided and contiguous axis; error vs FP64 stated)
    from twophaseflow_b200.kernel_cases import ccd_refined_case
    ccd_ref = [ccd_refined_case((256, 256, 256), ax, 2, 3) for ax in (0, 2)]
    # the FCCD matrix-free PPE operator (2-D 1025^2 wall, 3-D 257^3 wall)
    from twophaseflow_b200.kernel_cases import fccd_ppe_case
    fccd_b = [fccd_ppe_case((1024, 1024), "wall", 5), fccd_ppe_case((256, 256, 256), "wall", 3)]
    ccd3 = [c for c in ccd if len(c["N"]) == 3 and c["dtype"] == "f64"]
    ccd3_gbps = float(np.mean([c["GBps"] for c in ccd3]))
    ccd3_best = max(ccd3, key=lambda c: c["GBps"])

    # velocity corrector fused into the CCD solve (3-D 257^3 FP64 wall, per
    # axis; 32 B/point algorithmic: read p, u*, rho, write u) against the same
    # step as separate CCD + wall zeroing + elementwise operations
    from twophaseflow_b200.kernel_cases import corrector_case
    corr = []
    for axis in range(3):
        r = corrector_case((256, 256, 256), axis, "wall", "f64", 5)
        corr.append({"axis": axis, "us": r["us_per_call"], "GBps": r["GBps"], "separate_ops_us": r["separate_ops_us"]})

    # interface curvature from psi and the Rhie-Chow PPE right-hand side
    # (3-D 257^3 FP64 wall; whole calls and their own kernels, graph-replayed)
    from twophaseflow_b200.kernel_cases import curvature_case, rhiechow_case
    curv = curvature_case((256, 256, 256), "wall", "f64", 3)
    rcb = rhiechow_case((256, 256, 256), "wall", "f64", 3)
    # CLS transport (one TVD-RK3 step, FCCD flux form) and split reinitialization
    # (4 pseudo-steps + mass correction), 3-D 257^3 FP64
    from twophaseflow_b200.kernel_cases import advect_case, reinit_case
    advb = advect_case((256, 256, 256), "periodic", "f64", 2)
    reib = reinit_case((256, 256, 256), "f64", 2)
    from twophaseflow_b200.kernel_cases import viscous_case
    visb = viscous_case((256, 256, 256), "f64", 2)

    # whole two-phase time steps, 3-D 192^3 rising bubble (density ratio 1000):
    # CFL time step with the capillary bound, the step (pressure solve
    # included) replayed as one CUDA graph
    try:
        from twophaseflow_b200.kernel_cases import step_case
        stepb = step_case((192, 192, 192), 4)
    except Exception as exc:   # the headline line must still print
        stepb = {"error": f"{type(exc).__name__}: {exc}"[:200]}

    # many independent cases in one persistent launch (32 seeded grids, 128..512 per axis)
    from twophaseflow_b200.kernel_cases import batched_case
    bat = batched_case(n_cases=32, reps=2)
    bat_small = batched_case(n_cases=64, nmin=64, nmax=64, reps=3)
    bat.pop("grids", None)

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(rho, rhs, it64)

    c1 = time_c1(args.steps, args.warmup)

    clocks = clk.summary()
    if rank == 0:
        # the detail blocks first, on their own line; the headline line last and short
        detail = {
            "bench_detail": True,
            "learned_heldout": heldout,
            "learned_heldout_fgmres30": heldout30,
            "batched_32_cases": bat,
            "batched_64_cases_64x64": bat_small,
            "ccd": ccd,
            "ccd_fp32_refined_257cubed": ccd_ref,
            "fccd_ppe_apply": fccd_b,
            "corrector_257cubed_f64_wall": {"per_axis": corr, "peak": peak, "peak_kind": peak_kind,
                                            "frac_mean": round(float(np.mean([c["GBps"] for c in corr])) / peak, 3)},
            "curvature_257cubed_f64_wall": {k: v for k, v in curv.items() if k not in ("case", "N", "bc", "dtype")},
            "rhiechow_257cubed_f64_wall": {k: v for k, v in rcb.items() if k not in ("case", "N", "bc", "dtype")},
            "cls_transport_257cubed_f64_periodic": {k: v for k, v in advb.items() if k not in ("case", "N", "bc", "dtype")},
            "reinit_257cubed_f64": {k: v for k, v in reib.items() if k not in ("case", "N", "dtype")},
            "viscous_257cubed_f64_wall": {k: v for k, v in visb.items() if k not in ("case", "N", "dtype")},
            "two_phase_step_192cubed": {k: v for k, v in stepb.items() if k not in ("case", "N")},
            "mixed_detail": {"kernel": "band-resident FP32 (shared-memory vectors), FP64 residual replacement",
                             "inner_iterations": dmx["ppe_low_order_cg_iterations"],
                             "replacements": dmx["ppe_low_order_cg_refinements"],
                             "rel_residual": dmx["ppe_low_order_cg_relative_residual"],
                             "us_per_iteration": round(float(np.mean(tmx)) * 1e3
                                                       / max(1, dmx["ppe_low_order_cg_iterations"]), 2),
                             "fp64_us_per_iteration": round(float(np.mean(t64)) * 1e3 / max(1, it64), 2),
                             "global_fp32_kernel_ms": round(float(np.mean(tmg)), 3),
                             "global_fp32_kernel_iterations": dmg["ppe_low_order_cg_iterations"]},
            "learned_fgmres30": {"ms": round(float(np.mean(tgm)), 3), "iterations": dgm["ppe_learned_iterations"],
                                 "fell_back": bool(dgm["ppe_learned_fell_back"]),
                                 "max_rel_diff_vs_fp64": float(f"{float(torch.max(torch.abs(pgm - p64))) / float(torch.max(torch.abs(p64))):.3g}")},
            "learned_fcg8_smooth3": {"ms": round(float(np.mean(tfc)), 3), "iterations": dfc["ppe_learned_iterations"],
                                     "fell_back": bool(dfc["ppe_learned_fell_back"]),
                                     "max_rel_diff_vs_fp64": float(f"{float(torch.max(torch.abs(pfc - p64))) / float(torch.max(torch.abs(p64))):.3g}")},
            "learned_detail": {"method": "flexible GMRES(60), U-Net two-level preconditioner, 16 Jacobi sweeps",
                               "fallback_iterations": dlr["ppe_learned_fallback_iterations"],
                               "rel_residual": dlr["ppe_learned_relative_residual"],
                               "us_per_iteration": round(ms_lr * 1e3 / max(1, dlr["ppe_learned_iterations"]), 1)},
        }
        print(json.dumps(detail), flush=True)
        line = {
            "metric": METRIC, "value": round(ms_best, 3), "unit": "ms", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_best, 3), "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": {"fp64": "f64", "mixed": "f32 inner / f64 outer", "learned": "bf16 preconditioner / f64 Krylov"}[best],
            "data": "synthetic (seeded droplets, seeded velocity divergence)",
            "config": {"workload": WORKLOAD, "grid": list(N_PPE), "tol": TOL,
                       "method": {"fp64": "FP64 Jacobi-PCG, persistent single-reduction kernel",
                                  "mixed": "mixed: band-resident FP32 Jacobi-PCG with FP64 residual replacement",
                                  "learned": "two-level U-Net-preconditioned flexible GMRES(60)"}[best],
                       "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{ws}"},
            "plain_fp64_pcg_ms": round(ms_64, 3), "plain_fp64_iterations": it64,
            "mixed_ms": round(ms_mx, 3), "mixed_max_rel_diff_vs_fp64": float(f"{err:.3g}"),
            "learned_ms": round(ms_lr, 3), "learned_iterations": dlr["ppe_learned_iterations"],
            "learned_max_rel_diff_vs_fp64": float(f"{err_lr:.3g}"),
            "learned_speedup_vs_plain_fp64": round(ms_64 / ms_lr, 3),
            "mixed_speedup_vs_plain_fp64": round(ms_64 / ms_mx, 3),
            "c1_ms_per_step": c1["ms_per_step"], "c1": c1,
            "ccd_frac_3d_f64": round(ccd3_gbps / peak, 3),
            "e2e": {"value": round(e2e_ms, 3), "unit": "ms", "h2d_bytes_per_step": 2 * ndof * 8,
                    "d2h_bytes_per_step": ndof * 8, "wall_ms": round(e2e_wall, 3)},
            "roofline": roof_learned if best == "learned" else roof_plain,
            "roofline_plain_fp64": roof_plain,
            "gpu_launches": (launches_lr if best == "learned" else 4) * args.steps,
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
