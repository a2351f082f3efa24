"""Run single hot-path kernels on synthetic inputs for timing and profiling.

    python -m twophaseflow_b200.kernel_cases ccd --N 256 256 256 --axis 0 --bc wall [--dtype f64] [--reps 5]
    python -m twophaseflow_b200.kernel_cases ppe --N 512 512 [--precision fp64] [--reps 2]
    python -m twophaseflow_b200.kernel_cases learned --N 512 512 [--maxiter 16] [--reps 2]
    python -m twophaseflow_b200.kernel_cases batched --N 32 [--reps 3]     (32 cases, grids 128..512)
    python -m twophaseflow_b200.kernel_cases gmres --N 512 512 [--line thomas|pcr] [--maxiter 2] [--reps 1]
    python -m twophaseflow_b200.kernel_cases corrector --N 256 256 256 --axis 0 --bc wall [--reps 5]
    python -m twophaseflow_b200.kernel_cases curvature --N 256 256 256 --bc wall [--reps 3]
    python -m twophaseflow_b200.kernel_cases rhiechow --N 256 256 256 --bc wall [--reps 3]
    python -m twophaseflow_b200.kernel_cases advect --N 256 256 256 --bc periodic [--reps 3]
    python -m twophaseflow_b200.kernel_cases reinit --N 256 256 256 [--reps 2]
    python -m twophaseflow_b200.kernel_cases viscous --N 256 256 256 [--reps 2]
    python -m twophaseflow_b200.kernel_cases step --N 192 192 192 [--reps 3]    (rising bubble, whole step)

``ccd`` captures ``reps`` CCDSolver.differentiate calls in one CUDA graph and
replays it, so the reported time is device time per call (no Python launch
overhead), and prints achieved GB/s over the algorithmic 3 x field bytes.
``ppe`` runs full CG+Jacobi solves (one persistent kernel each).
Used for the ncu captures summarised under profiles/.
"""

from __future__ import annotations

import argparse
import json
import sys


def ccd_case(N, axis, bc, dtype, reps, warmup=3):
    import torch
    from . import CCDSolver, UniformGrid
    from .workloads import fourier_field
    dt = torch.float64 if dtype == "f64" else torch.float32
    f = torch.from_numpy(fourier_field(N, seed=0)).to("cuda").to(dt)
    ccd = CCDSolver(UniformGrid(N), None, bc_type=bc, dtype=dt)
    for _ in range(warmup):
        ccd.differentiate(f, axis)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        outs = []
        with torch.cuda.graph(g, stream=s):
            for _ in range(reps):
                outs.append(ccd.differentiate(f, axis))
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    g.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    nbytes = 3 * f.numel() * f.element_size()
    return {"case": "ccd", "N": list(N), "axis": axis, "bc": bc, "dtype": dtype, "us_per_call": round(ms * 1e3, 2),
            "GBps": round(nbytes / (ms * 1e-3) / 1e9, 1), "alg_bytes": nbytes}


def ccd_refined_case(N, axis, refinements=2, reps=5):
    """FP32 CCD line solves under FP64 iterative refinement against the direct
    FP64 solve (wall, FP64 field f = 32 seeded Fourier modes): device time per
    call (graph-replayed, the workspace allocated outside the graph) and the
    error of each against the FP64 result relative to max |d|."""
    import torch
    from . import CCDSolver, UniformGrid
    from .workloads import fourier_field
    f = torch.from_numpy(fourier_field(N, seed=0)).to("cuda")
    ccd = CCDSolver(UniformGrid(N), None, bc_type="wall")
    d1, d2 = ccd.differentiate(f, axis)
    r1, r2 = ccd.differentiate_refined(f, axis, refinements)
    e1 = float((r1 - d1).abs().max() / d1.abs().max())
    e2 = float((r2 - d2).abs().max() / d2.abs().max())
    t64 = _graph_time(lambda: ccd.differentiate(f, axis), reps)
    tref = _graph_time(lambda: ccd.differentiate_refined(f, axis, refinements), reps)
    return {"case": "ccd_refined", "N": list(N), "axis": axis, "refinements": refinements,
            "us_fp64": round(t64 * 1e3, 2), "us_refined": round(tref * 1e3, 2),
            "err_d1_vs_fp64": e1, "err_d2_vs_fp64": e2}


def fccd_ppe_case(N, bc="wall", reps=5):
    """FCCD matrix-free PPE operator application (the image gather on periodic
    axes, one CCD second-derivative solve per axis, the fused face-gradient /
    coefficient / divergence kernel), graph-replayed, with its algorithmic
    bytes: per axis 16 B/node for the CCD call (read p, write q) plus
    (3 + ndim) x 8 B/node for the fused kernel (p, rho, the q's, out)."""
    import torch
    from . import FCCDSolver, PPESolverFCCDMatrixFree, UniformGrid
    from .workloads import divergence_rhs, droplet_density

    class Cfg:
        pseudo_tol = 1e-8
        pseudo_maxiter = 500
        ppe_preconditioner = "jacobi"

    grid = UniformGrid(N)
    s = PPESolverFCCDMatrixFree(None, Cfg(), grid, FCCDSolver(grid, None, bc_type=bc))
    rho = torch.from_numpy(droplet_density(N, seed=0, rho_g=0.1)).cuda()
    p = torch.from_numpy(divergence_rhs(N, seed=1)).cuda()
    s.prepare_operator(rho)
    t = _graph_time(lambda: s.apply(p), reps)
    nd = len(N)
    nbytes = p.numel() * 8 * (2 * nd + 3 + nd) + (p.numel() * 16 if bc == "periodic" else 0)
    return {"case": "fccd_apply", "N": list(N), "bc": bc, "us_per_apply": round(t * 1e3, 2),
            "GBps": round(nbytes / (t * 1e-3) / 1e9, 1), "alg_bytes": nbytes}


def _graph_time(fn, reps, warmup=3):
    """Device time per call of ``fn`` from a CUDA graph of ``reps`` calls."""
    import torch
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        with torch.cuda.graph(g, stream=s):
            for _ in range(reps):
                fn()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    g.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def corrector_case(N, axis, bc, dtype, reps):
    """Velocity corrector along one axis: the fused CCD solve
    (tpf_ccd_apply_corrector: read p, u*, rho, write u) against the same step
    as separate operations (CCD differentiate, wall zeroing, elementwise
    update), both graph-replayed."""
    import ctypes as C
    import torch
    from . import CCDSolver, UniformGrid, _lib
    from .arrays import line_split
    from .workloads import fourier_field
    dt_ = torch.float64 if dtype == "f64" else torch.float32
    p = torch.from_numpy(fourier_field(N, seed=0)).to("cuda").to(dt_)
    gen = torch.Generator(device="cuda").manual_seed(3)
    rho = 1e-3 + torch.rand(p.shape, device="cuda", dtype=dt_, generator=gen)
    u = torch.randn(p.shape, device="cuda", dtype=dt_, generator=gen)
    out = torch.empty_like(u)
    ccd = CCDSolver(UniformGrid(N), None, bc_type=bc, dtype=dt_)
    lib = _lib.load()
    outer, n, inner = line_split(p.shape, axis)
    plan = ccd._plan(axis, ccd._axis_periodic(axis))
    dt = 0.01

    def fused():
        _lib.check(lib.tpf_ccd_apply_corrector(plan, outer, inner, _lib.dptr(p), _lib.dptr(u), _lib.dptr(rho),
                                               C.c_double(dt), _lib.dptr(out), 0, _lib.current_stream_handle()))

    def separate():
        d1, _ = ccd.differentiate(p, axis)
        ccd.enforce_wall_neumann(d1, axis)
        out.copy_(u - (dt / rho) * d1)

    ms = _graph_time(fused, reps)
    ms_sep = _graph_time(separate, reps)
    nbytes = 4 * p.numel() * p.element_size()
    return {"case": "corrector", "N": list(N), "axis": axis, "bc": bc, "dtype": dtype,
            "us_per_call": round(ms * 1e3, 2), "GBps": round(nbytes / (ms * 1e-3) / 1e9, 1), "alg_bytes": nbytes,
            "separate_ops_us": round(ms_sep * 1e3, 2)}


def curvature_case(N, bc, dtype, reps):
    """Curvature from psi (CurvatureCalculatorPsi.compute: CCD derivatives,
    DCCD filter, mixed derivatives, curvature formula) on a sphere, and its
    filter and formula kernels alone, all graph-replayed."""
    import ctypes as C
    import numpy as np
    import torch
    from . import CCDSolver, CurvatureCalculatorPsi, UniformGrid, _lib
    from .levelset import _filter_tensor
    dt_ = torch.float64 if dtype == "f64" else torch.float32
    nd = len(N)
    ax = [torch.linspace(0.0, 1.0, n + 1, dtype=torch.float64, device="cuda") for n in N]
    X = torch.meshgrid(*ax, indexing="ij")
    phi = torch.sqrt(sum((X[a] - 0.5 + 0.02 * a) ** 2 for a in range(nd))) - 0.3
    eps = 1.5 / max(N)
    psi = torch.sigmoid(phi / eps).to(dt_).contiguous()
    del X, phi
    ccd = CCDSolver(UniformGrid(N), None, bc_type=bc, dtype=dt_)
    calc = CurvatureCalculatorPsi(None, ccd)
    ms_all = _graph_time(lambda: calc.compute(psi), reps)
    sw = ((2.0 * psi - 1.0) ** 2).contiguous()
    g = torch.randn(psi.shape, device="cuda", dtype=dt_)
    ms_f = _graph_time(lambda: _filter_tensor(g, ccd.grid, 0.05, bc, sw), reps)
    d = [torch.randn(psi.shape, device="cuda", dtype=dt_) for _ in range(2 * nd + (1 if nd == 2 else 3))]
    kap = torch.empty_like(psi)
    P = C.c_void_p * 3
    nm = 1 if nd == 2 else 3
    pd1 = P(*([_lib.dptr(t) for t in d[:nd]] + [None] * (3 - nd)))
    pd2 = P(*([_lib.dptr(t) for t in d[nd:2 * nd]] + [None] * (3 - nd)))
    pmx = P(*([_lib.dptr(t) for t in d[2 * nd:]] + [None] * (3 - nm)))
    tdt = _lib.TPF_F64 if dt_ == torch.float64 else _lib.TPF_F32
    lib = _lib.load()

    def formula():
        _lib.check(lib.tpf_curvature_psi(nd, psi.numel(), _lib.dptr(psi), pd1, pd2, pmx, 0.01, _lib.dptr(kap), tdt,
                                         _lib.current_stream_handle()))

    ms_k = _graph_time(formula, reps)
    es = psi.element_size()
    # read f, sw; write out: once in 2-D (both passes in one kernel), per axis pass in 3-D
    filt_bytes = (3 if nd == 2 else 3 * nd) * psi.numel() * es
    form_bytes = (2 + 2 * nd + nm) * psi.numel() * es
    return {"case": "curvature", "N": list(N), "bc": bc, "dtype": dtype, "us_per_compute": round(ms_all * 1e3, 1),
            "filter_us": round(ms_f * 1e3, 1), "filter_GBps": round(filt_bytes / (ms_f * 1e-3) / 1e9, 1),
            "formula_us": round(ms_k * 1e3, 1), "formula_GBps": round(form_bytes / (ms_k * 1e-3) / 1e9, 1),
            "filters_per_compute": 2 * nd + (1 if nd == 2 else 0)}


def rhiechow_case(N, bc, dtype, reps):
    """Rhie-Chow face-velocity divergence (RhieChowInterpolator, plain and
    balanced-force: per axis a CCD first derivative + the divergence kernel)
    and the divergence kernel alone (axis 0), graph-replayed."""
    import ctypes as C
    import torch
    from . import CCDSolver, RhieChowInterpolator, UniformGrid, _lib
    dt_ = torch.float64 if dtype == "f64" else torch.float32
    gen = torch.Generator(device="cuda").manual_seed(7)
    shape = tuple(n + 1 for n in N)
    mk = lambda: torch.randn(shape, device="cuda", dtype=dt_, generator=gen)
    vel = [mk() for _ in N]
    p, kappa, psi, dp = mk(), mk(), mk(), mk()
    rho = 1e-3 + torch.rand(shape, device="cuda", dtype=dt_, generator=gen)
    grid = UniformGrid(N)
    rc = RhieChowInterpolator(None, grid, CCDSolver(grid, None, bc_type=bc, dtype=dt_), bc_type=bc)
    ms = _graph_time(lambda: rc.face_velocity_divergence(vel, p, rho, 0.01), reps)
    ms_bf = _graph_time(lambda: rc.face_velocity_divergence(vel, p, rho, 0.01, kappa=kappa, psi=psi, we=0.7), reps)
    div = torch.empty_like(p)
    sh = (C.c_int64 * len(shape))(*shape)
    lib = _lib.load()
    tdt = _lib.TPF_F64 if dt_ == torch.float64 else _lib.TPF_F32

    def kern(ax):
        _lib.check(lib.tpf_rc_divergence_axis(len(shape), sh, ax, 1 if bc == "periodic" else 0, 1.0 / N[ax], 0.01,
                                              _lib.dptr(vel[ax]), _lib.dptr(p), _lib.dptr(rho), _lib.dptr(dp), None,
                                              None, None, 0.0, 1, _lib.dptr(div), tdt, _lib.current_stream_handle()))

    nbytes = 6 * p.numel() * p.element_size()     # read u*, p, rho, dp, div; write div
    axes = []
    for ax in range(len(N)):
        ms_k = _graph_time(lambda: kern(ax), reps)
        axes.append({"axis": ax, "us": round(ms_k * 1e3, 1), "GBps": round(nbytes / (ms_k * 1e-3) / 1e9, 1)})
    return {"case": "rhiechow", "N": list(N), "bc": bc, "dtype": dtype, "us_per_call": round(ms * 1e3, 1),
            "us_per_call_bf": round(ms_bf * 1e3, 1), "axis_kernel": axes}


def advect_case(N, bc, dtype, reps):
    """One TVD-RK3 level-set step with the FCCD flux-form right-hand side
    (FCCDLevelSetAdvection.advance) on a sphere in a rotating-shear velocity,
    and the face-value + divergence kernel alone per axis, graph-replayed."""
    import ctypes as C
    import math
    import torch
    from . import CCDSolver, FCCDLevelSetAdvection, FCCDSolver, UniformGrid, _lib
    dt_ = torch.float64 if dtype == "f64" else torch.float32
    nd = len(N)
    ax = [torch.linspace(0.0, 1.0, n + 1, dtype=torch.float64, device="cuda") for n in N]
    X = torch.meshgrid(*ax, indexing="ij")
    r = torch.sqrt(sum((X[a] - 0.5) ** 2 for a in range(nd)))
    psi = torch.sigmoid((0.25 - r) / (1.5 / max(N))).to(dt_).contiguous()
    vel = [torch.sin(2 * math.pi * X[(a + 1) % nd]).to(dt_).contiguous() for a in range(nd)]
    del X, r
    grid = UniformGrid(N)
    fccd = FCCDSolver(grid, None, bc_type=bc, ccd_solver=CCDSolver(grid, None, bc_type=bc, dtype=dt_))
    adv = FCCDLevelSetAdvection(None, grid, fccd)
    dt = 0.2 / max(N)
    ms = _graph_time(lambda: adv.advance(psi, vel, dt), reps)
    prod, q = torch.randn_like(psi), torch.randn_like(psi)
    acc = torch.empty_like(psi)
    sh = (C.c_int64 * nd)(*[n + 1 for n in N])
    lib = _lib.load()
    tdt = _lib.TPF_F64 if dt_ == torch.float64 else _lib.TPF_F32
    nbytes = 4 * psi.numel() * psi.element_size()      # read prod, q, acc; write acc
    axes = []
    for a in range(nd):
        def kern(a=a):
            _lib.check(lib.tpf_fccd_flux_divergence_axis(nd, sh, a, 1 if bc == "periodic" else 0, 1.0 / N[a],
                                                         _lib.dptr(prod), _lib.dptr(q), 1, _lib.dptr(acc), tdt,
                                                         _lib.current_stream_handle()))
        ms_k = _graph_time(kern, reps)
        axes.append({"axis": a, "us": round(ms_k * 1e3, 1), "GBps": round(nbytes / (ms_k * 1e-3) / 1e9, 1)})
    return {"case": "advect", "N": list(N), "bc": bc, "dtype": dtype, "us_per_rk3_step": round(ms * 1e3, 1),
            "flux_kernel": axes}


def reinit_case(N, dtype, reps):
    """SplitReinitializer.reinitialize (4 pseudo-steps, zero padding, mass
    correction) on a noisy sphere, and its CN line-solve kernel alone per axis,
    graph-replayed."""
    import ctypes as C
    import torch
    from . import CCDSolver, SplitReinitializer, UniformGrid, _lib
    dt_ = torch.float64 if dtype == "f64" else torch.float32
    nd = len(N)
    ax = [torch.linspace(0.0, 1.0, n + 1, dtype=torch.float64, device="cuda") for n in N]
    X = torch.meshgrid(*ax, indexing="ij")
    r = torch.sqrt(sum((X[a] - 0.5) ** 2 for a in range(nd)))
    h = 1.0 / max(N)
    gen = torch.Generator(device="cuda").manual_seed(5)
    psi = torch.sigmoid((0.25 - r) / (2.5 * h)) + 0.02 * torch.randn(r.shape, device="cuda", dtype=torch.float64,
                                                                      generator=gen)
    psi = psi.clamp(0.0, 1.0).to(dt_).contiguous()
    del X, r
    grid = UniformGrid(N)
    rein = SplitReinitializer(None, grid, CCDSolver(grid, None, bc_type="wall", dtype=dt_), 1.5 * h)
    ms = _graph_time(lambda: rein.reinitialize(psi), reps)
    out = torch.empty_like(psi)
    sh = (C.c_int64 * nd)(*[n + 1 for n in N])
    lib = _lib.load()
    tdt = _lib.TPF_F64 if dt_ == torch.float64 else _lib.TPF_F32
    nbytes = 3 * psi.numel() * psi.element_size()      # read in; write d, read d, write x (d kept in out)
    axes = []
    for a in range(nd):
        cR, dR, f, m, sup = rein._cn[a]

        def kern(a=a, cR=cR, dR=dR, f=f, m=m, sup=sup):
            _lib.check(lib.tpf_reinit_cn_axis(nd, sh, a, cR, dR, _lib.dptr(f), _lib.dptr(m), _lib.dptr(sup),
                                              _lib.dptr(psi), _lib.dptr(out), tdt, _lib.current_stream_handle()))
        ms_k = _graph_time(kern, reps)
        axes.append({"axis": a, "us": round(ms_k * 1e3, 1), "GBps_min_traffic": round(nbytes / (ms_k * 1e-3) / 1e9, 1)})
    return {"case": "reinit", "N": list(N), "dtype": dtype, "n_steps": rein.n_steps,
            "us_per_reinitialize": round(ms * 1e3, 1), "cn_kernel": axes}


def viscous_case(N, dtype, reps):
    """ViscousTerm.compute_explicit (ccd_bulk: CCD velocity derivatives, the
    low-order stress derivative kernel) on random fields, graph-replayed, and
    the low-order kernel alone per axis."""
    import ctypes as C
    import torch
    from . import CCDSolver, UniformGrid, ViscousTerm, _lib
    dt_ = torch.float64 if dtype == "f64" else torch.float32
    nd = len(N)
    shape = tuple(n + 1 for n in N)
    gen = torch.Generator(device="cuda").manual_seed(9)
    mk = lambda: torch.randn(shape, device="cuda", dtype=dt_, generator=gen)
    vel = [mk() for _ in N]
    mu = 0.01 + torch.rand(shape, device="cuda", dtype=dt_, generator=gen)
    rho = 0.001 + torch.rand(shape, device="cuda", dtype=dt_, generator=gen)
    grid = UniformGrid(N)
    ccd = CCDSolver(grid, None, bc_type="wall", dtype=dt_)
    vt = ViscousTerm(None, 100.0)
    ms = _graph_time(lambda: vt.compute_explicit(vel, mu, rho, ccd), reps)
    a, b = mk(), mk()
    total = torch.empty_like(a)
    sh = (C.c_int64 * nd)(*shape)
    lib = _lib.load()
    tdt = _lib.TPF_F64 if dt_ == torch.float64 else _lib.TPF_F32
    nbytes = 5 * a.numel() * a.element_size()     # read a, b, mu, total; write total
    axes = []
    for ax in range(nd):
        (cl, cc, cr), dx0, dxl = vt._coefficients(grid, ax)

        def kern(ax=ax, cl=cl, cc=cc, cr=cr, dx0=dx0, dxl=dxl):
            _lib.check(lib.tpf_visc_lowfd_axis(nd, sh, ax, _lib.dptr(cl), _lib.dptr(cc), _lib.dptr(cr), dx0, dxl,
                                               _lib.dptr(a), _lib.dptr(b), _lib.dptr(mu), 1, 0, _lib.dptr(rho),
                                               100.0, _lib.dptr(total), tdt, _lib.current_stream_handle()))
        ms_k = _graph_time(kern, reps)
        axes.append({"axis": ax, "us": round(ms_k * 1e3, 1), "GBps": round(nbytes / (ms_k * 1e-3) / 1e9, 1)})
    return {"case": "viscous", "N": list(N), "dtype": dtype, "scheme": vt.spatial_scheme,
            "us_per_compute": round(ms * 1e3, 1), "lowfd_kernel": axes}


def step_case(N, reps, use_graphs=True):
    """Whole two-phase time steps (TwoPhaseStep): a gas bubble of radius 0.2 at
    (0.5, 0.5, 0.3) in liquid ((0.5, 0.3) in 2-D), density ratio 1000,
    viscosity ratio 100, Re 100, We 10, Fr 1, each step at the CFL time step
    with the capillary bound (time_integration/cfl.py:85-137).  The CG
    pressure solve is recorded in the same CUDA graph as the rest of the step,
    so a replayed step is one graph launch plus the read-back of the solve's
    status.  Two warm-up steps (eager + capture), then ``reps`` timed steps
    (CUDA events around each step)."""
    import torch
    from . import TwoPhaseStep, UniformGrid
    nd = len(N)
    ax = [torch.linspace(0.0, 1.0, n + 1, dtype=torch.float64, device="cuda") for n in N]
    X = torch.meshgrid(*ax, indexing="ij")
    c = [0.5] * (nd - 1) + [0.3]
    r = torch.sqrt(sum((X[a] - c[a]) ** 2 for a in range(nd)))
    h = 1.0 / max(N)
    psi = torch.sigmoid((r - 0.2) / (1.5 * h)).contiguous()   # liquid (psi = 1) outside the bubble
    del X, r
    stp = TwoPhaseStep(UniformGrid(N), psi, Re=100.0, Fr=1.0, We=10.0, rho_ratio=1e-3, mu_ratio=1e-2,
                       use_graphs=use_graphs)
    for _ in range(2):
        stp.step(stp.cfl_dt())
    torch.cuda.synchronize()
    ev = [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(reps)]
    its, dts = [], []
    for k in range(reps):
        dt = stp.cfl_dt()
        dts.append(dt)
        ev[k][0].record()
        stp.step(dt)
        ev[k][1].record()
        its.append(stp.last_ppe_iterations)
    torch.cuda.synchronize()
    t = [e[0].elapsed_time(e[1]) for e in ev]
    return {"case": "step", "N": list(N), "graphs": use_graphs, "one_graph_per_step": stp._g2 is None,
            "ms_per_step": round(sum(t) / reps, 2), "ppe_iterations": its, "dt": dts[-1],
            "steps_total": reps + 2,
            "psi_range": [round(float(stp.psi.min()), 6), round(float(stp.psi.max()), 6)],
            "u_max": round(float(max(v.abs().max() for v in stp.vel)), 6)}


def ppe_case(N, precision, reps, tol=1e-8):
    import torch
    from . import PPESolverFVMMatrixFree, UniformGrid
    from .workloads import divergence_rhs, droplet_density

    class Cfg:
        pseudo_tol = tol
        pseudo_maxiter = 1_000_000
        ppe_iteration_method = "cg"
        ppe_preconditioner = "jacobi"
        ppe_precision = precision

    rho = torch.from_numpy(droplet_density(N, seed=0)).cuda()
    rhs = torch.from_numpy(divergence_rhs(N, seed=1)).cuda()
    s = PPESolverFVMMatrixFree(None, Cfg(), UniformGrid(N))
    s.solve(rhs, rho)
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        s.solve(rhs, rho)
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    d = s.last_diagnostics
    it = d["ppe_low_order_cg_iterations"]
    ms = min(ts)
    return {"case": "ppe", "N": list(N), "precision": precision, "ms": round(ms, 3), "iterations": it,
            "us_per_iteration": round(ms * 1e3 / max(it, 1), 2)}


def learned_case(N, reps, maxiter=None, tol=1e-8, outer="fgmres"):
    """Network-preconditioned flexible GMRES (``outer='fgmres'``, the
    solver's default restart and sweeps) or flexible CG (``outer='fcg'``;
    shipped weights, two-level mode) on the droplet PPE; ``maxiter`` bounds
    the iterations (no fallback; whole restart cycles for GMRES) for profiling
    a fixed amount of work."""
    import torch
    from . import UniformGrid
    from .learned import PPESolverLearned
    from .workloads import divergence_rhs, droplet_density

    class Cfg:
        pseudo_tol = tol
        pseudo_maxiter = 20000
        ppe_learned_maxiter = maxiter if maxiter else 20000
        ppe_learned_fallback = False
        ppe_learned_outer = outer

    rho = torch.from_numpy(droplet_density(N, seed=0)).cuda()
    rhs = torch.from_numpy(divergence_rhs(N, seed=1)).cuda()
    s = PPESolverLearned(None, Cfg(), UniformGrid(N))

    def run():
        try:
            s.solve(rhs, rho)
        except RuntimeError:
            if not maxiter:
                raise

    run()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        run()
        e1.record()
        torch.cuda.synchronize()
        ts.append(e0.elapsed_time(e1))
    it = s.last_diagnostics["ppe_learned_iterations"]
    ms = min(ts)
    return {"case": "learned", "outer": outer, "N": list(N), "ms": round(ms, 3), "iterations": it,
            "us_per_iteration": round(ms * 1e3 / max(it, 1), 2)}


def smoother_case(N, sweeps=256, block=4):
    """The learned preconditioner's damped-Jacobi smoother alone on the droplet
    operator: ``sweeps`` sweeps, ``block`` per launch (temporally blocked
    kernel), timed from a CUDA graph.  Algorithmic bytes per launch: z, r,
    D^-1 and the two couplings read once, z written once (48 B per node)."""
    import torch
    from . import UniformGrid, _lib
    from .learned import PPESolverLearned
    from .workloads import divergence_rhs, droplet_density

    class Cfg:
        pseudo_tol = 1e-8
        pseudo_maxiter = 20000

    s = PPESolverLearned(None, Cfg(), UniformGrid(N))
    s.prepare_operator(torch.from_numpy(droplet_density(N, seed=0)).cuda())
    r = torch.from_numpy(divergence_rhs(N, seed=1)).cuda()
    z = torch.zeros_like(r)
    _lib.check(s.lib.tpf_lppe_set_smooth_block(s._lp, block))

    def call():
        _lib.check(s.lib.tpf_lppe_smooth(s._lp, _lib.dptr(z), _lib.dptr(r), _lib.dptr(z), sweeps, 0.8,
                                         _lib.current_stream_handle()))

    ms = _graph_time(call, 1)
    launches = (sweeps + block - 1) // block
    us = ms * 1e3 / launches
    ndof = r.numel()
    return {"case": "smoother", "N": list(N), "block": block, "launches": launches, "us_per_launch": round(us, 3),
            "GBps": round(48.0 * ndof / (us * 1e-6) / 1e9, 1)}


def batched_case(n_cases=32, nmin=128, nmax=512, reps=3, seed=0, tol=1e-8):
    """``n_cases`` independent 2-D droplet PPEs with seeded uneven grids
    (N_x, N_y uniform in [nmin, nmax]) solved in ONE persistent launch
    (solve_batched) against one solve after the other (each on the whole
    GPU, band-resident where it fits).  The batch is band-resident when the
    bands of all cases fit in shared memory at once, else all-global."""
    import numpy as np
    import torch
    from . import PPESolverFVMMatrixFree, UniformGrid, solve_batched
    from .workloads import divergence_rhs, droplet_density

    class Cfg:
        pseudo_tol = tol
        pseudo_maxiter = 1_000_000
        ppe_iteration_method = "cg"
        ppe_preconditioner = "jacobi"

    rng = np.random.default_rng(seed)
    shapes = [tuple(int(v) for v in rng.integers(nmin, nmax + 1, size=2)) for _ in range(n_cases)]
    solvers, rhs, rho = [], [], []
    for k, N in enumerate(shapes):
        solvers.append(PPESolverFVMMatrixFree(None, Cfg(), UniformGrid(N)))
        rho.append(torch.from_numpy(droplet_density(N, n_drops=8, seed=100 + k)).cuda())
        rhs.append(torch.from_numpy(divergence_rhs(N, seed=200 + k)).cuda())

    def timed(fn):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
        return min(ts)

    ms_b = timed(lambda: solve_batched(solvers, rhs, rho))
    its = [s.last_diagnostics["ppe_low_order_cg_iterations"] for s in solvers]
    ms_s = timed(lambda: [s.solve(rhs[k], rho[k]) for k, s in enumerate(solvers)])
    return {"case": "batched", "n_cases": n_cases, "grids": [list(g) for g in shapes], "ms_batched": round(ms_b, 3),
            "ms_sequential": round(ms_s, 3), "cases_per_s_batched": round(n_cases / (ms_b * 1e-3), 1),
            "cases_per_s_sequential": round(n_cases / (ms_s * 1e-3), 1), "iterations_max": int(max(its)),
            "iterations_total": int(sum(its))}


def gmres_case(N, line, reps, maxiter=None, tol=1e-8):
    """GMRES(80) with the shifted line preconditioner (the reference's default
    PPE route) on the droplet PPE; ``maxiter`` bounds the restart cycles (the
    solve then stops with the reference's non-convergence error, which is
    expected) for profiling a fixed amount of work."""
    import time
    import torch
    from . import PPESolverFVMMatrixFree, UniformGrid
    from .workloads import divergence_rhs, droplet_density

    class Cfg:
        pseudo_tol = tol
        pseudo_maxiter = maxiter if maxiter else 100000
        ppe_iteration_method = "gmres"
        ppe_preconditioner = "line_pcr"
        ppe_restart = 80
        ppe_line_solver = line

    rho = torch.from_numpy(droplet_density(N, seed=0)).cuda()
    rhs = torch.from_numpy(divergence_rhs(N, seed=1)).cuda()
    s = PPESolverFVMMatrixFree(None, Cfg(), UniformGrid(N))

    def run():
        try:
            s.solve(rhs, rho)
        except RuntimeError:
            if not maxiter:
                raise

    ts = []
    for _ in range(max(1, reps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        run()
        torch.cuda.synchronize()
        ts.append((time.perf_counter() - t0) * 1e3)
    d = s.last_diagnostics
    it = d.get("ppe_low_order_gmres_iterations", 0)
    ms = min(ts)
    return {"case": "gmres", "N": list(N), "line": line, "ms": round(ms, 2), "iterations": it,
            "us_per_iteration": round(ms * 1e3 / max(it, 1), 1)}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("case", choices=["ccd", "ppe", "learned", "smoother", "batched", "gmres", "corrector", "curvature", "rhiechow", "advect", "reinit", "viscous", "step"])
    ap.add_argument("--line", default="thomas", choices=["thomas", "pcr"], help="gmres: line solver")
    ap.add_argument("--N", type=int, nargs="+", required=True)
    ap.add_argument("--axis", type=int, default=0)
    ap.add_argument("--bc", default="wall")
    ap.add_argument("--dtype", default="f64", choices=["f64", "f32"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--nmin", type=int, default=128, help="batched: smallest nodes per axis")
    ap.add_argument("--nmax", type=int, default=512, help="batched: largest nodes per axis")
    ap.add_argument("--outer", default="fgmres", choices=["fcg", "fgmres"], help="learned: outer Krylov method")
    ap.add_argument("--maxiter", type=int, default=0,
                    help="learned: stop after this many iterations; gmres: after this many restart cycles")
    a = ap.parse_args(argv)
    if a.case == "ccd":
        r = ccd_case(tuple(a.N), a.axis, a.bc, a.dtype, a.reps)
    elif a.case == "ppe":
        r = ppe_case(tuple(a.N), a.precision, a.reps)
    elif a.case == "learned":
        r = learned_case(tuple(a.N), a.reps, a.maxiter or None, outer=a.outer)
    elif a.case == "smoother":
        r = smoother_case(tuple(a.N))
    elif a.case == "gmres":
        r = gmres_case(tuple(a.N), a.line, a.reps, a.maxiter or None)
    elif a.case == "corrector":
        r = corrector_case(tuple(a.N), a.axis, a.bc, a.dtype, a.reps)
    elif a.case == "curvature":
        r = curvature_case(tuple(a.N), a.bc, a.dtype, a.reps)
    elif a.case == "rhiechow":
        r = rhiechow_case(tuple(a.N), a.bc, a.dtype, a.reps)
    elif a.case == "advect":
        r = advect_case(tuple(a.N), a.bc, a.dtype, a.reps)
    elif a.case == "reinit":
        r = reinit_case(tuple(a.N), a.dtype, a.reps)
    elif a.case == "viscous":
        r = viscous_case(tuple(a.N), a.dtype, a.reps)
    elif a.case == "step":
        r = step_case(tuple(a.N), a.reps)
    else:
        r = batched_case(n_cases=a.N[0], nmin=a.nmin, nmax=a.nmax, reps=a.reps)
    print(json.dumps(r), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
