"""One two-phase flow time step on the GPU, composed from this package's
operators, with the work before and after the pressure solve captured as CUDA
graphs.

Order (the reference's projection step, src/twophase/simulation/ns_step_services.py):
CLS transport (FCCD flux form, TVD-RK3) -> split reinitialization -> rho, mu
from psi -> curvature from psi -> AB2 + IPC predictor (CCD convection,
gravity, CSF, -grad p^n, Picard-CN viscous) -> Rhie-Chow face-velocity
divergence / dt -> PPE for the pressure increment (FVM matrix-free CG, the
persistent kernel) -> velocity corrector, p += dp -> CFL maxima.

``TwoPhaseStep.step(dt)`` with the CG pressure route replays ONE graph that
holds the whole step, the solve included (its iteration count is read after
the replay).  With the GMRES route it replays graph 1 (everything up to the
PPE right-hand side), runs the host-driven solve, then replays graph 2
(corrector, pressure update, CFL maxima).  The first call for a given dt runs
the step eagerly (CCD plans, autotuning, allocator pools) and then captures.
With the quick-start selection the composition is pinned to six steps of the
reference's own pipeline; ``save_checkpoint`` / ``restore_checkpoint_state``
carry its state through the reference's restart format
(twophaseflow_b200.checkpoint).
"""

from __future__ import annotations

import ctypes as C
import math
from types import SimpleNamespace

import numpy as np

from . import _lib
from .advection import FCCDLevelSetAdvection, FCCDSolver, SplitReinitializer, UCCD6ConvectionTerm
from .ccd import CCDSolver
from .levelset import CurvatureCalculatorPsi, update_properties
from .ppe import PPESolverFVMMatrixFree
from .predictor import FlowState, Predictor
from .step import RhieChowInterpolator, VelocityCorrector


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("twophaseflow_b200 needs a CUDA device; there is no CPU fallback")
    return torch


class TwoPhaseStep:
    """State and operators of a wall-bounded two-phase flow on a uniform grid.

    psi: CLS field (1 = liquid); velocity zero at start; rho, mu from psi with
    rho_l = mu_l = 1, rho_g = rho_ratio, mu_g = mu_ratio."""

    def __init__(self, grid, psi, Re=100.0, Fr=1.0, We=10.0, rho_ratio=1e-3, mu_ratio=1e-2, cfl=0.3,
                 eps=None, reinit_steps=4, ppe_tol=1e-8, ppe_maxiter=20000, use_graphs=True,
                 convection="ccd", transport_mass_correction=False, reinit_bc="zero", ppe_method="cg",
                 no_slip=False, zero_velocity_shortcut=False, ppe_in_graph=None):
        """The keyword options after ``use_graphs`` select the reference
        quick-start pipeline's components (simulation/_core.py:126-172):
        ``convection="uccd6"``, ``transport_mass_correction=True``,
        ``reinit_bc="neumann"``, ``ppe_method="gmres"`` (GMRES(80) with the
        exact line preconditioner) and ``no_slip=True`` (every velocity
        component zeroed on every wall plane of u* and of the corrected u,
        simulation/boundary_condition.py:22-70).  ``zero_velocity_shortcut``
        skips the transport stages while the velocity is exactly zero (before
        the first step), as the reference's CPU backend does
        (levelset/fccd_advection.py:99-110).  The defaults keep the CCD
        convection, Jacobi-PCG composition.

        ``ppe_in_graph`` (default: True for the CG route) records the pressure
        solve inside the same CUDA graph as the rest of the step, so a step is
        ONE graph replay; the solve's iteration count and convergence are read
        back after the replay.  The GMRES route is host-driven and stays
        between two graphs.

        ``cfl_dt`` is the reference's CFLCalculator (time_integration/cfl.py:
        58-137) with Crank-Nicolson viscosity: the convective bound and the
        capillary bound cfl * sqrt((1 + rho_ratio) We h^3 / (2 pi))."""
        torch = _torch()
        self.options = dict(Re=Re, Fr=Fr, We=We, rho_ratio=rho_ratio, mu_ratio=mu_ratio, cfl=cfl, eps=eps,
                            reinit_steps=reinit_steps, ppe_tol=ppe_tol, ppe_maxiter=ppe_maxiter,
                            convection=convection, transport_mass_correction=bool(transport_mass_correction),
                            reinit_bc=reinit_bc, ppe_method=ppe_method, no_slip=bool(no_slip),
                            zero_velocity_shortcut=bool(zero_velocity_shortcut))
        self.grid = grid
        nd = grid.ndim
        self.nd = nd
        self.ccd = CCDSolver(grid, None, bc_type="wall")
        self.fccd = FCCDSolver(grid, None, bc_type="wall", ccd_solver=self.ccd)
        h = min(float(grid.L[a] / grid.N[a]) for a in range(nd))
        self.eps = 1.5 * h if eps is None else eps
        if convection not in ("ccd", "uccd6"):
            raise ValueError("convection must be 'ccd' or 'uccd6'")
        if ppe_method not in ("cg", "gmres"):
            raise ValueError("ppe_method must be 'cg' (Jacobi) or 'gmres' (line preconditioner)")
        self.transport = FCCDLevelSetAdvection(None, grid, self.fccd, mass_correction=transport_mass_correction)
        self.reinit = SplitReinitializer(None, grid, self.ccd, self.eps, n_steps=reinit_steps, bc=reinit_bc)
        self.curv = CurvatureCalculatorPsi(None, self.ccd)
        cfg = SimpleNamespace(grid=SimpleNamespace(ndim=nd), fluid=SimpleNamespace(Re=Re, Fr=Fr, We=We),
                              numerics=SimpleNamespace(cn_viscous=True, cn_mode="picard"))
        conv = UCCD6ConvectionTerm(None, grid, self.ccd) if convection == "uccd6" else None
        self.predictor = Predictor(None, cfg, self.ccd, convection=conv)
        self.rc = RhieChowInterpolator(None, grid, self.ccd, bc_type="wall")
        self.no_slip = bool(no_slip)
        ppe_cfg = SimpleNamespace(pseudo_tol=ppe_tol, pseudo_maxiter=ppe_maxiter, ppe_iteration_method=ppe_method,
                                  ppe_preconditioner="jacobi" if ppe_method == "cg" else "line_pcr",
                                  ppe_line_solver="thomas")
        self.ppe = PPESolverFVMMatrixFree(None, ppe_cfg, grid)
        self.corrector = VelocityCorrector(None, grid, self.ccd)
        self.rho_l, self.rho_g, self.mu_l, self.mu_g = 1.0, rho_ratio, 1.0, mu_ratio
        self.cfl = cfl
        self.h = h
        self._dt_sigma = math.sqrt((1.0 + rho_ratio) * We * h ** 3 / (2.0 * math.pi)) if We and We > 0.0 else None
        self.zero_velocity_shortcut = bool(zero_velocity_shortcut)
        self._vel_zero = True   # the velocity starts exactly zero
        dev = torch.device("cuda", torch.cuda.current_device())
        self.psi = torch.as_tensor(psi, dtype=torch.float64, device=dev).contiguous().clone()
        self.vel = [torch.zeros_like(self.psi) for _ in range(nd)]
        self.p = torch.zeros_like(self.psi)
        self.rho, self.mu = update_properties(None, self.psi, self.rho_l, self.rho_g, self.mu_l, self.mu_g)
        self.rhs = torch.zeros_like(self.psi)
        self.dp = torch.zeros_like(self.psi)
        self.maxima = torch.zeros(4, dtype=torch.float64, device=dev)
        self.use_graphs = use_graphs
        self.ppe_in_graph = (ppe_method == "cg") if ppe_in_graph is None else bool(ppe_in_graph)
        if self.ppe_in_graph and ppe_method != "cg":
            raise ValueError("ppe_in_graph needs the CG route (the GMRES route reads its residual on the host)")
        self._g1 = self._g2 = None
        self._dt_graph = None
        self._vel_star = None
        self.lib = _lib.load()
        self.last_ppe_iterations = 0

    # -- phases ---------------------------------------------------------------
    def _phase1(self, dt):
        """psi, rho, mu, kappa, u* and the PPE right-hand side (no host sync)."""
        skip = self.zero_velocity_shortcut and self._vel_zero
        psi = self.transport.advance(self.psi, self.vel, dt, velocity_is_zero=skip)
        psi = self.reinit.reinitialize(psi)
        self.psi.copy_(psi)
        rho, mu = update_properties(None, self.psi, self.rho_l, self.rho_g, self.mu_l, self.mu_g)
        self.rho.copy_(rho)
        self.mu.copy_(mu)
        kappa = self.curv.compute(self.psi)
        st = FlowState(velocity=self.vel, psi=self.psi, rho=self.rho, mu=self.mu, kappa=kappa, pressure=self.p)
        self._vel_star = self.predictor.compute(st, dt)
        if self.no_slip:
            self._wall_zero(self._vel_star)
        div = self.rc.face_velocity_divergence(self._vel_star, self.p, self.rho, dt)
        _lib.check(self.lib.tpf_ns_scaled(div.numel(), 2, _lib.dptr(div), None, float(dt), _lib.dptr(self.rhs),
                                          _lib.TPF_F64, _lib.current_stream_handle()))

    def _phase2(self, dt):
        """u = u* - dt/rho grad dp, p += dp, CFL maxima into a device buffer."""
        vel = self.corrector.correct(self._vel_star, self.dp, self.rho, dt)
        for c in range(self.nd):
            self.vel[c].copy_(vel[c])
        if self.no_slip:
            self._wall_zero(self.vel)
        st = _lib.current_stream_handle()
        _lib.check(self.lib.tpf_visc_accumulate(self.p.numel(), _lib.dptr(self.dp), 1, 0, None, 0.0,
                                                _lib.dptr(self.p), _lib.TPF_F64, st))
        self._update_maxima()

    def _update_maxima(self):
        ptrs = (C.c_void_p * self.nd)(*[_lib.dptr(v) for v in self.vel])
        _lib.check(self.lib.tpf_cfl_maxima(self.p.numel(), self.nd, ptrs, None, None, _lib.TPF_F64,
                                           _lib.dptr(self.maxima), _lib.current_stream_handle()))

    def _wall_zero(self, comps):
        """No-slip: every component zero on both planes of every (wall) axis."""
        for ax in range(self.nd):
            for c in comps:
                self.ccd.enforce_wall_neumann(c, ax)

    def _solve(self):
        dp = self.ppe.solve(self.rhs, self.rho)
        self.dp.copy_(dp)
        d = getattr(self.ppe, "last_diagnostics", {}) or {}
        self.last_ppe_iterations = int(d.get(f"ppe_low_order_{self.ppe.iteration_method}_iterations", 0))

    def _capture(self, dt):
        torch = _torch()
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            if self.ppe_in_graph:
                g1 = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g1, stream=s):
                    self._phase1(dt)
                    dp = self.ppe.solve(self.rhs, self.rho)
                    self.dp.copy_(dp)
                    self._phase2(dt)
                g2 = None
            else:
                g1 = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g1, stream=s):
                    self._phase1(dt)
                g2 = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g2, stream=s):
                    self._phase2(dt)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self._g1, self._g2, self._dt_graph = g1, g2, dt

    # -- public ----------------------------------------------------------------
    def step(self, dt: float):
        """Advance one step with time step dt (the graphs belong to one dt)."""
        first = self._vel_zero
        self._vel_zero = False
        if not self.use_graphs or (first and self.zero_velocity_shortcut):
            self._vel_zero = first   # read by _phase1 of this step only
            self._phase1(dt)
            self._vel_zero = False
            self._solve()
            self._phase2(dt)
            return
        if self._g1 is None or self._dt_graph != dt:
            self._phase1(dt)
            self._solve()
            self._phase2(dt)
            self._capture(dt)   # records only: the state has advanced by the eager step
            return
        if self._g2 is None:
            # the whole step, pressure solve included, as one graph
            self._g1.replay()
            d = self.ppe.read_result()
            self.last_ppe_iterations = int(d.get(f"ppe_low_order_{self.ppe.iteration_method}_iterations", 0))
            return
        self._g1.replay()
        self._solve()
        self._g2.replay()

    def cfl_dt(self) -> float:
        """CFL time step from the last step's velocity maxima (cfl.py:85-137):
        the smaller of the convective and the capillary bound, at least 1e-8."""
        m = self.maxima.cpu().tolist()
        u_sum = 0.0
        for v in m[:self.nd]:
            u_sum = u_sum + v
        cands = [self.cfl * self.h / max(u_sum, 1.0e-14)]
        if self._dt_sigma is not None:
            cands.append(self.cfl * self._dt_sigma)
        return max(min(cands), 1.0e-8)

    # -- restart checkpoints (twophaseflow_b200.checkpoint) --------------------------
    backend_device = "gpu"

    def checkpoint_config(self) -> dict:
        """The options that define this run (the config fingerprint of a
        checkpoint written without a YAML config)."""
        return {"N": list(self.grid.N), "L": list(self.grid.L), **self.options}

    def checkpoint_state(self) -> dict:
        """History the next step reads besides psi, u, p: p^n for the
        incremental pressure correction (after a step), the AB2 convection
        history and its ready flag."""
        pr = self.predictor
        return {"p_prev_dev": None if self._vel_zero else self.p,
                "conv_prev": pr._conv_prev if pr._ab2_ready else None,
                "conv_ab2_ready": bool(pr._ab2_ready and pr._conv_prev is not None)}

    def save_checkpoint(self, path, *, t: float, step: int, config_path=None, **kw) -> None:
        """``checkpoint.save_checkpoint`` with this step's own fields."""
        from .checkpoint import save_checkpoint
        save_checkpoint(path, solver=self, psi=self.psi, u=self.vel[0], v=self.vel[1], p=self.p,
                        w=self.vel[2] if self.nd == 3 else None, t=t, step=step, config_path=config_path, **kw)

    def restore_checkpoint_state(self, st: dict) -> dict:
        """Copy a checkpoint's state into this step's device tensors: psi, the
        velocity, p, the AB2 history; rho, mu and the CFL maxima are
        recomputed from them and the captured graphs are dropped (the next
        step runs eagerly and captures again)."""
        from .checkpoint import CheckpointError
        torch = _torch()
        for a, c in enumerate(st.get("grid_coords") or ()):
            if not np.array_equal(np.asarray(c, dtype=np.float64), np.asarray(self.grid.coords[a], dtype=np.float64)):
                raise CheckpointError("checkpoint grid coordinates differ from this step's uniform grid")
        if len(st["velocity"]) != self.nd:
            raise CheckpointError(f"checkpoint holds {len(st['velocity'])} velocity components, the grid has {self.nd}")
        dev = self.psi.device

        def put(dst, arr):
            dst.copy_(torch.as_tensor(np.asarray(arr, dtype=np.float64), device=dev))
        put(self.psi, st["psi"])
        for c in range(self.nd):
            put(self.vel[c], st["velocity"][c])
        put(self.p, st["p"])
        pr = self.predictor
        conv = st.get("conv_prev")
        if st.get("conv_ab2_ready") and conv is not None:
            if len(conv) != self.nd:
                raise CheckpointError("checkpoint AB2 history has the wrong number of components")
            if pr._conv_prev is None:
                pr._conv_prev = [torch.empty_like(self.psi) for _ in range(self.nd)]
            for c in range(self.nd):
                put(pr._conv_prev[c], conv[c])
            pr._ab2_ready = True
        else:
            pr._ab2_ready = False
        rho, mu = update_properties(None, self.psi, self.rho_l, self.rho_g, self.mu_l, self.mu_g)
        self.rho.copy_(rho)
        self.mu.copy_(mu)
        self._vel_zero = (not pr._ab2_ready) and all(float(v.abs().max()) == 0.0 for v in self.vel)
        self._g1 = self._g2 = None
        self._dt_graph = None
        self._update_maxima()
        fields = {"psi": self.psi, "u": self.vel[0], "v": self.vel[1], "p": self.p}
        if self.nd == 3:
            fields["w"] = self.vel[2]
        return fields
