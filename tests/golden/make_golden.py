"""Generate the golden fixtures by running the reference itself.

Run in a container that has the reference source tree (not needed at test time):

    PYTHONDONTWRITEBYTECODE=1 python tests/golden/make_golden.py <reference>/src [only ...]

or with the source directory in ``TWOPHASE_REFERENCE_SRC``.

It imports the reference's ``twophase`` package read-only, runs its own CPU
functions (``CCDSolver.differentiate``, ``PPESolverFVMMatrixFree``,
``PPESolverFVMSpsolve``, the batched tridiagonal helpers and the CCD
variable-density Laplacian) on small seeded inputs and stores inputs and
outputs in ``ccd_golden.npz`` / ``ppe_golden.npz`` next to this script;
``step_golden.npz`` holds the steps either side of the PPE
(``VelocityCorrector.correct``, ``ccd_pressure_gradient``,
``CFLCalculator.compute``).
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _ref_import(src):
    sys.path.insert(0, src)
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    import twophase  # noqa: F401
    return twophase


def make_ccd(out):
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.levelset.heaviside import heaviside

    be = Backend(use_gpu=False)
    rng = np.random.default_rng(2024)
    cases = [
        ("wall2d", (16, 12), "wall"),
        ("wall3d", (8, 10, 6), "wall"),
        ("per2d", (16, 10), "periodic"),
        ("per3d", (8, 6, 10), "periodic"),
        ("wall2d_big", (64, 40), "wall"),
    ]
    for name, N, bc in cases:
        grid = Grid(GridConfig(ndim=len(N), N=N, L=tuple(1.0 + 0.25 * a for a in range(len(N)))), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        f = rng.standard_normal(grid.shape)
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(grid.L, dtype=np.float64)
        out[f"{name}/f"] = f
        for ax in range(len(N)):
            d1, d2 = ccd.differentiate(f, ax)
            out[f"{name}/d1_ax{ax}"] = np.asarray(d1)
            out[f"{name}/d2_ax{ax}"] = np.asarray(d2)
            out[f"{name}/first_ax{ax}"] = np.asarray(ccd.first_derivative(f, ax))
            out[f"{name}/second_ax{ax}"] = np.asarray(ccd.second_derivative(f, ax))
        if bc == "wall":
            d1, d2 = ccd.differentiate(f, 0, bc_left=(0.3, -1.2), bc_right=(0.0, 2.5))
            out[f"{name}/bcov_d1"] = np.asarray(d1)
            out[f"{name}/bcov_d2"] = np.asarray(d2)
    # analytic case of the reference test suite: sin(2 pi x) on N=32, periodic and wall
    for bc in ("wall", "periodic"):
        grid = Grid(GridConfig(ndim=2, N=(32, 4), L=(1.0, 1.0)), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        x = np.asarray(grid.coords[0])
        f = np.broadcast_to(np.sin(2 * np.pi * x)[:, None], grid.shape).copy()
        d1, d2 = ccd.differentiate(f, 0)
        out[f"sin_{bc}/f"] = f
        out[f"sin_{bc}/d1"] = np.asarray(d1)
        out[f"sin_{bc}/d2"] = np.asarray(d2)
    # non-uniform (interface-fitted) grid: metric path
    N = 32
    grid = Grid(GridConfig(ndim=2, N=(N, N), L=(1.0, 1.0), alpha_grid=2.0, eps_g_factor=2.0), be)
    ccd = CCDSolver(grid, be, bc_type="wall")
    X, Y = grid.meshgrid()
    psi = heaviside(np, X - 0.5, 0.5 / N)
    grid.update_from_levelset(psi, 0.5 / N, ccd=ccd)
    ccd = CCDSolver(grid, be, bc_type="wall")
    X, Y = np.meshgrid(grid.coords[0], grid.coords[1], indexing="ij")
    f = np.sin(np.pi * X) * np.cos(np.pi * Y)
    out["nonuni/f"] = f
    for ax in range(2):
        out[f"nonuni/J{ax}"] = np.asarray(grid.J[ax], dtype=np.float64)
        out[f"nonuni/dJ{ax}"] = np.asarray(grid.dJ_dxi[ax], dtype=np.float64)
        out[f"nonuni/coords{ax}"] = np.asarray(grid.coords[ax])
        d1, d2 = ccd.differentiate(f, ax)
        out[f"nonuni/d1_ax{ax}"] = np.asarray(d1)
        out[f"nonuni/d2_ax{ax}"] = np.asarray(d2)
        out[f"nonuni/first_ax{ax}"] = np.asarray(ccd.first_derivative(f, ax))
        out[f"nonuni/second_ax{ax}"] = np.asarray(ccd.second_derivative(f, ax))
        r1, r2 = ccd.differentiate(f, ax, apply_metric=False)
        out[f"nonuni/raw_d1_ax{ax}"] = np.asarray(r1)
        out[f"nonuni/raw_d2_ax{ax}"] = np.asarray(r2)


def make_ppe(out):
    from twophase.backend import Backend
    from twophase.config import SimulationConfig, GridConfig, SolverConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.ppe.fvm_matrixfree import PPESolverFVMMatrixFree
    from twophase.ppe.fvm_spsolve import PPESolverFVMSpsolve
    from twophase.ppe.ccd_ppe_utils import compute_ccd_laplacian, precompute_density_gradients
    from twophase.linalg_backend import tridiag_variable_batched, _pcr_solve_variable_batched

    sys.path.insert(0, os.path.abspath(os.path.join(HERE, "..", "..")))
    from twophaseflow_b200.workloads import droplet_density, divergence_rhs

    be = Backend(use_gpu=False)

    def cfg_for(N, **solver):
        base = dict(ppe_solver_type="fvm_iterative", pseudo_tol=1e-10,
                    pseudo_maxiter=200, pseudo_c_tau=2.0)
        base.update(solver)
        cfg = SimulationConfig(grid=GridConfig(ndim=len(N), N=N, L=(1.0,) * len(N)),
                               solver=SolverConfig(**{k: v for k, v in base.items()
                                                      if k in ("ppe_solver_type", "pseudo_tol",
                                                               "pseudo_maxiter", "pseudo_c_tau")}))
        for k, v in base.items():
            if k not in ("ppe_solver_type", "pseudo_tol", "pseudo_maxiter", "pseudo_c_tau"):
                setattr(cfg.solver, k, v)
        return cfg

    # (name, N, seed, solver options, density kind)
    cases = [
        ("apply2d", (8, 8), 123, {}, "rand"),
        ("gmres_line2d", (8, 8), 456, {}, "rand"),
        ("gmres_jac2d", (8, 8), 789, {"ppe_preconditioner": "jacobi"}, "rand"),
        ("cg_jac2d", (8, 8), 987, {"ppe_iteration_method": "cg", "ppe_preconditioner": "jacobi"}, "rand"),
        ("cg_jac3d", (6, 7, 5), 11, {"ppe_iteration_method": "cg", "ppe_preconditioner": "jacobi"}, "rand"),
        ("gmres_line3d", (6, 5, 7), 12, {}, "rand"),
        ("cg_drop32", (32, 32), 0,
         {"ppe_iteration_method": "cg", "ppe_preconditioner": "jacobi", "pseudo_tol": 1e-8,
          "pseudo_maxiter": 20000}, "drop"),
        ("gmres_drop16", (16, 16), 0,
         {"pseudo_tol": 1e-8, "pseudo_maxiter": 500}, "drop"),
        ("cg_rect", (12, 20), 5, {"ppe_iteration_method": "cg", "ppe_preconditioner": "jacobi"}, "rand"),
    ]
    for name, N, seed, opts, kind in cases:
        cfg = cfg_for(N, **opts)
        grid = Grid(cfg.grid, be)
        rng = np.random.default_rng(seed)
        if kind == "rand":
            rho = 1.0 + rng.uniform(0.0, 1.0, grid.shape)
            rhs = rng.standard_normal(grid.shape)
        else:
            rho = droplet_density(N, seed=seed)
            rhs = divergence_rhs(N, seed=seed + 1)
        solver = PPESolverFVMMatrixFree(be, cfg, grid, bc_type="wall")
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/rho"] = rho
        out[f"{name}/rhs"] = rhs
        out[f"{name}/tol"] = np.array(solver.tol)
        out[f"{name}/maxiter"] = np.array(solver.maxiter)
        out[f"{name}/restart"] = np.array(solver.restart)
        out[f"{name}/method"] = np.array(solver.iteration_method)
        out[f"{name}/precond"] = np.array(solver.preconditioner)
        out[f"{name}/pin"] = np.array(solver._pin_dof)
        # operator apply
        solver.prepare_operator(rho)
        p_rand = rng.standard_normal(grid.shape)
        out[f"{name}/p_rand"] = p_rand
        out[f"{name}/apply"] = np.asarray(solver.apply(p_rand))
        # count operator applies inside the reference solve
        counter = {"n": 0}
        orig_apply = solver.apply

        def counting_apply(p, _orig=orig_apply):
            counter["n"] += 1
            return _orig(p)

        solver.apply = counting_apply
        p = solver.solve(rhs, rho, dt=1e-3)
        solver.apply = orig_apply
        out[f"{name}/p"] = np.asarray(p)
        out[f"{name}/applies"] = np.array(counter["n"])
        # preconditioner outputs on a random residual
        solver._prepare_preconditioner_state(rho)
        r_rand = rng.standard_normal(grid.shape)
        out[f"{name}/r_rand"] = r_rand
        if solver.preconditioner == "line_pcr":
            out[f"{name}/line_thomas"] = np.asarray(solver.apply_line_preconditioner(r_rand))
            # the GPU branch (truncated PCR, 4 stages) run through NumPy
            rw = r_rand.copy()
            rw.ravel()[solver._pin_dof] = 0.0
            z = np.zeros_like(rw)
            for ax, (lo, d, up) in enumerate(solver._precond_coeffs):
                z += tridiag_variable_batched(np, lo, d, up, rw, ax) * 0.0  # shape check
                n = rw.shape[ax]
                mv = lambda a: np.moveaxis(a, ax, 0).reshape(n, -1)
                x2 = _pcr_solve_variable_batched(np, mv(lo), mv(d), mv(up), mv(rw), max_stages=4)
                moved = np.moveaxis(rw, ax, 0)
                z += np.moveaxis(x2.reshape(moved.shape), 0, ax)
            z /= float(rw.ndim)
            z.ravel()[solver._pin_dof] = 0.0
            out[f"{name}/line_pcr4"] = z
        else:
            out[f"{name}/jacobi"] = np.asarray(solver.apply_jacobi_preconditioner(r_rand))
        # exact direct solution
        direct = PPESolverFVMSpsolve(be, grid, bc_type="wall")
        out[f"{name}/p_direct"] = np.asarray(direct.solve(rhs, rho, dt=1e-3))

    # defect correction (defect_correction.py) with an exact FVM base solve and
    # the CCD variable-density operator L_H as the target operator
    from twophase.ppe.defect_correction import PPESolverDefectCorrection

    class _LHOperator:
        """prepare_operator/apply/_pin_dof around the reference's compute_ccd_laplacian."""

        def __init__(self, grid, ccd, pin):
            self.grid, self.ccd, self._pin_dof = grid, ccd, pin
            self.last_diagnostics = {}

        def prepare_operator(self, rho):
            self.rho = np.asarray(rho)
            self.drho = precompute_density_gradients(self.rho, self.ccd, be)

        def apply(self, p):
            return compute_ccd_laplacian(np.asarray(p), self.rho, self.drho, self.ccd, be)

        def update_grid(self, grid):
            pass

        def invalidate_cache(self):
            pass

    N = (32, 32)
    grid = Grid(GridConfig(ndim=2, N=N, L=(1.0, 1.0)), be)
    ccd = CCDSolver(grid, be, bc_type="wall")
    base = PPESolverFVMSpsolve(be, grid, bc_type="wall")
    op = _LHOperator(grid, ccd, base.ppb._pin_dof)
    dc = PPESolverDefectCorrection(be, grid, base, op, max_corrections=3, tolerance=1e-10)
    rho = droplet_density(N, n_drops=3, rho_g=0.1, seed=2)
    rhs = divergence_rhs(N, seed=3)
    out["dc32/rho"] = rho
    out["dc32/rhs"] = rhs
    out["dc32/p"] = np.asarray(dc.solve(rhs, rho, dt=1e-3))
    out["dc32/history"] = np.asarray(dc.last_residual_history)

    # CCD variable-density Laplacian L_H (ccd_ppe_utils.compute_ccd_laplacian)
    for name, N in (("lh2d", (16, 12)), ("lh3d", (8, 9, 10))):
        grid = Grid(GridConfig(ndim=len(N), N=N, L=(1.0,) * len(N)), be)
        ccd = CCDSolver(grid, be, bc_type="wall")
        rng = np.random.default_rng(77)
        rho = 1.0 + rng.uniform(0.0, 1.0, grid.shape)
        p = rng.standard_normal(grid.shape)
        drho = precompute_density_gradients(rho, ccd, be)
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/rho"] = rho
        out[f"{name}/p"] = p
        out[f"{name}/Lp"] = np.asarray(compute_ccd_laplacian(p, rho, drho, ccd, be))


def make_step(out):
    """Velocity corrector and CFL time step of the reference on seeded fields."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.coupling.velocity_corrector import VelocityCorrector, ccd_pressure_gradient
    from twophase.time_integration.cfl import CFLCalculator

    be = Backend(use_gpu=False)
    rng = np.random.default_rng(4242)
    cases = [("wall2d", (16, 12), "wall"), ("per2d", (16, 10), "periodic"), ("wall3d", (8, 10, 6), "wall")]
    for name, N, bc in cases:
        grid = Grid(GridConfig(ndim=len(N), N=N, L=tuple(1.0 + 0.25 * a for a in range(len(N)))), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        p = rng.standard_normal(grid.shape)
        rho = 1e-3 + rng.uniform(0.0, 1.0, grid.shape)
        mu = 1e-2 + rng.uniform(0.0, 1.0, grid.shape)
        vel = [rng.standard_normal(grid.shape) for _ in range(len(N))]
        dt = 0.0137
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(grid.L, dtype=np.float64)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/p"] = p
        out[f"{name}/rho"] = rho
        out[f"{name}/mu"] = mu
        out[f"{name}/dt"] = np.array(dt)
        for ax in range(len(N)):
            out[f"{name}/u{ax}"] = vel[ax]
        grad = ccd_pressure_gradient(ccd, p, len(N))
        corr = VelocityCorrector(be, grid, ccd).correct(vel, p, rho, dt)
        for ax in range(len(N)):
            out[f"{name}/grad{ax}"] = np.asarray(grad[ax])
            out[f"{name}/unew{ax}"] = np.asarray(corr[ax])
        for tag, kw in (("cn", dict(cn_viscous=True)), ("expl", dict(cn_viscous=False)),
                        ("cap", dict(We=0.01, rho_ratio=0.1, cn_viscous=True))):
            out[f"{name}/dt_{tag}"] = np.array(CFLCalculator(be, grid, 0.3, **kw).compute(vel, mu, rho))


def make_levelset(out):
    """Curvature from psi, the DCCD filter and the material properties of the
    reference on seeded fields."""
    from types import SimpleNamespace
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.levelset.heaviside import heaviside, update_properties
    from twophase.levelset.curvature import _dccd_filter_nd
    from twophase.levelset.curvature_psi import CurvatureCalculatorPsi

    be = Backend(use_gpu=False)
    xp = be.xp
    rng = np.random.default_rng(777)
    # interface shapes on wall / periodic grids (circle, shifted ellipse, sphere)
    cases = [("circle2d", (32, 32), (1.0, 1.0), "wall"),
             ("ellipse2d", (24, 20), (1.2, 1.0), "periodic"),
             ("sphere3d", (12, 10, 14), (1.0, 0.9, 1.1), "wall")]
    for name, N, L, bc in cases:
        grid = Grid(GridConfig(ndim=len(N), N=N, L=L), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        axes = [np.linspace(0.0, L[a], N[a] + 1) for a in range(len(N))]
        X = np.meshgrid(*axes, indexing="ij")
        c = [0.5 * L[a] + 0.03 * (a + 1) for a in range(len(N))]
        r = [0.27 + 0.05 * a for a in range(len(N))]
        phi = np.sqrt(sum(((X[a] - c[a]) / r[a]) ** 2 for a in range(len(N)))) - 1.0
        phi = phi * min(r)
        eps = 1.5 * max(L[a] / N[a] for a in range(len(N)))
        psi = np.asarray(heaviside(xp, phi, eps))
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(L, dtype=np.float64)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/psi"] = psi
        for tag, kw in (("default", {}), ("nofilter", dict(dccd_eps=0.0)),
                        ("gauss", dict(gaussian_filter=True, psi_min=0.02))):
            if tag == "gauss" and len(N) != 2:
                continue
            out[f"{name}/kappa_{tag}"] = np.asarray(CurvatureCalculatorPsi(be, ccd, **kw).compute(psi.copy()))
    fcases = [("f_wall2d", (17, 13), "wall"), ("f_pw2d", (16, 11), "periodic_wall"),
              ("f_per3d", (9, 8, 7), "periodic"), ("f_wall3d", (7, 9, 8), "wall")]
    for name, shape, bc in fcases:
        f = rng.standard_normal(shape)
        sw = rng.uniform(0.0, 1.0, shape)
        g = SimpleNamespace(ndim=len(shape), N=tuple(n - 1 for n in shape))
        out[f"{name}/f"] = f
        out[f"{name}/sw"] = sw
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/plain"] = np.asarray(_dccd_filter_nd(xp, f.copy(), g, 0.05, bc_type=bc))
        out[f"{name}/switched"] = np.asarray(_dccd_filter_nd(xp, f.copy(), g, 0.05, bc_type=bc, switch=sw))
    psi = np.concatenate([[0.0, 0.5, 1.0], rng.uniform(0.0, 1.0, 61)])
    rho, mu = update_properties(xp, psi, 1.0, 0.001, 1.0, 0.0185)
    out["props/psi"] = psi
    out["props/rho"] = np.asarray(rho)
    out["props/mu"] = np.asarray(mu)


def make_rhiechow(out):
    """Rhie-Chow face-velocity divergence of the reference on seeded fields,
    plain and balanced-force."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.spatial.rhie_chow import RhieChowInterpolator

    be = Backend(use_gpu=False)
    rng = np.random.default_rng(9090)
    cases = [("wall2d", (16, 12), "wall"), ("per2d", (16, 10), "periodic"), ("wall3d", (8, 10, 6), "wall"),
             ("per3d", (6, 8, 7), "periodic")]
    for name, N, bc in cases:
        L = tuple(1.0 + 0.25 * a for a in range(len(N)))
        grid = Grid(GridConfig(ndim=len(N), N=N, L=L), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        rc = RhieChowInterpolator(be, grid, ccd, bc_type=bc)
        p = rng.standard_normal(grid.shape)
        rho = 1e-3 + rng.uniform(0.0, 1.0, grid.shape)
        vel = [rng.standard_normal(grid.shape) for _ in range(len(N))]
        kappa = rng.standard_normal(grid.shape)
        psi = rng.uniform(0.0, 1.0, grid.shape)
        dt, we = 0.0137, 0.7
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(L, dtype=np.float64)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/p"] = p
        out[f"{name}/rho"] = rho
        out[f"{name}/kappa"] = kappa
        out[f"{name}/psi"] = psi
        out[f"{name}/dt"] = np.array(dt)
        out[f"{name}/we"] = np.array(we)
        for ax in range(len(N)):
            out[f"{name}/u{ax}"] = vel[ax]
        out[f"{name}/div"] = np.asarray(rc.face_velocity_divergence(vel, p, rho, dt))
        out[f"{name}/div_bf"] = np.asarray(rc.face_velocity_divergence(vel, p, rho, dt, kappa=kappa, psi=psi, we=we))


def make_advect(out):
    """FCCD flux-form advection right-hand sides and one TVD-RK3 level-set
    step of the reference on seeded fields."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.ccd.fccd import FCCDSolver
    from twophase.levelset.fccd_advection import FCCDLevelSetAdvection
    from twophase.levelset.heaviside import heaviside

    be = Backend(use_gpu=False)
    xp = be.xp
    rng = np.random.default_rng(31337)
    cases = [("wall2d", (20, 16), (1.0, 0.8), "wall"), ("per2d", (16, 12), (1.0, 1.0), "periodic"),
             ("wall3d", (8, 10, 6), (1.0, 1.2, 0.8), "wall"), ("per3d", (8, 6, 10), (1.0, 1.0, 1.0), "periodic")]
    for name, N, L, bc in cases:
        grid = Grid(GridConfig(ndim=len(N), N=N, L=L), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        fccd = FCCDSolver(grid, be, bc_type=bc, ccd_solver=ccd)
        X = np.meshgrid(*[np.linspace(0.0, L[a], N[a] + 1) for a in range(len(N))], indexing="ij")
        phi = np.sqrt(sum((X[a] - 0.5 * L[a]) ** 2 for a in range(len(N)))) - 0.25
        psi = np.asarray(heaviside(xp, phi, 1.5 * max(L[a] / N[a] for a in range(len(N)))))
        vel = [0.5 * rng.standard_normal(grid.shape) + 0.3 * np.cos(2 * np.pi * X[(a + 1) % len(N)])
               for a in range(len(N))]
        if bc == "periodic":   # periodic fields carry equal image planes
            for v in vel + [psi]:
                for ax in range(len(N)):
                    src = [slice(None)] * len(N)
                    img = [slice(None)] * len(N)
                    src[ax] = 0
                    img[ax] = -1
                    v[tuple(img)] = v[tuple(src)]
        dt = 0.004
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(L, dtype=np.float64)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/psi"] = psi
        out[f"{name}/dt"] = np.array(dt)
        for a in range(len(N)):
            out[f"{name}/u{a}"] = vel[a]
        out[f"{name}/rhs_scalar"] = np.asarray(fccd.advection_rhs(vel, scalar=psi, mode="flux")[0])
        mom = fccd.advection_rhs(vel, mode="flux")
        for a in range(len(N)):
            out[f"{name}/rhs_mom{a}"] = np.asarray(mom[a])
        adv = FCCDLevelSetAdvection(be, grid, fccd, mode="flux")
        out[f"{name}/psi_new"] = np.asarray(adv.advance(psi.copy(), vel, dt))
        out[f"{name}/psi_new_noclip"] = np.asarray(adv.advance(psi.copy(), vel, dt, clip_bounds=None))
        adv_m = FCCDLevelSetAdvection(be, grid, fccd, mode="flux", mass_correction=True)
        out[f"{name}/psi_new_mass"] = np.asarray(adv_m.advance(psi.copy(), vel, dt))
        from twophase.ns_terms.uccd6_convection import UCCD6ConvectionTerm
        uc = UCCD6ConvectionTerm(be, grid, ccd, sigma=1.0e-3).compute(vel)
        for a in range(len(N)):
            out[f"{name}/uccd6_{a}"] = np.asarray(uc[a])
        # Option C (mode="node"): R_4 Hermite node gradients and the nodal
        # advection right-hand sides, and one TVD-RK3 step in that mode
        for a in range(len(N)):
            out[f"{name}/node_grad_psi{a}"] = np.asarray(fccd.node_gradient(psi, a))
        out[f"{name}/rhs_scalar_node"] = np.asarray(fccd.advection_rhs(vel, scalar=psi, mode="node")[0])
        mom = fccd.advection_rhs(vel, mode="node")
        for a in range(len(N)):
            out[f"{name}/rhs_mom_node{a}"] = np.asarray(mom[a])
        adv_n = FCCDLevelSetAdvection(be, grid, fccd, mode="node")
        out[f"{name}/psi_new_node"] = np.asarray(adv_n.advance(psi.copy(), vel, dt))


def make_reinit(out):
    """Split reinitialization (compression + CN-ADI + mass correction) of the
    reference on seeded interface fields."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.levelset.heaviside import heaviside
    from twophase.levelset.reinit_split import SplitReinitializer

    be = Backend(use_gpu=False)
    xp = be.xp
    rng = np.random.default_rng(4711)
    cases = [("zero2d", (24, 20), (1.0, 0.9), "wall", "zero", 4, True),
             ("per2d", (16, 16), (1.0, 1.0), "periodic", "periodic", 2, True),
             ("neu2d", (20, 18), (1.0, 1.0), "wall", "neumann", 3, False),
             ("zero3d", (10, 8, 12), (1.0, 0.8, 1.2), "wall", "zero", 2, True)]
    for name, N, L, ccd_bc, bc, n_steps, mass in cases:
        grid = Grid(GridConfig(ndim=len(N), N=N, L=L), be)
        ccd = CCDSolver(grid, be, bc_type=ccd_bc)
        h = max(L[a] / N[a] for a in range(len(N)))
        X = np.meshgrid(*[np.linspace(0.0, L[a], N[a] + 1) for a in range(len(N))], indexing="ij")
        phi = np.sqrt(sum(((X[a] - 0.5 * L[a]) / (0.3 + 0.05 * a)) ** 2 for a in range(len(N)))) - 1.0
        psi = np.asarray(heaviside(xp, 0.3 * phi, 2.5 * h)) + 0.02 * rng.standard_normal(grid.shape)
        psi = np.clip(psi, 0.0, 1.0)
        eps = 1.5 * h
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(L, dtype=np.float64)
        out[f"{name}/ccd_bc"] = np.array(ccd_bc)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/eps"] = np.array(eps)
        out[f"{name}/n_steps"] = np.array(n_steps)
        out[f"{name}/mass"] = np.array(mass)
        out[f"{name}/psi"] = psi
        r = SplitReinitializer(be, grid, ccd, eps, n_steps=n_steps, bc=bc, mass_correction=mass)
        out[f"{name}/psi_reinit"] = np.asarray(r.reinitialize(psi.copy()))


def make_viscous(out):
    """ViscousTerm.compute_explicit of the reference in its three spatial schemes."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.ns_terms.viscous import ViscousTerm

    be = Backend(use_gpu=False)
    rng = np.random.default_rng(2718)
    cases = [("wall2d", (18, 14), (1.0, 0.7), "wall"), ("per2d", (16, 12), (1.0, 1.0), "periodic"),
             ("wall3d", (8, 10, 6), (1.0, 1.2, 0.8), "wall")]
    for name, N, L, bc in cases:
        grid = Grid(GridConfig(ndim=len(N), N=N, L=L), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        vel = [rng.standard_normal(grid.shape) for _ in N]
        mu = 0.01 + rng.uniform(0.0, 1.0, grid.shape)
        rho = 0.001 + rng.uniform(0.0, 1.0, grid.shape)
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(L, dtype=np.float64)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/mu"] = mu
        out[f"{name}/rho"] = rho
        for a in range(len(N)):
            out[f"{name}/u{a}"] = vel[a]
        for scheme in ("ccd_bulk", "conservative_stress", "ccd_stress_legacy"):
            v = ViscousTerm(be, 100.0, spatial_scheme=scheme).compute_explicit(vel, mu, rho, ccd)
            for a in range(len(N)):
                out[f"{name}/{scheme}/v{a}"] = np.asarray(v[a])
        e = [rng.standard_normal(grid.shape) for _ in N]
        for a in range(len(N)):
            out[f"{name}/e{a}"] = e[a]
        for tag, cn in (("cn", True), ("fe", False)):
            u = ViscousTerm(be, 100.0, cn_viscous=cn).apply_cn_predictor(vel, e, mu, rho, ccd, 0.003)
            for a in range(len(N)):
                out[f"{name}/pred_{tag}{a}"] = np.asarray(u[a])
        # interface-band form of ccd_bulk (psi given): a thin sigmoid
        # interface (psi < 1e-6 deep inside, exactly 1 far outside)
        X = np.meshgrid(*[np.asarray(c) for c in grid.coords], indexing="ij")
        r = np.sqrt(sum((x - 0.45 * l) ** 2 for x, l in zip(X, L)))
        psi = 1.0 / (1.0 + np.exp(-(r - 0.3 * min(L)) / 0.02))
        out[f"{name}/psi"] = psi
        v = ViscousTerm(be, 100.0, spatial_scheme="ccd_bulk").compute_explicit(vel, mu, rho, ccd, psi=psi)
        for a in range(len(N)):
            out[f"{name}/ccd_bulk_band/v{a}"] = np.asarray(v[a])
        u = ViscousTerm(be, 100.0, cn_viscous=True).apply_cn_predictor(vel, e, mu, rho, ccd, 0.003, psi=psi)
        for a in range(len(N)):
            out[f"{name}/pred_band{a}"] = np.asarray(u[a])
        # Richardson extrapolation around Picard (cn_mode='richardson_picard')
        from twophase.time_integration.cn_advance import make_cn_advance
        u = ViscousTerm(be, 100.0, cn_viscous=True, cn_advance=make_cn_advance(be, "richardson_picard")
                        ).apply_cn_predictor(vel, e, mu, rho, ccd, 0.003)
        for a in range(len(N)):
            out[f"{name}/pred_rich{a}"] = np.asarray(u[a])


def make_viscous_nonuniform(out):
    """ViscousTerm.compute_explicit on an interface-fitted (non-uniform) 2-D
    wall grid, the three spatial schemes (separate file so the uniform
    cases' arrays stay as they are)."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.levelset.heaviside import heaviside
    from twophase.ns_terms.viscous import ViscousTerm

    be = Backend(use_gpu=False)
    N = 32
    grid = Grid(GridConfig(ndim=2, N=(N, N), L=(1.0, 1.0), alpha_grid=2.0, eps_g_factor=2.0), be)
    ccd = CCDSolver(grid, be, bc_type="wall")
    X, Y = grid.meshgrid()
    grid.update_from_levelset(heaviside(np, X - 0.5, 0.5 / N), 0.5 / N, ccd=ccd)
    ccd = CCDSolver(grid, be, bc_type="wall")
    rng = np.random.default_rng(4242)
    vel = [rng.standard_normal(grid.shape) for _ in range(2)]
    mu = 0.01 + rng.uniform(0.0, 1.0, grid.shape)
    rho = 0.001 + rng.uniform(0.0, 1.0, grid.shape)
    out["N"] = np.array((N, N))
    for ax in range(2):
        out[f"J{ax}"] = np.asarray(grid.J[ax], dtype=np.float64)
        out[f"dJ{ax}"] = np.asarray(grid.dJ_dxi[ax], dtype=np.float64)
        out[f"coords{ax}"] = np.asarray(grid.coords[ax])
        out[f"u{ax}"] = vel[ax]
    out["mu"] = mu
    out["rho"] = rho
    for scheme in ("ccd_bulk", "conservative_stress", "ccd_stress_legacy"):
        v = ViscousTerm(be, 100.0, spatial_scheme=scheme).compute_explicit(vel, mu, rho, ccd)
        for a in range(2):
            out[f"{scheme}/v{a}"] = np.asarray(v[a])


def make_fccd_nonuniform(out):
    """FCCD advection right-hand sides (flux and node forms), node gradients
    and one TVD-RK3 step (both forms) on an interface-fitted (non-uniform)
    2-D wall grid."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.ccd.fccd import FCCDSolver
    from twophase.levelset.fccd_advection import FCCDLevelSetAdvection
    from twophase.levelset.heaviside import heaviside

    be = Backend(use_gpu=False)
    N = 32
    grid = Grid(GridConfig(ndim=2, N=(N, N), L=(1.0, 1.0), alpha_grid=2.0, eps_g_factor=2.0), be)
    ccd = CCDSolver(grid, be, bc_type="wall")
    X, Y = grid.meshgrid()
    grid.update_from_levelset(heaviside(np, np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2) - 0.25, 0.5 / N), 0.5 / N,
                              ccd=ccd)
    ccd = CCDSolver(grid, be, bc_type="wall")
    fccd = FCCDSolver(grid, be, bc_type="wall", ccd_solver=ccd)
    X, Y = np.meshgrid(grid.coords[0], grid.coords[1], indexing="ij")
    psi = np.asarray(heaviside(np, np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2) - 0.25, 1.5 / N))
    rng = np.random.default_rng(777)
    vel = [0.5 * rng.standard_normal(grid.shape) + 0.3 * np.cos(2 * np.pi * (Y if a == 0 else X)) for a in range(2)]
    out["N"] = np.array((N, N))
    for ax in range(2):
        out[f"J{ax}"] = np.asarray(grid.J[ax], dtype=np.float64)
        out[f"dJ{ax}"] = np.asarray(grid.dJ_dxi[ax], dtype=np.float64)
        out[f"coords{ax}"] = np.asarray(grid.coords[ax])
        out[f"u{ax}"] = vel[ax]
        out[f"node_grad_psi{ax}"] = np.asarray(fccd.node_gradient(psi, ax))
    out["psi"] = psi
    for mode in ("flux", "node"):
        out[f"rhs_scalar_{mode}"] = np.asarray(fccd.advection_rhs(vel, scalar=psi, mode=mode)[0])
        mom = fccd.advection_rhs(vel, mode=mode)
        for a in range(2):
            out[f"rhs_mom_{mode}{a}"] = np.asarray(mom[a])
        out[f"psi_new_{mode}"] = np.asarray(FCCDLevelSetAdvection(be, grid, fccd, mode=mode).advance(psi.copy(), vel,
                                                                                                    0.004))


def make_reinit_nonuniform(out):
    """Split reinitialization on an interface-fitted (non-uniform) 2-D wall
    grid: zero and Neumann ghost padding, with and without mass correction."""
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.levelset.heaviside import heaviside
    from twophase.levelset.reinit_split import SplitReinitializer

    be = Backend(use_gpu=False)
    N = 32
    grid = Grid(GridConfig(ndim=2, N=(N, N), L=(1.0, 1.0), alpha_grid=2.0, eps_g_factor=2.0), be)
    ccd = CCDSolver(grid, be, bc_type="wall")
    X, Y = grid.meshgrid()
    grid.update_from_levelset(heaviside(np, np.sqrt((X - 0.5) ** 2 + (Y - 0.45) ** 2) - 0.3, 0.5 / N), 0.5 / N,
                              ccd=ccd)
    ccd = CCDSolver(grid, be, bc_type="wall")
    X, Y = np.meshgrid(grid.coords[0], grid.coords[1], indexing="ij")
    rng = np.random.default_rng(9191)
    psi = np.asarray(heaviside(np, np.sqrt((X - 0.5) ** 2 + (Y - 0.45) ** 2) - 0.3, 2.5 / N))
    psi = np.clip(psi + 0.02 * rng.standard_normal(grid.shape), 0.0, 1.0)
    eps = 1.5 / N
    out["N"] = np.array((N, N))
    for ax in range(2):
        out[f"J{ax}"] = np.asarray(grid.J[ax], dtype=np.float64)
        out[f"dJ{ax}"] = np.asarray(grid.dJ_dxi[ax], dtype=np.float64)
        out[f"coords{ax}"] = np.asarray(grid.coords[ax])
        out[f"h{ax}"] = np.asarray(grid.h[ax], dtype=np.float64)
    out["psi"] = psi
    out["eps"] = np.array(eps)
    for tag, bc, mass in (("zero_mass", "zero", True), ("neumann", "neumann", False)):
        r = SplitReinitializer(be, grid, ccd, eps, n_steps=3, bc=bc, mass_correction=mass)
        out[f"{tag}/dtau"] = np.array(r.dtau)
        out[f"{tag}/psi_reinit"] = np.asarray(r.reinitialize(psi.copy()))


def make_predictor(out):
    """Two consecutive AB2 + IPC predictor steps of the reference (forward Euler
    convection, then AB2), CN and explicit viscous, CSF and GFM."""
    from twophase.backend import Backend
    from twophase.config import FluidConfig, GridConfig, NumericsConfig, SimulationConfig
    from twophase.core.grid import Grid
    from twophase.core.flow_state import FlowState
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.time_integration.ab2_predictor import Predictor

    be = Backend(use_gpu=False)
    rng = np.random.default_rng(1618)
    cases = [("wall2d", (16, 12), (1.0, 0.8), "wall", True, False), ("per2d", (12, 14), (1.0, 1.0), "periodic", False, False),
             ("wall3d", (8, 6, 10), (1.0, 0.8, 1.2), "wall", True, True)]
    for name, N, L, bc, cn, gfm in cases:
        cfg = SimulationConfig(grid=GridConfig(ndim=len(N), N=N, L=L), fluid=FluidConfig(Re=50.0, Fr=0.8, We=4.0),
                               numerics=NumericsConfig(cn_viscous=cn, bc_type=bc))
        grid = Grid(cfg.grid, be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        pred = Predictor(be, cfg, ccd, use_gfm=gfm)
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(L, dtype=np.float64)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/cn"] = np.array(cn)
        out[f"{name}/gfm"] = np.array(gfm)
        for step, dt in enumerate((0.002, 0.0025)):
            vel = [0.3 * rng.standard_normal(grid.shape) for _ in N]
            psi = rng.uniform(0.0, 1.0, grid.shape)
            rho = 0.1 + 0.9 * psi
            mu = 0.01 + 0.99 * psi
            kappa = rng.standard_normal(grid.shape)
            p = rng.standard_normal(grid.shape)
            for a in range(len(N)):
                out[f"{name}/s{step}/u{a}"] = vel[a]
            out[f"{name}/s{step}/psi"] = psi
            out[f"{name}/s{step}/kappa"] = kappa
            out[f"{name}/s{step}/p"] = p
            out[f"{name}/s{step}/dt"] = np.array(dt)
            u = pred.compute(FlowState(velocity=vel, psi=psi, rho=rho, mu=mu, kappa=kappa, pressure=p), dt)
            for a in range(len(N)):
                out[f"{name}/s{step}/ustar{a}"] = np.asarray(u[a])


def make_fccd_ppe(out):
    """The FCCD matrix-free PPE of the reference on its default path
    (phase_density coefficients, full faces): operator applies, the Jacobi
    inverse and GMRES solutions."""
    from types import SimpleNamespace
    from twophase.backend import Backend
    from twophase.config import GridConfig
    from twophase.core.grid import Grid
    from twophase.ccd.ccd_solver import CCDSolver
    from twophase.ccd.fccd import FCCDSolver
    from twophase.ppe.fccd_matrixfree import PPESolverFCCDMatrixFree

    be = Backend(use_gpu=False)
    rng = np.random.default_rng(5151)
    cases = [("wall2d", (16, 12), (1.0, 0.8), "wall", "jacobi"), ("per2d", (12, 12), (1.0, 1.0), "periodic", "none"),
             ("wall3d", (8, 6, 10), (1.0, 0.8, 1.2), "wall", "jacobi")]
    for name, N, L, bc, pre in cases:
        grid = Grid(GridConfig(ndim=len(N), N=N, L=L), be)
        ccd = CCDSolver(grid, be, bc_type=bc)
        fccd = FCCDSolver(grid, be, bc_type=bc, ccd_solver=ccd)
        cfg = SimpleNamespace(pseudo_tol=1e-9, pseudo_maxiter=500, ppe_restart=None, ppe_preconditioner=pre)
        solver = PPESolverFCCDMatrixFree(be, cfg, grid, fccd)
        rho = 0.5 + rng.uniform(0.0, 1.0, grid.shape)
        if bc == "periodic":
            for ax in range(len(N)):
                src = [slice(None)] * len(N)
                img = [slice(None)] * len(N)
                src[ax] = 0
                img[ax] = -1
                rho[tuple(img)] = rho[tuple(src)]
        p = rng.standard_normal(grid.shape)
        rhs = rng.standard_normal(grid.shape)
        solver.prepare_operator(rho)
        out[f"{name}/N"] = np.array(N)
        out[f"{name}/L"] = np.array(L, dtype=np.float64)
        out[f"{name}/bc"] = np.array(bc)
        out[f"{name}/pre"] = np.array(pre)
        out[f"{name}/rho"] = rho
        out[f"{name}/p"] = p
        out[f"{name}/rhs"] = rhs
        out[f"{name}/apply"] = np.asarray(solver.apply(p))
        if pre == "jacobi":
            out[f"{name}/diag_inv"] = np.asarray(solver._diag_inv)
        out[f"{name}/sol"] = np.asarray(solver.solve(rhs, rho))


def make_c1(out):
    """The reference's stable quick-start (64^2 bubble, R = 0.25 at the centre,
    Re 100, Fr 1, We 10, density and viscosity ratios 0.1, extension_method
    'none'): six steps of SimulationBuilder(cfg).build().step_forward(dt) with
    the reference's CFL time step, fields after each step."""
    from twophase.config import FluidConfig, GridConfig, NumericsConfig, SimulationConfig
    from twophase.simulation.builder import SimulationBuilder

    cfg = SimulationConfig(grid=GridConfig(ndim=2, N=(64, 64), L=(1.0, 1.0)),
                           fluid=FluidConfig(Re=100.0, Fr=1.0, We=10.0, rho_ratio=0.1, mu_ratio=0.1),
                           numerics=NumericsConfig(extension_method="none"))
    sim = SimulationBuilder(cfg).build()
    X, Y = sim.grid.meshgrid()
    sim.psi.data[:] = 1.0 / (1.0 + np.exp(-(np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2) - 0.25) / (1.5 / 64)))
    out["psi0"] = np.array(sim.psi.data)
    for k in range(6):
        dt = float(sim.cfl_calc.compute([sim.velocity[0], sim.velocity[1]], sim.mu.data, sim.rho.data))
        sim.step_forward(dt)
        out[f"s{k}/dt"] = np.array(dt)
        out[f"s{k}/psi"] = np.array(sim.psi.data)
        out[f"s{k}/u"] = np.array(sim.velocity[0])
        out[f"s{k}/v"] = np.array(sim.velocity[1])
        out[f"s{k}/p"] = np.array(sim.pressure.data)


C1_CHECKPOINT_YAML = """\
run:
  T_final: 0.05
  cfl: 0.3
grid:
  ndim: 2
  N: [64, 64]
  L: [1.0, 1.0]
fluid:
  Re: 100.0
  Fr: 1.0
  We: 10.0
  rho_ratio: 0.1
  mu_ratio: 0.1
numerics:
  extension_method: none
output:
  dir: results/c1
"""


def make_checkpoint(out):
    """A restart checkpoint written by the reference's own writer
    (simulation/checkpoint.py save_checkpoint) after three quick-start steps
    (the make_c1 run): state/psi, u, v, p, the grid, p^n as
    solver/p_prev_dev and the predictor's AB2 convection history as
    solver/conv_prev.  Writes c1_checkpoint_ref.npz and c1_checkpoint.yaml
    (the config the fingerprint covers) next to this script; ``out`` stays
    empty."""
    from types import SimpleNamespace
    from twophase.config import FluidConfig, GridConfig, NumericsConfig, SimulationConfig
    from twophase.simulation.builder import SimulationBuilder
    from twophase.simulation.checkpoint import save_checkpoint

    cfg = SimulationConfig(grid=GridConfig(ndim=2, N=(64, 64), L=(1.0, 1.0)),
                           fluid=FluidConfig(Re=100.0, Fr=1.0, We=10.0, rho_ratio=0.1, mu_ratio=0.1),
                           numerics=NumericsConfig(extension_method="none"))
    sim = SimulationBuilder(cfg).build()
    X, Y = sim.grid.meshgrid()
    sim.psi.data[:] = 1.0 / (1.0 + np.exp(-(np.sqrt((X - 0.5) ** 2 + (Y - 0.5) ** 2) - 0.25) / (1.5 / 64)))
    t = 0.0
    for _ in range(3):
        dt = float(sim.cfl_calc.compute([sim.velocity[0], sim.velocity[1]], sim.mu.data, sim.rho.data))
        sim.step_forward(dt)
        t += dt
    yaml_path = os.path.join(HERE, "c1_checkpoint.yaml")
    with open(yaml_path, "w") as fh:
        fh.write(C1_CHECKPOINT_YAML)
    solver = SimpleNamespace(_backend=sim.backend, _grid=sim.grid, _p_prev_dev=np.array(sim.pressure.data),
                             _conv_prev=sim.predictor._conv_prev, _conv_ab2_ready=sim.predictor._ab2_ready)
    save_checkpoint(os.path.join(HERE, "c1_checkpoint_ref.npz"), solver=solver, psi=sim.psi.data,
                    u=sim.velocity[0], v=sim.velocity[1], p=sim.pressure.data, t=t, step=3,
                    config_path=yaml_path, state_phase="post_step", dt_candidate=dt, dt_effective=dt)


def main():
    """Usage: make_golden.py <reference src dir> [only: ccd|ppe|step|levelset|rhiechow|advect|reinit|reinit_nonuniform|viscous|viscous_nonuniform|fccd_nonuniform|predictor|fccd_ppe|c1|checkpoint ...].

    The source directory comes from the first argument or, when the
    argument list is empty, from the TWOPHASE_REFERENCE_SRC environment variable."""
    args = sys.argv[1:]
    if args and os.path.isdir(os.path.join(args[0], "twophase")):
        src, only = args[0], set(args[1:])
    else:
        src, only = os.environ.get("TWOPHASE_REFERENCE_SRC", ""), set(args)
    if not src or not os.path.isdir(os.path.join(src, "twophase")):
        raise SystemExit("make_golden.py: give the reference's src directory as the first argument "
                         "or in TWOPHASE_REFERENCE_SRC")
    _ref_import(src)
    makers = {"ccd": make_ccd, "ppe": make_ppe, "step": make_step, "levelset": make_levelset,
              "rhiechow": make_rhiechow, "advect": make_advect, "reinit": make_reinit,
              "viscous": make_viscous, "predictor": make_predictor,
              "fccd_ppe": make_fccd_ppe, "c1": make_c1, "checkpoint": make_checkpoint,
              "viscous_nonuniform": make_viscous_nonuniform, "fccd_nonuniform": make_fccd_nonuniform,
              "reinit_nonuniform": make_reinit_nonuniform}
    for key, fn in makers.items():
        if only and key not in only:
            continue
        arrays = {}
        fn(arrays)
        if not arrays:      # the maker wrote its own files
            print("wrote", key, "files")
            continue
        np.savez_compressed(os.path.join(HERE, f"{key}_golden.npz"), **arrays)
        print("wrote", len(arrays), key, "arrays")


if __name__ == "__main__":
    main()
