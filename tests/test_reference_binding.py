"""The reference-side binding: the reference's own PPE registry and builder
resolve to this package's solver once it is registered.

Runs on the CPU against the reference's Python package, read in place
(``TWOPHASE_REFERENCE_SRC``, default: the reference's source mount); skipped
where the reference is not importable.  The B200 solver's construction is let
past its CUDA checks (``torch.cuda.is_available`` and the device-side handle
creation are patched): no solve is run, only the wiring is checked.

Reference call sites: ``ppe/factory.py:31-39`` (``register_ppe_solver``),
``:90-120`` (``create_ppe_solver``), ``simulation/legacy_builder_runtime.py:140-146``
(the builder asks the registry for ``config.solver.ppe_solver_type``),
``simulation/builder.py:66-74`` (``with_ppe_solver``), ``ppe/interfaces.py:28-86``
(``IPPESolver``).
"""

from __future__ import annotations

import inspect
import os
import sys

import numpy as np
import pytest

REF_SRC = os.environ.get("TWOPHASE_REFERENCE_SRC", "/root/reference/src")


@pytest.fixture()
def reference(monkeypatch):
    if not os.path.isdir(os.path.join(REF_SRC, "twophase")):
        pytest.skip("the reference package is not available on this machine")
    monkeypatch.setattr(sys, "dont_write_bytecode", True)   # the reference tree is read-only
    monkeypatch.syspath_prepend(REF_SRC)
    try:
        import twophase  # noqa: F401
        from twophase.ppe import factory
    except Exception as exc:   # pragma: no cover - depends on the machine
        pytest.skip(f"the reference package does not import here: {exc}")
    saved = dict(factory._SOLVER_REGISTRY)
    yield factory
    factory._SOLVER_REGISTRY.clear()
    factory._SOLVER_REGISTRY.update(saved)


@pytest.fixture()
def no_device(monkeypatch):
    """Let PPESolverFVMMatrixFree construct without a GPU: the CUDA check
    passes and the device-side handle is not created."""
    import torch

    from twophaseflow_b200 import ppe as bppe
    monkeypatch.setattr(torch.cuda, "is_available", lambda: True)
    monkeypatch.setattr(bppe.PPESolverFVMMatrixFree, "_create", lambda self: None)
    monkeypatch.setattr(bppe.PPESolverFVMMatrixFree, "__del__", lambda self: None)


def _config(N=(16, 16), **solver):
    from twophase.config import FluidConfig, GridConfig, NumericsConfig, SimulationConfig, SolverConfig
    return SimulationConfig(grid=GridConfig(ndim=len(N), N=N, L=(1.0,) * len(N)),
                            fluid=FluidConfig(Re=100.0, Fr=1.0, We=10.0),
                            numerics=NumericsConfig(t_end=0.1, cfl_number=0.3),
                            solver=SolverConfig(ppe_solver_type="fvm_iterative", **solver))


def _reference_grid(cfg):
    from twophase.backend import Backend
    from twophase.core.grid import Grid
    backend = Backend(use_gpu=False)
    return backend, Grid(cfg.grid, backend)


def test_registry_resolves_to_b200_solver(reference, no_device):
    from twophaseflow_b200 import PPESolverFVMMatrixFree, register_with_reference
    factory = reference
    register_with_reference(factory.register_ppe_solver)
    for key in ("fvm_iterative", "fvm_matrixfree"):
        assert factory._SOLVER_REGISTRY[key].__module__ == "twophaseflow_b200.ppe"
    cfg = _config()
    backend, grid = _reference_grid(cfg)
    s = factory.create_ppe_solver(cfg, backend, grid)
    assert isinstance(s, PPESolverFVMMatrixFree)
    # the pinned gauge is the reference BoundarySpec's (core/boundary.py:182-191)
    bc_spec = factory._make_bc_spec(cfg, grid)
    assert s._pin_dof == int(bc_spec.pin_dof)
    # options read from the reference config with the reference defaults
    # (fvm_matrixfree.py:90-127)
    assert (s.tol, s.maxiter, s.restart, s.c_tau) == (1e-8, 500, 80, 2.0)
    assert s.iteration_method == "gmres" and s.preconditioner == "line_pcr"
    # the reference grid object is read as-is
    assert tuple(s.grid.shape) == (17, 17)
    np.testing.assert_array_equal(np.asarray(grid.coords[0]), np.linspace(0.0, 1.0, 17))


def test_registry_passes_cg_options(reference, no_device):
    """SolverConfig's own fields reach the B200 solver: tolerance, budget and
    the CG route, whose default preconditioner is Jacobi (fvm_matrixfree.py:100-118)."""
    from twophaseflow_b200 import register_with_reference
    factory = reference
    register_with_reference(factory.register_ppe_solver)
    cfg = _config(pseudo_tol=1e-10, pseudo_maxiter=4000, ppe_iteration_method="cg")
    backend, grid = _reference_grid(cfg)
    s = factory.create_ppe_solver(cfg, backend, grid)
    assert (s.tol, s.maxiter, s.restart) == (1e-10, 4000, 80)
    assert s.iteration_method == "cg" and s.preconditioner == "jacobi"


def test_class_covers_ippesolver_surface(reference):
    from twophase.ppe.interfaces import IPPESolver

    from twophaseflow_b200 import PPESolverFVMMatrixFree
    assert IPPESolver.__abstractmethods__ == frozenset({"solve"})
    ref_params = list(inspect.signature(IPPESolver.solve).parameters)
    ours = list(inspect.signature(PPESolverFVMMatrixFree.solve).parameters)
    assert ours[:len(ref_params)] == ref_params   # self, rhs, rho, dt, p_init
    for name in ("get_matrix", "update_grid", "invalidate_cache", "clear_interface_jump_context", "apply",
                 "prepare_operator"):
        assert callable(getattr(PPESolverFVMMatrixFree, name, None)), name


def test_builder_wires_registered_solver(reference, no_device):
    """SimulationBuilder(cfg).build() takes its PPE from the registry; with the
    B200 solver registered, the built simulation holds it."""
    from twophase.simulation.builder import SimulationBuilder

    from twophaseflow_b200 import PPESolverFVMMatrixFree, register_with_reference
    factory = reference
    register_with_reference(factory.register_ppe_solver)
    sim = SimulationBuilder(_config()).build()
    held = [v for v in vars(sim).values() if isinstance(v, PPESolverFVMMatrixFree)]
    if not held:   # components may sit one level down
        for v in vars(sim).values():
            held += [w for w in getattr(v, "__dict__", {}).values() if isinstance(w, PPESolverFVMMatrixFree)]
    assert held, "the built simulation does not hold the registered B200 PPE solver"


def test_builder_accepts_injected_solver(reference, no_device):
    """SimulationBuilder(cfg).with_ppe_solver(s) keeps the B200 instance."""
    from twophase.simulation.builder import SimulationBuilder

    from twophaseflow_b200 import PPESolverFVMMatrixFree, create_fvm_matrixfree
    cfg = _config()
    backend, grid = _reference_grid(cfg)
    s = create_fvm_matrixfree(cfg, backend, grid)
    b = SimulationBuilder(cfg).with_ppe_solver(s)
    assert b._ppe_solver is s and isinstance(s, PPESolverFVMMatrixFree)
