"""twophaseflow_b200: B200 (sm_100a) implementation of TwoPhaseFlow's hot path.

* ``CCDSolver`` -- drop-in for ``twophase.ccd.ccd_solver.CCDSolver``
* ``PPESolverFVMMatrixFree`` -- drop-in for
  ``twophase.ppe.fvm_matrixfree.PPESolverFVMMatrixFree`` (an ``IPPESolver``)
* ``CCDVariableDensityOperator`` / ``PPESolverDefectCorrection`` -- the CCD
  variable-density operator L_H and the defect-correction PPE loop
* ``PPESolverFCCDMatrixFree`` -- drop-in for
  ``twophase.ppe.fccd_matrixfree.PPESolverFCCDMatrixFree`` (default path)
* ``register_with_reference`` -- installs the PPE solver in the reference's
  ``register_ppe_solver`` registry.
* ``VelocityCorrector`` / ``CFLCalculator`` / ``ccd_pressure_gradient`` -- the
  steps either side of the PPE (velocity correction fused into the CCD line
  solve; CFL maxima in one reduction).
* ``TwoPhaseStep`` -- the whole two-phase step; ``save_checkpoint`` /
  ``load_checkpoint`` -- restart files in the reference's ``.npz`` format.

All arithmetic runs in the in-tree CUDA library ``libtpf.so`` (C ABI:
``include/tpf.h``); build it with ``python -m twophaseflow_b200.build``.
"""

from . import checkpoint
from .advection import FCCDLevelSetAdvection, FCCDSolver, SplitReinitializer, UCCD6ConvectionTerm
from .ccd import CCDSolver
from .ccd_ppe import CCDVariableDensityOperator, PPESolverDefectCorrection
from .fccd_ppe import PPESolverFCCDMatrixFree
from .grid import BoundarySpec, UniformGrid
from .ppe import (MatrixAssemblyUnavailable, PPESolverFVMMatrixFree, create_fvm_matrixfree, register_with_reference,
                  solve_batched)
from .levelset import CurvatureCalculatorPsi, dccd_filter_nd, update_properties
from .viscous import PicardCNAdvance, RichardsonCNAdvance, ViscousTerm, make_cn_advance
from .predictor import ConvectionTerm, FlowState, GravityTerm, NSComputeContext, Predictor, SurfaceTensionTerm
from .ns_step import TwoPhaseStep
from .step import CFLCalculator, RhieChowInterpolator, VelocityCorrector, ccd_pressure_gradient
from .checkpoint import CheckpointError, load_checkpoint, save_checkpoint

__all__ = [
    "CCDSolver",
    "FCCDSolver",
    "FCCDLevelSetAdvection",
    "SplitReinitializer",
    "UCCD6ConvectionTerm",
    "CCDVariableDensityOperator",
    "PPESolverDefectCorrection",
    "PPESolverFVMMatrixFree",
    "PPESolverFCCDMatrixFree",
    "MatrixAssemblyUnavailable",
    "create_fvm_matrixfree",
    "register_with_reference",
    "solve_batched",
    "UniformGrid",
    "BoundarySpec",
    "VelocityCorrector",
    "CFLCalculator",
    "ViscousTerm",
    "PicardCNAdvance",
    "RichardsonCNAdvance",
    "make_cn_advance",
    "ConvectionTerm",
    "GravityTerm",
    "SurfaceTensionTerm",
    "NSComputeContext",
    "FlowState",
    "Predictor",
    "TwoPhaseStep",
    "RhieChowInterpolator",
    "ccd_pressure_gradient",
    "CurvatureCalculatorPsi",
    "dccd_filter_nd",
    "update_properties",
    "checkpoint",
    "CheckpointError",
    "save_checkpoint",
    "load_checkpoint",
]
