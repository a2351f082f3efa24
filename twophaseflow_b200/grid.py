"""Minimal grid and boundary descriptors with the attributes the hot path reads.

The reference's own ``twophase.core.grid.Grid`` (src/twophase/core/grid.py:36-120)
and ``BoundarySpec`` (src/twophase/core/boundary.py:143-204) can be passed
wherever these are accepted: only ``ndim``, ``N``, ``L``, ``shape``,
``uniform``, ``coords``, ``h`` (checkpoints) and, for non-uniform grids, ``J`` / ``dJ_dxi`` are read.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


class UniformGrid:
    """Node-centred uniform grid: coords = linspace(0, L, N+1) per axis."""

    def __init__(self, N, L=None):
        self.N = tuple(int(n) for n in N)
        self.ndim = len(self.N)
        self.L = tuple(float(v) for v in (L if L is not None else (1.0,) * self.ndim))
        self.shape = tuple(n + 1 for n in self.N)
        self.coords = [np.linspace(0.0, l, n + 1) for n, l in zip(self.N, self.L)]
        self.uniform = True
        self.J = [np.full(n + 1, n / l) for n, l in zip(self.N, self.L)]
        # per-node spacing, the reference grid's ``h`` (core/grid.py:60-68)
        self.h = [np.full(n + 1, l / n) for n, l in zip(self.N, self.L)]
        self.dJ_dxi = [np.zeros(n + 1) for n in self.N]


def boundary_axes(bc_type, ndim: int) -> tuple:
    """Per-axis 'wall'/'periodic' labels (semantics of tp/core/boundary.py:40-62)."""
    if isinstance(bc_type, (tuple, list)):
        axes = tuple(str(v).strip().lower() for v in bc_type)
        if len(axes) != ndim:
            raise ValueError(f"len(boundary axes)={len(axes)} != ndim={ndim}")
        if any(a not in ("wall", "periodic") for a in axes):
            raise ValueError(f"boundary axes must be wall|periodic, got {axes!r}")
        return axes
    value = str(getattr(bc_type, "value", bc_type)).strip().lower()
    if value == "wall":
        return ("wall",) * ndim
    if value == "periodic":
        return ("periodic",) * ndim
    if value in ("periodic_wall", "x_periodic_y_wall") and ndim == 2:
        return ("periodic", "wall")
    if value in ("wall_periodic", "x_wall_y_periodic") and ndim == 2:
        return ("wall", "periodic")
    raise ValueError(f"unsupported boundary type {bc_type!r} for ndim={ndim}")


@dataclass(frozen=True)
class BoundarySpec:
    """pin_dof of the wall case: ravel index of (N//2, ...) (boundary.py:182-191)."""

    bc_type: str
    shape: tuple
    N: tuple

    @property
    def pin_dof(self) -> int:
        if all(a == "periodic" for a in boundary_axes(self.bc_type, len(self.N))):
            return 0
        return int(np.ravel_multi_index(tuple(n // 2 for n in self.N), tuple(self.shape)))
