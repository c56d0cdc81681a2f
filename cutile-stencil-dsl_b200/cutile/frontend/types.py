"""Boundary condition types of the user API (reference: cutile/frontend/types.py:10-65)."""

from __future__ import annotations

from dataclasses import dataclass
from enum import Enum
from typing import Union


class BoundaryType(Enum):
    DIRICHLET = "dirichlet"
    NEUMANN = "neumann"
    PERIODIC = "periodic"
    REFLECTING = "reflecting"


@dataclass(frozen=True)
class BoundaryCondition:
    """A single boundary condition (type + optional value)."""

    bc_type: BoundaryType
    value: float = 0.0


@dataclass
class BoundarySpec:
    """Boundary specification per dimension: ``(low, high)`` condition pairs.

    A single-entry list means "the same condition on every side of every
    dimension" (the reference's ``uniform`` sentinel, types.py:37-53).
    """

    conditions: list[tuple[BoundaryCondition, BoundaryCondition]]

    @classmethod
    def uniform(cls, bc_type: Union[str, BoundaryType], value: float = 0.0) -> "BoundarySpec":
        if isinstance(bc_type, str):
            bc_type = BoundaryType(bc_type)
        bc = BoundaryCondition(bc_type=bc_type, value=value)
        return cls(conditions=[(bc, bc)])

    @classmethod
    def periodic(cls) -> "BoundarySpec":
        return cls.uniform(BoundaryType.PERIODIC)

    @classmethod
    def dirichlet(cls, value: float = 0.0) -> "BoundarySpec":
        return cls.uniform(BoundaryType.DIRICHLET, value)

    @classmethod
    def neumann(cls) -> "BoundarySpec":
        return cls.uniform(BoundaryType.NEUMANN)

    @classmethod
    def reflecting(cls) -> "BoundarySpec":
        return cls.uniform(BoundaryType.REFLECTING)

    def is_uniform(self) -> bool:
        if len(self.conditions) == 0:
            return False
        first = self.conditions[0][0]
        return all(lo == first and hi == first for lo, hi in self.conditions)

    def to_dict(self) -> dict:
        """``{"type": ..., "value": ...}`` for a uniform spec (what ``@stencil``
        records); raises for mixed specs, which the kernels do not take."""
        if not self.is_uniform():
            raise ValueError("only uniform boundary specs can be attached to a stencil")
        bc = self.conditions[0][0]
        d = {"type": bc.bc_type.value}
        if bc.bc_type is BoundaryType.DIRICHLET:
            d["value"] = float(bc.value)
        return d
