"""The node contract the LBM step plugs into.

When MADDENING itself is importable (``maddening.core.node``; it needs JAX),
its ``SimulationNode`` / ``BoundaryInputSpec`` / ``NodeMeta`` are used, so the
node registers with ``GraphManager`` unchanged.  Otherwise this module
provides minimal stand-ins with the same names and semantics
(``src/maddening/core/node.py:23-45, 70-480``;
``src/maddening/core/compliance/metadata.py``), enough for the node to be used
and tested on its own.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from dataclasses import dataclass, field
from enum import Enum
from typing import Any, ClassVar, Optional

try:  # the real contract, when MADDENING (and JAX) are installed
    from maddening.core.node import BoundaryInputSpec, SimulationNode  # type: ignore
    from maddening.core.compliance.metadata import (  # type: ignore
        NodeMeta, StabilityLevel, ValidatedRegime)
    HAVE_MADDENING = True
except Exception:  # noqa: BLE001 -- any import failure means "not available"
    HAVE_MADDENING = False

    class StabilityLevel(Enum):
        EXPERIMENTAL = "experimental"
        STABLE = "stable"

    @dataclass(frozen=True)
    class ValidatedRegime:
        parameter: str
        min_value: float
        max_value: float
        notes: str = ""

    @dataclass(frozen=True)
    class NodeMeta:
        algorithm_id: str = ""
        algorithm_version: str = ""
        stability: StabilityLevel = StabilityLevel.EXPERIMENTAL
        description: str = ""
        governing_equations: str = ""
        discretization: str = ""
        assumptions: tuple = ()
        limitations: tuple = ()
        validated_regimes: tuple = ()
        hazard_hints: tuple = ()
        extra: dict = field(default_factory=dict)

    @dataclass(frozen=True)
    class BoundaryInputSpec:
        """Expected boundary input (mirror of core/node.py:23-45)."""
        shape: tuple = ()
        dtype: Any = None
        default: Any = None
        coupling_type: str = "replacive"
        description: str = ""
        expected_units: Optional[str] = None

    class MigrationError(TypeError):
        pass

    class SimulationNode(ABC):
        """Minimal mirror of the reference ABC (core/node.py:70-480)."""

        meta: ClassVar[Optional[NodeMeta]] = None

        def __init_subclass__(cls, **kwargs):
            super().__init_subclass__(**kwargs)
            if "requires_halo" in cls.__dict__ and "halo_width" not in cls.__dict__:
                raise MigrationError(
                    "SimulationNode.requires_halo was removed; override "
                    "halo_width() -> dict[int, int] instead")

        def __init__(self, name: str, timestep: float, **params):
            self.name = name
            self.delta_t = float(timestep)
            self.geometry_source = params.pop("geometry_source", None)
            self.params = dict(params)

        @abstractmethod
        def initial_state(self) -> dict: ...

        @abstractmethod
        def update(self, state: dict, boundary_inputs: dict, dt: float) -> dict: ...

        def state_fields(self) -> list:
            return list(self.initial_state().keys())

        def halo_width(self) -> dict:
            return {}

        def update_padded(self, state_padded, boundary_inputs, dt, *,
                          static_padded=None, shard_info=None):
            if self.halo_width():
                raise NotImplementedError(
                    f"{type(self).__name__} declares halo_width={self.halo_width()} "
                    "but does not override `update_padded`. Required for sharded "
                    "stencil execution.")
            return self.update(state_padded, boundary_inputs, dt)

        def boundary_input_spec(self) -> dict:
            return {}

        def compute_boundary_fluxes(self, state, boundary_inputs, dt) -> dict:
            return {}

        def derivatives(self, state, boundary_inputs):
            raise NotImplementedError(
                f"{type(self).__name__} does not implement derivatives().")

        def to_dict(self) -> dict:
            return {"type": type(self).__name__, "name": self.name,
                    "timestep": self.delta_t, "params": self.params}

__all__ = ["BoundaryInputSpec", "SimulationNode", "NodeMeta", "StabilityLevel",
           "ValidatedRegime", "HAVE_MADDENING"]
