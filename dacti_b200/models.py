"""Model tables shared by the host code: state sizes, index layout and boundary-condition types.

Follows the compile-time constants of DACTI's model policies:
- ``euler<D>``: model/euler.hpp:26-34 (E = D+2, iu = 1, ip = E-1, gamma = 1.4 constexpr);
- ``navier_stokes<D>``: model/navier_stokes.hpp:19-31 (adds NumGrad = D+1, cp = 1005, R = 287);
- ``multi<D>``: model/multi.hpp:27-62 (E = D+4, NumFlux = E+D+1, NumParm = D+4, NumGrad = D+3).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass


class ModelId(enum.IntEnum):
    EULER = 0
    NAVIER_STOKES = 1
    MULTI = 2


class BcType(enum.IntEnum):
    """Boundary::Type order of integrator/boundary.hpp:23-32."""

    ZERO_GRADIENT = 0
    FREESLIP = 1
    NOSLIP = 2
    INFLOW = 3
    INFLOW_R = 4
    OUTFLOW = 5
    DIRICHLET = 6
    NEUMANN = 7


@dataclass(frozen=True)
class ModelShape:
    model: ModelId
    dims: int

    @property
    def E(self) -> int:  # NumEqns
        return self.dims + (4 if self.model == ModelId.MULTI else 2)

    @property
    def F(self) -> int:  # NumFlux
        return self.E + (self.dims + 1 if self.model == ModelId.MULTI else 0)

    @property
    def G(self) -> int:  # NumGrad
        if self.model == ModelId.MULTI:
            return self.dims + 3
        if self.model == ModelId.NAVIER_STOKES:
            return self.dims + 1
        return 0

    @property
    def P(self) -> int:  # NumParm
        return self.dims + 4 if self.model == ModelId.MULTI else 0

    @property
    def C(self) -> int:  # children per node
        return 1 << self.dims

    @property
    def NF(self) -> int:  # faces per cell
        return 2 * self.dims

    @property
    def iu(self) -> int:
        return 2 if self.model == ModelId.MULTI else 1

    @property
    def ip(self) -> int:
        return self.E - 2 if self.model == ModelId.MULTI else self.E - 1

    @property
    def ia(self) -> int:
        if self.model != ModelId.MULTI:
            raise ValueError("only the multiphase model carries a volume fraction")
        return self.E - 1

    @property
    def name(self) -> str:
        return {ModelId.EULER: "euler", ModelId.NAVIER_STOKES: "navier_stokes", ModelId.MULTI: "multi"}[
            self.model
        ] + f"<{self.dims}>"


# Node flag bits of the flat tree (mirror the bool members of integrator/node.hpp:60-66).
F_LEAF = 1 << 0
F_ACTIVE = 1 << 1
F_GARBAGE = 1 << 2
F_CAN_SPLIT = 1 << 3
F_CAN_UNSPLIT = 1 << 4
F_SHOULD_SPLIT = 1 << 5
F_IS_BOUNDARY = 1 << 6
