"""Host snapshot of the macroscopic fields (reference ``src/lbm/diagnostics.py:25-70``).

The CUDA solver computes rho = 1 + sum f~* and rho u = sum c f* - F/2 on the
device (``macro_kernel`` in ``csrc/aux.cu``) and copies the result into this container.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True, eq=False)
class MacroscopicFields:
    rho: np.ndarray
    u: tuple[np.ndarray, ...]
    solid: np.ndarray

    def __post_init__(self) -> None:
        object.__setattr__(self, "u", tuple(self.u))
        for array in (self.rho, self.solid, *self.u):
            array.setflags(write=False)

    @property
    def d(self) -> int:
        return len(self.u)

    @property
    def ux(self) -> np.ndarray:
        return self.u[0]

    @property
    def uy(self) -> np.ndarray:
        return self.u[1]

    @property
    def uz(self) -> np.ndarray:
        if self.d < 3:
            raise AttributeError("2D fields have no uz component")
        return self.u[2]

    @property
    def speed(self) -> np.ndarray:
        return np.sqrt(sum(c * c for c in self.u))

    @property
    def total_mass(self) -> float:
        return float(self.rho[~self.solid].sum(dtype=np.float64))
