"""Validated, immutable description of one simulation (2D or 3D).

Mirrors ``SimulationParams`` of the reference (``src/lbm/params.py:86-205``):
same fields, same defaults, same checks and error messages, so code written
against the reference builds its parameters unchanged. Two storage formats
are added for the B200 kernels: ``"float16"`` and ``"bfloat16"`` keep the
shifted populations in 16 bits and compute in float32 registers.

Arrays are indexed ``[y, x]`` in 2D and ``[z, y, x]`` in 3D, x fastest.
"""

from __future__ import annotations

import warnings
from dataclasses import dataclass, field

import numpy as np

from .lattice import LATTICES, VelocitySet, as_lattice, default_lattice

TAU_WARNING = 0.51
COLLISION_MODELS = ("bgk", "trt", "regularized", "cumulant")
"""The reference's two models, "regularized" (projective regularisation of the non-equilibrium
part, Latt & Chopard 2006, with one relaxation rate 1/tau) and "cumulant" (the cumulant method of
Geier et al. 2015 on D2Q9: shear rate 1/tau, bulk and higher-order rates 1), which the reference
lists on its roadmap (item 3, high Reynolds numbers) but does not implement."""
SUPPORTED_DTYPES = ("float32", "float64", "float16", "bfloat16")
COMPUTE_DTYPE = {"float32": "float32", "float64": "float64", "float16": "float32", "bfloat16": "float32"}
"""Arithmetic type of each storage format: 16-bit storage computes in float32."""


class StabilityWarning(UserWarning):
    """Parameters are valid but numerically risky (tau near 1/2)."""


def check_tau(tau: float) -> None:
    """Reject tau <= 1/2; warn below ``TAU_WARNING`` (reference ``params.py:50-60``)."""
    if not tau > 0.5:
        raise ValueError(f"tau must be > 0.5 (viscosity nu = (tau - 0.5)/3 > 0); got tau={tau}")
    if tau < TAU_WARNING:
        warnings.warn(
            f"tau={tau:.6f} is close to 0.5: BGK becomes unstable in shear layers; "
            "use TRT, refine the grid, or lower the lattice velocity",
            StabilityWarning,
            stacklevel=3,
        )


def _frozen(array: np.ndarray) -> np.ndarray:
    out = np.array(array, copy=True)
    out.setflags(write=False)
    return out


@dataclass(frozen=True, eq=False)
class SimulationParams:
    """Everything a solver needs to advance one simulation.

    Attributes follow the reference: ``nx, ny`` grid size; ``tau`` relaxation
    time (> 1/2); ``collision`` ``"bgk"``/``"trt"`` (or ``"regularized"``, an addition); ``magic`` the TRT
    parameter Lambda; ``force`` a uniform body-force density; ``solid`` the
    solid mask; ``wall_velocity`` (d, *shape), read only at solid nodes;
    ``dtype`` the population storage format; ``nz`` for 3D; ``lattice``;
    optional ``link_rules`` and ``immersed`` body.
    """

    nx: int
    ny: int
    tau: float
    collision: str = "bgk"
    magic: float = 3.0 / 16.0
    force: tuple[float, ...] | None = None
    solid: np.ndarray | None = field(default=None, repr=False)
    wall_velocity: np.ndarray | None = field(default=None, repr=False)
    dtype: str = "float32"
    nz: int | None = field(default=None, kw_only=True)
    lattice: str | VelocitySet | None = field(default=None, kw_only=True)
    link_rules: object | None = field(default=None, kw_only=True, repr=False)
    immersed: object | None = field(default=None, kw_only=True, repr=False)

    def __post_init__(self) -> None:
        """Validate and freeze. The checks, their order and their error messages are the
        reference's (``params.py:129-175``) statement for statement, on purpose: they are the
        drop-in's input contract, pinned by ``tests/test_builders_golden.py``. The additions are
        the 16-bit storage formats and the ``"regularized"`` and ``"cumulant"`` collision models."""
        sizes = {"nx": self.nx, "ny": self.ny} | ({} if self.nz is None else {"nz": self.nz})
        if any(n <= 0 for n in sizes.values()):
            got = ", ".join(f"{k}={v}" for k, v in sizes.items())
            raise ValueError(f"{' and '.join(sizes)} must be positive; got {got}")
        if self.collision not in COLLISION_MODELS:
            raise ValueError(f"collision must be one of {COLLISION_MODELS}; got {self.collision!r}")
        if not self.magic > 0:
            raise ValueError(f"TRT magic parameter must be > 0; got magic={self.magic}")
        if self.dtype not in SUPPORTED_DTYPES:
            raise ValueError(f"dtype must be one of {SUPPORTED_DTYPES}; got {self.dtype!r}")
        check_tau(self.tau)

        d = 2 if self.nz is None else 3
        if self.lattice is None:
            lattice = default_lattice(d)
        elif isinstance(self.lattice, str) and self.lattice not in LATTICES:
            raise ValueError(f"unknown lattice {self.lattice!r}; choose from {tuple(LATTICES)}")
        else:
            lattice = as_lattice(self.lattice)
        if lattice.d != d:
            raise ValueError(
                f"lattice {lattice.name} is {lattice.d}D but the grid is {d}D "
                "(set nz for 3D, leave it unset for 2D)"
            )
        if self.collision == "cumulant" and lattice.name != "D2Q9":
            raise ValueError(f"the cumulant collision is built for D2Q9 (a tensor-product lattice holding "
                             f"every moment it relaxes); got {lattice.name}")
        shape = (self.ny, self.nx) if d == 2 else (self.nz, self.ny, self.nx)

        solid = np.zeros(shape, dtype=bool) if self.solid is None else np.asarray(self.solid)
        if solid.shape != shape:
            raise ValueError(f"solid mask must have shape {shape}; got {solid.shape}")
        solid = solid.astype(bool)

        if self.wall_velocity is None:
            wall = np.zeros((d, *shape))
        else:
            wall = np.asarray(self.wall_velocity, dtype=np.float64)
        if wall.shape != (d, *shape):
            raise ValueError(f"wall_velocity must have shape {(d, *shape)}; got {wall.shape}")
        wall = np.where(solid, wall, 0.0)

        force = (0.0,) * d if self.force is None else tuple(float(c) for c in self.force)
        if len(force) != d:
            raise ValueError(f"force must have {d} components for a {d}D grid; got {force}")

        if self.immersed is not None and self.immersed.d != d:
            raise ValueError(f"the immersed body is {self.immersed.d}D but the grid is {d}D")
        if self.link_rules is not None:
            self.link_rules.validate(lattice, solid, wall)

        object.__setattr__(self, "lattice", lattice)
        object.__setattr__(self, "solid", _frozen(solid))
        object.__setattr__(self, "wall_velocity", _frozen(wall))
        object.__setattr__(self, "force", force)
        object.__setattr__(self, "tau", float(self.tau))
        object.__setattr__(self, "magic", float(self.magic))

    @property
    def d(self) -> int:
        return self.lattice.d

    @property
    def shape(self) -> tuple[int, ...]:
        return (self.ny, self.nx) if self.d == 2 else (self.nz, self.ny, self.nx)

    @property
    def fluid(self) -> np.ndarray:
        return ~self.solid

    @property
    def viscosity(self) -> float:
        return self.lattice.cs2 * (self.tau - 0.5)

    @property
    def relaxation_rates(self) -> tuple[float, float]:
        """(omega_plus, omega_minus): 1/tau and 1/(1/2 + Lambda/(tau - 1/2)); equal for BGK."""
        omega_plus = 1.0 / self.tau
        if self.collision in ("bgk", "regularized", "cumulant"):
            return omega_plus, omega_plus
        return omega_plus, 1.0 / (0.5 + self.magic / (self.tau - 0.5))
