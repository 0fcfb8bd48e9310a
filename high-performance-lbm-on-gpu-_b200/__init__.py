"""B200-native lattice Boltzmann time step: a drop-in ``cuda`` backend.

Mirrors the public API of the reference ``lbm`` package
(``src/lbm/__init__.py``, ``src/lbm/backends/__init__.py:23-83``)::

    import lbm_b200 as lbm
    params = lbm.SimulationParams(nx=256, ny=256, nz=256, tau=0.9, collision="trt")
    solver = lbm.make_solver(params, backend="cuda")        # or "cuda-aa"
    solver.run(1000)
    fields = solver.macroscopic()

Populations live in PyTorch CUDA tensors; every step runs hand-written
sm_100a kernels from ``liblbm_b200.so`` through a C ABI (``include/lbm_b200.h``).
There is no CPU path: without the library or a GPU the solver raises
``BackendUnavailable``.

The directory name is not a Python identifier, so the package registers itself
as ``lbm_b200`` on import (``lbm_b200.py`` at the repository root imports it).
"""

from __future__ import annotations

import sys as _sys

from . import build, device_rules, diagnostics, forces, geometry, ibm, lattice, link_rules, open_boundaries, params
from .diagnostics import MacroscopicFields
from .forces import ForceProbe
from .geometry import Ball, WallLinks, cavity_walls, channel_walls, circle, duct_walls, sphere, voxelize, wall_links
from .ibm import ImmersedBoundary, roma
from .lattice import D2Q9, D3Q19, LATTICES, VelocitySet, default_lattice
from .link_rules import LAYOUTS, AffineSet, CompiledAffine, LinkRules, bouzidi_rules, compile_affine
from .open_boundaries import open_channel, zou_he_inlet_derivative
from .params import SimulationParams, StabilityWarning
from .solver import (
    BACKENDS,
    BackendUnavailable,
    CudaSolver,
    SimulationDiverged,
    Solver,
    available_backends,
    gpu_available,
    make_solver,
)

__version__ = "0.1.0"

_ALIAS = "lbm_b200"
if __name__ != _ALIAS:
    _sys.modules.setdefault(_ALIAS, _sys.modules[__name__])
    for _name, _mod in list(_sys.modules.items()):
        if _name.startswith(__name__ + "."):
            _sys.modules.setdefault(_ALIAS + _name[len(__name__):], _mod)

__all__ = [
    "BACKENDS", "Ball", "BackendUnavailable", "CudaSolver", "D2Q9", "D3Q19", "ForceProbe",
    "ImmersedBoundary", "LATTICES", "LAYOUTS", "AffineSet", "CompiledAffine", "LinkRules",
    "MacroscopicFields", "SimulationDiverged", "SimulationParams", "Solver", "StabilityWarning",
    "VelocitySet", "WallLinks", "available_backends", "bouzidi_rules", "cavity_walls",
    "channel_walls", "circle", "compile_affine", "default_lattice", "duct_walls", "gpu_available",
    "make_solver", "open_channel", "roma", "sphere", "voxelize", "wall_links", "zou_he_inlet_derivative",
]
