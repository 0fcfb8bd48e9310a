"""The unmodified reference package (``lbm``) in ``baseline/_ref/`` -- TEST AND BASELINE INFRASTRUCTURE.

The reference is pure Python + NumPy (its CUDA backends need CuPy, which is
not installed). ``pip install --target baseline/_ref`` of the reference fails
here because its build backend (hatchling) is not in the offline wheelhouse,
so ``install`` places what that wheel would contain -- the ``src/lbm``
package directory (``pyproject.toml``: ``packages = ["src/lbm"]``), unmodified
-- into ``baseline/_ref/lbm``. ``baseline/_ref/`` is git-ignored (nothing of
the reference enters this repository's history) but travels with the
working tree to a GPU host, where the build container's reference checkout
does not exist.

Users: ``bench.py --impl reference`` and the bench's ``cpu_baseline`` time the
reference's own ``ReferenceSolver(params, xp=numpy)`` through this module;
``tests/test_gpu_reference_objects.py`` builds cases with the reference's own
``SimulationParams``, rule builders, immersed boundaries and force probes and
runs them on this package's CUDA solver. The product package never imports it.
"""

from __future__ import annotations

import os
import shutil
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
TARGET = ROOT / "baseline" / "_ref"
SOURCE = Path(os.environ.get("LBM_REFERENCE_SRC", "/root/reference/src")) / "lbm"


def install(verbose: bool = False) -> bool:
    """Copy the reference package into ``baseline/_ref/lbm``; False when the reference tree is absent."""
    if not (SOURCE / "__init__.py").is_file():
        return False
    dest = TARGET / "lbm"
    if dest.exists():
        shutil.rmtree(dest)
    TARGET.mkdir(parents=True, exist_ok=True)
    shutil.copytree(SOURCE, dest, ignore=shutil.ignore_patterns("__pycache__", "*.pyc"))
    if verbose:
        print(f"installed the reference package into {dest}")
    return True


def available() -> bool:
    return (TARGET / "lbm" / "__init__.py").is_file()


def load():
    """The reference ``lbm`` package from ``baseline/_ref`` (None when it is not installed).

    The package is imported under its own name, ``lbm``; an ``lbm`` already
    imported from elsewhere (the build container's checkout) is the same code
    and is returned as it is.
    """
    if not available():
        return None
    path = str(TARGET)
    if path not in sys.path:
        sys.path.append(path)
    import lbm  # noqa: PLC0415

    return lbm


def modules():
    """The reference modules the test cases and the bench use, as a namespace (None if absent)."""
    import types

    lbm = load()
    if lbm is None:
        return None
    import lbm.backends as backends  # noqa: PLC0415
    import lbm.forces as forces  # noqa: PLC0415
    import lbm.geometry as geometry  # noqa: PLC0415
    import lbm.ibm as ibm  # noqa: PLC0415
    import lbm.lattice as lattice  # noqa: PLC0415
    import lbm.link_rules as link_rules  # noqa: PLC0415
    import lbm.open_boundaries as open_boundaries  # noqa: PLC0415
    import lbm.params as params  # noqa: PLC0415
    import lbm.solver as solver  # noqa: PLC0415

    return types.SimpleNamespace(
        lbm=lbm, backends=backends, forces=forces, geometry=geometry, ibm=ibm, lattice=lattice,
        link_rules=link_rules, open_boundaries=open_boundaries, params=params, solver=solver,
    )
