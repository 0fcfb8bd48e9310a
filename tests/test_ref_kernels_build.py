"""The reference's CUDA kernels compiled into oracle/_ref/ load and export their launchers (CPU).

No kernel runs here (no GPU); ``tests/test_gpu_reference_kernels.py`` runs them.
"""

from __future__ import annotations

import ctypes

import pytest

from oracle import ref_kernels


@pytest.mark.skipif(not ref_kernels.available(), reason="oracle/_ref holds no compiled reference kernels")
@pytest.mark.parametrize("lattice", ref_kernels.LATTICES)
@pytest.mark.parametrize("dtype", sorted(ref_kernels.DTYPES))
def test_reference_kernel_library_exports_its_launchers(lattice, dtype):
    try:
        lib = ctypes.CDLL(str(ref_kernels.library_path(lattice, dtype)))
    except OSError as e:  # the CUDA runtime may be absent without a driver
        pytest.skip(f"cannot load without the CUDA driver: {e}")
    for name in ("ref_step_naive", "ref_step_aa") + (("ref_step_tiled",) if lattice == "D2Q9" else ()):
        assert hasattr(lib, name)
