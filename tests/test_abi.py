"""The C ABI without a GPU: build, load, exported symbols, device lattice tables."""

from __future__ import annotations

import ctypes
import re
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

import lbm_b200 as lbm
from lbm_b200 import _native as N

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "lbm_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(lbm_[a-z0-9_]+)\s*\(", text)))


def test_library_builds_and_exports_every_declared_symbol():
    lbm.build.build()
    lib = ctypes.CDLL(str(N.LIBRARY))
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(N.EXPORTED), "the ctypes binding must cover exactly the header"


def test_abi_version_and_argument_checks_without_a_gpu():
    lib = N.load()
    assert lib.lbm_abi_version() == N.ABI_VERSION
    # invalid descriptors are rejected before any CUDA call
    bad = N.Grid(7, 0, 4, 4, 1, 4, 16)
    assert lib.lbm_step_pull(ctypes.byref(bad), None, None, None, None, None, None, None) == N.LBM_ERR_INVALID
    grid = N.Grid(N.LBM_D2Q9, N.LBM_F32, 4, 4, 1, 3, 12)  # pitch < nx
    assert lib.lbm_unpack(ctypes.byref(grid), None, 0, None, None) == N.LBM_ERR_INVALID
    assert lib.lbm_affine_reduce(0, None, None, None, None, None, 0, 0, 1, None, None, None, None) == N.LBM_ERR_INVALID


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc")
def test_device_lattice_tables_match_python(tmp_path):
    """The constexpr tables in csrc/lbm_common.cuh are host-callable: print them on the CPU."""
    src = tmp_path / "tables.cu"
    src.write_text(
        '#include "lbm_common.cuh"\n#include <cstdio>\n'
        "template <class L> void dump() { for (int i = 0; i < L::Q; ++i) "
        'printf("%d %d %d %d %.17g\\n", L::cx(i), L::cy(i), L::cz(i), L::opp(i), L::w(i)); }\n'
        "int main() { dump<lbm::D2Q9>(); dump<lbm::D3Q19>(); return 0; }\n"
    )
    exe = tmp_path / "tables"
    csrc = ROOT / "high-performance-lbm-on-gpu-_b200" / "csrc"
    subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", f"-I{csrc}", str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    rows = [line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.splitlines()]
    for vs, block in ((lbm.D2Q9, rows[:9]), (lbm.D3Q19, rows[9:])):
        c = np.array([[int(r[0]), int(r[1]), int(r[2])] for r in block])
        np.testing.assert_array_equal(c, vs.c3)
        assert [int(r[3]) for r in block] == list(vs.opposite)
        np.testing.assert_array_equal([float(r[4]) for r in block], vs.w)


def test_backend_registry_and_errors():
    params = lbm.SimulationParams(nx=8, ny=8, tau=0.8)
    with pytest.raises(ValueError, match="backend"):
        lbm.make_solver(params, backend="opencl")
    assert lbm.BACKENDS == ("cuda", "cuda-naive", "cuda-tiled", "cuda-aa")
    with pytest.raises(ValueError, match="2D only"):
        lbm.make_solver(lbm.SimulationParams(nx=8, ny=8, nz=8, tau=0.8), backend="cuda-tiled")


def test_solver_without_gpu_raises_backend_unavailable():
    import torch

    if torch.cuda.is_available():
        pytest.skip("checks the error raised on machines without a GPU")
    with pytest.raises(lbm.BackendUnavailable):
        lbm.make_solver(lbm.SimulationParams(nx=8, ny=8, tau=0.8))


def test_checked_step_partial_count_without_a_gpu():
    """lbm_health_partials is host arithmetic: the bulk grid's blocks, then the boundary warps'
    (split) or the fused grid's extra planes."""
    lib = N.load()
    grid = N.Grid(N.LBM_D3Q19, N.LBM_F32, 64, 20, 16, 64, 64 * 20 * 16)
    sp = N.Special()
    bulk = N.Launch(32, 4, N.LAUNCH_BULK)
    assert lib.lbm_health_partials(ctypes.byref(grid), ctypes.byref(sp), ctypes.byref(bulk)) == 2 * 5 * 16
    sp.n_special = 100
    sp.node = sp.rule_mask = sp.rule_first = sp.force_slot = 8  # non-null; never dereferenced here
    assert lib.lbm_health_partials(ctypes.byref(grid), ctypes.byref(sp), ctypes.byref(bulk)) == 160 + 4
    fused = N.Launch(32, 4, N.LAUNCH_FUSED)
    assert lib.lbm_health_partials(ctypes.byref(grid), ctypes.byref(sp), ctypes.byref(fused)) == 2 * 5 * 17
    bad = N.Launch(48, 4, N.LAUNCH_BULK)
    assert lib.lbm_health_partials(ctypes.byref(grid), ctypes.byref(sp), ctypes.byref(bad)) == N.LBM_ERR_INVALID


@pytest.mark.parametrize("change", ["grid", "solid", "layer", "sign", "column", "layer_x", "inlet_without_velocity",
                                    "outlet_with_velocity", "scratch"])
def test_zou_he_builder_rejects_invalid_arguments_without_a_gpu(change):
    """Every rejection returns before any CUDA call, so it runs on a machine without a GPU."""
    lib = N.load()
    grid = N.Grid(N.LBM_D3Q19, N.LBM_F64, 12, 9, 5, 12, 12 * 9 * 5)
    if change == "grid":
        grid = N.Grid(N.LBM_D3Q19, N.LBM_F64, 12, 9, 5, 11, 12 * 9 * 5)  # pitch < nx
    one = ctypes.c_void_p(16)  # stands in for a device pointer; never dereferenced on these paths
    args = {"solid": one, "column": 1, "sign": 1, "layer_x": 0, "layer": one, "velocity": one, "scratch": one}
    if change in ("solid", "layer", "scratch"):
        args[change] = None
    if change == "sign":
        args["sign"] = 0
    if change == "column":
        args["column"] = 12
    if change == "layer_x":
        args["layer_x"] = -1
    if change == "inlet_without_velocity":
        args["velocity"] = None
    if change == "outlet_with_velocity":
        args["sign"] = -1
    a = args
    common = (ctypes.byref(grid), a["solid"], a["column"], a["sign"], a["layer_x"], a["layer"], a["velocity"], 1.0)
    assert lib.lbm_zou_he_count(*common, a["scratch"], None) == N.LBM_ERR_INVALID
    assert lib.lbm_zou_he_write(*common, a["scratch"], 14, one, one, one, one, one, one, None) == N.LBM_ERR_INVALID


@pytest.mark.parametrize("storage,nx,pitch", [
    ("float32", 256, 256), ("float32", 250, 256), ("float32", 2050, 2056), ("float32", 880, 880),
    ("float32", 244, 248), ("float32", 10, 10),  # 16 columns would add more than a quarter
    ("float64", 40, 40), ("float64", 30, 32), ("float64", 250, 252), ("float64", 5, 5),
    ("float16", 200, 208), ("bfloat16", 250, 256), ("float16", 10, 16),
])
def test_default_row_pitch(storage, nx, pitch):
    """4- and 8-byte rows start on 32-byte boundaries when that adds at most a quarter to the row;
    16-bit rows are padded to 16 nodes (the pair and TMA kernels' 16-byte row strides)."""
    from lbm_b200.solver import row_pitch

    assert row_pitch(nx, storage) == pitch


@pytest.mark.parametrize("change", ["null_batch", "same_buffers", "no_domains", "no_kind", "no_nbr", "n_domains",
                                    "n_tiles", "no_tiles", "tile_x", "tile_y", "tile_size", "blocks", "no_seed_16bit",
                                    "lattice", "storage"])
def test_batch_step_rejects_invalid_arguments_without_a_gpu(change):
    """Every rejection of lbm_batch_step returns before any CUDA call (each case breaks one
    argument of an otherwise complete batch), so it runs on a machine without a GPU."""
    lib = N.load()
    one = 16  # stands in for a device pointer; never dereferenced on these paths
    fields = {"lattice": N.LBM_D2Q9, "storage": N.LBM_F32, "n_domains": 2, "domains": one, "n_tiles": 4, "tiles": one,
              "tile_x": 32, "tile_y": 4, "blocks": 8, "kind": one, "solid_nbr": one, "wall_u": None,
              "round_seed": None}
    src, dst = one, 32
    bad = {"no_domains": ("domains", None), "no_kind": ("kind", None), "no_nbr": ("solid_nbr", None),
           "n_domains": ("n_domains", 0), "n_tiles": ("n_tiles", -1), "no_tiles": ("tiles", None),
           "tile_x": ("tile_x", 48), "tile_y": ("tile_y", 0), "tile_size": ("tile_y", 9), "blocks": ("blocks", 0),
           "lattice": ("lattice", 7), "storage": ("storage", 9)}
    if change in bad:
        key, value = bad[change]
        fields[key] = value
    if change == "no_seed_16bit":
        fields["storage"] = N.LBM_F16
    if change == "same_buffers":
        dst = src
    batch = N.Batch(**fields)
    arg = None if change == "null_batch" else ctypes.byref(batch)
    assert lib.lbm_batch_step(arg, ctypes.c_void_p(src), ctypes.c_void_p(dst), None) == N.LBM_ERR_INVALID
    assert lib.lbm_batch_occupancy(N.LBM_D2Q9, N.LBM_F32, 32, 4, None) == N.LBM_ERR_INVALID
    assert lib.lbm_batch_occupancy(N.LBM_D2Q9, N.LBM_F32, 0, 4, ctypes.byref(ctypes.c_int32())) == N.LBM_ERR_INVALID


def _grid_entry_points():
    names = [n for n, a in N._SIGNATURES.items() if a and a[0] is ctypes.POINTER(N.Grid)]
    return sorted(set(names) | {"lbm_health_partials", "lbm_ball_links_scratch", "lbm_zou_he_scratch"})


@pytest.mark.parametrize("name", _grid_entry_points())
def test_every_grid_entry_point_rejects_an_invalid_grid_without_a_gpu(name):
    """Each entry point that takes a grid checks it before any CUDA call: a grid with pitch < nx
    (every other argument present, distinct stand-in pointers that are never dereferenced)
    returns LBM_ERR_INVALID, so this runs on a machine without a GPU."""
    lib = N.load()
    fn = getattr(lib, name)
    bad = N.Grid(N.LBM_D3Q19, N.LBM_F32, 12, 9, 5, 11, 12 * 9 * 5)  # pitch < nx
    args, keep = [], []
    for k, t in enumerate(fn.argtypes or [ctypes.POINTER(N.Grid)]):
        if t is ctypes.POINTER(N.Grid):
            args.append(ctypes.byref(bad))
        elif isinstance(t, type) and issubclass(t, ctypes._Pointer) and issubclass(t._type_, ctypes.Structure):
            s = t._type_()
            keep.append(s)
            args.append(ctypes.byref(s))
        elif t is ctypes.c_void_p:
            args.append(ctypes.c_void_p(4096 * (k + 1)))
        elif t in (ctypes.c_double, ctypes.c_float):
            args.append(1.0)
        else:
            args.append(1)
    assert fn(*args) == N.LBM_ERR_INVALID
