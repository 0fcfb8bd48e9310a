"""The reference's own CUDA kernels, compiled for sm_100a -- TEST INFRASTRUCTURE ONLY.

Recipe (``build``): each kernel module is assembled the way the reference's
``build_kernel_source`` assembles it (``src/lbm/backends/cuda_solver.py:65-87``):
the lattice preamble that ``lbm.lattice.cuda_preamble`` generates
(``src/lbm/lattice.py:174-214``), ``TILE_X``/``TILE_Y``, ``kernels/common.cuh``,
then the variant's source. Here the kernel files are ``#include``d where they
lie in the reference tree, so none of them is copied into this repository; a C
launcher of this module's own is appended. Everything it writes goes to
``oracle/_ref/`` (git-ignored): the generated preamble, the wrapper ``.cu`` and
``libref_<lattice>_<dtype>.so``. It needs the reference tree, which only the
build container has; a GPU host uses the prebuilt libraries.

Users: ``tests/test_gpu_reference_kernels.py`` checks this repository's CUDA
path against these kernels on the same inputs, and ``python -m
oracle.ref_kernels`` times both on one GPU (the same-box baseline). The
product package never loads them.

The launchers mirror ``CudaSolver._advance`` (``cuda_solver.py:267-284``):
grid (ceil(nx/bx), ceil(ny/by), nz), block (bx, by), default block (32, 8);
``stream_collide_naive`` (and, 2D only, ``stream_collide_tiled``, whose block
is its tile) between two buffers; ``aa_odd`` then ``aa_even`` on one buffer
that starts in the post-even layout (slot opp(i) holds f_i); before every
launch the link-rule pre-pass of that launch's layout (``rules_evaluate``,
``rules_write`` from ``kernels/link_rules.cu``), as ``_pre_pass`` runs it.
"""

from __future__ import annotations

import ctypes
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
DEFAULT_REFERENCE_SRC = "/root/reference/src"
REFERENCE_SRC = Path(os.environ.get("LBM_REFERENCE_SRC", DEFAULT_REFERENCE_SRC))
"""The reference's ``src`` directory (the ``LBM_REFERENCE_SRC`` environment variable, else the
build container's read-only checkout)."""
KERNELS = REFERENCE_SRC / "lbm" / "backends" / "kernels"
LATTICES = ("D2Q9", "D3Q19")
DTYPES = {"float32": "float", "float64": "double"}
DEFAULT_BLOCK = (32, 8)

_LAUNCHERS = r"""
#include <cuda_runtime.h>

extern "C" int ref_step_naive(const void* f_src, void* f_dst, const unsigned char* solid, const void* wall_u,
                              const void* force_field, int nx, int ny, int nz, double omega_plus,
                              double omega_minus, double fx, double fy, double fz, int bx, int by, void* stream)
{
    const dim3 grid((nx + bx - 1) / bx, (ny + by - 1) / by, nz), block(bx, by, 1);
    stream_collide_naive<<<grid, block, 0, (cudaStream_t)stream>>>(
        (const real_t*)f_src, (real_t*)f_dst, solid, (const real_t*)wall_u, (const real_t*)force_field, nx, ny, nz,
        (real_t)omega_plus, (real_t)omega_minus, (real_t)fx, (real_t)fy, (real_t)fz);
    return (int)cudaGetLastError();
}

extern "C" int ref_step_aa(void* f, int odd, const unsigned char* solid, const void* wall_u, const void* force_field,
                           int nx, int ny, int nz, double omega_plus, double omega_minus, double fx, double fy,
                           double fz, int bx, int by, void* stream)
{
    const dim3 grid((nx + bx - 1) / bx, (ny + by - 1) / by, nz), block(bx, by, 1);
    if (odd)
        aa_odd<<<grid, block, 0, (cudaStream_t)stream>>>((real_t*)f, solid, (const real_t*)wall_u,
                                                         (const real_t*)force_field, nx, ny, nz, (real_t)omega_plus,
                                                         (real_t)omega_minus, (real_t)fx, (real_t)fy, (real_t)fz);
    else
        aa_even<<<grid, block, 0, (cudaStream_t)stream>>>((real_t*)f, solid, (const real_t*)force_field, nx, ny, nz,
                                                          (real_t)omega_plus, (real_t)omega_minus, (real_t)fx,
                                                          (real_t)fy, (real_t)fz);
    return (int)cudaGetLastError();
}
"""

# the link-rule pre-pass (kernels/link_rules.cu needs only real_t), launched as
# _RulePass launches it: RULES_BLOCK threads per block (cuda_solver.py:98-176)
_RULE_LAUNCHERS = r"""
extern "C" int ref_rules_evaluate(const void* f, const long long* slot, const void* coeff, const void* constant,
                                  void* out, int n_rules, int n_terms, void* stream)
{
    if (n_rules <= 0) return 0;
    rules_evaluate<<<(n_rules + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        (const real_t*)f, slot, (const real_t*)coeff, (const real_t*)constant, (real_t*)out, n_rules, n_terms);
    return (int)cudaGetLastError();
}

extern "C" int ref_rules_write(void* f, const long long* target, const void* value, int n_rules, void* stream)
{
    if (n_rules <= 0) return 0;
    rules_write<<<(n_rules + 127) / 128, 128, 0, (cudaStream_t)stream>>>((real_t*)f, target, (const real_t*)value,
                                                                        n_rules);
    return (int)cudaGetLastError();
}
"""

# 2D only: the tiled kernel's block must be its tile (TILE_X x TILE_Y)
_TILED_LAUNCHER = r"""
extern "C" int ref_step_tiled(const void* f_src, void* f_dst, const unsigned char* solid, const void* wall_u,
                              const void* force_field, int nx, int ny, int nz, double omega_plus,
                              double omega_minus, double fx, double fy, double fz, int bx, int by, void* stream)
{
    if (bx != TILE_X || by != TILE_Y || nz != 1) return (int)cudaErrorInvalidValue;
    const dim3 grid((nx + bx - 1) / bx, (ny + by - 1) / by, 1), block(bx, by, 1);
    stream_collide_tiled<<<grid, block, 0, (cudaStream_t)stream>>>(
        (const real_t*)f_src, (real_t*)f_dst, solid, (const real_t*)wall_u, (const real_t*)force_field, nx, ny, nz,
        (real_t)omega_plus, (real_t)omega_minus, (real_t)fx, (real_t)fy, (real_t)fz);
    return (int)cudaGetLastError();
}
"""


def library_path(lattice: str, dtype: str) -> Path:
    return OUT / f"libref_{lattice}_{dtype}.so"


def available() -> bool:
    return all(library_path(lat, dt).exists() for lat in LATTICES for dt in DTYPES)


def build(verbose: bool = False) -> bool:
    """Compile the reference kernels into oracle/_ref/; False when the reference tree is absent."""
    if not KERNELS.is_dir():
        return False
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    sys.path.insert(0, str(REFERENCE_SRC))
    try:
        from lbm.lattice import LATTICES as REF_LATTICES
        from lbm.lattice import cuda_preamble
    finally:
        sys.path.remove(str(REFERENCE_SRC))
    OUT.mkdir(exist_ok=True)
    for lat in LATTICES:
        for dtype, ctype in DTYPES.items():
            stem = f"{lat}_{dtype}"
            preamble = OUT / f"preamble_{stem}.h"
            preamble.write_text(cuda_preamble(REF_LATTICES[lat], ctype))
            wrapper = OUT / f"ref_{stem}.cu"
            wrapper.write_text("\n".join([
                "// Generated by oracle/ref_kernels.py: the reference's kernels, included unmodified, plus a launcher.",
                f'#include "{preamble.name}"',
                f"#define TILE_X {DEFAULT_BLOCK[0]}",
                f"#define TILE_Y {DEFAULT_BLOCK[1]}",
                f'#include "{KERNELS / "common.cuh"}"',
                f'#include "{KERNELS / "stream_collide_naive.cu"}"',
                f'#include "{KERNELS / "stream_collide_aa.cu"}"',
                f'#include "{KERNELS / "stream_collide_tiled.cu"}"' if lat == "D2Q9" else "",
                f'#include "{KERNELS / "link_rules.cu"}"',
                _LAUNCHERS,
                _RULE_LAUNCHERS,
                _TILED_LAUNCHER if lat == "D2Q9" else "",
            ]))
            target = library_path(lat, dtype)
            cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-shared",
                   "-Xcompiler", "-fPIC", "-o", str(target), str(wrapper), "-lcudart"]
            proc = subprocess.run(cmd, capture_output=True, text=True, cwd=OUT)
            if proc.returncode != 0:
                raise RuntimeError(f"nvcc failed for {wrapper.name}:\n{proc.stderr}")
            if verbose:
                print(f"built {target}")
    return True


class RefKernels:
    """ctypes handle on one compiled module (lattice, dtype)."""

    def __init__(self, lattice: str, dtype: str):
        path = library_path(lattice, dtype)
        if not path.exists():
            raise FileNotFoundError(f"{path} is missing: run oracle.ref_kernels.build() where the reference tree is")
        lib = ctypes.CDLL(str(path))
        c = ctypes
        common = [c.c_void_p, c.c_void_p, c.c_void_p, c.c_int, c.c_int, c.c_int, c.c_double, c.c_double,
                  c.c_double, c.c_double, c.c_double, c.c_int, c.c_int, c.c_void_p]
        lib.ref_step_naive.argtypes = [c.c_void_p, c.c_void_p] + common
        lib.ref_step_naive.restype = c.c_int
        lib.ref_step_aa.argtypes = [c.c_void_p, c.c_int] + common
        lib.ref_step_aa.restype = c.c_int
        if lattice == "D2Q9":
            lib.ref_step_tiled.argtypes = [c.c_void_p, c.c_void_p] + common
            lib.ref_step_tiled.restype = c.c_int
        lib.ref_rules_evaluate.argtypes = [c.c_void_p] * 5 + [c.c_int, c.c_int, c.c_void_p]
        lib.ref_rules_evaluate.restype = c.c_int
        lib.ref_rules_write.argtypes = [c.c_void_p] * 3 + [c.c_int, c.c_void_p]
        lib.ref_rules_write.restype = c.c_int
        self.lib = lib


class RulePass:
    """The reference's link-rule pre-pass for one layout (``_RulePass``, ``cuda_solver.py:114-176``):
    rules compiled to flat slots of the layout, grouped by their number of non-zero terms, each
    group trimmed to that length and stored term-major, evaluated group by group into one buffer,
    then written back by one launch. Slots come from this package's ``compile_rules``, which
    follows the reference's ``compile_rules`` (``link_rules.py:203-250``)."""

    def __init__(self, params, layout: str, kernels: RefKernels, torch, device, t_real):
        import numpy as np

        from lbm_b200.link_rules import compile_rules

        compiled = compile_rules(params.lattice, params.link_rules, layout, params.solid, params.wall_velocity)
        values = compiled.values
        lengths = np.count_nonzero(values.coeff, axis=1)
        order = np.argsort(lengths, kind="stable")
        self.groups = []
        start = 0
        for length in np.unique(lengths):
            rows = order[lengths[order] == length]
            nonzero_first = np.argsort(values.coeff[rows] == 0, axis=1, kind="stable")
            take = nonzero_first[:, : max(int(length), 1)]
            slots = np.take_along_axis(values.slots[rows], take, axis=1)
            coeff = np.take_along_axis(values.coeff[rows], take, axis=1)
            self.groups.append((
                start, len(rows),
                torch.from_numpy(np.ascontiguousarray(slots.T).astype(np.int64)).to(device),
                torch.from_numpy(np.ascontiguousarray(coeff.T)).to(device, t_real),
                torch.from_numpy(np.array(values.constant[rows])).to(device, t_real),
            ))
            start += len(rows)
        self.target = torch.from_numpy(np.array(compiled.target[order], dtype=np.int64)).to(device)
        self.buffer = torch.empty(len(order), dtype=t_real, device=device)
        self.n = len(order)
        self.lib = kernels.lib
        self.itemsize = self.buffer.element_size()

    def __call__(self, f, stream) -> None:
        base = self.buffer.data_ptr()
        for start, count, slots, coeff, constant in self.groups:
            err = self.lib.ref_rules_evaluate(f.data_ptr(), slots.data_ptr(), coeff.data_ptr(), constant.data_ptr(),
                                              base + start * self.itemsize, count, slots.shape[0], stream)
            if err:
                raise RuntimeError(f"reference rule evaluation failed ({err})")
        if self.lib.ref_rules_write(f.data_ptr(), self.target.data_ptr(), base, self.n, stream):
            raise RuntimeError("reference rule write-back failed")


class RefSolver:
    """The reference's CudaSolver state handling on torch tensors (``cuda_solver.py:188-305``):
    populations in the reference's layout (natural order, unpadded), a uint8 kind mask (0 fluid,
    1 solid), the full wall-velocity array, a one-element placeholder force field."""

    def __init__(self, params, variant: str = "naive", block=DEFAULT_BLOCK, device="cuda"):
        import numpy as np
        import torch

        if variant not in ("naive", "tiled", "aa") or (variant == "tiled" and params.d != 2):
            raise ValueError(f"variant {variant!r} is not available for a {params.d}D grid")
        if variant == "tiled" and tuple(block) != DEFAULT_BLOCK:
            raise ValueError(f"the tiled kernel is compiled for blocks of {DEFAULT_BLOCK}")

        self.torch = torch
        self.params = params
        self.variant = variant
        self.block = tuple(int(b) for b in block)
        self.kernels = RefKernels(params.lattice.name, params.dtype)
        t_real = torch.float32 if params.dtype == "float32" else torch.float64
        self.t_real = t_real
        self.device = device
        self.opp = list(params.lattice.opposite)
        self.solid = torch.from_numpy(np.asarray(params.solid, dtype=np.uint8).copy()).to(device)
        self.wall = torch.from_numpy(np.array(params.wall_velocity, dtype=np.float64)).to(device, t_real).contiguous()
        self.field = torch.zeros(1, dtype=t_real, device=device)
        self.rule_passes = {}
        if getattr(params, "link_rules", None) is not None and len(params.link_rules):
            layouts = ("aa_odd", "aa_even") if variant == "aa" else ("pull",)
            self.rule_passes = {lay: RulePass(params, lay, self.kernels, torch, device, t_real) for lay in layouts}
        if getattr(params, "immersed", None) is not None:
            raise ValueError("the reference drives immersed bodies with CuPy array code, not with these kernels")
        self.scalars = (params.nx, params.ny, params.nz or 1, *params.relaxation_rates,
                        *(tuple(float(v) for v in params.force) + (0.0,) * (3 - params.d))[:3])
        self.f = self.f_next = None
        self.time_step = 0

    def set_populations(self, f) -> None:
        """f: (Q, *shape) shifted populations in natural direction order."""
        torch = self.torch
        f = torch.as_tensor(f).to(self.device, self.t_real)
        if self.variant == "aa":
            self.f = f[self.opp].contiguous()  # post-even layout
        else:
            self.f = f.contiguous()
            self.f_next = self.f.clone()
        self.time_step = 0

    def advance(self, steps: int) -> None:
        stream = self.torch.cuda.current_stream().cuda_stream
        bx, by = self.block
        lib = self.kernels.lib
        p = self.f.data_ptr
        if self.variant == "aa":
            if steps % 2:
                raise ValueError("the AA kernels advance in pairs of steps")
            for _ in range(steps // 2):
                for odd in (1, 0):
                    if self.rule_passes:
                        self.rule_passes["aa_odd" if odd else "aa_even"](self.f, stream)
                    err = lib.ref_step_aa(p(), odd, self.solid.data_ptr(), self.wall.data_ptr(),
                                          self.field.data_ptr(), *self.scalars, bx, by, stream)
                    if err:
                        raise RuntimeError(f"reference AA kernel launch failed ({err})")
        else:
            step = lib.ref_step_tiled if self.variant == "tiled" else lib.ref_step_naive
            for _ in range(steps):
                if self.rule_passes:
                    self.rule_passes["pull"](self.f, stream)
                err = step(self.f.data_ptr(), self.f_next.data_ptr(), self.solid.data_ptr(),
                           self.wall.data_ptr(), self.field.data_ptr(), *self.scalars, bx, by, stream)
                if err:
                    raise RuntimeError(f"reference kernel launch failed ({err})")
                self.f, self.f_next = self.f_next, self.f
        self.time_step += steps

    def populations(self):
        f = self.f[self.opp] if self.variant == "aa" else self.f
        return f.cpu().numpy()


def time_reference(params, variant: str, steps: int) -> float:
    """MLUPS of the reference's kernels alone on `params` (from the rest state), CUDA events;
    the same number of steps runs untimed first."""
    import numpy as np
    import torch

    ref = RefSolver(params, variant)
    ref.set_populations(torch.zeros((params.lattice.q, *params.shape), dtype=ref.t_real))
    ref.advance(steps)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    ref.advance(steps)
    b.record()
    b.synchronize()
    mlups = int(np.prod(params.shape)) * steps / a.elapsed_time(b) / 1e3
    del ref
    torch.cuda.empty_cache()
    return mlups


def _time_pair(lbm, torch, params, steps: int, variant: str):
    """MLUPS of the reference kernel and of this repository's step on the same grid (CUDA events);
    each side first runs the same number of steps untimed (so this repository's CUDA graphs for
    that step count exist before the timed run)."""
    import numpy as np

    backend = "cuda-aa" if variant == "aa" else "cuda-naive"  # tiled: against this build's pull step
    ours = lbm.make_solver(params, backend=backend)
    ours.initialize()
    ref = RefSolver(params, variant)
    ref.set_populations(ours.populations())
    nodes = int(np.prod(params.shape))
    out = {}
    for name, advance in (("reference", ref.advance), ("ours", ours._advance)):
        advance(steps)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        advance(steps)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b)
        out[name] = round(nodes * steps / ms / 1e3, 1)
    del ours, ref
    torch.cuda.empty_cache()
    return out


def main() -> None:
    """Same-box baseline: the reference's kernels and this repository's step, one GPU, MLUPS."""
    import json

    import torch

    sys.path.insert(0, str(HERE.parent))
    import lbm_b200 as lbm

    duct = lbm.SimulationParams(nx=256, ny=256, nz=256, tau=0.9, collision="trt", force=(1e-6, 0.0, 0.0),
                                solid=lbm.duct_walls(256, 256, 256), dtype="float32")
    tgv = lbm.SimulationParams(nx=2048, ny=2048, tau=0.8, collision="trt", dtype="float32")
    result = {
        "duct_256_d3q19_float32": {v: _time_pair(lbm, torch, duct, 200, v) for v in ("naive", "aa")},
        "periodic_2048_d2q9_float32": {v: _time_pair(lbm, torch, tgv, 400, v) for v in ("naive", "tiled", "aa")},
        "unit": "MLUPS (all nodes, CUDA events, inputs larger than L2)",
        "device": torch.cuda.get_device_name(0),
    }
    print(json.dumps(result), flush=True)


def small_case(steps: int = 10) -> None:
    """A profiling case: the reference's pull kernel alone on a 128^3 duct in float32
    (2 x 159 MB of populations, larger than L2), `steps` launches."""
    import torch

    sys.path.insert(0, str(HERE.parent))
    import lbm_b200 as lbm

    n = 128
    p = lbm.SimulationParams(nx=n, ny=n, nz=n, tau=0.9, collision="trt", force=(1e-6, 0.0, 0.0),
                             solid=lbm.duct_walls(n, n, n), dtype="float32")
    ref = RefSolver(p, "naive")
    ref.set_populations(torch.zeros((p.lattice.q, *p.shape), dtype=torch.float32))
    ref.advance(steps)
    torch.cuda.synchronize()
    print(f"reference stream_collide_naive: {steps} steps on a {n}^3 duct")


if __name__ == "__main__":
    if "--build" in sys.argv:
        sys.exit(0 if build(verbose=True) else 1)
    if "--small" in sys.argv:
        small_case()
    else:
        main()
