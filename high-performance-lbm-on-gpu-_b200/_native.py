"""ctypes binding of ``liblbm_b200.so`` (declarations in ``include/lbm_b200.h``).

The library is loaded lazily on first use and never silently replaced: if it
is missing or cannot be loaded the caller gets ``NativeUnavailable``.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "liblbm_b200.so"
ABI_VERSION = 9

LBM_OK, LBM_ERR_INVALID, LBM_ERR_UNSUPPORTED, LBM_ERR_LAUNCH, LBM_ERR_TOO_LARGE = 0, -1, -2, -3, -4
AFFINE_REDUCE_STATIC_MAX_ROWS = 1048576
DENSE_TERMS = 32
# lbm_ibm_force: one block with node and marker arrays (and, when they fit
# too, the body's tables) in shared memory up to IBM_SMEM_BYTES, one block on
# global arrays up to IBM_FUSED_MAX nodes and markers, else a launch per pass
# (the constants of csrc/ibm.cu)
IBM_SMEM_BYTES = 48 * 1024
IBM_FUSED_MAX = 4096
LBM_D2Q9, LBM_D3Q19 = 0, 1
LBM_F32, LBM_F64, LBM_F16, LBM_BF16 = 0, 1, 2, 3
LBM_PULL, LBM_AA_EVEN, LBM_AA_ODD = 0, 1, 2
COLLIDE_TRT, COLLIDE_REGULARIZED, COLLIDE_CUMULANT = 0, 1, 2
COLLISION_CODE = {"bgk": COLLIDE_TRT, "trt": COLLIDE_TRT, "regularized": COLLIDE_REGULARIZED,
                  "cumulant": COLLIDE_CUMULANT}
LAYOUT_PULL, LAYOUT_AA_ODD, LAYOUT_AA_EVEN = 0, 1, 2
KIND_SOLID, KIND_SPECIAL, KIND_NEAR, KIND_EDGE = 1, 2, 4, 8
LAUNCH_FUSED, LAUNCH_BULK, LAUNCH_BOUNDARY = 0, 1, 2
LAUNCH_MODES = (LAUNCH_FUSED, LAUNCH_BULK, LAUNCH_BOUNDARY)
TMA_WAIT_NONE = 0xFFFFFFFF

STORAGE_CODE = {"float32": LBM_F32, "float64": LBM_F64, "float16": LBM_F16, "bfloat16": LBM_BF16}
LATTICE_CODE = {"D2Q9": LBM_D2Q9, "D3Q19": LBM_D3Q19}

vp = C.c_void_p
i32, i64, u32 = C.c_int32, C.c_int64, C.c_uint32


class NativeUnavailable(RuntimeError):
    pass


class NativeError(RuntimeError):
    pass


class Grid(C.Structure):
    _fields_ = [("lattice", i32), ("storage", i32), ("nx", i32), ("ny", i32), ("nz", i32), ("pitch", i32), ("qstride", i64)]


class Physics(C.Structure):
    _fields_ = [
        ("omega_plus", C.c_double), ("omega_minus", C.c_double), ("force", C.c_double * 3),
        ("wall_u", vp), ("force_field", vp), ("solid_nbr", vp), ("collision", i32), ("round_seed", vp),
    ]


class Special(C.Structure):
    _fields_ = [
        ("n_special", i32), ("node", vp), ("rule_mask", vp), ("rule_first", vp), ("force_slot", vp),
        ("export_mask", vp), ("export_first", vp), ("n_rules", i32), ("n_terms", i32), ("term_start", vp),
        ("rule_const", vp), ("term_dir", vp), ("term_node", vp), ("term_export", vp), ("term_coeff", vp),
        ("local_force", vp), ("n_local", i32), ("n_export", i32), ("export_in", vp), ("export_out", vp),
        ("ut_start", vp), ("ut_slot", vp), ("ut_export", vp), ("rule_row", vp), ("rule_dense", vp),
    ]


class Health(C.Structure):
    _fields_ = [("words", vp), ("partial", vp), ("n_partial", i64), ("rho", vp), ("u", vp)]


class Launch(C.Structure):
    _fields_ = [("tile_x", i32), ("tile_y", i32), ("mode", i32), ("tma_wait_limit", u32), ("health", C.POINTER(Health))]


class Ibm(C.Structure):
    _fields_ = [
        ("n_nodes", i32), ("n_markers", i32), ("stencil_size", i32), ("node", vp), ("stencil", vp),
        ("weight", vp), ("area", vp), ("inv_start", vp), ("inv_marker", vp), ("inv_weight", vp),
        ("rho", vp), ("u_star", vp), ("marker_force", vp), ("marker_scratch", vp),
    ]


class Adjoint(C.Structure):
    _fields_ = [
        ("gather_start", vp), ("gather_dir", vp), ("gather_slot", vp), ("gather_coeff", vp), ("rule_dconst", vp),
        ("term_dcoeff", vp), ("rule_du", vp), ("force_grad", vp), ("local_force_grad", vp), ("rule_ddense", vp),
    ]


class Domain(C.Structure):
    _fields_ = [
        ("nx", i32), ("ny", i32), ("nz", i32), ("pitch", i32), ("offset", i64), ("qstride", i64),
        ("kind_offset", i64), ("wall_offset", i64), ("omega_plus", C.c_double), ("omega_minus", C.c_double),
        ("force", C.c_double * 3),
    ]


class Batch(C.Structure):
    _fields_ = [
        ("lattice", i32), ("storage", i32), ("n_domains", i32), ("domains", vp), ("n_tiles", i32), ("tiles", vp),
        ("tile_x", i32), ("tile_y", i32), ("blocks", i32), ("kind", vp), ("solid_nbr", vp), ("wall_u", vp),
        ("round_seed", vp),
    ]


P = C.POINTER
_SIGNATURES = {
    "lbm_adjoint_step": [P(Grid), P(Physics), P(Special), P(Adjoint), P(Launch), vp, vp, vp, vp, C.c_double, vp],
    "lbm_adjoint_initial": [P(Grid), P(Physics), P(Special), P(Adjoint), vp, vp, vp, vp, C.c_double, vp],
    "lbm_batch_step": [P(Batch), vp, vp, vp],
    "lbm_batch_occupancy": [i32, i32, i32, i32, vp],
    "lbm_step_pull": [P(Grid), P(Physics), P(Special), P(Launch), vp, vp, vp, vp],
    "lbm_step_aa": [P(Grid), P(Physics), P(Special), P(Launch), vp, vp, i32, vp],
    "lbm_export_prime": [P(Grid), P(Special), vp, i32, vp, vp],
    "lbm_classify": [P(Grid), vp, vp, i32, vp, vp, vp],
    "lbm_init_equilibrium": [P(Grid), P(Physics), vp, vp, i32, vp, vp],
    "lbm_unpack": [P(Grid), vp, i32, vp, vp],
    "lbm_pack": [P(Grid), vp, i32, vp, vp],
    "lbm_macroscopic": [P(Grid), P(Physics), vp, vp, i32, vp, vp, i32, vp, vp, vp],
    "lbm_health_reset": [vp, vp],
    "lbm_health_finish": [P(Health), vp, vp],
    "lbm_health": [P(Grid), vp, vp, vp, vp],
    "lbm_affine_gather": [i32, vp, vp, vp, vp, i64, i32, vp, vp],
    "lbm_affine_reduce": [i32, vp, vp, vp, vp, vp, i64, i32, i32, vp, vp, vp, vp],
    "lbm_affine_reduce_static": [i32, vp, vp, vp, vp, vp, i64, i32, i32, vp, vp],
    "lbm_ibm_moments": [P(Grid), P(Physics), P(Ibm), vp, i32, vp],
    "lbm_ibm_iteration": [P(Grid), P(Ibm), i32, vp, vp, vp],
    "lbm_ibm_force": [P(Grid), P(Physics), P(Ibm), vp, i32, i32, vp, vp],
    "lbm_step_pull_ibm": [P(Grid), P(Physics), P(Special), P(Ibm), i32, vp, vp, vp, vp, vp],
    "lbm_ibm_body_force": [P(Grid), P(Ibm), i32, vp, vp],
    "lbm_ibm_adjoint_iteration": [P(Grid), P(Ibm), vp, vp, i32, C.c_double, vp, vp, vp],
    "lbm_ibm_adjoint_moments": [P(Grid), P(Ibm), vp, vp, vp],
    "lbm_kernel_resources": [i32, i32, i32, vp],
    "lbm_ball_voxelize": [P(Grid), C.c_double, C.c_double, C.c_double, C.c_double, vp, vp],
    "lbm_ball_links_count": [P(Grid), vp, C.c_double, C.c_double, C.c_double, C.c_double, vp, vp],
    "lbm_ball_links_write": [P(Grid), vp, C.c_double, C.c_double, C.c_double, C.c_double, vp, vp, vp, vp, vp],
    "lbm_bouzidi_links": [P(Grid), vp, i64, vp, vp, vp, vp, vp, vp, vp, vp],
    "lbm_compile_terms": [P(Grid), i32, vp, vp, i64, vp, vp, vp, vp, vp, vp],
    "lbm_zou_he_count": [P(Grid), vp, i32, i32, i32, vp, vp, C.c_double, vp, vp],
    "lbm_zou_he_write": [P(Grid), vp, i32, i32, i32, vp, vp, C.c_double, vp, i32, vp, vp, vp, vp, vp, vp, vp],
}
EXPORTED = (*_SIGNATURES, "lbm_health_partials", "lbm_ball_links_scratch", "lbm_zou_he_scratch",
            "lbm_last_cuda_error", "lbm_abi_version")

_lib = None


def load(path: Path | None = None):
    """Load the library once; raise ``NativeUnavailable`` if it cannot be loaded."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    target = Path(path) if path is not None else LIBRARY
    if not target.exists():
        raise NativeUnavailable(f"{target.name} is not built; run build() from __graft_entry__ or build.py")
    try:
        lib = C.CDLL(str(target))
    except OSError as exc:
        raise NativeUnavailable(f"cannot load {target}: {exc}") from exc
    for name, args in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = C.c_int
    lib.lbm_health_partials.argtypes = [P(Grid), P(Special), P(Launch)]
    lib.lbm_health_partials.restype = i64
    lib.lbm_ball_links_scratch.argtypes = [P(Grid)]
    lib.lbm_ball_links_scratch.restype = i64
    lib.lbm_zou_he_scratch.argtypes = [P(Grid)]
    lib.lbm_zou_he_scratch.restype = i64
    lib.lbm_last_cuda_error.restype = C.c_char_p
    lib.lbm_last_cuda_error.argtypes = []
    lib.lbm_abi_version.restype = i32
    lib.lbm_abi_version.argtypes = []
    if lib.lbm_abi_version() != ABI_VERSION:
        raise NativeUnavailable(f"{target.name} has ABI {lib.lbm_abi_version()}, expected {ABI_VERSION}")
    if path is None:
        _lib = lib
    return lib


def check(status: int, what: str) -> None:
    if status == LBM_OK:
        return
    lib = load()
    if status == LBM_ERR_LAUNCH:
        raise NativeError(f"{what}: CUDA launch failed ({lib.lbm_last_cuda_error().decode()})")
    if status == LBM_ERR_UNSUPPORTED:
        raise NativeError(f"{what}: unsupported configuration")
    if status == LBM_ERR_TOO_LARGE:
        raise NativeError(f"{what}: size beyond the library's fixed scratch limit")
    raise NativeError(f"{what}: invalid argument (status {status})")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args), name)


def ptr(tensor) -> int | None:
    """Device address of a torch tensor (None for None)."""
    return None if tensor is None else tensor.data_ptr()
