"""lbm_affine_reduce_static: the force-probe reduction with its scratch inside the library (GPU).

Called through the C ABI and compared with lbm_affine_reduce (caller-provided
scratch) on the same inputs, twice in a row so the second call runs on the
scratch the first one left behind.
"""

from __future__ import annotations

import numpy as np
import pytest

from lbm_b200 import _native as N

pytestmark = pytest.mark.gpu

TORCH_DTYPE = {"float32": "float32", "float64": "float64", "float16": "float16", "bfloat16": "bfloat16"}


def probe_inputs(storage: str, n_rows: int, n_terms: int, d: int, seed: int):
    import torch

    gen = torch.Generator().manual_seed(seed)
    n_slots = 40_000
    f = (0.01 * torch.randn(n_slots, generator=gen, dtype=torch.float64)).to(getattr(torch, TORCH_DTYPE[storage]))
    slots = torch.randint(0, n_slots, (n_rows * n_terms,), generator=gen, dtype=torch.int64)
    coeff = torch.randn(n_rows * n_terms, generator=gen, dtype=torch.float64)
    constant = 1e-3 * torch.randn(n_rows, generator=gen, dtype=torch.float64)
    weight = torch.randn(n_rows * d, generator=gen, dtype=torch.float64)
    return [t.cuda() for t in (f, slots, coeff, constant, weight)]


def reduce_with_buffers(lib, storage, f, slots, coeff, constant, weight, n_rows, n_terms, d, stream):
    import torch

    partial = torch.empty((n_rows + 255) // 256 * d, dtype=torch.float64, device="cuda")
    counter = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.empty(d, dtype=torch.float64, device="cuda")
    status = lib.lbm_affine_reduce(N.STORAGE_CODE[storage], N.ptr(f), N.ptr(slots), N.ptr(coeff), N.ptr(constant),
                                   N.ptr(weight), n_rows, n_terms, d, N.ptr(partial), N.ptr(counter), N.ptr(out),
                                   stream)
    N.check(status, "lbm_affine_reduce")
    return out


@pytest.mark.parametrize("storage,n_rows,n_terms,d", [
    ("float64", 1_000, 3, 2),
    ("float32", 70_001, 2, 3),
    ("float16", 257, 4, 3),
    ("bfloat16", 4_096, 1, 2),
    ("float64", N.AFFINE_REDUCE_STATIC_MAX_ROWS, 2, 3),
])
def test_static_reduce_matches_the_buffered_reduce_twice_in_a_row(storage, n_rows, n_terms, d):
    """Same kernel and summation order: agreement to 1e-12 relative (observed: identical bits)."""
    import torch

    lib = N.load()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    args = probe_inputs(storage, n_rows, n_terms, d, seed=n_rows)
    want = reduce_with_buffers(lib, storage, *args, n_rows, n_terms, d, stream)
    outs = []
    for _ in range(2):
        out = torch.full((d,), float("nan"), dtype=torch.float64, device="cuda")
        status = lib.lbm_affine_reduce_static(N.STORAGE_CODE[storage], *(N.ptr(t) for t in args), n_rows, n_terms, d,
                                              N.ptr(out), stream)
        N.check(status, "lbm_affine_reduce_static")
        outs.append(out)
    torch.cuda.synchronize()
    w = want.cpu().numpy()
    assert np.all(np.isfinite(w))
    for out in outs:
        np.testing.assert_allclose(out.cpu().numpy(), w, rtol=1e-12, atol=1e-12 * np.abs(w).max())


def test_static_reduce_rejects_more_rows_than_its_scratch_holds():
    import torch

    lib = N.load()
    args = probe_inputs("float64", 4, 1, 3, seed=1)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    n_rows = N.AFFINE_REDUCE_STATIC_MAX_ROWS + 1
    status = lib.lbm_affine_reduce_static(N.LBM_F64, *(N.ptr(t) for t in args), n_rows, 1, 3, N.ptr(out),
                                          torch.cuda.current_stream().cuda_stream)
    assert status == N.LBM_ERR_TOO_LARGE
    with pytest.raises(N.NativeError, match="scratch limit"):
        N.check(status, "lbm_affine_reduce_static")
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0  # nothing was launched


@pytest.mark.parametrize("change", [
    {"n_rows": 0}, {"n_rows": -5}, {"d": 0}, {"d": 4}, {"storage": 7}, {"storage": -1}, {"n_terms": -1},
    {"null": 0}, {"null": 1}, {"null": 2}, {"null": 3}, {"null": 4}, {"out_null": True},
])
def test_static_reduce_rejects_invalid_arguments_and_launches_nothing(change):
    """Every early return: LBM_ERR_INVALID and an untouched output (nothing is launched)."""
    import torch

    lib = N.load()
    torch.cuda.set_device(0)
    args = [N.ptr(t) for t in probe_inputs("float64", 4, 2, 3, seed=2)]
    if "null" in change:
        args[change["null"]] = None
    n_rows, n_terms, d = change.get("n_rows", 4), change.get("n_terms", 2), change.get("d", 3)
    storage = change.get("storage", N.LBM_F64)
    out = torch.zeros(3, dtype=torch.float64, device="cuda")
    status = lib.lbm_affine_reduce_static(storage, *args, n_rows, n_terms, d,
                                          None if change.get("out_null") else N.ptr(out),
                                          torch.cuda.current_stream().cuda_stream)
    assert status == N.LBM_ERR_INVALID
    torch.cuda.synchronize()
    assert torch.count_nonzero(out).item() == 0
