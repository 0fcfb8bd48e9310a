"""Stochastic rounding of 16-bit stored populations: the oracle's emulation and the device hash (CPU)."""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import lowbias32, stochastic_round
from oracle.lbm_oracle import FP16_SCALE, SR_MULT, sr_keys

ROOT = Path(__file__).resolve().parent.parent


def between(lo: np.ndarray, hi: np.ndarray, frac: float) -> np.ndarray:
    return (lo.astype(np.float64) + frac * (hi.astype(np.float64) - lo.astype(np.float64))).astype(np.float32)


@pytest.mark.parametrize("frac", [0.1, 0.25, 0.5, 0.9])
def test_float16_rounds_up_with_probability_equal_to_the_fraction(frac):
    """Over 2^16 nodes the share rounded up is frac within 5 standard deviations."""
    n = 1 << 16
    lo16 = np.linspace(0.1, 60.0, n).astype(np.float16)  # scaled values, normal float16 range
    hi16 = np.nextafter(lo16, np.float16(np.inf))
    lo = lo16.astype(np.float32) / np.float32(FP16_SCALE)
    hi = hi16.astype(np.float32) / np.float32(FP16_SCALE)
    x = between(lo, hi, frac)[None, :]
    out = stochastic_round(x, "float16", step=7)[0]
    assert np.all((out == lo) | (out == hi))
    up = np.mean(out == hi)
    assert abs(up - frac) < 5 * np.sqrt(frac * (1 - frac) / n)


def test_bfloat16_is_unbiased_on_average():
    rng = np.random.default_rng(0)
    x = rng.normal(0.0, 1e-3, size=(19, 4096)).astype(np.float32)
    errs = [stochastic_round(x, "bfloat16", step=t) - x for t in range(16)]
    mean_err = np.mean(errs)
    spread = np.std(errs) / np.sqrt(np.size(errs))
    assert abs(mean_err) < 5 * spread
    for e in errs:  # never more than one bfloat16 gap away
        assert np.all(np.abs(e) <= np.abs(x) * 2.0**-7 + 1e-30)


@pytest.mark.parametrize("dtype", ["float16", "bfloat16"])
def test_representable_values_are_unchanged_and_runs_reproduce(dtype):
    rng = np.random.default_rng(1)
    x = rng.normal(0.0, 1e-2, size=(9, 500)).astype(np.float32)
    once = stochastic_round(x, dtype, step=3)
    np.testing.assert_array_equal(stochastic_round(once, dtype, step=11), once)
    np.testing.assert_array_equal(stochastic_round(x, dtype, step=3), once)
    assert np.any(stochastic_round(x, dtype, step=4) != once)


def test_wider_formats_are_not_rounded():
    x = np.linspace(-1, 1, 90, dtype=np.float32).reshape(9, 10)
    assert stochastic_round(x, "float32", step=0) is x


@pytest.mark.skipif(shutil.which("nvcc") is None, reason="needs nvcc")
def test_device_hash_matches_the_oracle(tmp_path):
    """lowbias32, the direction keys and the multiplier of lbm_common.cuh, run on the host, equal the NumPy ones."""
    src = tmp_path / "hash.cu"
    src.write_text(
        '#include "lbm_common.cuh"\n#include <cstdio>\n'
        "int main() { const unsigned xs[] = {0u, 1u, 2u, 12345u, 4000000000u, 0xffffffffu};\n"
        '  for (unsigned x : xs) printf("%u\\n", lbm::lowbias32(x));\n'
        '  for (int i = 0; i < 19; ++i) printf("%u\\n", lbm::sr_key(i));\n'
        '  printf("%u\\n", lbm::SR_MULT);\n  return 0; }\n'
    )
    exe = tmp_path / "hash"
    csrc = ROOT / "high-performance-lbm-on-gpu-_b200" / "csrc"
    subprocess.run(["nvcc", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", f"-I{csrc}", str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    vals = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    xs = np.array([0, 1, 2, 12345, 4000000000, 0xFFFFFFFF], dtype=np.uint64).astype(np.uint32)
    assert vals[:6] == [int(v) for v in lowbias32(xs)]
    assert vals[6:25] == [int(v) for v in sr_keys(19)]
    assert vals[25] == SR_MULT


def test_pairs_share_a_word_but_not_their_bits():
    """Neighbouring nodes of a pair round with different halves of the same random word."""
    x = np.full((19, 2, 4096), 1.0 + 0.5 * 2.0**-10, dtype=np.float32) / np.float32(2.0**14)
    out = stochastic_round(x.reshape(19, 2 * 4096), "float16", step=5).reshape(19, 2, 4096)
    up = out > x
    assert abs(up.mean() - 0.5) < 0.02
    assert abs(np.mean(up[:, 0] == up[:, 1]) - 0.5) < 0.03  # even and odd nodes decide independently
