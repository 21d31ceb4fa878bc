"""The guiding network's tensor-core path (tcgen05 BF16 MMA, FP32 accumulation in TMEM)."""
import ctypes

import numpy as np
import pytest

import xenon_b200 as xb


def bf16_bits(x: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even float32 -> bfloat16 bit patterns."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def bf16_to_f32(b: np.ndarray) -> np.ndarray:
    return (b.astype(np.uint32) << 16).view(np.float32)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 48, 64])
@pytest.mark.parametrize("rows", [128, 300])
def test_tc_gemm_matches_fp64(n, rows):
    rng = np.random.default_rng(n * 1000 + rows)
    a = bf16_bits(rng.normal(size=(rows, 64)))
    b = bf16_bits(rng.normal(size=(n, 64)))
    d = np.zeros((rows, n), np.float32)
    p = lambda x: x.ctypes.data_as(ctypes.c_void_p)
    xb.native.check(xb.lib().xb_tc_gemm_bf16(p(a), p(b), rows, n, p(d)))
    want = bf16_to_f32(a).astype(np.float64) @ bf16_to_f32(b).astype(np.float64).T
    err = np.abs(d - want) / (np.abs(want) + 1.0)
    assert err.max() < 1e-4, (err.max(), np.unravel_index(err.argmax(), err.shape))
