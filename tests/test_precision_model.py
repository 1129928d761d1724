"""The arithmetic model behind the mixed-precision LU (host only, numpy): each FP32 operand is split
into hi = bf16(x) and lo = bf16(x - hi) (round to nearest even, as __float2bfloat16_rn), and a product
is taken as hi_a hi_b + hi_a lo_b + lo_a hi_b with FP32 accumulation.  The split keeps 16 significand
bits, so a product is good to about 2^-16 relative (the dropped lo_a lo_b term and the bits below lo),
against 2^-8 for a single bf16 product; that is why factors from the tensor-core path carry a backward
error near 1e-5 and are refined against FP64 residuals."""
from __future__ import annotations

import numpy as np


def _bf16(x: np.ndarray) -> np.ndarray:
    """Round float32 to the nearest bfloat16 (ties to even), returned as float32."""
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    rounded = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return rounded.astype(np.uint32).view(np.float32)


def test_bf16_rounding_is_nearest_even():
    assert _bf16(np.float32(1.0)) == 1.0
    step = np.float32(2.0 ** -7)                                   # bf16 spacing at 1
    assert _bf16(np.float32(1.0) + step / 2) == 1.0                # tie -> even (1.0)
    assert _bf16(np.float32(1.0) + 3 * step / 2) == 1.0 + 2 * step # tie -> even (1 + 2 step)
    assert _bf16(np.float32(1.0) + step * 0.51) == 1.0 + step


def test_three_product_split_keeps_sixteen_bits():
    rng = np.random.default_rng(7)
    a = rng.normal(size=200_000).astype(np.float32)
    b = rng.normal(size=200_000).astype(np.float32)
    exact = a.astype(np.float64) * b.astype(np.float64)
    ah, bh = _bf16(a), _bf16(b)
    al, bl = _bf16(a - ah), _bf16(b - bh)
    three = (ah.astype(np.float64) * bh + ah.astype(np.float64) * bl + al.astype(np.float64) * bh)
    one = ah.astype(np.float64) * bh
    rel3 = np.abs(three - exact) / np.abs(exact)
    rel1 = np.abs(one - exact) / np.abs(exact)
    assert rel3.max() < 2.0 ** -15 and np.median(rel3) < 2.0 ** -17
    assert rel1.max() > 2.0 ** -9 and np.median(rel1) > 2.0 ** -11
    # a K = 64 complex block update accumulated in FP32 stays near FP32-sum accuracy
    K = 64
    A = rng.normal(size=(256, K)).astype(np.float32)
    B = rng.normal(size=(K, 256)).astype(np.float32)
    split = lambda x: (_bf16(x), _bf16(x - _bf16(x)))
    (Ah, Al), (Bh, Bl) = split(A), split(B)
    C3 = (Ah @ Bh + Ah @ Bl + Al @ Bh).astype(np.float32)
    C = A.astype(np.float64) @ B.astype(np.float64)
    assert np.linalg.norm(C3 - C) / np.linalg.norm(C) < 3e-5
