"""The gradient kernel's integer-pipe widening (widen_scaled in autan_b200/csrc/euler_device.cu),
restated in numpy: the float's bits moved into a double with a signed 32 x 32 -> 64 multiply by
2^29 and an AND of the high word's bits 28-30. Checked here against exact scaling by 2^-896, and
FP64 sums of such values against 2^-896 times the sums of the cvt-widened products, on every
class of finite float (normal, subnormal, zero of either sign) and on stencil-like sequences."""

import numpy as np


def widen_scaled(p: np.ndarray) -> np.ndarray:
    bits = p.astype(np.float32).view(np.int32).astype(np.int64)
    wide = bits * (1 << 29)  # the signed 32 x 32 -> 64 product
    lo = wide & 0xFFFFFFFF
    hi = (wide >> 32) & 0x8FFFFFFF
    return ((hi << 32) | lo).astype(np.uint64).view(np.float64)


def finite_floats(rng, n):
    """Normal, subnormal and zero floats of both signs, all exponents."""
    bits = rng.integers(0, 2**32, size=n, dtype=np.uint64).astype(np.uint32)
    x = bits.view(np.float32)
    x = x[np.isfinite(x)]
    special = np.array([0.0, -0.0, 1e-45, -1e-45, 1.1754942e-38, -1.1754942e-38, 1.1754944e-38,
                        3.4028235e38, -3.4028235e38, 1.0, -1.0], dtype=np.float32)
    return np.concatenate([x, special])


def test_widening_is_exact_scaling():
    rng = np.random.default_rng(3)
    x = finite_floats(rng, 200_000)
    got = widen_scaled(x)
    want = np.ldexp(x.astype(np.float64), -896)
    assert np.array_equal(got.view(np.uint64), want.view(np.uint64))


def test_scaled_sums_equal_the_cvt_sums():
    """Sequential FP64 sums (the stencil order) of scaled values, times 2^896, equal the sums of
    the cvt-widened values bit for bit: random products of stencil magnitudes, products that cancel
    to subnormal scaled sums, and tiny products near the float subnormal range."""
    rng = np.random.default_rng(4)
    cases = []
    for _ in range(2000):
        n = int(rng.integers(1, 40))
        scale = 10.0 ** rng.uniform(-40, 30)
        dw = (rng.standard_normal(n) * scale).astype(np.float32)
        w = (rng.standard_normal(n) * 10.0 ** rng.uniform(-3, 3)).astype(np.float32)
        cases.append(dw * w)
    # cancellation: a product and its negation with small leftovers
    for _ in range(500):
        a = (rng.standard_normal(8) * 10.0 ** rng.uniform(-38, -30)).astype(np.float32)
        cases.append(np.concatenate([a, -a[::-1], a[:3] * np.float32(1e-3)]).astype(np.float32))
    cases.append(finite_floats(rng, 64)[:64])
    for p in cases:
        p = p.astype(np.float32)
        ref = np.float64(0.0)
        for v in p.astype(np.float64):
            ref = ref + v
        acc = np.float64(0.0)
        for v in widen_scaled(p):
            acc = acc + v
        got = acc * np.float64(2.0**896)
        if np.isfinite(ref) and abs(ref) < 2.0**120:
            assert got.view(np.uint64) == ref.view(np.uint64), (p, got, ref)


def test_integer_multiply_equals_the_two_shifts():
    """The multiply's high word is the arithmetic shift right by 3 and its low word the shift left
    by 29: the restatement does not depend on how a compiler lowers the multiply."""
    rng = np.random.default_rng(5)
    b = rng.integers(-(2**31), 2**31, size=100_000, dtype=np.int64)
    wide = b * (1 << 29)
    assert np.array_equal((wide >> 32) & 0xFFFFFFFF, (b >> 3) & 0xFFFFFFFF)
    assert np.array_equal(wide & 0xFFFFFFFF, (b << 29) & 0xFFFFFFFF)
