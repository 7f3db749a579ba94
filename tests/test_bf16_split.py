"""The split-precision pre-pass (split_store4 in mojoblas_b200/csrc/tc_gemm.cu),
restated in numpy and checked on the CPU.

Each fp32 element x is split into bf16 terms by repeated round-to-nearest-even:
x1 = bf16(x), x2 = bf16(x - x1), x3 = bf16(x - x1 - x2), every difference
formed in fp32.  Checked here, over magnitudes 2^-60..2^60 and the values
where rounding carries into the exponent:

* every fp32 difference is exact (x_t - h_t equals the float64 difference);
* three terms (BF16x6) represent x exactly: x1 + x2 + x3 == x;
* two terms (BF16x3) leave |x - x1 - x2| <= 2^-16 |x|, the residual that makes
  BF16x3's error independent of k and above plain fp32's at short k.
The bf16 products of the terms are exact in the tensor cores' fp32
accumulation (8-bit by 8-bit significands); the GPU parity tests check the rest.
"""
import numpy as np
import pytest


def bf16_rn(x):
    """float32 -> bf16 (round to nearest, ties to even), returned as float32."""
    b = x.astype(np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) >> 16 << 16
    return r.astype(np.uint32).view(np.float32)


def split(x, terms):
    x = x.astype(np.float32)
    out = []
    for _ in range(terms):
        h = bf16_rn(x)
        d = x - h  # fp32, as the kernel forms it
        assert np.array_equal(d.astype(np.float64), x.astype(np.float64) - h.astype(np.float64))
        out.append(h)
        x = d
    return out, x


def samples():
    rng = np.random.default_rng(7)
    x = (rng.uniform(1, 2, 200000) * 2.0 ** rng.integers(-60, 61, 200000)).astype(np.float32)
    x *= np.where(rng.random(x.size) < 0.5, -1, 1).astype(np.float32)
    # significands just below a power of two (bf16 rounding carries into the exponent) and exact bf16 values
    edge = np.array([1.9999999, 1.99609375, 1.0, 1.00390625, 1.0039063, 1.5, 1.2345678], np.float32)
    return np.concatenate([x, edge, -edge, edge * np.float32(2.0 ** 40)])


def test_bf16_rounding_is_ties_to_even():
    x = np.array([1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, 1.0 + 2 ** -9], np.float32)  # two ties, one below half
    assert np.array_equal(bf16_rn(x), np.array([1.0, 1.0 + 2 ** -6, 1.0], np.float32))


def test_three_terms_are_exact():
    x = samples()
    terms, rest = split(x, 3)
    assert np.all(rest == 0)
    total = sum(t.astype(np.float64) for t in terms)
    assert np.array_equal(total, x.astype(np.float64))


@pytest.mark.parametrize("terms,bound", [(1, 2.0 ** -8), (2, 2.0 ** -16)])
def test_truncated_split_residual(terms, bound):
    x = samples()
    _, rest = split(x, terms)
    assert np.all(np.abs(rest.astype(np.float64)) <= bound * np.abs(x.astype(np.float64)))
