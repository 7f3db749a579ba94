"""The integer steps of the Ozaki slicing kernel (slice_i8_kernel and oz_fixed in
mojoblas_b200/csrc/tc_gemm.cu), restated in Python and checked on the CPU.

For a value v in a row whose largest magnitude is below 2^er, the kernel forms
G = trunc(v 2^(B - er)) with B = 8s - 2 from the double's bits, then writes the
s signed base-256 digits of G, most significant first, as int8 slices: byte j
of H = G + 0x80...80 (s bytes, modulo 2^64), XOR 0x80.  Checked here:

* the closed form equals the carry-propagating signed-digit expansion
  (every G for s = 2, seeded samples with the extremes for s = 3..8);
* digits lie in [-128, 127] and the leading one in [-65, 65] (|G| < 2^(8s-2));
* sum_p d_p 2^(er - 6 - 8p) reconstructs v to within 2^(er - B), the
  truncation bound the error analysis uses, over exponents -60..60, signed
  zeros and subnormals.
The GPU parity tests check the kernel's planes through the products they feed.
"""
import math
import random
import struct

import pytest


def oz_fixed(v, er, B):
    """trunc(v 2^(B - er)) from the bits of v, as the kernel computes it (a Python int)."""
    b = struct.unpack("<Q", struct.pack("<d", v))[0]
    E = (b >> 52) & 0x7FF
    M = (b & ((1 << 52) - 1)) | ((1 << 52) if E else 0)
    sh = (E if E else 1) - 1075 - er + B
    if sh >= 0:
        F = (M << sh) if sh < 64 else 0
    else:
        F = (M >> -sh) if sh > -64 else 0
    return -F if b >> 63 else F


def signed_digits(G, s):
    """Signed base-256 digits of G, most significant first, by carry propagation."""
    out = [0] * s
    for p in range(s - 1, -1, -1):
        d = G & 255
        d = d - 256 if d >= 128 else d
        G = (G - d) // 256
        out[p] = d
    assert G == 0
    return out


def kernel_digits(G, s):
    """The kernel's closed form: bytes of G + 0x80..80 (mod 2^64), each XOR 0x80, as int8."""
    bias = 0x8080808080808080 >> (64 - 8 * s)
    H = (G + bias) % (1 << 64)
    out = []
    for p in range(s):
        byte = ((H >> (8 * (s - 1 - p))) & 255) ^ 0x80
        out.append(byte - 256 if byte >= 128 else byte)
    return out


def test_closed_form_every_value_two_slices():
    s, B = 2, 14
    for G in range(-(1 << B) + 1, 1 << B):
        assert kernel_digits(G, s) == signed_digits(G, s), G


@pytest.mark.parametrize("s", range(3, 9))
def test_closed_form_sampled(s):
    B = 8 * s - 2
    rng = random.Random(100 + s)
    extremes = [0, 1, -1, (1 << B) - 1, -(1 << B) + 1, 127, -128, 128, -129]
    for G in extremes + [rng.randint(-(1 << B) + 1, (1 << B) - 1) for _ in range(20000)]:
        d = kernel_digits(G, s)
        assert d == signed_digits(G, s), (s, G)
        assert all(-128 <= x <= 127 for x in d) and abs(d[0]) <= 65
        assert sum(x * 256 ** (s - 1 - p) for p, x in enumerate(d)) == G


@pytest.mark.parametrize("s", range(2, 9))
def test_reconstruction_within_truncation_bound(s):
    B = 8 * s - 2
    rng = random.Random(200 + s)
    for _ in range(5000):
        mx = rng.uniform(0.5, 1.0) * 2.0 ** rng.randint(-60, 60)
        er = math.frexp(mx)[1]  # the row maximum is below 2^er
        v = rng.choice([1, -1]) * rng.uniform(0, 1) * mx
        if rng.random() < 0.05:
            v = rng.choice([mx, -mx, 0.0, -0.0, 5e-324, -5e-324])
        G = oz_fixed(v, er, B)
        assert abs(G) < 1 << B
        d = kernel_digits(G, s)
        val = sum(x * 2.0 ** (er - 6 - 8 * p) for p, x in enumerate(d))
        assert abs(val - v) <= 2.0 ** (er - B) * (1 + 1e-12), (s, v, val)
