"""The slicer's bit-field digits equal repeated truncation (host model of k_slice's arithmetic).

k_slice (shtensor_b200/csrc/split.cu) cuts y = v * 2^-e, |y| < 1, into S signed 7-bit slices.
The definition is repeated truncation, s_t = trunc(128 * remainder).  The kernel instead reads
the 7-bit fields of the mantissa of z = 1 + |y| rounded toward zero, negates them for negative
v, and negates four packed bytes at once with ((b ^ 0x7f) + 1) ^ 0x80.  These tests model that
arithmetic in numpy and check it against the definition, for S = 1..8.
"""
import math

import numpy as np
import pytest


def trunc_slices(y, S):
    out, v = [], y.copy()
    for _ in range(S):
        Y = v * 128.0
        tr = np.trunc(Y)
        out.append(tr.astype(np.int64))
        v = Y - tr
    return out


def field_slices(y, S):
    a = np.abs(y)
    # z = 1 + |y| rounded toward zero: 1 + floor(|y| 2^52) 2^-52 (exact)
    frac = np.array([math.floor(math.ldexp(x, 52)) for x in a], dtype=np.int64)
    z = 1.0 + frac.astype(np.float64) * 2.0 ** -52
    W = z.view(np.uint64)
    zl = W & np.uint64(0xFFFFFFFF)
    out = []
    for t in range(1, S + 1):
        if t <= 7:
            d = ((W >> np.uint64(52 - 7 * t)) & np.uint64(127)).astype(np.int64)
        else:
            tail = a - (z - 1.0)  # the bits of |y| below 2^-52, exact
            d = ((zl & np.uint64(7)) << np.uint64(4)).astype(np.int64) | np.trunc(tail * 2.0 ** 56).astype(np.int64)
        out.append(np.where(np.signbit(y), -d, d))
    return out


@pytest.mark.parametrize("S", range(1, 9))
def test_field_slices_equal_truncation(S):
    rng = np.random.default_rng(11 + S)
    n = 20000
    y = rng.uniform(-1, 1, n) * 2.0 ** rng.integers(-60, 1, n)
    top = np.nextafter(1.0, 0.0)
    y = np.clip(y, -top, top)
    y[:10] = [0.0, -0.0, 0.5, -0.5, top, -top, 2.0 ** -49, 2.0 ** -50, 2.0 ** -53, -(2.0 ** -56)]
    for a, b in zip(trunc_slices(y, S), field_slices(y, S)):
        assert np.array_equal(a, b)


def test_packed_negation():
    # per byte: b in [0, 127] (bit 7 may hold another field's bit), mask 0x00 or 0xff
    for b in range(256):
        for m in (0x00, 0xFF):
            got = ((((b ^ m) & 0x7F) + (m & 0x01)) ^ (m & 0x80)) & 0xFF
            want = ((b & 0x7F) if m == 0 else -(b & 0x7F)) & 0xFF
            assert got == want
    # four bytes at once: no carry between bytes
    rng = np.random.default_rng(3)
    for _ in range(2000):
        bs = rng.integers(0, 256, 4)
        ms = rng.choice([0, 0xFF], 4)
        pk = int(sum(int(x) << (8 * i) for i, x in enumerate(bs)))
        sm = int(sum(int(x) << (8 * i) for i, x in enumerate(ms)))
        w = ((((pk ^ sm) & 0x7F7F7F7F) + (sm & 0x01010101)) ^ (sm & 0x80808080)) & 0xFFFFFFFF
        for i in range(4):
            b = int(bs[i]) & 0x7F
            assert (w >> (8 * i)) & 0xFF == ((b if ms[i] == 0 else -b) & 0xFF)
