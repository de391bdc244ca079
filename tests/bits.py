"""Bitwise comparison helpers for the bit-exact parity tests."""
import numpy as np


def bits_equal(a, b) -> bool:
    """True when both arrays hold the same floating-point bit patterns (signed zeros and NaN
    payloads included)."""
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    if a.shape != b.shape or a.dtype != b.dtype:
        return False
    iv = np.int64 if a.dtype == np.float64 else np.int32
    return bool(np.array_equal(a.view(iv), b.view(iv)))
