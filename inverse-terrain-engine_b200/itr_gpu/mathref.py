"""Python copy of csrc/itr_math.h (deterministic exp / log1p / softplus), same operation
sequence in IEEE double, so host-side J equals the device's bit for bit."""
from __future__ import annotations

import struct


def _b2d(b: int) -> float:
    return struct.unpack("<d", struct.pack("<Q", b & 0xFFFFFFFFFFFFFFFF))[0]


def _d2b(d: float) -> int:
    return struct.unpack("<Q", struct.pack("<d", d))[0]


_LN2_HI = _b2d(0x3FE62E42FEFA39EF & ~((1 << 21) - 1))
_LN2_LO = (_b2d(0x3FE62E42FEFA39EF) - _LN2_HI) + 2.3190468138462996e-17


def _pow2i(k: int) -> float:
    return _b2d((k + 1023) << 52)


_EXP_C = [1.0 / 479001600.0, 1.0 / 39916800.0, 1.0 / 3628800.0, 1.0 / 362880.0, 1.0 / 40320.0, 1.0 / 5040.0,
          1.0 / 720.0, 1.0 / 120.0, 1.0 / 24.0, 1.0 / 6.0, 0.5]


def exp_ref(x: float) -> float:
    if x != x:
        return x
    if x > 709.782712893384:
        return float("inf")
    if x < -745.1332191019412:
        return 0.0
    kf = x * 1.4426950408889634
    kf = float(int(kf - 0.5)) if kf < 0.0 else float(int(kf + 0.5))
    k = int(kf)
    r = (x - kf * _LN2_HI) - kf * _LN2_LO
    p = 1.0 / 6227020800.0
    for c in _EXP_C:
        p = p * r + c
    e = 1.0 + (r + (r * r) * p)
    if k > 1023:
        return (e * 2.0) * _pow2i(k - 1)
    if k < -1022:
        return (e * _pow2i(k + 600)) * _pow2i(-600)
    return e * _pow2i(k)


_ATANH_C = [1.0 / 23.0, 1.0 / 21.0, 1.0 / 19.0, 1.0 / 17.0, 1.0 / 15.0, 1.0 / 13.0, 1.0 / 11.0, 1.0 / 9.0, 1.0 / 7.0,
            1.0 / 5.0, 1.0 / 3.0]


def _two_atanh(s: float) -> float:
    s2 = s * s
    p = 1.0 / 25.0
    for c in _ATANH_C:
        p = p * s2 + c
    return 2.0 * s + 2.0 * (s * (s2 * p))


def log1p_ref(x: float) -> float:
    if x != x:
        return x
    if x == 0.0:
        return x
    if x < -1.0:
        return float("nan")
    if x == -1.0:
        return float("-inf")
    if x > 1.7976931348623157e308:
        return x
    if -0.25 < x < 0.25:
        return _two_atanh(x / (2.0 + x))
    u = 1.0 + x
    c = (x - (u - 1.0)) / u
    b = _d2b(u)
    e = ((b >> 52) & 0x7FF) - 1023
    m = _b2d((b & 0x000FFFFFFFFFFFFF) | 0x3FF0000000000000)
    if m > 1.4142135623730951:
        m = m * 0.5
        e += 1
    lm = _two_atanh((m - 1.0) / (m + 1.0))
    ef = float(e)
    return ef * _LN2_HI + ((ef * _LN2_LO + lm) + c)


def softplus(x: float) -> float:
    """softplus of objective.rs:70-75 on the shared exp/log1p."""
    if x > 30.0:
        return x
    if x < -30.0:
        return exp_ref(x)
    return log1p_ref(exp_ref(x))
